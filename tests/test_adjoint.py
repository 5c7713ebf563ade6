"""Adjoint gradients of a receiver misfit (coseis_b200/adjoint.py,
sord_adjoint_* in include/sordgpu.h) against central finite differences of
the FP64 oracle forward run, along seeded random directions.

The misfit is L = 1/2 sum (v_receiver - v_observed)^2 over 4 receivers x 3
components x every step, the observed traces coming from a second seeded
model.  FD step h = 1e-3 relative; the bound enforced is 1e-3 relative."""
import math
import os
import shutil

import numpy as np
import pytest

import sordcases as sc

from coseis_b200 import adjoint

SHAPE = (18, 16, 14)
NT = 40
H_FD = 1e-3
TOL = 1e-3


def problem(segment=7, pml=False, snapshots=None):
    """Free surfaces on every face, or (pml) a free surface at l = 1 and a
    4-node PML on the other five faces with a fixed damping velocity (vpml
    derived from the material's extremes would move with the material)."""
    prm = {
        'shape': list(SHAPE) + [NT], 'delta': [100.0, 100.0, 100.0, 0.008],
        'bc1': ['free'] * 3, 'bc2': ['free'] * 3, 'npml': 0, 'hourglass': [1.0, 0.5], 'gam': [0.0],
        'tm0': -0.15, 'itstats': 10, 'itio': 20,
    }
    if pml:
        prm.update({'bc1': ['pml', 'pml', 'free'], 'bc2': ['pml'] * 3, 'npml': 4, 'vpml': 4500.0})
    src = {'x': [8.3, 7.6, 6.4], 'pulse': 'ricker2', 'tau': 0.05}
    rng = np.random.default_rng(7)
    rec = [[float(rng.uniform(2, SHAPE[0] - 3)), float(rng.uniform(2, SHAPE[1] - 3)), 0.0] for _ in range(4)]
    return adjoint.Problem(prm, src, rec, segment=segment, snapshots=snapshots)


def model(seed):
    """Background 2700 / 6000 / 3464 with a 10 % Gaussian blob at a seeded place."""
    rng = np.random.default_rng(seed)
    nc = tuple(n - 1 for n in SHAPE)
    j, k, l = np.meshgrid(*[np.arange(n) + 0.5 for n in nc], indexing='ij')
    c = [rng.uniform(0.3, 0.7) * n for n in nc]
    b = np.exp(-((j - c[0]) ** 2 + (k - c[1]) ** 2 + (l - c[2]) ** 2) / (2 * 3.0 ** 2))
    amp = rng.uniform(-0.1, 0.1, 3)
    m = rng.standard_normal(6)
    m *= 1e15 / math.sqrt((m[:3] ** 2).sum() + 2 * (m[3:] ** 2).sum())
    return (2700.0 * (1 + amp[0] * b), 6000.0 * (1 + amp[1] * b), 3464.0 * (1 + amp[2] * b), m)


def oracle_traces(p, rho, vp, vs, mom, path, exe):
    shutil.rmtree(path, ignore_errors=True)
    p.stage(rho, vp, vs, mom, path, realsize=8)
    sc.run_oracle(path, exe)
    return p.read_traces(path, '<f8')


def test_material_chain_matches_finite_differences():
    """The chain rule of the material setup, against central differences of a
    direct evaluation of lambda, mu, yy (cells) and mr (nodes)."""
    rng = np.random.default_rng(3)
    nc = (4, 3, 5)
    rho = 2500 + 300 * rng.random(nc)
    vp = 5500 + 800 * rng.random(nc)
    vs = 3000 + 500 * rng.random(nc)
    delta = [100.0, 80.0, 120.0]
    g = {'lam': rng.standard_normal(nc), 'mu': rng.standard_normal(nc), 'yy': rng.standard_normal(nc),
         'mr': rng.standard_normal(tuple(n + 1 for n in nc)) * 1e12}
    s = math.sqrt(sum(d * d for d in delta) / 3) / 12
    V = delta[0] * delta[1] * delta[2]

    def F(r, a, b):
        mu = r * b * b
        lam = r * a * a - 2 * mu
        yy = mu * (lam + mu) * s / (lam + 2 * mu)
        S = np.zeros(tuple(n + 1 for n in nc))
        for dj in (0, 1):
            for dk in (0, 1):
                for dl in (0, 1):
                    S[dj:dj + nc[0], dk:dk + nc[1], dl:dl + nc[2]] += r * V
        mr = 8.0 / S
        return (g['lam'] * lam).sum() + (g['mu'] * mu).sum() + (g['yy'] * yy).sum() + (g['mr'] * mr).sum()

    grads = adjoint.material_chain(rho, vp, vs, g, delta)
    for x, gx in zip(range(3), grads):
        d = rng.standard_normal(nc)
        h = 1e-6
        args = [rho, vp, vs]
        ap = list(args); ap[x] = args[x] * (1 + h * d)
        am = list(args); am[x] = args[x] * (1 - h * d)
        fd = (F(*ap) - F(*am)) / (2 * h)
        an = (gx * args[x] * d).sum()
        assert abs(fd - an) <= 1e-6 * max(abs(fd), 1e-30), (x, fd, an)


def test_problem_stages_moment_and_receivers(tmp_path):
    p = problem()
    rho, vp, vs, m = model(1)
    p.stage(rho, vp, vs, m, str(tmp_path))
    text = open(str(tmp_path / 'sord.in')).read()
    assert sorted(adjoint.MOMENT[c] for c in p.moment_order(str(tmp_path))) == sorted(adjoint.MOMENT)
    assert text.count('.>') == 12
    assert os.path.getsize(str(tmp_path / 'rho.bin')) == 4 * np.prod([n - 1 for n in SHAPE])


@pytest.mark.gpu
@pytest.mark.parametrize('segment', [7, 1], ids=['recompute', 'stored'])
def test_adjoint_gradient_vs_finite_differences(segment, tmp_path, oracle_bins, gpu_lib):
    fd_check(problem(segment), tmp_path, oracle_bins)


@pytest.mark.gpu
@pytest.mark.parametrize('segment', [7, 1], ids=['recompute', 'stored'])
def test_adjoint_pml_gradient_vs_finite_differences(segment, tmp_path, oracle_bins, gpu_lib):
    """The PML adjoint (cell and node memories carried backwards, the
    viscous PML hourglass), with receivers inside and outside the damped
    bands, against central differences of the FP64 oracle."""
    fd_check(problem(segment, pml=True), tmp_path, oracle_bins)


def fd_check(p, tmp_path, oracle_bins):
    import torch
    exe = oracle_bins['f64']
    rho0, vp0, vs0, m0 = model(11)
    obs = oracle_traces(p, *model(12), str(tmp_path / 'obs'), exe)

    rho = torch.tensor(rho0, dtype=torch.float32, requires_grad=True)
    vp = torch.tensor(vp0, dtype=torch.float32, requires_grad=True)
    vs = torch.tensor(vs0, dtype=torch.float32, requires_grad=True)
    mom = torch.tensor(m0, dtype=torch.float32, requires_grad=True)
    tr = adjoint.ReceiverTraces.apply(rho, vp, vs, mom, p)
    # the forward traces are the oracle's within FP32 rounding
    ref = oracle_traces(p, rho0, vp0, vs0, m0, str(tmp_path / 'fwd'), exe)
    assert np.abs(tr.detach().numpy() - ref).max() <= 1e-4 * np.abs(ref).max()
    loss = 0.5 * ((tr.double() - torch.as_tensor(obs)) ** 2).sum()
    loss.backward()
    G = [rho.grad.numpy().astype(np.float64), vp.grad.numpy().astype(np.float64),
         vs.grad.numpy().astype(np.float64), mom.grad.numpy().astype(np.float64)]

    def L(r, a, b, m, tag):
        t = oracle_traces(p, r, a, b, m, str(tmp_path / tag), exe)
        return 0.5 * ((t - obs) ** 2).sum()

    rng = np.random.default_rng(2024)
    base = [rho0, vp0, vs0, m0]
    # one direction per variable (rho, vp, vs, moment), then all together
    for k, group in enumerate([[0], [1], [2], [3], [0, 1, 2, 3]]):
        d = [rng.standard_normal(x.shape) if i in group else np.zeros(np.shape(x)) for i, x in enumerate(base)]
        plus = [x * (1 + H_FD * dx) for x, dx in zip(base, d)]
        minus = [x * (1 - H_FD * dx) for x, dx in zip(base, d)]
        fd = (L(*plus, tag='p%d' % k) - L(*minus, tag='m%d' % k)) / (2 * H_FD)
        an = sum((g * x * dx).sum() for g, x, dx in zip(G, base, d))
        assert abs(an - fd) <= TOL * abs(fd), (k, an, fd)


@pytest.mark.gpu
@pytest.mark.parametrize('change,msg', [({'gridnoise': 0.05}, 'rectilinear')])
def test_adjoint_rejects_unsupported_runs(change, msg, tmp_path, gpu_lib):
    """Non-rectilinear meshes stay forward-only: the adjoint forward refuses
    them with SORD_E_PARAM before running."""
    from coseis_b200 import _lib
    p = problem()
    p.prm.update(change)
    rho, vp, vs, m = model(1)
    d = str(tmp_path)
    p.stage(rho, vp, vs, m, d)
    s = _lib.Solver(d, open(os.path.join(d, 'sord.in')).read())
    try:
        with pytest.raises(_lib.SordError) as e:
            s.adjoint_forward(1)
        assert e.value.code == _lib.SORD_E_PARAM and msg in str(e.value)
    finally:
        s.close()


@pytest.mark.gpu
def test_source_position_and_delay_gradients(tmp_path, oracle_bins, gpu_lib):
    """dL/d(source position) and dL/d(source delay) (sord_adjoint_source_gradients)
    against central differences of the FP64 oracle: all six moment ops moved
    together along each axis (h = 1e-3 cell, inside one cell, where the
    trilinear weights are linear), and the source delayed through the clock
    origin tm0 (dL/dt0 = -dL/dtm0, h = 1e-4 s)."""
    from coseis_b200 import _lib
    exe = oracle_bins['f64']
    p = problem(7)
    rho, vp, vs, m = model(11)
    obs = oracle_traces(p, *model(12), str(tmp_path / 'obs'), exe)
    d = str(tmp_path / 'adj')
    files = p.stage(rho, vp, vs, m, d)
    s = _lib.Solver(d, open(os.path.join(d, 'sord.in')).read())
    try:
        s.adjoint_forward(7)
        tr = p.read_traces(d)
        dtr = {f: (tr[i // 3, i % 3].astype(np.float64) - obs[i // 3, i % 3]).astype(np.float32)
               for i, f in enumerate(files)}
        g = s.adjoint_backward(dtr, 6)
    finally:
        s.close()
    delta = p.prm['delta']

    def L(tag, shift=(0.0, 0.0, 0.0), tm0=None):
        q = adjoint.Problem(dict(p.prm), dict(p.source), p.receivers, segment=7)
        q.source['x'] = [a + b for a, b in zip(p.source['x'], shift)]
        if tm0 is not None:
            q.prm['tm0'] = tm0
        t = oracle_traces(q, rho, vp, vs, m, str(tmp_path / tag), exe)
        return 0.5 * ((t - obs) ** 2).sum()

    h = 1e-3
    for ax in range(3):
        e = [0.0, 0.0, 0.0]
        e[ax] = h
        fd = (L('xp%d' % ax, e) - L('xm%d' % ax, [-x for x in e])) / (2 * h)
        an = g['position'][:, ax].sum() * delta[ax]
        assert abs(an - fd) <= TOL * abs(fd), (ax, an, fd)
    ht = 1e-4
    tm0 = p.prm['tm0']
    fd = (L('tp', tm0=tm0 + ht) - L('tm', tm0=tm0 - ht)) / (2 * ht)
    an = -g['delay'].sum()
    assert abs(an - fd) <= TOL * abs(fd), (an, fd)


@pytest.mark.gpu
def test_autograd_source_position_and_delay(tmp_path, oracle_bins, gpu_lib):
    """ReceiverTraces with the source position and delay as inputs: their
    gradients are the handle's (already held to finite differences) summed
    over the six moment ops, in node-index units and seconds."""
    import torch
    from coseis_b200 import _lib
    p = problem(7)
    rho0, vp0, vs0, m0 = model(11)
    obs = oracle_traces(p, *model(12), str(tmp_path / 'obs'), oracle_bins['f64'])
    args = [torch.tensor(a, dtype=torch.float32, requires_grad=True) for a in (rho0, vp0, vs0, m0)]
    pos = torch.tensor(p.source['x'], dtype=torch.float32, requires_grad=True)
    delay = torch.tensor(0.0, dtype=torch.float32, requires_grad=True)
    tr = adjoint.ReceiverTraces.apply(*args, p, pos, delay)
    loss = 0.5 * ((tr.double() - torch.as_tensor(obs)) ** 2).sum()
    loss.backward()
    d = str(tmp_path / 'ref')
    files = p.stage(rho0, vp0, vs0, m0, d)
    s = _lib.Solver(d, open(os.path.join(d, 'sord.in')).read())
    try:
        s.adjoint_forward(7)
        t = p.read_traces(d)
        g = s.adjoint_backward({f: (t[i // 3, i % 3].astype(np.float64) - obs[i // 3, i % 3]).astype(np.float32)
                                for i, f in enumerate(files)}, 6)
    finally:
        s.close()
    ref = g['position'].sum(0) * np.asarray(p.prm['delta'][:3])
    assert np.allclose(pos.grad.numpy(), ref, rtol=1e-5), (pos.grad, ref)
    assert abs(float(delay.grad) - g['delay'].sum()) <= 1e-5 * abs(g['delay'].sum())
    assert np.abs(args[0].grad.numpy()).max() > 0


def test_binomial_cost_is_the_optimal_recursion():
    """sord_adjoint_binomial_cost (the binomial schedule's forward steps, the
    forward run included) against an exhaustive search over every split of
    the checkpointing recursion: reversing steps (lo, hi] with S_lo and S_hi
    kept and c free records costs min over m of (m - lo) + cost(m, hi, c - 1)
    + cost(lo, m, c); with no free record each state is recomputed from
    S_lo."""
    from coseis_b200 import _lib
    L, C = 60, 6
    D = [[0] * (C + 1) for _ in range(L + 1)]
    for l in range(2, L + 1):
        D[l][0] = l * (l - 1) // 2
        for c in range(1, C + 1):
            D[l][c] = min(m + D[l - m][c - 1] + D[m][c] for m in range(1, l))
    for l in range(1, L + 1):
        for c in range(0, C + 1):
            # snapshots = c + 1: S_0 and the c records the recursion may fill
            assert _lib.binomial_cost(l, c + 1) == D[l][c], (l, c)
    # with a record for every state each state is computed once
    assert _lib.binomial_cost(600, 600) == 599


def binomial_vs_stored(p_of, tmp_path, snapshots):
    """Gradients of the binomial schedule equal those of keeping every state."""
    from coseis_b200 import _lib
    rho, vp, vs, m = model(11)
    out = []
    for tag, kw in (('stored', {'segment': 1}), ('binomial', {'snapshots': snapshots})):
        p = p_of(**kw)
        d = str(tmp_path / tag)
        files = p.stage(rho, vp, vs, m, d)
        s = _lib.Solver(d, open(os.path.join(d, 'sord.in')).read())
        try:
            p.forward(s)
            tr = p.read_traces(d)
            dtr = {f: (0.1 * tr[i // 3, i % 3]).astype(np.float32) for i, f in enumerate(files)}
            out.append(s.adjoint_backward(dtr, 6))
        finally:
            s.close()
    a, b = out
    for k in ('lam', 'mu', 'yy', 'mr', 'moment'):
        x, y = np.asarray(a[k], np.float64), np.asarray(b[k], np.float64)
        assert np.linalg.norm(x - y) <= 1e-6 * np.linalg.norm(x), k


@pytest.mark.gpu
@pytest.mark.parametrize('pml', [False, True], ids=['free', 'pml'])
@pytest.mark.parametrize('snapshots', [3, 6])
def test_binomial_checkpointing_matches_stored_states(pml, snapshots, tmp_path, gpu_lib):
    """Binomial checkpointing with 3 and 6 kept states over 40 steps (deep
    recursions, records recomputed with no free record left) gives the
    gradients of the run that keeps every state: the recomputed states are
    the forward run's."""
    binomial_vs_stored(lambda **kw: problem(pml=pml, **kw), tmp_path, snapshots)


@pytest.mark.gpu
def test_adjoint_eight_directions_larger_run(tmp_path, oracle_bins, gpu_lib):
    """The adjoint configuration's check at a larger size: 48^3 nodes, 240
    steps, a 10 % Gaussian blob in rho, vp and vs, a seeded moment tensor
    with a 2 Hz Ricker wavelet, 16 surface receivers, binomial
    checkpointing with 35 kept states; the gradient along 8 seeded random
    directions in (rho, vp, vs, moment) together against central
    differences (h = 1e-3 relative) of the FP64 oracle, bound 1e-3."""
    import torch
    exe = oracle_bins['f64']
    threads = max(1, min(16, os.cpu_count() or 1))
    n, nt = 48, 240
    rng = np.random.default_rng(48)
    prm = {'shape': [n, n, n, nt], 'delta': [100.0, 100.0, 100.0, 0.008], 'bc1': ['free'] * 3,
           'bc2': ['free'] * 3, 'npml': 0, 'hourglass': [1.0, 1.0], 'gam': [0.0], 'tm0': -0.25,
           'itstats': 10, 'itio': 60}
    src = {'x': [n * 0.5 + 0.3, n * 0.5 - 0.2, n * 0.5 + 0.1], 'pulse': 'ricker2',
           'tau': 1.0 / (math.sqrt(2.0) * math.pi * 2.0)}
    rec = [[float(rng.uniform(2, n - 3)), float(rng.uniform(2, n - 3)), 0.0] for _ in range(16)]
    p = adjoint.Problem(prm, src, rec, snapshots=35)
    nc = (n - 1,) * 3
    j, k, l = np.meshgrid(*[np.arange(c) + 0.5 for c in nc], indexing='ij')

    def blob_model(seed):
        r = np.random.default_rng(seed)
        c = [r.uniform(0.3, 0.7) * m for m in nc]
        b = np.exp(-((j - c[0]) ** 2 + (k - c[1]) ** 2 + (l - c[2]) ** 2) / (2 * 5.0 ** 2))
        amp = r.choice([-0.1, 0.1], 3)
        m = r.standard_normal(6)
        m *= 1e16 / math.sqrt((m[:3] ** 2).sum() + 2 * (m[3:] ** 2).sum())
        return [base * (1 + a * b) for base, a in zip((2700.0, 6000.0, 3464.0), amp)] + [m]

    def traces(model, tag):
        path = str(tmp_path / tag)
        shutil.rmtree(path, ignore_errors=True)
        p.stage(*model, path, realsize=8)
        sc.run_oracle(path, exe, threads)
        return p.read_traces(path, '<f8')

    obs = traces(blob_model(2), 'obs')
    base = blob_model(1)
    t = [torch.tensor(x, dtype=torch.float32, requires_grad=True) for x in base]
    tr = adjoint.ReceiverTraces.apply(t[0], t[1], t[2], t[3], p)
    loss = 0.5 * ((tr.double() - torch.as_tensor(obs)) ** 2).sum()
    loss.backward()
    G = [x.grad.numpy().astype(np.float64) for x in t]
    d_rng = np.random.default_rng(2025)
    for q in range(8):
        d = [d_rng.standard_normal(np.shape(x)) for x in base]
        lp = 0.5 * ((traces([x * (1 + H_FD * dx) for x, dx in zip(base, d)], 'p') - obs) ** 2).sum()
        lm = 0.5 * ((traces([x * (1 - H_FD * dx) for x, dx in zip(base, d)], 'm') - obs) ** 2).sum()
        fd = (lp - lm) / (2 * H_FD)
        an = sum((g * x * dx).sum() for g, x, dx in zip(G, base, d))
        assert abs(an - fd) <= TOL * abs(fd), (q, an, fd)
