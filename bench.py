"""Benchmark of the SORD time loop on the large wave-propagation workload.

Workload "wave226" (N = 768 x 768 x 384 = 226,492,416 nodes, dx = 50 m,
dt = 0.004 s): layered half-space (vs 1000 / 2500 / 3500 m/s above 1 km,
1-4 km, below 4 km; vp = sqrt(3) vs; rho 2200 / 2500 / 2700) with a seeded
von Karman perturbation (5 % std, correlation length 1 km, Hurst 0.3) on
vp, vs and rho; terrain-following mesh from a seeded Gaussian hill (peak
500 m, sigma 5 km) stretched linearly to a flat bottom; free surface at the
l = 1 face, 12-node PML on the other five; seeded random moment-tensor
point source at 5 km depth (Brune, 0.1 s); 64 seeded surface receivers
(vx, vy, vz).  All inputs go through the cst.sord-compatible front end as
'=<' files and '.' / '.>' ops, exactly like a user run.

A step is one time step of the whole mesh.  `value` is node-updates/s with
every input resident in HBM; `e2e` is the same metric for the user call
(staged files on the host -> setup -> K steps -> outputs written); the
reference arm (--impl reference) runs the CPU oracle, the restatement of the
Fortran solver, on a bounded sample of the same workload.

The interior step kernel runs in fast arithmetic by default (--arithmetic
fast: fused multiply-adds and fewer operations, relative L2 error ~1e-6
against the FP64 oracle, tested to <= 1e-4); the same handle then times the
reference-order kernel (bit-identical to the FP32 oracle), reported as
`reference_order`.
"""
import argparse
import copy
import json
import math
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SHAPE = (768, 768, 384)
DX, DT = 50.0, 0.004
NPML = 12
SEED = 20261203
HBM_FALLBACK = 6650.0


# ------------------------------------------------------------------ workload
def von_karman(shape, dx, a, hurst, std, seed, use_torch=True):
    """Seeded von Karman random field on a cell grid (numpy order (l,k,j))."""
    n = shape
    if use_torch:
        try:
            import torch
            if torch.cuda.is_available():
                dev = torch.device('cuda')
                g = torch.Generator(device=dev).manual_seed(seed)
                w = torch.randn(n, generator=g, device=dev, dtype=torch.float32)
                F = torch.fft.rfftn(w)
                del w
                k0 = torch.fft.fftfreq(n[0], d=dx, device=dev) * 2 * math.pi
                k1 = torch.fft.fftfreq(n[1], d=dx, device=dev) * 2 * math.pi
                k2 = torch.fft.rfftfreq(n[2], d=dx, device=dev) * 2 * math.pi
                k2sq = (k0[:, None, None] ** 2 + k1[None, :, None] ** 2 + k2[None, None, :] ** 2)
                F *= (1.0 + k2sq * a * a) ** (-(hurst + 1.5) / 2.0)
                del k2sq
                f = torch.fft.irfftn(F, s=n)
                del F
                f = f - f.mean()
                f = f * (std / f.std())
                out = f.cpu().numpy().astype(np.float32)
                del f
                torch.cuda.empty_cache()
                return out
        except Exception:
            pass
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(n).astype(np.float32)
    F = np.fft.rfftn(w)
    k0 = np.fft.fftfreq(n[0], d=dx) * 2 * np.pi
    k1 = np.fft.fftfreq(n[1], d=dx) * 2 * np.pi
    k2 = np.fft.rfftfreq(n[2], d=dx) * 2 * np.pi
    k2sq = k0[:, None, None] ** 2 + k1[None, :, None] ** 2 + k2[None, None, :] ** 2
    F *= (1.0 + k2sq * a * a) ** (-(hurst + 1.5) / 2.0)
    f = np.fft.irfftn(F, s=n, axes=(0, 1, 2))
    f -= f.mean()
    f *= std / f.std()
    return f.astype(np.float32)


def make_inputs(shape, outdir, seed=SEED, use_torch=True, hill=500.0):
    """Write rho.bin, vp.bin, vs.bin (cells) and z.bin (nodes), j fastest."""
    os.makedirs(outdir, exist_ok=True)
    mark = os.path.join(outdir, 'ok.json')
    if os.path.exists(mark):
        return
    nx, ny, nz = shape
    # terrain-following z: surface elevation h(x, y), flat bottom
    x = DX * np.arange(nx, dtype=np.float32)
    y = DX * np.arange(ny, dtype=np.float32)
    xc, yc = x[-1] * 0.5, y[-1] * 0.5
    sig = 5000.0 * min(1.0, min(nx, ny) / 768.0)
    h = hill * np.exp(-((x[None, :] - xc) ** 2 + (y[:, None] - yc) ** 2) / (2 * sig * sig))
    h = h.astype(np.float32)
    with open(os.path.join(outdir, 'z.bin'), 'wb') as fh:
        for l in range(nz):
            frac = np.float32(1.0 - l / (nz - 1.0))
            zl = np.float32(DX * l) - h * frac
            fh.write(zl.astype(np.float32).tobytes())
    # layered model + perturbation on cells
    cshape = (nz - 1, ny - 1, nx - 1)
    dv = von_karman(cshape, DX, 1000.0, 0.3, 0.05, seed, use_torch=use_torch)
    depth = DX * (np.arange(nz - 1, dtype=np.float32) + 0.5)
    vs_l = np.where(depth < 1000.0, 1000.0, np.where(depth < 4000.0, 2500.0, 3500.0)).astype(np.float32)
    rho_l = np.where(depth < 1000.0, 2200.0, np.where(depth < 4000.0, 2500.0, 2700.0)).astype(np.float32)
    for name, base in (('vs', vs_l), ('vp', vs_l * np.float32(math.sqrt(3.0))), ('rho', rho_l)):
        with open(os.path.join(outdir, name + '.bin'), 'wb') as fh:
            for l in range(nz - 1):
                fh.write((base[l] * (1.0 + dv[l])).astype(np.float32).tobytes())
    del dv
    json.dump({'shape': list(shape), 'seed': seed}, open(mark, 'w'))


def wave_prm(shape, nt, seed=SEED, nrec=64):
    """cst.sord parameter dict of the wave226 workload (any shape)."""
    nx, ny, nz = shape
    rng = np.random.default_rng(seed + 1)
    m = rng.standard_normal(6)
    m *= 1e16 / math.sqrt((m[:3] ** 2).sum() + 2 * (m[3:] ** 2).sum())
    zsrc = min(5000.0 / DX, nz - NPML - 3)
    src = [nx * 0.5 + 0.37, ny * 0.5 - 0.21, zsrc + 0.13]
    prm = {
        'shape': [nx, ny, nz, nt], 'delta': [DX, DX, DX, DT],
        'bc1': ['pml', 'pml', 'free'], 'bc2': ['pml', 'pml', 'pml'], 'npml': NPML,
        'hourglass': [1.0, 1.0], 'gam': [0.0],
        'rho': [([], '=<', 'rho.bin')], 'vp': [([], '=<', 'vp.bin')], 'vs': [([], '=<', 'vs.bin')],
        'z': [([], '=<', 'z.bin')],
        'vp_max': 6800.0, 'vs_max': 6800.0 / math.sqrt(3.0), 'vs_min': 600.0, 'vp_min': 1000.0,
        'itstats': 10, 'itio': 50,
    }
    for f, v in zip(('mxx', 'myy', 'mzz', 'myz', 'mzx', 'mxy'), m):
        prm[f] = [([src[0], src[1], src[2], []], '.', float(v), 'brune', 0.1)]
    lo = NPML + 1
    for r in range(nrec):
        xr = float(rng.uniform(lo, nx - 1 - lo))
        yr = float(rng.uniform(lo, ny - 1 - lo))
        for f in ('vx', 'vy', 'vz'):
            prm.setdefault(f, []).append(([xr, yr, 0.0, []], '.>', 'r%02d-%s.bin' % (r, f)))
    return prm


def stage_in(prm, workdir, inputs):
    from coseis_b200 import sord
    os.makedirs(workdir, exist_ok=True)
    for f in ('rho.bin', 'vp.bin', 'vs.bin', 'z.bin'):
        dst = os.path.join(workdir, f)
        if not os.path.exists(dst):
            os.symlink(os.path.join(inputs, f), dst)
    cwd = os.getcwd()
    os.chdir(workdir)
    try:
        sord.stage(prm)
    finally:
        os.chdir(cwd)
    return open(os.path.join(workdir, 'sord.in')).read()


# ------------------------------------------------------- rupture ensemble
ENS_DX, ENS_DT, ENS_NT, ENS_NPML = 100.0, 0.008, 600, 10


def gaussian_field_2d(shape, dx, corr, std, rng):
    """Seeded Gaussian random field on a (nx, ny) plane with a Gaussian
    correlation of length `corr`, zero mean and standard deviation `std`."""
    w = rng.standard_normal(shape)
    k0 = np.fft.fftfreq(shape[0], d=dx) * 2 * np.pi
    k1 = np.fft.rfftfreq(shape[1], d=dx) * 2 * np.pi
    F = np.fft.rfft2(w) * np.exp(-(k0[:, None] ** 2 + k1[None, :] ** 2) * corr * corr / 8.0)
    f = np.fft.irfft2(F, s=shape)
    f -= f.mean()
    f *= std / f.std()
    return f


def rupture_scenario(i, seed=SEED, nt=ENS_NT, shape=None):
    """Scenario `i` of the batched rupture ensemble: a spontaneous
    slip-weakening rupture on the k-midplane ('+z' double-node fault) of a
    seeded grid between 64x64x64 and 192x96x96 nodes (dx 100 m, dt 0.008 s,
    homogeneous rho 2670, vp 6000, vs 3464, 10-node PML on all faces).
    Seeded per scenario: mu_s in [0.6, 0.7], mu_d in [0.45, 0.55], Dc in
    [0.2, 0.5] m, normal stress in [-120, -60] MPa; initial shear stress
    0.58 |tn| (58 MPa at -100 MPa) plus a Gaussian random field of std
    0.03 |tn| (3 MPa at -100 MPa) and correlation length 1 km; frictional
    region the central 2/3 x 2/3 of the fault (mu_s = 1e4 outside), and a
    square nucleation patch (3 km, at most a third of the region) at
    1.02 mu_s |tn|.  Outputs: final slip, slip rate and shear traction
    magnitude and the rupture time on the fault.

    Returns (cst.sord parameter dict, {file name: float32 array}) where the
    arrays are the '=<' input files (Fortran order, j fastest)."""
    rng = np.random.default_rng([seed, 5, i])
    if shape is None:
        shape = (16 * int(rng.integers(4, 13)), 16 * int(rng.integers(4, 7)), 16 * int(rng.integers(4, 7)))
    nx, ny, nz = shape
    mus = float(rng.uniform(0.6, 0.7))
    mud = float(rng.uniform(0.45, 0.55))
    dc = float(rng.uniform(0.2, 0.5))
    tn = -float(rng.uniform(60e6, 120e6))
    ts = 0.58 * abs(tn) + gaussian_field_2d((nx, ny), ENS_DX, 1000.0, 0.03 * abs(tn), rng)
    # frictional region and nucleation patch, in fault-plane node indices
    rj, rk = max(1, nx // 6), max(1, ny // 6)
    reg = [[rj, nx - rj], [rk, ny - rk]]
    half = max(1, min(int(1500.0 / ENS_DX), (nx - 2 * rj) // 6, (ny - 2 * rk) // 6))
    jc, kc = nx // 2, ny // 2
    ts[jc - half:jc + half, kc - half:kc + half] = 1.02 * mus * abs(tn)
    prm = {
        'shape': [nx, ny, nz, nt], 'delta': [ENS_DX, ENS_DX, ENS_DX, ENS_DT],
        'rho': [2670.0], 'vp': [6000.0], 'vs': [3464.0], 'gam': [0.1], 'hourglass': [1.0, 2.0],
        'bc1': ['pml'] * 3, 'bc2': ['pml'] * 3, 'npml': ENS_NPML,
        'faultnormal': '+z', 'hypocenter': [float(jc), float(kc), nz * 0.5 - 0.5], 'vrup': -1.0,
        'mus': [1e4, (reg, '=', mus)], 'mud': [mud], 'dc': [dc], 'tn': [tn],
        'ts': [([], '=<', 'ts.bin')],
        'itstats': 10, 'itio': 100,
    }
    for f in ('sum', 'svm', 'tsm', 'trup'):
        prm[f] = [([[], [], -1], '=>', f + '.bin')]
    # the file holds the plane in Fortran order: j fastest
    return prm, {'ts.bin': np.ascontiguousarray(ts.T, dtype='<f4')}


def stage_scenarios(indices, root, seed=SEED, nt=ENS_NT, shape=None):
    """Stage ensemble scenarios into root/s<i>; returns the directories."""
    from coseis_b200 import sord
    dirs = []
    cwd = os.getcwd()
    try:
        for i in indices:
            d = os.path.join(root, 's%03d' % i)
            os.makedirs(d, exist_ok=True)
            prm, files = rupture_scenario(i, seed, nt, shape)
            for f, a in files.items():
                a.tofile(os.path.join(d, f))
            os.chdir(d)
            sord.stage(prm)
            os.chdir(cwd)
            dirs.append(d)
    finally:
        os.chdir(cwd)
    return dirs


# ------------------------------------------------------- explosion and rupture configs
def explosion_prm(nt=200, seed=SEED):
    """Plain point-source explosion: 61^3 rectilinear nodes, dx 100 m,
    dt 0.008 s, 200 steps; rho 2670, vp 6000, vs 3464; isotropic moment
    source (M0 1e16 N m, Brune, tau 0.1 s) at the centre node, spread over
    its 8 cells; 10-node PML on all six faces; default hourglass constants;
    vx, vy, vz on the k mid-plane every 10 steps and at 8 seeded interior
    nodes."""
    n, c = 61, 30
    prm = {'shape': [n, n, n, nt], 'delta': [100.0, 100.0, 100.0, 0.008],
           'rho': [2670.0], 'vp': [6000.0], 'vs': [3464.0], 'gam': [0.0], 'hourglass': [1.0, 1.0],
           'bc1': ['pml'] * 3, 'bc2': ['pml'] * 3, 'npml': 10, 'itstats': 10, 'itio': 50}
    for f in ('mxx', 'myy', 'mzz'):
        prm[f] = [([c, c, c, []], '.', 1e16, 'brune', 0.1)]
    rng = np.random.default_rng([seed, 1])
    rec = rng.integers(12, n - 12, size=(8, 3))
    for f in ('vx', 'vy', 'vz'):
        prm[f] = [([[], c, [], [0, None, 10]], '=>', 'snap-%s.bin' % f)]
        prm[f] += [([int(j), int(k), int(l), []], '=>', 'rec%d-%s.bin' % (r, f)) for r, (j, k, l) in enumerate(rec)]
    return prm


RUP_SHAPE = (600, 300, 300)


def rupture3_prm(nt=1500, shape=RUP_SHAPE, seed=SEED, dx=50.0, dt=0.004):
    """Spontaneous rupture on a planar fault: 600 x 300 x 300 nodes, dx 50 m,
    dt 0.004 s, 1500 steps, homogeneous rho 2670, vp 6000, vs 3464;
    double-node fault ('+y') at the k mid-plane; 20 km x 10 km frictional
    region (mu_s = 1e4 outside); linear slip weakening mu_s 0.65, mu_d 0.50,
    Dc 0.30 m; normal stress -100 MPa; initial shear stress 58 MPa plus a
    seeded Gaussian random field (std 3 MPa, correlation 1 km); 3 km square
    nucleation patch at 1.02 mu_s |tn|; 10-node PML; final slip, slip rate,
    shear traction and rupture time on the fault.  Smaller shapes keep the
    physical sizes where they fit (region and patch clipped to the plane).
    Returns (parameter dict, {file name: float32 array})."""
    nx, ny, nz = shape
    rng = np.random.default_rng([seed, 7])
    ts = 58e6 + gaussian_field_2d((nx, nz), dx, 1000.0, 3e6, rng)
    jc, lc = nx // 2, nz // 2
    rj, rl = min(int(10000.0 / dx), nx // 2 - 2), min(int(5000.0 / dx), nz // 2 - 2)
    half = max(1, min(int(1500.0 / dx), rj // 3, rl // 3))
    ts[jc - half:jc + half, lc - half:lc + half] = 1.02 * 0.65 * 100e6
    prm = {
        'shape': [nx, ny, nz, nt], 'delta': [dx, dx, dx, dt],
        'rho': [2670.0], 'vp': [6000.0], 'vs': [3464.0], 'gam': [0.0], 'hourglass': [1.0, 1.0],
        'bc1': ['pml'] * 3, 'bc2': ['pml'] * 3, 'npml': 10,
        'faultnormal': '+y', 'hypocenter': [float(jc), ny * 0.5 - 0.5, float(lc)], 'vrup': -1.0,
        'mus': [1e4, ([[jc - rj, jc + rj], [lc - rl, lc + rl]], '=', 0.65)], 'mud': [0.5], 'dc': [0.3],
        'tn': [-100e6], 'ts': [([], '=<', 'ts.bin')],
        'itstats': 10, 'itio': 100,
    }
    for f in ('sum', 'svm', 'tsm', 'trup'):
        prm[f] = [([[], [], -1], '=>', f + '.bin')]
    return prm, {'ts.bin': np.ascontiguousarray(ts.T, dtype='<f4')}


def stage_files(prm, files, d, realsize=4):
    from coseis_b200 import sord
    os.makedirs(d, exist_ok=True)
    for f, a in files.items():
        a.astype('<f8' if realsize == 8 else '<f4').tofile(os.path.join(d, f))
    cwd = os.getcwd()
    os.chdir(d)
    try:
        sord.stage(prm, realsize=realsize)
    finally:
        os.chdir(cwd)
    return open(os.path.join(d, 'sord.in')).read()


def run_config_bench(name, prm, files, steps, warmup, device, full_steps):
    """Device node-updates/s of one configuration (its own handle, inputs
    resident, CUDA events around one sord_step call of `steps` steps after
    `warmup`), and end to end: sord_run_directory of the whole run
    (`full_steps` steps, setup and output files included, host clock)."""
    from coseis_b200 import _lib
    nodes = float(np.prod(prm['shape'][:3]))
    work = tempfile.mkdtemp(prefix='sord_%s_' % name)
    try:
        p = dict(prm)
        p['shape'] = list(prm['shape'][:3]) + [warmup + steps]
        text = stage_files(p, files, os.path.join(work, 'dev'))
        s = _lib.Solver(os.path.join(work, 'dev'), text, device=device)
        try:
            s.step(warmup)
            s.step(steps)
            ms = s.last_step_ms()
        finally:
            s.close()
        out = {'value': nodes * steps / (ms / 1e3), 'unit': 'node-updates/s', 'ms_per_step': ms / steps,
               'nodes': int(nodes), 'timed_steps': steps}
        if full_steps:
            p = dict(prm)
            p['shape'] = list(prm['shape'][:3]) + [full_steps]
            stage_files(p, files, os.path.join(work, 'e2e'))
            t0 = time.time()
            _lib.run_directory(os.path.join(work, 'e2e'), device)
            wall = time.time() - t0
            out['e2e'] = {'value': nodes * full_steps / wall, 'unit': 'node-updates/s', 'steps': full_steps,
                          'wall_s': round(wall, 3), 'includes': 'setup, all steps, output files, teardown'}
        return out
    finally:
        shutil.rmtree(work, ignore_errors=True)


def oracle_config_rate(prm, files, steps, warmup, threads):
    """CPU oracle node-updates/s on a configuration (steps after warm-up)."""
    exe = oracle_exe()
    work = tempfile.mkdtemp(prefix='sord_cpucfg_')
    try:
        p = dict(prm)
        p['shape'] = list(prm['shape'][:3]) + [warmup + steps]
        stage_files(p, files, work)
        r = subprocess.run([exe, '--threads', str(threads), '--timed-from', str(warmup)], cwd=work,
                           capture_output=True, text=True, timeout=1800)
        if r.returncode:
            raise RuntimeError(r.stderr[-2000:])
        info = json.loads(r.stdout.strip().splitlines()[-1])
        return float(np.prod(prm['shape'][:3])) * steps / info['timed_seconds']
    finally:
        shutil.rmtree(work, ignore_errors=True)


def run_other_configs(device, cpu=True):
    """node-updates/s of the explosion (61^3, all 200 steps timed) and of the
    600 x 300 x 300 rupture (30 steps after 5, of its 1500), each beside the
    CPU oracle on all host threads on the same configuration (explosion: the
    whole run; rupture: 2 steps after 1)."""
    thr = os.cpu_count() or 1
    res = {}
    prm = explosion_prm()
    r = run_config_bench('explosion', prm, {}, 200, 3, device, 200)
    r['workload'] = 'explosion: 61^3 rectilinear nodes, 200 steps, moment source, 10-node PML, snapshots + 8 receivers'
    if cpu:
        r['cpu_oracle'] = {'value': oracle_config_rate(prm, {}, 199, 1, thr), 'cores': thr, 'steps': 199}
    res['explosion'] = r
    prm, files = rupture3_prm()
    r = run_config_bench('rupture', prm, files, 30, 5, device, 0)
    r['workload'] = ('rupture: 600x300x300 nodes, slip-weakening +y fault (20 x 10 km region, 3 km patch, '
                     'seeded 3 MPa stress field), 10-node PML; 30 of 1500 steps timed')
    if cpu:
        r['cpu_oracle'] = {'value': oracle_config_rate(prm, files, 2, 1, thr), 'cores': thr, 'steps': 2}
    res['rupture'] = r
    return res


# ------------------------------------------------------- adjoint
def adjoint_problem(shape=(128, 128, 128), nt=1200, nrec=32, seed=SEED, segment=35):
    """The adjoint workload: 128^3 nodes, dx 100 m, dt 0.008 s, 1200 steps;
    rho / vp / vs 2700 / 6000 / 3464 with a 10 % seeded Gaussian blob
    (2 km wide, seeded place and signs); seeded moment tensor (M0 1e16 N m)
    at the centre with a Ricker wavelet of 2 Hz peak frequency ('ricker2',
    tau = 1 / (sqrt(2) pi f0), start time -0.25 s); 32 seeded surface
    receivers (vx, vy, vz every step); free surfaces on all faces (the
    configuration names no boundary); checkpoints every 35 steps."""
    from coseis_b200 import adjoint
    nx, ny, nz = shape
    rng = np.random.default_rng([seed, 3])
    prm = {'shape': [nx, ny, nz, nt], 'delta': [100.0, 100.0, 100.0, 0.008], 'bc1': ['free'] * 3,
           'bc2': ['free'] * 3, 'npml': 0, 'hourglass': [1.0, 1.0], 'gam': [0.0], 'tm0': -0.25,
           'itstats': 10, 'itio': 100}
    tau = 1.0 / (math.sqrt(2.0) * math.pi * 2.0)
    src = {'x': [nx * 0.5 + 0.3, ny * 0.5 - 0.2, nz * 0.5 + 0.1], 'pulse': 'ricker2', 'tau': tau}
    rec = [[float(rng.uniform(2, nx - 3)), float(rng.uniform(2, ny - 3)), 0.0] for _ in range(nrec)]
    nc = (nx - 1, ny - 1, nz - 1)
    j, k, l = np.meshgrid(*[np.arange(n, dtype=np.float32) + 0.5 for n in nc], indexing='ij', sparse=True)
    c = [rng.uniform(0.3, 0.7) * n for n in nc]
    blob = np.exp(-((j - c[0]) ** 2 + (k - c[1]) ** 2 + (l - c[2]) ** 2) / (2 * 10.0 ** 2)).astype(np.float32)
    amp = rng.choice([-0.1, 0.1], 3)
    m = rng.standard_normal(6)
    m *= 1e16 / math.sqrt((m[:3] ** 2).sum() + 2 * (m[3:] ** 2).sum())
    mat = [base * (1 + a * blob) for base, a in zip((2700.0, 6000.0, 3464.0), amp)]
    return adjoint.Problem(prm, src, rec, segment=segment), mat[0], mat[1], mat[2], m


def run_adjoint_bench(device, nt=1200):
    """Cost of the misfit gradient against the forward run alone, all on the
    device clock: (adjoint forward with checkpoints + backward) / plain
    forward of the same problem; `value` with a checkpoint every 35 steps
    (35 checkpoints, each segment recomputed while the adjoint pass runs
    over the next), `stored` keeping every state instead (no
    recomputation; 9.5 GB here), `binomial` binomial checkpointing with 35
    kept states (the revolve schedule, recomputation and adjoint steps on
    one stream); `pml` the same problem with a free surface at l = 1 and a
    10-node PML on the other faces (the two-pass PML adjoint), a checkpoint
    every 35 steps, against its own forward."""
    from coseis_b200 import _lib
    p, rho, vp, vs, m = adjoint_problem(nt=nt)
    pp = copy.deepcopy(p)
    pp.prm.update({'bc1': ['pml', 'pml', 'free'], 'bc2': ['pml'] * 3, 'npml': 10, 'vpml': 6000.0})
    work = tempfile.mkdtemp(prefix='sord_adjb_')

    def forward_ms(prob, tag):
        d = os.path.join(work, tag)
        prob.stage(rho, vp, vs, m, d)
        s = _lib.Solver(d, open(os.path.join(d, 'sord.in')).read(), device=device)
        # the adjoint kernels transpose the reference-order step; forward and
        # recomputation use that arithmetic here, so the ratio compares like with like
        s.set_arithmetic('reference')
        s.step(nt)
        t = s.last_step_ms()
        s.close()
        return t

    try:
        t_fwd = forward_ms(p, 'fwd')
        t_fwd_pml = forward_ms(pp, 'fwd_pml')
        res = {}
        for tag, seg in (('checkpointed', 35), ('stored', 1), ('binomial', -35), ('pml', 35)):
            prob, tf = (pp, t_fwd_pml) if tag == 'pml' else (p, t_fwd)
            d = os.path.join(work, tag)
            prob.stage(rho, vp, vs, m, d)
            s = _lib.Solver(d, open(os.path.join(d, 'sord.in')).read(), device=device)
            s.set_arithmetic('reference')
            try:
                if seg > 0:
                    s.adjoint_forward(seg)
                else:
                    s.adjoint_forward_binomial(-seg)
                t_af = s.last_step_ms()
                tr = prob.read_traces(d)
                # misfit against observed traces 0.9 x the computed ones
                dtr = {f: 0.1 * tr[i // 3, i % 3] for i, f in enumerate(prob.files())}
                g = s.adjoint_backward(dtr, 6)
                t_b = s.last_step_ms()
            finally:
                s.close()
            ok = bool(np.isfinite(g['lam']).all() and np.abs(g['mu']).max() > 0)
            res[tag] = {'ratio': (t_af + t_b) / tf, 'adjoint_forward_ms': t_af, 'backward_ms': t_b,
                        'finite_gradients': ok}
            if tag == 'pml':
                res[tag]['forward_ms'] = tf
            if seg > 0:
                res[tag]['segment'] = seg
            else:
                res[tag]['snapshots'] = -seg
                res[tag]['schedule_forward_steps'] = _lib.binomial_cost(nt, -seg)
        return {'metric': 'adjoint gradient cost / forward', 'value': res['checkpointed']['ratio'], 'unit': 'x',
                'higher_is_better': False, 'forward_ms': t_fwd, 'arithmetic': 'reference',
                'checkpointed': res['checkpointed'],
                'stored': res['stored'],
                'binomial': res['binomial'],
                'pml': res['pml'],
                'workload': 'adjoint: 128^3 nodes, %d steps, seeded 10%% blob in rho/vp/vs, 32 receivers, '
                            'moment tensor with 2 Hz Ricker, free surfaces' % nt}
    finally:
        shutil.rmtree(work, ignore_errors=True)


def pml_memberships(shape):
    """Node and cell PML slab memberships (one per node/cell per PML face)."""
    nn = np.array(shape)
    faces = [(0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]  # (axis, side): l=1 face is free
    nodes = cells = 0
    for ax, _ in faces:
        other = int(np.prod(nn)) // nn[ax]
        otherc = int(np.prod(nn - 1)) // (nn[ax] - 1)
        nodes += NPML * other
        cells += NPML * otherc
    return nodes, cells


def algorithmic_bytes_per_node(shape):
    """Compulsory FP32 traffic per node-update with perfect on-chip reuse:
    v, u read + write (48 B), node statics mr, gam (8 B), cell statics lam,
    mu, yy, 1/V (16 B), node coordinates x, y, z (12 B) = 84 B, plus 24 B
    (3-component r/w) per node PML-slab membership (p memory) and per cell
    membership (g memory)."""
    n = float(np.prod(shape))
    pn, pc = pml_memberships(shape)
    return 84.0 + 24.0 * (pn + pc) / n


# ------------------------------------------------------------------ helpers
class Clocks(object):
    """nvidia-smi sampling during the timed region."""
    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
         'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
         'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.p = None
        self.lines = []

    def start(self):
        try:
            self.p = subprocess.Popen(['nvidia-smi', '-i', str(self.index), '--query-gpu=' + self.Q,
                                       '--format=csv,noheader,nounits', '-lms', '200'],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.p = None

    def _read(self):
        for line in self.p.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.p:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for line in self.lines:
            f = [x.strip() for x in line.split(',')]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith('active'):
                    reasons.add(n)
        if not sm:
            return None
        return {'sm_mhz': statistics.median(sm), 'sm_max_mhz': max(mx), 'reasons': sorted(reasons),
                'samples': len(sm)}


def peaks():
    try:
        p = json.load(open(os.path.join(ROOT, 'MEASURED_PEAKS.json')))
        return float(p['hbm_gbs']), 'measured'
    except Exception:
        return HBM_FALLBACK, 'fallback'


def traffic_per_node():
    """DRAM bytes per node-update of the step kernels from the committed ncu summary."""
    try:
        t = json.load(open(os.path.join(ROOT, 'profiles', 'traffic_wave.json')))
        return float(t['dram_bytes_per_node_update'])
    except Exception:
        return None


def oracle_exe():
    from oracle import build as ob
    return ob.build()['f32']


def cpu_sample(shape_s, steps, warm, threads):
    """Run the oracle on a scaled sample of the workload; node-updates/s."""
    exe = oracle_exe()
    d = tempfile.mkdtemp(prefix='sord_cpu_')
    try:
        inp = os.path.join(d, 'in')
        make_inputs(shape_s, inp, use_torch=False)
        prm = wave_prm(shape_s, warm + steps)
        stage_in(prm, os.path.join(d, 'run'), inp)
        r = subprocess.run([exe, '--threads', str(threads), '--timed-from', str(warm)],
                           cwd=os.path.join(d, 'run'), capture_output=True, text=True, timeout=900)
        if r.returncode:
            raise RuntimeError(r.stderr[-2000:])
        info = json.loads(r.stdout.strip().splitlines()[-1])
        nodes = float(np.prod(shape_s))
        return nodes * steps / info['timed_seconds'], info
    finally:
        shutil.rmtree(d, ignore_errors=True)


# ------------------------------------------------------------------ arms
def dist_init(backend='nccl'):
    """World size, rank, this rank's device and the process group (None for
    one rank).  backend 'gloo' moves the halo planes through host memory and
    lets several ranks share a device (their kernels never wait on one
    another: the ranks meet on the host between steps)."""
    ws = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    pg = None
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        os.environ.setdefault('MASTER_ADDR', '127.0.0.1')
        local = local % max(torch.cuda.device_count(), 1)
        torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        pg = dist
    return ws, rank, local, pg


def reduce_sum(pg, v):
    if pg is None:
        return v
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64, device='cuda' if pg.get_backend() == 'nccl' else 'cpu')
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def reduce_max(pg, v):
    """Maximum of v over all ranks (the slowest rank's device time)."""
    if pg is None:
        return v
    import torch
    dev = 'cuda' if pg.get_backend() == 'nccl' else 'cpu'
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def job_rate(nodes, steps, ms_max):
    """Whole-job node-updates/s: the ranks advance one mesh of `nodes` nodes
    by `steps` steps, each its slab of l planes; the job takes the slowest
    rank's time."""
    return nodes * steps / (ms_max / 1e3)


def shared_workdir(pg, rank, prefix):
    """A scratch directory that every rank of the job sees (one node)."""
    d = [tempfile.mkdtemp(prefix=prefix) if rank == 0 else None]
    if pg is not None:
        pg.broadcast_object_list(d, src=0)
    return d[0]


def split_prm(prm, ws):
    """The parameters of a run split into ws slabs of l planes."""
    if ws > 1:
        prm = dict(prm)
        prm['nproc3'] = [1, 1, ws]
    return prm


def open_solver(work, text, local, rank, ws, pg=None):
    from coseis_b200 import _lib
    if ws == 1:
        return _lib.Solver(work, text, device=local)
    from coseis_b200 import parallel
    transport = 'device' if pg.get_backend() == 'nccl' else 'host'
    return _lib.Solver(work, text, device=local, part=rank, exchange=parallel.DistExchange(transport))


def barrier(pg):
    if pg is not None:
        pg.barrier()


def run_ours(args):
    from coseis_b200 import build as cb
    cb.build()
    from coseis_b200 import _lib
    # read by every handle this process creates (timed run, e2e, ensemble, adjoint)
    os.environ['SORD_ARITHMETIC'] = args.arithmetic
    ws, rank, local, pg = dist_init(args.backend)
    shape = tuple(args.shape)
    nodes = float(np.prod(shape))
    inputs = os.path.join(args.cache, 'wave_%dx%dx%d_%d_%g' % (shape + (SEED, args.hill)))
    if rank == 0:
        make_inputs(shape, inputs, hill=args.hill)
    barrier(pg)
    prof_steps = 6
    # with fast arithmetic the same handle then times the reference-order
    # kernel too (2 warm-up steps + the same number of timed steps)
    other = args.arithmetic == 'fast' and not args.no_reference_order
    nt = args.warmup + args.steps + prof_steps + ((2 + args.steps) if other else 0)
    # N > 1: the mesh split into N slabs of l planes, one per rank, halo
    # planes exchanged over NCCL every step (strong scaling)
    work = shared_workdir(pg, rank, 'sord_bench_')
    try:
        if rank == 0:
            stage_in(split_prm(wave_prm(shape, nt), ws), work, inputs)
        barrier(pg)
        text = open(os.path.join(work, 'sord.in')).read()
        t0 = time.time()
        s = open_solver(work, text, local, rank, ws, pg)
        setup_s = time.time() - t0
        s.step(args.warmup)
        barrier(pg)
        clk = Clocks(local)
        clk.start()
        l0 = s.kernel_launches()
        w0 = time.time()
        s.step(args.steps)
        wall = time.time() - w0
        ms = s.last_step_ms()
        launches = s.kernel_launches() - l0
        clocks = clk.stop()
        ms_max = reduce_max(pg, ms)
        launches = reduce_sum(pg, launches)
        s.set_profiling(True)
        s.step(prof_steps)
        kt = s.kernel_times()
        s.set_profiling(False)
        ref_order = None
        if other:
            s.set_arithmetic('reference')
            s.step(2)
            barrier(pg)
            s.step(args.steps)
            r_ms = reduce_max(pg, s.last_step_ms())
            ref_order = {'ms_per_step': r_ms / args.steps, 'value': job_rate(nodes, args.steps, r_ms)}
        s.close()
        barrier(pg)
        e2e = None
        if not args.no_e2e:
            e2e = run_e2e(args, shape, inputs, local, pg, ws, rank)
            barrier(pg)
        ens = None
        if ws == 1 and args.ensemble > 0:
            ens = run_ensemble_bench(args.ensemble, args.ensemble_threads, local)
        adj = None
        if ws == 1 and args.adjoint_steps > 0:
            adj = run_adjoint_bench(local, args.adjoint_steps)
        cfgs = None
        if ws == 1 and not args.no_configs:
            cfgs = run_other_configs(local, cpu=not args.no_cpu)
    finally:
        if rank == 0:
            shutil.rmtree(work, ignore_errors=True)
    if rank != 0:
        return
    value = job_rate(nodes, args.steps, ms_max)
    hbm, src = peaks()
    alg = algorithmic_bytes_per_node(shape)
    # dominant kernel: the fused whole-step kernel, average launch duration
    k_ms, k_n = kt.get('step', (0.0, 0))
    if k_n:
        kernel, launch_ms = 'k_interior + k_shell (one fused step, concurrent)', k_ms / k_n
    else:
        kernel = 'k_time + k_stress + k_accel (separate-kernel step)'
        launch_ms = sum(kt[k][0] for k in ('time', 'stress', 'accel', 'mass')) / prof_steps
    # rank 0's kernels advance its slab only
    knodes = nodes
    if ws > 1:
        from coseis_b200 import parallel
        a, b = parallel.part_planes(shape[2], ws)[0]
        knodes = float(shape[0] * shape[1] * (b - a + 1))
    achieved = alg * knodes / (launch_ms / 1e3) / 1e9
    tr = traffic_per_node()
    out = {
        'metric': 'node-updates/s', 'value': value, 'unit': 'node-updates/s',
        'n_gpus': ws, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': ms_max / args.steps, 'higher_is_better': True, 'scaling': 'strong',
        'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic (seeded)',
        'config': {'workload': wave_workload(shape),
                   'nodes': int(nodes), 'dx_m': DX, 'dt_s': DT,
                   'parallelism': ('l-slabs x %d (nproc3 = [1, 1, %d], NCCL halo exchange)' % (ws, ws)) if ws > 1
                   else 'single',
                   'arithmetic': args.arithmetic,
                   'l2': 'inputs larger than L2 (%.1f GB resident)' % (nodes * 100 / 1e9),
                   'setup_s': round(setup_s, 2), 'host_wall_s': round(wall, 4)},
        'roofline': {'bound': 'hbm', 'kernel': kernel, 'launch_ms': launch_ms,
                     'achieved': achieved, 'peak': hbm, 'unit': 'GB/s', 'frac': achieved / hbm,
                     'peak_source': src, 'algorithmic_bytes_per_node': alg,
                     'algorithmic_bytes_per_launch': alg * knodes,
                     'traffic': (tr * knodes if tr else None)},
        'kernels_ms_per_step': {k: v[0] / prof_steps for k, v in kt.items() if v[1]},
        'reference_order': ref_order,
        'gpu_launches': int(launches),
        'clocks': clocks,
        'e2e': e2e,
        'ensemble': ens,
        'adjoint': adj,
        'configs': cfgs,
    }
    if ws == 1 and not args.no_cpu:
        try:
            thr = os.cpu_count() or 1
            v, info = cpu_sample(tuple(args.cpu_shape), args.cpu_steps, 1, thr)
            out['cpu_baseline'] = {'value': v, 'unit': 'node-updates/s', 'cores': thr, 'kind': 'port',
                                   'sample': 'oracle on the same workload at %dx%dx%d nodes, %d timed steps'
                                             % (tuple(args.cpu_shape) + (args.cpu_steps,))}
        except Exception as e:
            out['cpu_baseline'] = {'value': None, 'error': str(e)[:200]}
    print(json.dumps(out))


def run_e2e(args, shape, inputs, device, pg=None, ws=1, rank=0):
    """User call end to end: staged files on the host -> sord_run_directory
    (N > 1: every rank runs its slab, coseis_b200.parallel.run_dist, into
    one shared directory; the job takes the slowest rank's host time)."""
    from coseis_b200 import _lib
    nodes = float(np.prod(shape))
    work = shared_workdir(pg, rank, 'sord_e2e_')
    try:
        if rank == 0:
            stage_in(split_prm(wave_prm(shape, args.steps), ws), work, inputs)
        h2d = sum(os.path.getsize(os.path.join(inputs, f)) for f in ('rho.bin', 'vp.bin', 'vs.bin', 'z.bin'))
        h2d += os.path.getsize(os.path.join(work, 'sord.in')) if rank == 0 else 0
        # start from an idle device: the memory of the handles before is back with the driver
        _lib.trim_memory(device)
        barrier(pg)
        t0 = time.time()
        if ws > 1:
            from coseis_b200 import parallel
            parallel.run_dist(work, device, transport='device' if pg.get_backend() == 'nccl' else 'host')
        else:
            _lib.run_directory(work, device)
        wall = reduce_max(pg, time.time() - t0)
        barrier(pg)
        d2h = sum(os.path.getsize(os.path.join(work, f)) for f in os.listdir(work)
                  if f.endswith('.bin') and not os.path.islink(os.path.join(work, f)))
        if ws > 1:
            return {'value': nodes * args.steps / wall, 'unit': 'node-updates/s',
                    'h2d_bytes_per_step': h2d / args.steps, 'd2h_bytes_per_step': d2h / args.steps,
                    'wall_s': round(wall, 3), 'includes': 'setup of every slab from the staged host files, '
                                                          '%d steps, output files, teardown' % args.steps}
        # where the time goes: the same run again through the handle calls
        part = os.path.join(work, 'parts')
        text = stage_in(wave_prm(shape, args.steps), part, inputs)
        t0 = time.time()
        s = _lib.Solver(part, text, device=device)
        t1 = time.time()
        s.run()
        t2 = time.time()
        s.close()
        t3 = time.time()
        _lib.trim_memory(device)
        t4 = time.time()
        return {'value': nodes * args.steps / wall, 'unit': 'node-updates/s',
                'h2d_bytes_per_step': h2d / args.steps, 'd2h_bytes_per_step': d2h / args.steps,
                'wall_s': round(wall, 3), 'includes': 'setup from staged host files, %d steps, output files, '
                                                      'teardown' % args.steps,
                'parts_s': {'setup': round(t1 - t0, 3), 'steps_and_outputs': round(t2 - t1, 3),
                            'teardown': round(t3 - t2, 3),
                            'memory_return_after_teardown': round(t4 - t3, 3)}}
    finally:
        if rank == 0:
            shutil.rmtree(work, ignore_errors=True)


def run_ensemble_bench(n, nthreads, device, nt=ENS_NT, seed=SEED):
    """Batched rupture ensemble: scenarios 0..n-1 run one at a time by the
    plain solver (one sord_run_directory call each), then the same scenarios
    through one sord_run_ensemble call with `nthreads` concurrent scenarios.
    Each arm is timed by the host clock around all its calls (setup from
    staged files, nt steps, outputs written): the metric is scenarios/s of
    finished runs."""
    from coseis_b200 import _lib
    work = tempfile.mkdtemp(prefix='sord_ens_')
    try:
        ser = stage_scenarios(range(n), os.path.join(work, 'serial'), seed, nt)
        ens = stage_scenarios(range(n), os.path.join(work, 'batched'), seed, nt)
        _lib.run_ensemble(stage_scenarios([n], os.path.join(work, 'warm'), seed, 20), device, 1)
        t0 = time.time()
        for d in ser:
            _lib.run_directory(d, device)
        t_ser = time.time() - t0
        t0 = time.time()
        _lib.run_ensemble(ens, device, nthreads)
        t_ens = time.time() - t0
        # every output file but the wall-clock timers (prof-*.bin)
        keep = lambda f: f.endswith('.bin') and f != 'ts.bin' and not f.startswith('prof-')
        outs = [sorted(f for f in os.listdir(a) if keep(f)) for a in ser]
        same = all(o == sorted(f for f in os.listdir(b) if keep(f)) and
                   all(open(os.path.join(a, f), 'rb').read() == open(os.path.join(b, f), 'rb').read() for f in o)
                   for a, b, o in zip(ser, ens, outs))
        nfiles = sum(len(o) for o in outs)
        nodes = [int(np.prod(rupture_scenario(i, seed, nt)[0]['shape'][:3])) for i in range(n)]
        account = ensemble_account(stage_scenarios(range(0, n, 8), os.path.join(work, 'account'), seed, nt),
                                   device, nt)
        return {'metric': 'scenarios/s', 'value': n / t_ens, 'unit': 'scenarios/s',
                'one_at_a_time': n / t_ser, 'speedup': t_ser / t_ens, 'scenarios': n,
                'concurrent': nthreads, 'steps': nt, 'wall_s': round(t_ens, 3), 'serial_wall_s': round(t_ser, 3),
                'node_updates_per_s': float(sum(nodes)) * nt / t_ens, 'outputs_identical': bool(same),
                'files_compared': nfiles, 'account': account,
                'arithmetic': os.environ.get('SORD_ARITHMETIC', 'reference'),
                'workload': 'rupture ensemble: seeded grids 64x64x64..192x96x96, dx 100 m, dt 0.008 s, '
                            'slip-weakening +z fault, seeded friction / stresses (scenarios 0..%d)' % (n - 1)}
    finally:
        shutil.rmtree(work, ignore_errors=True)


def ensemble_account(dirs, device, nt):
    """Where one scenario's time goes, on a sample of freshly staged
    scenarios run one after another through the handle calls: setup from the staged
    files (host clock), the nt steps on the device (CUDA events around one
    sord_step call), the rest of the call (output files, host clock) and
    teardown.  Per scenario, averaged over the sample."""
    from coseis_b200 import _lib
    t = {'setup': 0.0, 'steps_device': 0.0, 'steps_host': 0.0, 'teardown': 0.0}
    for d in dirs:
        text = open(os.path.join(d, 'sord.in')).read()
        t0 = time.time()
        s = _lib.Solver(d, text, device=device)
        t1 = time.time()
        s.step(nt)
        t2 = time.time()
        dev = s.last_step_ms() / 1e3
        s.close()
        t3 = time.time()
        t['setup'] += t1 - t0
        t['steps_device'] += dev
        t['steps_host'] += t2 - t1
        t['teardown'] += t3 - t2
    n = max(len(dirs), 1)
    out = {k + '_ms': round(1e3 * v / n, 2) for k, v in t.items()}
    out['sample'] = len(dirs)
    return out


def wave_workload(shape):
    return ('wave226: %dx%dx%d nodes curvilinear terrain, layered von Karman medium, '
            '12-node PML on 5 faces, moment-tensor source, 64 receivers' % tuple(shape))


def host_memory_available():
    try:
        for line in open('/proc/meminfo'):
            if line.startswith('MemAvailable:'):
                return int(line.split()[1]) * 1024
    except Exception:
        pass
    return 0


def run_reference(args):
    """The reference arm: the CPU oracle (the C++ OpenMP restatement of
    sord/*.f90; the Fortran cannot be built here) on all host threads, on the
    same workload as the GPU arm: the full mesh when the host holds it (23
    FP32 arrays of the mesh with halos), timing --steps whole time steps
    after --warmup (each about 20 s on 16 threads at 768 x 768 x 384);
    otherwise the --cpu-shape sample for --steps steps."""
    ws = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return
    thr = os.cpu_count() or 1
    shape = tuple(args.shape)
    need = 23 * 4 * float(np.prod([n + 2 for n in shape])) * 1.15 + 6e9
    full = host_memory_available() >= need
    if full:
        steps = args.steps if args.ref_steps <= 0 else max(1, min(args.steps, args.ref_steps))
        warm = args.warmup
        exe = oracle_exe()
        inputs = os.path.join(args.cache, 'wave_%dx%dx%d_%d_%g' % (shape + (SEED, args.hill)))
        make_inputs(shape, inputs, hill=args.hill)
        d = tempfile.mkdtemp(prefix='sord_ref_')
        try:
            stage_in(wave_prm(shape, warm + steps), d, inputs)
            r = subprocess.run([exe, '--threads', str(thr), '--timed-from', str(warm)], cwd=d,
                               capture_output=True, text=True, timeout=3600)
            if r.returncode:
                raise RuntimeError(r.stderr[-2000:])
            info = json.loads(r.stdout.strip().splitlines()[-1])
        finally:
            shutil.rmtree(d, ignore_errors=True)
        nodes = float(np.prod(shape))
        v = nodes * steps / info['timed_seconds']
        sample = ('CPU oracle (C++ restatement of sord/*.f90, OpenMP, %d threads) on the whole %dx%dx%d mesh: '
                  '%d timed time steps after %d warm-up steps (setup %.0f s untimed)'
                  % ((thr,) + shape + (steps, warm, info['seconds'] - info['timed_seconds'])))
        cfg_shape = shape
    else:
        shape_s = tuple(args.cpu_shape)
        steps = args.steps
        v, info = cpu_sample(shape_s, args.steps, args.warmup, thr)
        sample = ('CPU oracle on the same workload at %dx%dx%d nodes, %d timed steps after %d warm-up steps '
                  '(the host has %.0f GB available, the whole mesh needs %.0f GB)'
                  % (shape_s + (args.steps, args.warmup, host_memory_available() / 1e9, need / 1e9)))
        cfg_shape = shape_s
    out = {
        'impl': 'reference', 'metric': 'node-updates/s', 'value': v, 'unit': 'node-updates/s',
        'n_gpus': ws, 'steps': steps, 'warmup': args.warmup,
        'ms_per_step': float(np.prod(cfg_shape)) / v * 1e3, 'higher_is_better': True,
        'scaling': 'strong', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic (seeded)',
        'config': {'workload': wave_workload(cfg_shape), 'nodes': int(np.prod(cfg_shape)), 'dx_m': DX, 'dt_s': DT},
        'cpu_baseline': {'value': v, 'unit': 'node-updates/s', 'cores': thr, 'kind': 'port', 'sample': sample},
        'e2e': {'value': v, 'unit': 'node-updates/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=100)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='ours')
    ap.add_argument('--shape', type=int, nargs=3, default=list(SHAPE))
    ap.add_argument('--cpu-shape', type=int, nargs=3, default=[192, 192, 96])
    ap.add_argument('--cpu-steps', type=int, default=8)
    ap.add_argument('--cache', default=os.environ.get('SORD_BENCH_CACHE', os.path.join(tempfile.gettempdir(), 'sord_bench')))
    ap.add_argument('--no-e2e', action='store_true')
    ap.add_argument('--no-cpu', action='store_true')
    ap.add_argument('--ensemble', type=int, default=256, help='rupture-ensemble scenarios (0: skip)')
    ap.add_argument('--no-configs', action='store_true', help='skip the explosion and rupture throughput lines')
    ap.add_argument('--ref-steps', type=int, default=0,
                    help='reference arm: cap on the timed steps of the full mesh (0: all --steps)')
    ap.add_argument('--ensemble-threads', type=int, default=8)
    ap.add_argument('--adjoint-steps', type=int, default=1200, help='adjoint workload steps (0: skip)')
    ap.add_argument('--hill', type=float, default=500.0, help='topography peak (m); 0 gives a rectilinear mesh')
    ap.add_argument('--arithmetic', choices=['reference', 'fast'], default='fast',
                    help='interior step kernel arithmetic (sord_set_arithmetic)')
    ap.add_argument('--backend', choices=['nccl', 'gloo'], default='nccl',
                    help='N > 1: halo planes over NCCL from device memory, or over gloo through host memory')
    ap.add_argument('--no-reference-order', action='store_true',
                    help='with --arithmetic fast, skip timing the reference-order kernel on the same handle')
    args = ap.parse_args()
    if args.impl == 'reference':
        run_reference(args)
    else:
        run_ours(args)


if __name__ == '__main__':
    main()
