"""Receiver-misfit gradients through the CUDA adjoint of the SORD time loop.

    problem = adjoint.Problem(prm, source, receivers)
    traces = adjoint.ReceiverTraces.apply(rho, vp, vs, moment, problem)
    loss = 0.5 * ((traces - observed) ** 2).sum()
    loss.backward()   # rho.grad, vp.grad, vs.grad per cell; moment.grad (6)

The reference computes no derivatives; the forward run is the one
``cst.sord.run`` would make with ``rho``, ``vp``, ``vs`` as '=<' cell files
and the moment tensor as six '.' point ops.  The backward pass is the
library's discrete adjoint (``sord_adjoint_forward`` / ``_backward`` in
include/sordgpu.h): it returns dL/d(lambda), dL/d(mu), dL/d(yy) per cell and
dL/d(mr) per node, and this module applies the chain rule of the material
setup (sord/material_model.f90:65-76, 120-134: mu = rho vs^2,
lambda = rho vp^2 - 2 mu, yy = mu (lambda + mu) s / (lambda + 2 mu) with
s = sqrt((dx^2 + dy^2 + dz^2) / 3) / 12; sord/material_resample.f90:16-18:
mr = 1 / mean of rho V over the 8 cells around a node).  Material limits
(``vp_min`` ...) are not differentiated; leave them unset.  With PML
faces the damping profile is held fixed: give ``vpml`` a value (by default
it follows the material's extremes).

Supported runs: rectilinear mesh, no fault, boundary conditions that need
no plane copies (free, PML), every step a plain step.
"""
import math
import os
import shutil
import tempfile

import numpy as np

from . import _lib, sord

MOMENT = ('mxx', 'myy', 'mzz', 'myz', 'mzx', 'mxy')
COMPONENTS = ('x', 'y', 'z')


def _write_cells(path, a, dtype):
    np.asarray(a, dtype=dtype).ravel(order='F').tofile(path)


class Problem(object):
    """A forward problem whose material and moment tensor are the variables.

    prm        cst.sord parameters without rho/vp/vs/m** entries
    source     dict(x=[x, y, z] position of the '.' ops (cell registration),
               pulse=time function name, tau=its parameter)
    receivers  list of [x, y, z] node positions; each records vx, vy, vz
               at every step ('.>' ops)
    segment    steps between checkpoints: 1 keeps every state (no
               recomputation), 0 or None lets the library choose (1 when
               the states fit in half of the free device memory, else about
               sqrt(nt))
    snapshots  if given, binomial checkpointing with at most this many
               kept states instead of uniform segments
    """

    def __init__(self, prm, source, receivers, segment=None, device=0, snapshots=None):
        self.prm = dict(prm)
        self.source = dict(source)
        self.receivers = [list(r) for r in receivers]
        self.segment = int(segment or 0)
        self.snapshots = int(snapshots or 0)
        self.device = device

    def forward(self, solver):
        """The adjoint forward run on `solver` with this problem's schedule."""
        if self.snapshots > 0:
            solver.adjoint_forward_binomial(self.snapshots)
        else:
            solver.adjoint_forward(self.segment)

    @property
    def cells(self):
        return tuple(n - 1 for n in self.prm['shape'][:3])

    def files(self):
        return ['r%03d-v%s.bin' % (r, c) for r in range(len(self.receivers)) for c in COMPONENTS]

    def stage(self, rho, vp, vs, moment, path, realsize=4):
        """Write the material files and sord.in into `path`; returns the
        receiver file names in (receiver, component) order."""
        os.makedirs(path, exist_ok=True)
        dt = '<f4' if realsize == 4 else '<f8'
        for name, a in (('rho', rho), ('vp', vp), ('vs', vs)):
            a = np.asarray(a)
            if a.shape != self.cells:
                raise ValueError('%s has shape %s, cells are %s' % (name, a.shape, self.cells))
            _write_cells(os.path.join(path, name + '.bin'), a, dt)
        prm = dict(self.prm)
        prm['rho'] = [([], '=<', 'rho.bin')]
        prm['vp'] = [([], '=<', 'vp.bin')]
        prm['vs'] = [([], '=<', 'vs.bin')]
        x = list(self.source['x'])
        for f, m in zip(MOMENT, np.asarray(moment, dtype=np.float64).ravel()):
            prm[f] = [([x[0], x[1], x[2], []], '.', float(m), self.source['pulse'], float(self.source['tau']))]
        for r, xr in enumerate(self.receivers):
            for c in COMPONENTS:
                prm['v' + c] = list(prm.get('v' + c, [])) + [([xr[0], xr[1], xr[2], []], '.>', 'r%03d-v%s.bin' % (r, c))]
        cwd = os.getcwd()
        os.chdir(path)
        try:
            sord.stage(prm, realsize=realsize)
        finally:
            os.chdir(cwd)
        return self.files()

    def moment_order(self, path):
        """Component index of each '.' moment op in sord.in order."""
        order = []
        for line in open(os.path.join(path, 'sord.in')).read().splitlines()[1:]:
            t = line.split()
            if t and t[0] in MOMENT and t[-2] == '.':
                order.append(MOMENT.index(t[0]))
        return order

    def read_traces(self, path, dtype='<f4'):
        a = [np.fromfile(os.path.join(path, f), dtype) for f in self.files()]
        return np.stack(a).reshape(len(self.receivers), 3, -1)


def material_chain(rho, vp, vs, g, delta):
    """Chain rule of the material setup: gradients with respect to
    (lambda, mu, yy) per cell and mr per node -> (rho, vp, vs) per cell.
    Arrays are indexed [j, k, l]; computed in float64."""
    rho = np.asarray(rho, np.float64)
    vp = np.asarray(vp, np.float64)
    vs = np.asarray(vs, np.float64)
    mu = rho * vs * vs
    lam = rho * vp * vp - 2.0 * mu
    s = math.sqrt((delta[0] ** 2 + delta[1] ** 2 + delta[2] ** 2) / 3.0) / 12.0
    r = lam + 2.0 * mu
    with np.errstate(divide='ignore', invalid='ignore'):
        dl = np.where(r != 0, s * mu * mu / (r * r), 0.0)
        dm = np.where(r != 0, s * (lam * lam + 2.0 * lam * mu + 2.0 * mu * mu) / (r * r), 0.0)
    gl = g['lam'].astype(np.float64) + g['yy'] * dl
    gm = g['mu'].astype(np.float64) + g['yy'] * dm
    grho = gl * (vp * vp - 2.0 * vs * vs) + gm * vs * vs
    gvp = gl * 2.0 * rho * vp
    gvs = gl * (-4.0 * rho * vs) + gm * 2.0 * rho * vs
    # nodal mass: mr(n) = 1 / (sum over the 8 cells around n of rho V / 8)
    V = float(delta[0] * delta[1] * delta[2])
    nx, ny, nz = (n + 1 for n in rho.shape)
    S = np.zeros((nx, ny, nz))
    rv = rho * V
    for dj in (0, 1):
        for dk in (0, 1):
            for dl_ in (0, 1):
                S[dj:dj + nx - 1, dk:dk + ny - 1, dl_:dl_ + nz - 1] += rv
    with np.errstate(divide='ignore'):
        mr = np.where(S != 0, 8.0 / S, 0.0)
    gn = g['mr'].astype(np.float64) * (-mr * mr) * 0.125 * V
    for dj in (0, 1):
        for dk in (0, 1):
            for dl_ in (0, 1):
                grho += gn[dj:dj + nx - 1, dk:dk + ny - 1, dl_:dl_ + nz - 1]
    return grho, gvp, gvs


def _function():
    import torch

    class ReceiverTraces(torch.autograd.Function):
        """traces[r, c, t] = v_c at receiver r, sample t, of the forward run
        with cell fields rho, vp, vs ([j, k, l]) and moment tensor
        (xx yy zz yz zx xy); optionally the source position (3, node-index
        coordinates like the problem's source 'x') and a delay of the source
        time function (seconds) as differentiable inputs too."""

        @staticmethod
        def forward(ctx, rho, vp, vs, moment, problem, position=None, delay=None):
            ctx.has_source = (position is not None, delay is not None)
            if position is not None or delay is not None:
                problem = Problem(problem.prm, problem.source, problem.receivers, problem.segment, problem.device,
                                  problem.snapshots)
                if position is not None:
                    problem.source['x'] = [float(a) for a in position.detach().cpu().numpy().ravel()]
                if delay is not None:
                    # a delay of the time function is an earlier clock origin
                    problem.prm['tm0'] = float(problem.prm.get('tm0', 0.0)) - float(delay.detach().cpu())
            d = tempfile.mkdtemp(prefix='sord_adj_')
            try:
                problem.stage(rho.detach().cpu().numpy(), vp.detach().cpu().numpy(), vs.detach().cpu().numpy(),
                              moment.detach().cpu().numpy(), d)
                s = _lib.Solver(d, open(os.path.join(d, 'sord.in')).read(), device=problem.device)
                try:
                    problem.forward(s)
                    tr = problem.read_traces(d)
                except Exception:
                    s.close()
                    raise
            except Exception:
                shutil.rmtree(d, ignore_errors=True)
                raise
            ctx.solver, ctx.dir, ctx.problem = s, d, problem
            ctx.order = problem.moment_order(d)
            ctx.save_for_backward(rho, vp, vs, moment)
            return torch.as_tensor(tr, dtype=rho.dtype, device=rho.device)

        @staticmethod
        def backward(ctx, gtr):
            rho, vp, vs, moment = ctx.saved_tensors
            p = ctx.problem
            g = gtr.detach().cpu().numpy().astype(np.float32)
            files = p.files()
            dtr = {f: g[i // 3, i % 3] for i, f in enumerate(files)}
            try:
                res = ctx.solver.adjoint_backward(dtr, len(ctx.order))
            finally:
                ctx.solver.close()
                shutil.rmtree(ctx.dir, ignore_errors=True)
            grho, gvp, gvs = material_chain(rho.detach().cpu().numpy(), vp.detach().cpu().numpy(),
                                            vs.detach().cpu().numpy(), res, p.prm['delta'])
            gmom = np.zeros(6)
            for m, c in enumerate(ctx.order):
                gmom[c] += res['moment'][m]
            t = lambda a, like: torch.as_tensor(a, dtype=like.dtype, device=like.device)
            # source position per node-index unit, summed over the six ops; delay per second
            gpos = (res['position'].sum(0) * np.asarray(p.prm['delta'][:3], np.float64)
                    if ctx.has_source[0] else None)
            gdel = float(res['delay'].sum()) if ctx.has_source[1] else None
            like = rho
            return (t(grho, rho), t(gvp, vp), t(gvs, vs), t(gmom, moment), None,
                    None if gpos is None else t(gpos, like), None if gdel is None else t(gdel, like))

    return ReceiverTraces


class _Lazy(object):
    """``ReceiverTraces`` is built on first use so that importing this module
    does not import torch."""
    _f = None

    def __getattr__(self, name):
        if _Lazy._f is None:
            _Lazy._f = _function()
        return getattr(_Lazy._f, name)


ReceiverTraces = _Lazy()
