"""Generate the golden fixtures in this directory from the reference.

Run in a checkout that has the Coseis reference (shineusn/coseis) on disk:

    python tests/golden/make_golden.py /path/to/coseis

It imports only pure functions of the reference's Python package and writes
small JSON files; nothing here is read by the tests at run time except those
files.

* kostrov.json -- analytic slip rate of the Kostrov circular crack at the
  four receivers of cst/tests/sord_kostrov.py (cst/kostrov.py:31-47, the C
  constant from the Dahlen integral).
* explosion.json -- analytic radial velocity of the explosion point source
  of scripts/Explosion-sim.py at its receiver p2 (M0 = 3 rho vp^2 -
  4 rho vs^2 per unit potency, moment history = integral of the Brune
  pulse), sampled on the solver's output times, unfiltered and after the
  lowpass of scripts/Explosion-plot.py:54-58 (cst/dsp.py:107-142), plus a
  probe vector through the same filter to pin its restatement.
* srf.json -- a small synthetic SRF rupture read and written by the
  reference (cst/srf.py:13-194) and the fault geometry of its points
  (cst/coord.py:190-202 slip_vectors, 336-351 potency_tensor).
* loh1_fk.npz -- the Prose frequency-wavenumber solution of the PEER
  LOH.1 problem (layer over a half-space, buried double couple) shipped
  with the reference as data/LOH1-ProseFK-{Time,V-Radial,V-Transverse,
  V-Vertical}.npy, the traces scripts/PEER-LOH1-plot.py compares SORD
  with (receiver 9, 10 km from the epicentre), copied unchanged (float32).
* tpv3_bi.npz -- the boundary-integral solution of SCEC TPV3 shipped with
  the reference as data/TPV3-BI-*.npy (time, slip, slip rate and shear
  traction at the mode II station P1 and the mode III station P2, rupture
  time on a 300 x 150 grid of 0.1 km cells), the traces
  scripts/TPV3-plot.py compares SORD with, copied unchanged (float32).
* frontend.json -- for several parameter sets, the sord.in text and the
  metadata (indices, shapes, deltas) that the reference front end produces:
  cst/sord.py:prepare (cst/sord.py:296-468) followed by the sord.in
  serialisation of cst/sord.py:538-544.  cst/sord.py:stage() itself cannot
  be used: it builds the Fortran solver first (cst/sord.py:495).  Two
  defects of the shipped front end are bypassed as the CUDA front end fixes
  them: typed_dict (cst/sord.py:219-223) is replaced by a plain dict, and
  expand_slices (cst/sord.py:226-238) maps [] to the whole axis and returns
  lists; the parameter sets use nx == nz so the node-shape defect of
  cst/sord.py:355 does not change the result.
"""
import copy
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# ------------------------------------------------------------ parameter sets
# Kostrov: cst/tests/sord_kostrov.py:12-49
KOSTROV = dict(dx=100.0, dt=0.0075, shape=[51, 51, 24, 200], rho=2670.0, vp=6000.0, vs=3464.0,
               dtau=10e6, r=2000.0, vrup_frac=0.9)

# Explosion: scripts/Explosion-sim.py with its last step-size option (dx 200 m,
# dt 0.016 s) and its '+node' registration option (reg 0).  Its other
# registration, '+cell' at reg 0.5, puts the point source in the boundary cell
# that scalar_bc overwrites with its neighbour after every op
# (sord/input_output.f90:256-257, boundary_cond.f90 scalar_bc), so that
# configuration radiates nothing.
EXPLOSION = dict(dx=200.0, dt=0.016, rho=2670.0, vp=6000.0, vs=3464.0, tau=0.1, reg=0.0, bc='+node')


def explosion_grid():
    dx, dt = EXPLOSION['dx'], EXPLOSION['dt']
    nx = int(6000.0 / dx + 1.0001)
    nt = int(3.0 / dt + 1.0001)
    return nx, nt


def frontend_cases():
    """Parameter sets for the front-end fixtures (nx == nz)."""
    cases = {}
    cases['explosion'] = {
        'shape': [21, 17, 21, 30], 'delta': [100.0, 100.0, 100.0, 0.008],
        'bc1': ['pml', 'pml', 'free'], 'bc2': ['pml', 'pml', 'pml'], 'npml': 4,
        'hourglass': [1.0, 0.5], 'itstats': 5, 'itio': 10,
        'mxx': [([10.25, 8.5, 10.0, []], '.', 1e16, 'brune', 0.1)],
        'myy': [([10.25, 8.5, 10.0, []], '.', 1e16, 'brune', 0.1)],
        'mxy': [([10.25, 8.5, 10.0, [0, 20]], '.', -3e15, 'ricker1', 0.2)],
        'vx': [([12.5, 3.25, 0.0, []], '.>', 'r1-vx.bin'),
               ([[], 8, [], [0, None, 5]], '=>', 'snap-vx.bin')],
        'vz': [([[2, 19, 3], [1, -1], -1, [4, 25, 2]], '=>', 'sub-vz.bin')],
        'rho': [2500.0, ([[0, 10], [], []], '*', 1.1), ([], '+~', 5.0)],
        'vs': [([], '*@', [0.0, 0.0, 0.0], [900.0, 900.0, 500.0], 0.9)],
    }
    cases['rupture'] = {
        'shape': [31, 21, 31, 40], 'delta': [100.0, 100.0, 100.0, 0.0075],
        'bc1': ['pml', 'pml', 'pml'], 'bc2': ['-node', '+node', 'pml'], 'npml': 5,
        'faultnormal': '+z', 'hypocenter': [-1.0, -1.0, 15.5], 'vrup': 3000.0, 'rcrit': 1000.0,
        'trelax': 0.05, 'gam': [0.1],
        'mus': [0.7, ([[0, 10], [0, 10]], '=', 10000.0)], 'mud': [0.5], 'dc': [0.4],
        'tn': [-70e6], 'ts': [-40e6, ([[-5, None], [-5, None]], '=', -45e6)],
        'svm': [([-1, -11, []], '=>', 'p-svm.bin')],
        'sux': [([[], [], [0, None, 10]], '=>', 'sux.bin')],
        'trup': [([[], [], []], '=>', 'trup.bin')],
    }
    cases['inputs'] = {
        'shape': [13, 11, 13, 6], 'delta': [50.0, 50.0, 50.0, 0.004],
        'bc1': ['+cell', '-cell', 'rigid'], 'bc2': ['+node', '-node', 'free'], 'npml': 0,
        'rho': [([], '=<', 'rho.bin')], 'vp': [([], '=<', 'vp.bin')], 'vs': [3000.0],
        'z': [([], '=<', 'z.bin')], 'gridnoise': 0.1,
        'fz': [([6.0, 5.0, 6.0, []], '.', 1e10, 'hann', 0.02)],
        'ux': [([[1, -1], [], [], -1], '=>', 'ux-last.bin')],
        'um2': [([6, 5, 6, []], '=>', 'um2.bin')],
        'source': 'force',
    }
    return cases


# ------------------------------------------------------------- generators
def reference_front_end(ref):
    sys.dont_write_bytecode = True
    sys.path.insert(0, ref)
    import cst.sord as S

    def expand_slices(shape, slices):
        n = len(shape)
        if len(slices) == 0:
            slices = n * [[]]
        elif len(slices) != n:
            raise Exception('error in indices: %r' % (slices,))
        out = []
        for m, s in zip(shape, slices):
            if isinstance(s, (list, tuple)):
                s = list((slice(*s) if s else slice(None)).indices(m))
            else:
                s = [s % m, s % m + 1, 1]
            out.append(s)
        return out
    S.expand_slices = expand_slices
    return S


def sord_in(prm, fio):
    """The sord.in wire format: sorted parameter values on line 1, one op per
    line, JSON with '"', ',', '[' and ']' removed."""
    text = json.dumps([prm[k] for k in sorted(prm)]) + '\n'
    for op in fio:
        text += json.dumps(op) + '\n'
    for c in '",[]':
        text = text.replace(c, '')
    return text


def make_frontend(S):
    out = {}
    for name, args in frontend_cases().items():
        prm, fio = {}, {}
        for k, v in S.parameters.items():
            (fio if k in S.fieldnames else prm)[k] = copy.deepcopy(v)
        for k, v in copy.deepcopy(args).items():
            (fio if k in S.fieldnames else prm)[k] = v
        prm, fio, meta = S.prepare(prm, fio)
        out[name] = {'args': args, 'sord_in': sord_in(prm, fio), 'meta': meta}
    return out


def make_kostrov(ref):
    sys.path.insert(0, ref)
    from cst import kostrov
    k = KOSTROV
    nt = k['shape'][3]
    vr = k['vrup_frac'] * k['vs']
    t = (nt - 1.5) * k['dt'] - k['r'] / vr
    v = float(kostrov.slip_rate(k['rho'], k['vp'], k['vs'], vr, k['dtau'], k['r'], t))
    c = float(kostrov.cee(vr / k['vp'], vr / k['vs']))
    return dict(k, vrup=vr, t=t, slip_rate=v, C=c, reference_tolerance=0.015)


def make_explosion(ref):
    sys.path.insert(0, ref)
    import cst.dsp
    e = EXPLOSION
    nx, nt = explosion_grid()
    dx, dt, reg = e['dx'], e['dt'], e['reg']
    # receiver p2 of scripts/Explosion-sim.py: (reg, reg + 3 km / dx, reg + 4 km / dx)
    x, y, z = 0.0, 3000.0, 4000.0
    r = math.sqrt(x * x + y * y + z * z)
    rho, vp, vs, tau = e['rho'], e['vp'], e['vs'], e['tau']
    m0 = 3 * rho * vp * vp - 4 * rho * vs * vs
    # scripts/Explosion-plot.py:43-49: va(t) is the radial velocity at time t + r / vp
    t = np.arange(0.5, nt) * dt
    va = m0 * np.exp(-t / tau) * (t * vp / r - t / tau + 1) / (4 * math.pi * rho * vp ** 3 * tau * tau * r)
    # the same signal on the solver's sample times: sample i is at t_i
    s = np.arange(0.5, nt) * dt - r / vp
    vs_ = np.where(s > 0, m0 * np.exp(-s / tau) * (s * vp / r - s / tau + 1) /
                   (4 * math.pi * rho * vp ** 3 * tau * tau * r), 0.0)
    cutoff = vp / (20.0 * dx)
    vf = cst.dsp.filter(vs_, dt, cutoff, 'lowpass', 2, 1)
    probe = np.linspace(-1, 1, 64) ** 3
    return dict(e, nx=nx, nt=nt, receiver=[x, y, z], r=r, m0=m0, cutoff=cutoff,
                analytic=vs_.tolist(), analytic_filtered=vf.tolist(),
                filter_probe=probe.tolist(),
                filter_probe_out=cst.dsp.filter(probe, dt, cutoff, 'lowpass', 2, 1).tolist(),
                plot_analytic_first=float(va[0]))


# A small synthetic SRF rupture (one plane of 3 x 2 points) for the SRF
# reader / writer / geometry fixtures; all numbers are made up here.
SRF_TEXT = """1.0
PLANE 1
-118.0 34.0 3 2 3.0 2.0
30.0 60.0 0.5 1.0 0.8
POINTS 6
-118.01 34.00 1.0 30.0 60.0 100000000.0 0.10 0.01
90.0 20.0 3 5.0 2 0.0 0
1.0 2.0 3.0 4.0 5.0
-118.00 34.00 1.0 30.0 60.0 100000000.0 0.15 0.01
45.0 30.0 4 0.0 0 10.0 1
0.5 1.5 2.5 3.5 7.0
-117.99 34.00 1.0 31.0 61.0 100000000.0 0.20 0.02
0.0 10.0 2 0.0 0 0.0 0
6.0 8.0
-118.01 34.01 1.9 30.0 60.0 100000000.0 0.30 0.01
-30.0 0.0 0 12.0 3 0.0 0
1.0 1.0 1.0
-118.00 34.01 1.9 29.0 59.0 100000000.0 0.35 0.01
170.0 15.0 1 15.0 1 1.0 1
2.0 3.0 4.0
-117.99 34.01 1.9 30.0 60.0 100000000.0 0.40 0.01
90.0 0.0 0 0.0 0 0.0 0

"""


def make_srf(ref):
    """Reference SRF read of SRF_TEXT, its write, and the fault geometry of
    every point (cst/srf.py:13-194, cst/coord.py:190-202, 336-351)."""
    import io
    sys.path.insert(0, ref)
    from cst import coord, srf
    fh = io.StringIO(SRF_TEXT)
    fh.name = 'synthetic.srf'
    meta, data = srf.read(fh)
    # the reference writer indexes the arrays by point, so it needs them in
    # file order (read reshapes single-plane files to the plane grid)
    fdata = {k: (np.asarray(v).T.ravel() if np.ndim(v) > 1 else v) for k, v in data.items()}
    out = io.StringIO()
    srf.write(out, (meta, fdata))
    flat = {k: np.asarray(v).T.ravel().tolist() for k, v in data.items() if not k.startswith('sv')}
    R = coord.slip_vectors(np.asarray(flat['stk']), np.asarray(flat['dip']), np.asarray(flat['rake']))
    R = np.asarray([[np.asarray(c, dtype=float) for c in row] for row in R])
    pot = [coord.potency_tensor(R[2], R[0]), coord.potency_tensor(R[2], R[1]), coord.potency_tensor(R[2], R[2])]
    return {'text': SRF_TEXT, 'meta': meta, 'data': flat,
            'sv': [np.asarray(data['sv%d' % c]).tolist() for c in (1, 2, 3)],
            'written': out.getvalue(), 'slip_vectors': R.tolist(),
            'potency': [[np.asarray(a, dtype=float).tolist() for a in part] for p_ in pot for part in p_]}


def write_loh1(ref):
    import numpy as np
    names = {'t': 'Time', 'radial': 'V-Radial', 'transverse': 'V-Transverse', 'vertical': 'V-Vertical'}
    arrs = {k: np.load(os.path.join(ref, 'data', 'LOH1-ProseFK-%s.npy' % v)) for k, v in names.items()}
    np.savez_compressed(os.path.join(HERE, 'loh1_fk.npz'), **arrs)


def write_tpv3(ref):
    import numpy as np
    names = {'t': 'P-Time', 'trup': 'Rupture-Time'}
    for sta in ('P1', 'P2'):
        for k, v in (('slip', 'Slip'), ('sv', 'Slip-Velocity'), ('ts', 'Traction')):
            names['%s_%s' % (sta.lower(), k)] = '%s-%s' % (sta, v)
    arrs = {k: np.load(os.path.join(ref, 'data', 'TPV3-BI-%s.npy' % v)) for k, v in names.items()}
    np.savez_compressed(os.path.join(HERE, 'tpv3_bi.npz'), **arrs)


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('COSEIS_REFERENCE', '')
    if not ref or not os.path.isdir(os.path.join(ref, 'cst')):
        raise SystemExit('usage: make_golden.py /path/to/coseis')
    S = reference_front_end(ref)
    with open(os.path.join(HERE, 'frontend.json'), 'w') as fh:
        json.dump(make_frontend(S), fh, indent=1, sort_keys=True)
    with open(os.path.join(HERE, 'kostrov.json'), 'w') as fh:
        json.dump(make_kostrov(ref), fh, indent=1, sort_keys=True)
    with open(os.path.join(HERE, 'explosion.json'), 'w') as fh:
        json.dump(make_explosion(ref), fh, indent=1, sort_keys=True)
    with open(os.path.join(HERE, 'srf.json'), 'w') as fh:
        json.dump(make_srf(ref), fh, indent=1, sort_keys=True, default=lambda o: o.item())
    write_loh1(ref)
    write_tpv3(ref)


if __name__ == '__main__':
    main()
