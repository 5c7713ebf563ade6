"""Small SORD configurations used by the parity tests, and a runner that
stages one configuration twice (oracle / CUDA solver) and compares every
output file.  Sizes are chosen so the oracle finishes in seconds."""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from coseis_b200 import sord  # noqa: E402


def all_outputs(prm, fields='nc', step=None):
    """Add a '=>' output of every node/cell field (cst/tests/sord_mpi.py:27-29)."""
    for k, v in sord.fieldnames.items():
        if v[0][0] in fields and k[0] != '_':
            t = [] if step is None else [[], [], [], [None, None, step]]
            if '~' not in v[0] and step is not None:
                t = []
            prm[k] = list(prm.get(k, [])) + [(t, '=>', k + '.bin')]
    return prm


def case_mpi():
    """cst/tests/sord_mpi.py:14-31: 5x4x2 nodes, 2 steps, potency '=' at node 0."""
    prm = {
        'itstats': 1, 'shape': [5, 4, 2, 2], 'delta': [100.0, 100.0, 100.0, 0.0075],
        'rho': [2670.0], 'vp': [6000.0], 'vs': [3464.0], 'gam': [0.3],
        'hourglass': [1.0, 1.0], 'bc1': ['free'] * 3, 'bc2': ['free'] * 3,
    }
    all_outputs(prm)
    for f in 'pxx', 'pyy', 'pzz':
        prm[f] = prm[f] + [([0, 0, 0, 0], '=', 1e10)]
    return prm


def case_pml(n=22, nt=11):
    """cst/tests/sord_pml.py:14-31: PML on all faces, potency '=' at (10,10,10)."""
    prm = {
        'itstats': 1, 'shape': [n, n, n, nt], 'delta': [100.0, 100.0, 100.0, 0.0075],
        'rho': [2670.0], 'vp': [6000.0], 'vs': [3464.0], 'gam': [0.3],
        'hourglass': [1.0, 1.0], 'bc1': ['pml'] * 3, 'bc2': ['pml'] * 3, 'npml': 5,
    }
    all_outputs(prm)
    for f in 'pxx', 'pyy', 'pzz':
        prm[f] = prm[f] + [([10, 10, 10, 0], '=', 1e10)]
    return prm


def case_explosion(n=25, nt=40, npml=6):
    """Scaled-down explosion: isotropic moment '.' source (Brune), PML, receivers."""
    c = (n - 1) // 2
    prm = {
        'shape': [n, n, n, nt], 'delta': [100.0, 100.0, 100.0, 0.008],
        'rho': [2670.0], 'vp': [6000.0], 'vs': [3464.0], 'gam': [0.0],
        'hourglass': [1.0, 1.0], 'bc1': ['pml'] * 3, 'bc2': ['pml'] * 3, 'npml': npml,
        'itstats': 5, 'itio': 20,
    }
    for f in 'mxx', 'myy', 'mzz':
        prm[f] = [([c + 0.5, c + 0.5, c + 0.5, []], '.', 1e16, 'brune', 0.1)]
    for f in 'vx', 'vy', 'vz':
        prm[f] = [([[], [], c, [None, None, 5]], '=>', 'snap-%s.bin' % f)]
        for r, (x, y, z) in enumerate([(c - 5, c, c), (c, c + 4, c - 3), (c + 0.3, c - 2.6, c + 1.2)]):
            prm[f] += [([x, y, z, []], '.>', 'rec%d-%s.bin' % (r, f))]
    prm['am2'] = [([c, c, c, []], '=>', 'am2.bin')]
    prm['wm2'] = [([c, [], c, [None, None, 3]], '=>', 'wm2.bin')]
    return prm


def case_curvilinear(n=16, nt=12):
    """Random mesh (gridnoise) with PML and viscosity: general bracket path."""
    prm = case_pml(n, nt)
    prm['gridnoise'] = 0.1
    prm['npml'] = 3
    return prm


def case_bc():
    """Every boundary type on some face, hourglass viscosity, mixed PML."""
    prm = {
        'itstats': 2, 'shape': [14, 12, 10, 10], 'delta': [100.0, 100.0, 100.0, 0.0075],
        'rho': [2670.0], 'vp': [6000.0], 'vs': [3464.0], 'gam': [0.2],
        'hourglass': [1.0, 2.0], 'bc1': ['-node', '+cell', 'rigid'], 'bc2': ['pml', '-cell', '+node'],
        'npml': 3,
    }
    all_outputs(prm, step=2)
    prm['mxy'] = [([6.5, 5.5, 4.5, []], '.', 1e14, 'ricker1', 0.02)]
    return prm


def case_rupture(nx=21, ny=21, nz=10, nt=30):
    """Small Kostrov-like forced rupture (cst/tests/sord_kostrov.py:16-52)."""
    prm = {
        'delta': [100.0, 100.0, 100.0, 0.0075], 'shape': [nx, ny, nz, nt],
        'rho': [2670.0], 'vp': [6000.0], 'vs': [3464.0], 'gam': 1.0,
        'hourglass': [1.0, 1.0], 'bc1': ['pml'] * 3, 'bc2': ['-node', '+node', '-cell'],
        'npml': 4, 'faultnormal': '+z', 'hypocenter': [-1.0, -1.0, -1.5],
        'vrup': 0.9 * 3464.0, 'rcrit': 1e9, 'trelax': 0.0,
        'mud': 1.0, 'mus': 1e9, 'dc': 1e9, 'tn': -90e6, 'ts': -90e6 - 10e6,
        'itstats': 3, 'itio': 10,
    }
    for f in ('svm', 'sux', 'suy', 'sum', 'sl', 'psv', 'trup', 'tarr', 'tsm', 'tnm', 'fr',
              'tx', 'ty', 'tz', 'sax', 'sam', 'nsz'):
        prm[f] = [([], '=>', f + '.bin')]
    prm['vx'] = [([[], [], -1, []], '=>', 'vx.bin')]
    prm['svx'] = [([5.5, -1, []], '.>', 'p-svx.bin')]
    return prm


def case_slipweak(nt=40):
    """Spontaneous slip-weakening rupture with a nucleation patch (TPV3-like)."""
    prm = {
        'delta': [100.0, 100.0, 100.0, 0.008], 'shape': [30, 18, 24, 40],
        'rho': [2670.0], 'vp': [6000.0], 'vs': [3464.0], 'gam': [0.1],
        'hourglass': [1.0, 2.0], 'bc1': ['pml'] * 3, 'bc2': ['pml'] * 3, 'npml': 4,
        'faultnormal': '+y', 'hypocenter': [14.0, 8.5, 11.0], 'faultopening': 1,
        'mus': [1e4, ([[5, 25], [5, 18]], '=', 0.65)], 'mud': [0.5], 'dc': [0.3],
        'tn': [-100e6], 'ts': [58e6, ([[12, 17], [9, 14]], '=', 1.02 * 0.65 * 100e6)],
        'itstats': 4, 'itio': 20, 'vrup': -1.0,
    }
    for f in ('svm', 'sux', 'suz', 'sl', 'psv', 'trup', 'tsx', 'tsz', 'tnm', 'fr', 'sam'):
        prm[f] = [([], '=>', f + '.bin')]
    prm['vy'] = [([[], 9, [], [None, None, 4]], '=>', 'vy.bin')]
    return prm


def case_visc(n=23, nt=30):
    """Viscosity, viscous hourglass in the PML, receivers only (every step fused)."""
    prm = case_explosion(n, nt, npml=5)
    prm['gam'] = [0.4]
    prm['hourglass'] = [1.0, 2.0]
    prm.pop('am2')
    prm.pop('wm2')
    prm['bc1'] = ['pml', 'pml', 'free']
    return prm


def case_noise(n=18, nt=16):
    """Random mesh (gridnoise), PML, moment source, receivers only: general fused path."""
    prm = case_visc(n, nt)
    prm['gridnoise'] = 0.15
    prm['npml'] = 4
    return prm


def case_wave(shape=(40, 36, 30), nt=24):
    """The benchmark workload (terrain mesh, layered random medium read from
    '=<' files, moment tensor, surface receivers) at a small size."""
    import bench
    return bench.wave_prm(shape, nt, nrec=6)


def wave_inputs(path, shape=(40, 36, 30)):
    import bench
    inp = os.path.join(os.path.dirname(path), 'wave_inputs_%dx%dx%d' % tuple(shape))
    bench.make_inputs(shape, inp, use_torch=False)
    for f in ('rho.bin', 'vp.bin', 'vs.bin', 'z.bin'):
        dst = os.path.join(path, f)
        if not os.path.exists(dst):
            os.symlink(os.path.join(inp, f), dst)


def case_interior(shape=(72, 40, 28), nt=14, gridnoise=0.0):
    """A mesh large enough to hold interior tiles, so the fused interior
    kernel runs next to the PML kernel; one moment source inside an interior
    tile column and one inside the PML, viscous hourglass, every step fused."""
    nx, ny, nz = shape
    prm = {
        'shape': [nx, ny, nz, nt], 'delta': [100.0, 100.0, 100.0, 0.008],
        'rho': [2670.0], 'vp': [6000.0], 'vs': [3464.0], 'gam': [0.2],
        'hourglass': [1.0, 2.0], 'bc1': ['pml', 'pml', 'free'], 'bc2': ['pml'] * 3, 'npml': 4,
        'itstats': 3, 'itio': 10, 'gridnoise': gridnoise,
    }
    for f, v in (('mxx', 1e16), ('myy', 8e15), ('mzz', 1.2e16), ('mxy', -3e15)):
        prm[f] = [([45.3, 21.6, 13.2, []], '.', v, 'brune', 0.1),
                  ([2.5, 20.5, 6.5, []], '.', 0.5 * v, 'brune', 0.1)]
    for f in 'vx', 'vy', 'vz':
        prm[f] = [([[], 20, [], [None, None, 4]], '=>', 'snap-%s.bin' % f)]
        for r, (x, y, z) in enumerate([(40.0, 18.0, 0.0), (50.5, 25.25, 10.0), (3.0, 5.0, 20.0)]):
            prm[f] += [([x, y, z, []], '.>', 'rec%d-%s.bin' % (r, f))]
    return prm


def case_interior_noise():
    """The interior-tile case on a random (general) mesh."""
    return case_interior(gridnoise=0.1)


WAVE_INTERIOR = (80, 48, 32)


def case_interior_wave():
    """The benchmark workload (terrain mesh) at a size with interior tiles."""
    return case_wave(WAVE_INTERIOR, nt=16)


def interior_wave_inputs(path):
    wave_inputs(path, WAVE_INTERIOR)


def case_fault_x(nt=20):
    """x-normal slip-weakening fault with forced nucleation, PML on every
    face (the fused step with its fault kernels), a moment point source and
    fault outputs at every step."""
    prm = {
        'delta': [100.0, 100.0, 100.0, 0.008], 'shape': [44, 40, 30, nt],
        'rho': [2670.0], 'vp': [6000.0], 'vs': [3464.0], 'gam': [0.2],
        'hourglass': [1.0, 2.0], 'bc1': ['pml'] * 3, 'bc2': ['pml'] * 3, 'npml': 5,
        'faultnormal': '+x', 'slipvector': [0.0, 1.0, 0.0], 'hypocenter': [21.5, 19.0, 14.0],
        'vrup': 3000.0, 'rcrit': 1500.0,
        'trelax': 0.05, 'mus': [1e4, ([[6, 34], [6, 24]], '=', 0.6)], 'mud': [0.5], 'dc': [0.2],
        'tn': [-80e6], 'ts': [45e6, ([[16, 22], [11, 17]], '=', 50e6)],
        'itstats': 3, 'itio': 7,
        'mxy': [([30.3, 12.2, 20.6, []], '.', 1e14, 'brune', 0.05)],
    }
    for f in ('svm', 'sux', 'svy', 'tsm', 'trup', 'sam', 'tnm', 'psv', 'sl', 'tx', 'fr', 'tarr'):
        prm[f] = [([], '=>', f + '.bin')]
    prm['vx'] = [([[], [], 14, [None, None, 3]], '=>', 'vx.bin')]
    prm['am2'] = [([21, [], [], -1], '=>', 'am2.bin')]
    return prm


def case_fault_noise(nt=16):
    """z-normal spontaneous fault on a randomly perturbed (general) mesh."""
    prm = case_fault_x(nt)
    prm.update({'shape': [40, 36, 32, nt], 'faultnormal': '+z', 'slipvector': [1.0, 0.0, 0.0],
                'hypocenter': [19.0, 17.0, 15.5],
                'gridnoise': 0.05, 'vrup': -1.0,
                'mus': [1e4, ([[5, 34], [5, 30]], '=', 0.6)],
                'ts': [45e6, ([[15, 23], [13, 21]], '=', 50e6)]})
    prm['vx'] = [([[], 17, [], [None, None, 4]], '=>', 'vx.bin')]
    prm['am2'] = [([[], [], 16, -1], '=>', 'am2.bin')]
    prm['mxy'] = [([10.3, 12.2, 25.6, []], '.', 1e14, 'brune', 0.05)]
    return prm


def case_free(nt=24):
    """Free surfaces on all six faces, no PML: interior tiles reach every
    boundary (cells outside the mesh add zero); moment and force-free point
    source, snapshots and receivers."""
    prm = {
        'delta': [100.0, 100.0, 100.0, 0.008], 'shape': [44, 38, 30, nt],
        'rho': [2670.0], 'vp': [6000.0], 'vs': [3464.0], 'gam': [0.1], 'hourglass': [1.0, 0.7],
        'bc1': ['free'] * 3, 'bc2': ['free'] * 3, 'npml': 0, 'tm0': -0.1,
        'mxx': [([4.3, 5.6, 3.2, []], '.', 1e12, 'ricker2', 0.05)],
        'myz': [([4.3, 5.6, 3.2, []], '.', -4e11, 'ricker2', 0.05)],
        'itstats': 3, 'itio': 8,
    }
    prm['vx'] = [([[], [], 0, [None, None, 3]], '=>', 'vx-top.bin'), ([[], 0, [], -1], '=>', 'vx-side.bin')]
    prm['vz'] = [([[], [], -1, -1], '=>', 'vz-bottom.bin'), ([0.0, 5.5, 3.25, []], '.>', 'vz-corner.bin')]
    prm['uy'] = [([-1, [], [], -1], '=>', 'uy-far.bin')]
    prm['am2'] = [([[], [], [], -1], '=>', 'am2.bin')]
    return prm


def case_io_ops(nt=6):
    """Every field-I/O op kind on a node field (ax) and a cell field (wxx),
    after cst/tests/sord_io.py: '#', '= + *', the random '=~ +~ *~', the
    cube '=@ +@ *@', '=' with every time function, a '.' point op and the
    file reads '.< =< +< *<'; outputs of several fields by '.>' and '=>'."""
    from coseis_b200 import sord
    prm = {'shape': [9, 10, 11, nt], 'delta': [100.0, 100.0, 100.0, 0.008], 'itstats': 1, 'itio': 3,
           'bc1': ['free'] * 3, 'bc2': ['free'] * 3, 'npml': 0, 'gam': [0.1], 'hourglass': [1.0, 0.5],
           'mxx': [([4.0, 4.5, 5.0, []], '.', 1e14, 'brune', 0.05)]}
    x1, x2 = [110.0, 110.0, 110.0], [590.0, 690.0, 790.0]
    ii = [4.4, 5.5, 6.6, 1]
    for k in ('ax', 'wxx'):
        ops = [([], '#')]
        for op in ('=', '+', '*', '=~', '+~', '*~'):
            ops.append(([], op, 2.2))
        for op in ('=@', '+@', '*@'):
            ops.append(([], op, x1, x2, 2.2))
        for func in sorted(sord.time_functions):
            ops.append(([], '=', 2.2, func, 0.033))
        ops.append((ii, '.', 2.2))
        for i, op in enumerate(('.<', '=<', '+<', '*<')):
            ops.append((ii if op == '.<' else [4, 5, 6, 1], op, '%s_i%d.bin' % (k, i)))
        prm[k] = ops
    # ops whose results last (the sequences above end in plain sets)
    prm['gam'] = [([], '=~', 0.2)]
    prm['rho'] = [2670.0, ([], '+@', x1, x2, 100.0)]
    prm['vx'] = [([], '+~', 1e-4)]
    prm['vy'] = [([], '*@', x1, x2, 0.5)]
    prm['vz'] = [([], '*~', 1.0)]
    for k in ('vx', 'vy', 'uz', 'ax', 'wxx', 'wyz', 'am2', 'wm2'):
        prm[k] = list(prm.get(k, [])) + [([4.4, 5.5, 6.6, []], '.>', 'o1-%s.bin' % k),
                                          ([[], [], 5, []], '=>', 'o0-%s.bin' % k)]
    return prm


def io_ops_inputs(path):
    for k in ('ax', 'wxx'):
        for i in range(4):
            np.array([1.5 + i], '<f4').tofile(os.path.join(path, '%s_i%d.bin' % (k, i)))


CASES = {
    'mpi': case_mpi,
    'pml': case_pml,
    'explosion': case_explosion,
    'curvilinear': case_curvilinear,
    'bc': case_bc,
    'rupture': case_rupture,
    'slipweak': case_slipweak,
    'visc': case_visc,
    'noise': case_noise,
    'wave': case_wave,
    'interior': case_interior,
    'interior_noise': case_interior_noise,
    'interior_wave': case_interior_wave,
    'fault_x': case_fault_x,
    'fault_noise': case_fault_noise,
    'free': case_free,
    'io_ops': case_io_ops,
}
INPUTS = {'wave': wave_inputs, 'interior_wave': interior_wave_inputs, 'io_ops': io_ops_inputs}


def stage(prm, path, realsize=4, inputs=None):
    os.makedirs(path, exist_ok=True)
    if inputs:
        inputs(path)
    cwd = os.getcwd()
    os.chdir(path)
    try:
        sord.stage(prm, realsize=realsize)
    finally:
        os.chdir(cwd)


def run_oracle(path, exe, threads=4):
    r = subprocess.run([exe, '--threads', str(threads)], cwd=path, capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError('oracle failed: ' + r.stderr)
    return json.loads(r.stdout.strip().splitlines()[-1])


def run_gpu(path, fused=True, arithmetic='reference'):
    """Run the CUDA solver through the C ABI; SORD_FUSED and SORD_ARITHMETIC
    (read when a handle is created) select the fused step kernel or the
    per-stage kernels, and the interior kernel's arithmetic."""
    from coseis_b200 import _lib
    env = {'SORD_FUSED': '1' if fused else '0', 'SORD_ARITHMETIC': arithmetic}
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        _lib.run_directory(path)
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


def outputs(path):
    skip = ('prof-',)
    return sorted(f for f in os.listdir(path) if f.endswith('.bin') and not f.startswith(skip))


def compare(path_a, path_b, dtype_a='<f4', dtype_b='<f4'):
    """Per-file max |a-b| / max |a| and exact-equality flag."""
    res = {}
    fa, fb = outputs(path_a), outputs(path_b)
    assert fa == fb, (set(fa) ^ set(fb))
    for f in fa:
        a = np.fromfile(os.path.join(path_a, f), dtype_a).astype(np.float64)
        b = np.fromfile(os.path.join(path_b, f), dtype_b).astype(np.float64)
        assert a.shape == b.shape, (f, a.shape, b.shape)
        scale = np.abs(a).max() if a.size else 0.0
        d = np.abs(a - b).max() if a.size else 0.0
        res[f] = (d / scale if scale > 0 else d, bool(np.array_equal(a, b)))
    return res
