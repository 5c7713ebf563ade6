"""Fast arithmetic of the interior step kernel (sord_set_arithmetic mode 1,
SORD_ARITHMETIC=fast): fused multiply-adds, brackets scaled once per cell,
divergence brackets taken as negated gradient brackets, closed-form terrain
brackets.  Not bit-identical to the reference's FP32 arithmetic, so it is
held to the accuracy bound of the wave workload instead: relative L2 error
<= 1e-4 of every velocity, displacement, slip and slip-rate output against
the FP64 oracle (and against the FP32 oracle), of the same order as the FP32
oracle's own error, and rupture times within one time step."""
import os

import numpy as np
import pytest

import sordcases as sc

TOL_L2 = 1e-4
# interior tiles on rectilinear, general and terrain meshes, all-free
# boundaries, and a fault
# and meshes without interior tiles (the shell kernel alone)
CASES = ['interior', 'interior_noise', 'interior_wave', 'free', 'fault_x', 'fault_noise', 'explosion', 'visc',
         'noise', 'wave']
# cases whose output steps read stress (separate-kernel path there)
MIXED = {'explosion'}


def rel_l2(a, b, floor=0.0):
    """||a - b|| / ||b||, with the RMS of b raised to `floor` (the RMS of the
    vector quantity a component belongs to: a component that is zero up to
    rounding, like the opening of a fault, is measured against the size of
    the field, as a relative error of the vector field)."""
    n = max(np.linalg.norm(b), floor * np.sqrt(b.size))
    return float(np.linalg.norm(a - b) / n) if n > 0 else float(np.linalg.norm(a - b))


# component files -> magnitude files of the same quantity (fault outputs)
FAMILY = {'su': ('sl.bin',), 'sv': ('svm.bin', 'psv.bin'), 'sa': ('sam.bin',), 't': ('tsm.bin', 'tnm.bin')}


def floor_of(path, f, dtype):
    for pre, mags in FAMILY.items():
        if f.startswith(pre):
            return max([np.sqrt(np.mean(load(path, m, dtype) ** 2)) for m in mags
                        if os.path.exists(os.path.join(path, m))] + [0.0])
    # volume and receiver components ('snap-vx', 'snap-vy', 'snap-vz'): the
    # RMS of the largest component of the same output
    if len(f) > 6 and f[-5] in 'xyz' and f[-6] in 'vua':
        comps = [f[:-5] + c + '.bin' for c in 'xyz']
        return max([np.sqrt(np.mean(load(path, m, dtype) ** 2)) for m in comps
                    if os.path.exists(os.path.join(path, m))] + [0.0])
    return 0.0


def load(path, f, dtype):
    return np.fromfile(os.path.join(path, f), dtype).astype(np.float64)


@pytest.mark.gpu
@pytest.mark.parametrize('name', CASES)
def test_fast_arithmetic_accuracy(name, tmp_path, oracle_bins, gpu_lib):
    prm = sc.CASES[name]()
    # the whole volume at the last step: every interior tile's nodes
    prm.setdefault('vz', []).append(([[], [], [], -1], '=>', 'vol-vz.bin'))
    prm.setdefault('ux', []).append(([[], [], [], -1], '=>', 'vol-ux.bin'))
    inputs = sc.INPUTS.get(name)
    o64, o32, fast, ref = (str(tmp_path / t) for t in ('o64', 'o32', 'fast', 'ref'))
    sc.stage(prm, o64, realsize=8, inputs=inputs)
    for d in (o32, fast, ref):
        sc.stage(prm, d, inputs=inputs)
    # the FP64 build reads its '=<' input files as FP64
    for f in os.listdir(o64):
        p = os.path.join(o64, f)
        if os.path.islink(p):
            x = np.fromfile(p, '<f4').astype('<f8')
            os.unlink(p)
            x.tofile(p)
    sc.run_oracle(o64, oracle_bins['f64'])
    sc.run_oracle(o32, oracle_bins['f32'])
    sc.run_gpu(fast, arithmetic='fast')
    sc.run_gpu(ref, arithmetic='reference')
    files = [f for f in sc.outputs(fast) if not f.startswith('stats-')]
    assert files
    worst, differs = {}, False
    for f in files:
        b = load(o64, f, '<f8')
        a = load(fast, f, '<f4')
        r = load(ref, f, '<f4')
        differs = differs or not np.array_equal(a, r)
        if f == 'trup.bin' or f == 'tarr.bin':
            # rupture / arrest times within one time step where both ruptured
            dt = prm['delta'][3]
            m = (b < 1e8) | (a < 1e8)
            assert np.all(np.abs(a[m] - b[m]) <= dt * (1 + 1e-6)), f
            continue
        fl = floor_of(o64, f, '<f8')
        e_fast = rel_l2(a, b, fl)
        e_o32 = rel_l2(load(o32, f, '<f4'), b, fl)
        worst[f] = (e_fast, e_o32)
        assert e_fast <= TOL_L2, (f, e_fast, e_o32)
        # no worse than the FP32 reference-order solution by more than a
        # small factor (both are FP32 rounding of the same operators)
        assert e_fast <= max(10 * e_o32, 1e-6), (f, e_fast, e_o32)
        assert rel_l2(a, load(o32, f, '<f4'), fl) <= TOL_L2, f
    # the fast kernel ran: its outputs are not the reference-order ones
    assert differs or name in MIXED, 'fast arithmetic gave bit-identical outputs'
    print(name, {f: ('%.2e' % e[0], '%.2e' % e[1]) for f, e in sorted(worst.items())})
    # statistics maxima within the same bound, or no worse than the FP32
    # oracle's by more than a small factor (the fault traction maxima are
    # small differences of large stresses)
    for f in sc.outputs(fast):
        if f.startswith('stats-') and f not in ('stats-efric.bin', 'stats-estrain.bin', 'stats-moment.bin',
                                                'stats-mw.bin'):
            b = load(o64, f, '<f8')
            e_fast, e_o32 = rel_l2(load(fast, f, '<f4'), b), rel_l2(load(o32, f, '<f4'), b)
            assert e_fast <= max(TOL_L2, 10 * e_o32), (f, e_fast, e_o32)


def test_arithmetic_mode_api(tmp_path):
    """Mode values and the Python names; without a device sord_create fails
    before a handle exists, so only the binding is checked here."""
    from coseis_b200 import _lib
    lib = _lib.load()
    assert _lib.ARITHMETIC == {'reference': 0, 'fast': 1}
    assert lib.sord_set_arithmetic(None, 1) == _lib.SORD_E_PARAM
    assert lib.sord_get_arithmetic(None) == _lib.SORD_E_PARAM


@pytest.mark.gpu
def test_arithmetic_mode_switch(tmp_path, gpu_lib):
    from coseis_b200 import _lib
    prm = sc.case_explosion(n=15, nt=4, npml=3)
    d = str(tmp_path)
    sc.stage(prm, d)
    s = _lib.Solver(d, open(os.path.join(d, 'sord.in')).read())
    try:
        assert s.arithmetic() == 'reference'
        s.set_arithmetic('fast')
        assert s.arithmetic() == 'fast'
        s.step(2)
        s.set_arithmetic('reference')
        s.step(2)
        with pytest.raises(_lib.SordError) as e:
            _lib._check(_lib.load().sord_set_arithmetic(s._h, 2), s._h)
        assert e.value.code == _lib.SORD_E_PARAM
    finally:
        s.close()
