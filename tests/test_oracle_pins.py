"""Pins of the oracle (the C++ restatement of sord/*.f90) against the
reference's own known answers, on the CPU.

The reference ships no solver output, so the oracle is pinned through the
physics checks the reference itself uses, with the analytic values computed
by the reference's own code into tests/golden/ (make_golden.py):

* the Kostrov crack test, cst/tests/sord_kostrov.py:12-76, at the
  reference's resolution and refined twofold (where it meets the
  reference's 1.5 % per receiver), and with the reference's own fault
  geometry (which fails it);
* the explosion point source of scripts/Explosion-sim.py against the analytic
  solution of scripts/Explosion-plot.py:41-58;
* the decomposition-identity tests cst/tests/sord_mpi.py:49-71 and
  sord_pml.py:49-71 (a run split across workers must give identical
  output), here across OpenMP thread counts;
* FP32 against the FP64 build of the same restatement.
"""
import json
import math
import os
import subprocess

import numpy as np
import pytest

import sordcases as sc

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def _golden(name):
    return json.load(open(os.path.join(GOLDEN, name)))


def kostrov_prm(refine=1):
    """cst/tests/sord_kostrov.py:12-49 (serial).  refine > 1 divides dx and
    dt by it and keeps the physical problem: the same domain, PML thickness,
    fault plane half a cell below the last node, and receivers 2 km from the
    hypocentre."""
    g = _golden('kostrov.json')
    nx, ny, nz, nt = g['shape']
    f = refine
    prm = {
        'delta': [g['dx'] / f, g['dx'] / f, g['dx'] / f, g['dt'] / f],
        'shape': [(nx - 1) * f + 1, (ny - 1) * f + 1, (nz - 2) * f + 2, nt * f],
        'rho': [g['rho']], 'vp': [g['vp']], 'vs': [g['vs']], 'gam': 1.0, 'hourglass': [1.0, 1.0],
        'bc1': ['pml', 'pml', 'pml'], 'bc2': ['-node', '+node', '-cell'], 'npml': 10 * f,
        'faultnormal': '+z', 'hypocenter': [-1.0, -1.0, -1.5], 'vrup': g['vrup'],
        'rcrit': 1e9, 'trelax': 0.0, 'mud': 1.0, 'mus': 1e9, 'dc': 1e9,
        'tn': -90e6, 'ts': -90e6 - g['dtau'],
        'svm': [([-1, -1 - 20 * f, []], '=>', 'p20a.bin'), ([-1 - 12 * f, -1 - 16 * f, []], '=>', 'p20b.bin'),
                ([-1 - 16 * f, -1 - 12 * f, []], '=>', 'p20c.bin'), ([-1 - 20 * f, -1, []], '=>', 'p20d.bin')],
    }
    return prm, g


def kostrov_errors(d, g, nt, dtype='<f4'):
    """Relative error of the final slip rate at the four receivers
    (cst/tests/sord_kostrov.py:70-76)."""
    errs = []
    for p in 'abcd':
        v = np.fromfile(os.path.join(d, 'p20%s.bin' % p), dtype)
        assert v.shape == (nt,)
        errs.append((g['slip_rate'] - float(v[-1])) / g['slip_rate'])
    return errs


def run_kostrov(tmp_path, exe, refine=1, extra=()):
    prm, g = kostrov_prm(refine)
    d = str(tmp_path / ('k%d' % refine))
    sc.stage(prm, d)
    r = subprocess.run([exe, '--threads', str(os.cpu_count() or 1)] + list(extra), cwd=d,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return kostrov_errors(d, g, prm['shape'][3])


def test_kostrov_reference_geometry_fails(tmp_path, oracle_bins):
    """The reference as shipped computes fault normals and the hypocentral
    radius from w1 (dynamic_rupture.f90:120,186,197-199), which holds cell
    centres with a zeroed halo at that point (grid_generation.f90:127-132).
    The Kostrov hypocentre sits on the last node row, so its interpolated
    position is the origin (the far PML corner): the forced rupture starts
    there and never reaches the receivers within the run.  The oracle's
    --w1-geometry switch reproduces that; the slip rate stays near zero and
    the reference's own 1.5 % assertion fails at every receiver (measured
    error 0.9999-1.0000).  The oracle therefore uses the node coordinates."""
    errs = run_kostrov(tmp_path, oracle_bins['f32'], extra=['--w1-geometry'])
    assert min(abs(e) for e in errs) > 0.99, errs


def test_kostrov_slip_rate(tmp_path, oracle_bins):
    """Final slip rate 2 km from the hypocentre vs Kostrov's solution at the
    reference test's resolution (dx 100 m): 1.2, 2.1, 1.5 and 1.7 % on the
    four receivers, against the reference test's 1.5 %.  The error is
    discretisation error: at dx 50 m (test_kostrov_slip_rate_refined) every
    receiver is within 1.5 %.  Bound here 2.5 %."""
    errs = run_kostrov(tmp_path, oracle_bins['f32'])
    assert max(abs(e) for e in errs) < 0.025, errs
    assert min(abs(e) for e in errs) < 0.015, errs


def test_kostrov_slip_rate_refined(tmp_path, oracle_bins):
    """The same crack at dx = 50 m (twice the resolution, 101 x 101 x 46
    nodes, 400 steps): every receiver within the reference test's own bound
    of 1.5 % (cst/tests/sord_kostrov.py:76); measured 1.1, 1.25, 1.3 and
    0.85 %, each below its dx = 100 m error."""
    errs = run_kostrov(tmp_path, oracle_bins['f32'], refine=2)
    assert max(abs(e) for e in errs) < 0.015, errs


@pytest.mark.gpu
def test_kostrov_slip_rate_gpu_refined(tmp_path, gpu_lib):
    """The CUDA solver (reference order, bit-identical to the oracle) on the
    crack at dx = 50 m and 25 m (201 x 201 x 90 nodes, 800 steps, too long
    for the CPU suite): every receiver within 1.5 % at both resolutions, and
    the largest error smaller at 25 m than at 50 m."""
    worst = []
    for refine in (2, 4):
        prm, g = kostrov_prm(refine)
        d = str(tmp_path / ('g%d' % refine))
        sc.stage(prm, d)
        sc.run_gpu(d)
        errs = kostrov_errors(d, g, prm['shape'][3])
        print('Kostrov dx = %g m: %s' % (g['dx'] / refine, ', '.join('%.4f' % e for e in errs)))
        assert max(abs(e) for e in errs) < 0.015, (refine, errs)
        worst.append(max(abs(e) for e in errs))
    assert worst[1] < worst[0], worst


def lowpass2(x, dt, cutoff):
    """Second-order Butterworth lowpass applied twice, causal
    (cst/dsp.py:130-141 with order 2, repeat 1)."""
    import scipy.signal
    b, a = scipy.signal.butter(2, 2.0 * dt * cutoff, 'lowpass')
    return scipy.signal.lfilter(b, a, scipy.signal.lfilter(b, a, x))


def test_filter_restatement():
    g = _golden('explosion.json')
    y = lowpass2(np.array(g['filter_probe']), g['dt'], g['cutoff'])
    np.testing.assert_allclose(y, g['filter_probe_out'], rtol=0, atol=1e-12)
    y = lowpass2(np.array(g['analytic']), g['dt'], g['cutoff'])
    np.testing.assert_allclose(y, g['analytic_filtered'], rtol=0, atol=1e-20)


def explosion_prm(g, realsize=4):
    """scripts/Explosion-sim.py (dx 200 m, '+node' registration) with receiver
    p2.  A '.' op adds its value to the strain array (input_output.f90:182-190)
    where a physical potency is subtracted (kinematic_source.f90:110-113), so
    an explosion of unit potency is the value -1; its moment history is the
    integral of the Brune pulse, as the analytic solution assumes."""
    nx, nt, dx, dt, reg = g['nx'], g['nt'], g['dx'], g['dt'], g['reg']
    prm = {'shape': [nx, nx, nx, nt], 'delta': [dx, dx, dx, dt], 'bc1': [g['bc']] * 3, 'bc2': ['pml'] * 3,
           'hourglass': [1.0, 1.0], 'rho': [g['rho']], 'vp': [g['vp']], 'vs': [g['vs']], 'gam': [0.0]}
    for f in ('pxx', 'pyy', 'pzz'):
        prm[f] = [([reg, reg, reg, []], '.', -1.0, 'integral_brune', g['tau'])]
    x, y, z = g['receiver']
    for f in ('vx', 'vy', 'vz'):
        prm[f] = [([reg + x / dx, reg + y / dx, reg + z / dx, []], '.>', 'p2-%s.bin' % f)]
    return prm


def _radial(d, g, dtype):
    v = np.array([np.fromfile(os.path.join(d, 'p2-v%s.bin' % c), dtype).astype(np.float64) for c in 'xyz'])
    n = np.array(g['receiver']) / g['r']
    return n @ v


def test_explosion_analytic(tmp_path, oracle_bins):
    """Radial velocity at 5 km vs the analytic explosion after the lowpass of
    scripts/Explosion-plot.py.  The solver's velocity sample n follows the
    source evaluated at step n by one step, so the trace is compared one
    sample earlier; misfit bound 8 % (measured 5.5 %), peak within 3 %."""
    g = _golden('explosion.json')
    d = str(tmp_path / 'e')
    sc.stage(explosion_prm(g), d)
    sc.run_oracle(d, oracle_bins['f32'], threads=os.cpu_count() or 1)
    vr = lowpass2(_radial(d, g, '<f4'), g['dt'], g['cutoff'])
    ref = np.array(g['analytic_filtered'])
    assert vr.shape == ref.shape
    sim = vr[1:]
    ana = ref[:-1]
    mis = np.linalg.norm(sim - ana) / np.linalg.norm(ana)
    assert mis < 0.08, mis
    assert abs(sim.max() / ana.max() - 1.0) < 0.03
    assert abs(int(np.argmax(sim)) - int(np.argmax(ana))) <= 1


def test_fp32_vs_fp64(tmp_path, oracle_bins):
    """The FP32 restatement against its FP64 build on the explosion case."""
    g = _golden('explosion.json')
    a, b = str(tmp_path / 'f32'), str(tmp_path / 'f64')
    sc.stage(explosion_prm(g), a)
    sc.stage(explosion_prm(g), b, realsize=8)
    sc.run_oracle(a, oracle_bins['f32'], threads=os.cpu_count() or 1)
    sc.run_oracle(b, oracle_bins['f64'], threads=os.cpu_count() or 1)
    x, y = _radial(a, g, '<f4'), _radial(b, g, '<f8')
    rel = np.linalg.norm(x - y) / np.linalg.norm(y)
    assert rel < 1e-4, rel


@pytest.mark.parametrize('name', ['pml', 'curvilinear', 'rupture'])
def test_thread_count_identity(name, tmp_path, oracle_bins):
    """sord_mpi.py / sord_pml.py: splitting the work gives identical output."""
    prm = sc.CASES[name]()
    inputs = sc.INPUTS.get(name)
    a, b = str(tmp_path / 't1'), str(tmp_path / 't4')
    sc.stage(prm, a, inputs=inputs)
    sc.stage(prm, b, inputs=inputs)
    sc.run_oracle(a, oracle_bins['f32'], threads=1)
    sc.run_oracle(b, oracle_bins['f32'], threads=4)
    res = sc.compare(a, b)
    assert res
    bad = {f: r for f, r in res.items() if not r[1] and not f.startswith('stats-e') and f not in
           ('stats-moment.bin', 'stats-mw.bin')}
    assert not bad, bad
