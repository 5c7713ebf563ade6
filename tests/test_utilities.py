"""Host utilities of the cst package kept for users of the solver:
coseis_b200.dsp (cst/dsp.py), coseis_b200.kostrov (cst/kostrov.py) and
coseis_b200.bin2npy (cst/bin2npy.py), against the reference's outputs
(tests/golden/dsp.json, kostrov.json; make_golden.py)."""
import json
import os

import numpy as np
import pytest

from coseis_b200 import bin2npy, dsp, kostrov, sord

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
DSP = json.load(open(os.path.join(GOLDEN, 'dsp.json')))
KOSTROV = json.load(open(os.path.join(GOLDEN, 'kostrov.json')))


@pytest.mark.parametrize('pulse', sorted(DSP['time_function']))
def test_time_function_matches_reference(pulse):
    f = dsp.time_function(pulse, np.asarray(DSP['t']), DSP['tau'])
    assert np.array_equal(f, np.asarray(DSP['time_function'][pulse]))


def test_filters_match_reference():
    x = np.asarray(DSP['x'])
    cases = {'low2': (5.0, 'lowpass', 2, 0), 'high4': (3.0, 'highpass', 4, 1),
             'band': ((2.0, 8.0), 'bandpass', 2, -1), 'hann': (4.0, 'hann', 2, 1)}
    for name, (fc, bt, order, rep) in cases.items():
        y = dsp.filter(x, 0.01, fc, bt, order, rep)
        assert np.allclose(y, DSP['filter'][name], rtol=0, atol=1e-12), name
    assert np.allclose(dsp.brune2gauss(x, 0.01, 0.05), DSP['brune2gauss'], rtol=0, atol=1e-12)


def test_kostrov_matches_reference():
    k = KOSTROV
    c = kostrov.cee(k['vrup'] / k['vp'], k['vrup'] / k['vs'])
    assert abs(float(c) - k['C']) <= 1e-12 * abs(k['C'])
    v = kostrov.slip_rate(k['rho'], k['vp'], k['vs'], k['vrup'], k['dtau'], k['r'], k['t'])
    assert abs(float(v) - k['slip_rate']) <= 1e-12 * abs(k['slip_rate'])


def test_bin2npy_load_with_staged_meta(tmp_path):
    """Arrays come back indexed [j, k, l, t] with the shapes of meta.json."""
    cwd = os.getcwd()
    os.chdir(str(tmp_path))
    try:
        sord.stage({'shape': [6, 5, 4, 3], 'vx': [([], '=>', 'vx.bin')], 'rho': [([], '=>', 'rho.bin')]})
    finally:
        os.chdir(cwd)
    meta = json.load(open(str(tmp_path / 'meta.json')))
    shp = meta['shapes']['vx.bin']
    a = np.arange(np.prod(shp), dtype='f').reshape(shp[::-1]).T
    a.T.tofile(str(tmp_path / 'vx.bin'))
    (x,) = bin2npy.load([str(tmp_path / 'meta.json'), str(tmp_path / 'vx.bin')])
    assert x.shape == tuple(shp) and np.array_equal(x, a)
    bin2npy.convert([str(tmp_path / 'meta.json'), str(tmp_path / 'vx.bin')])
    assert np.array_equal(np.load(str(tmp_path / 'vx.npy')), a)
