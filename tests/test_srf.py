"""SRF utilities (coseis_b200/srf.py) against the reference (tests/golden/
srf.json, made by make_golden.py from cst/srf.py and cst/coord.py), and a
finite-source run driven by write_sord on the CUDA solver against the
oracle."""
import io
import json
import os

import numpy as np
import pytest

import sordcases as sc
from coseis_b200 import srf

GOLDEN = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'srf.json')))


def _read():
    fh = io.StringIO(GOLDEN['text'])
    fh.name = 'synthetic.srf'
    return srf.read(fh)


def test_read_matches_reference():
    meta, data = _read()
    for k in ('version', 'plane', 'nsource', 'nsource_nonzero', 'hypocenter', 'area', 'potency', 'displacement'):
        assert meta[k] == GOLDEN['meta'][k], k
    for k, v in GOLDEN['data'].items():
        a = np.asarray(data[k]).T.ravel()
        assert np.array_equal(a, np.asarray(v, dtype=a.dtype)), k
    assert np.asarray(data['lon']).shape == (3, 2)  # one plane: the plane grid, [j, k]
    for c in range(3):
        assert np.array_equal(data['sv%d' % (c + 1)], np.asarray(GOLDEN['sv'][c], 'f'))


def test_write_matches_reference():
    out = io.StringIO()
    srf.write(out, _read())
    assert out.getvalue() == GOLDEN['written']
    back = io.StringIO(out.getvalue())
    back.name = 'rewritten.srf'
    m2, d2 = srf.read(back)
    m1, d1 = _read()
    # the text keeps about 7 significant digits
    for k in d1:
        assert np.allclose(d1[k], d2[k], rtol=1e-6, atol=0), k


def test_geometry_matches_reference():
    d = GOLDEN['data']
    R = srf.slip_vectors(np.asarray(d['stk']), d['dip'], d['rake'])
    assert np.array_equal(R, np.asarray(GOLDEN['slip_vectors']))
    pot = [srf.potency_tensor(R[2], R[0]), srf.potency_tensor(R[2], R[1]), srf.potency_tensor(R[2], R[2])]
    flat = [np.asarray(a) for p in pot for part in p for a in [part]]
    ref = [np.asarray(a) for a in GOLDEN['potency']]
    assert len(flat) == len(ref)
    for a, b in zip(flat, ref):
        assert np.array_equal(a, b)


def test_rotation_of_a_plain_projection():
    """A projection that is a scaled, rotated copy of lon/lat gives that
    rotation back (cst/coord.py:205-230)."""
    ang = np.radians(20.0)

    def proj(lon, lat):
        x = np.asarray(lon) * 1e5
        y = np.asarray(lat) * 1e5
        return np.cos(ang) * x + np.sin(ang) * y, -np.sin(ang) * x + np.cos(ang) * y
    mat, theta = srf.rotation(np.array([0.0]), np.array([0.0]), proj)
    assert abs(theta[0] - 20.0) < 1e-6


def synthetic_rupture(shape=(20, 18, 16), dx=100.0, seed=5):
    """A small SRF-like rupture (meta, data) with positions in metres inside
    a mesh of `shape` nodes (no projection): 4 points, mixed slip components."""
    rng = np.random.default_rng(seed)
    n = 4
    data = {
        'lon': (rng.uniform(6, shape[0] - 7, n) * dx).astype('f'),
        'lat': (rng.uniform(6, shape[1] - 7, n) * dx).astype('f'),
        'dep': (rng.uniform(6, shape[2] - 7, n) * dx).astype('f'),
        'stk': rng.uniform(0, 360, n).astype('f'), 'dip': rng.uniform(30, 90, n).astype('f'),
        'rake': rng.uniform(-180, 180, n).astype('f'), 'area': np.full(n, 1e4, 'f'),
        't0': rng.uniform(0.0, 0.05, n).astype('f'), 'dt': np.full(n, 0.004, 'f'),
        'slip1': np.ones(n, 'f'), 'slip2': np.ones(n, 'f'), 'slip3': np.zeros(n, 'f'),
        'nt1': np.array([5, 3, 0, 4], 'i'), 'nt2': np.array([0, 2, 4, 0], 'i'), 'nt3': np.zeros(n, 'i'),
    }
    for c in (1, 2, 3):
        m = int(data['nt%d' % c].sum())
        data['sv%d' % c] = rng.uniform(0.1, 1.0, m).astype('f')
    return {'version': '1.0', 'nsource': n}, data


def test_write_sord_files(tmp_path):
    meta, data = synthetic_rupture()
    n = srf.write_sord(str(tmp_path / 'source-'), (meta, data), delta=(100.0, 100.0, 100.0))
    sel = [data['nt%d' % c] > 0 for c in (1, 2, 3)]
    assert n == sum(int(s.sum()) for s in sel)
    nt = np.fromfile(str(tmp_path / 'source-nt.bin'), 'i4')
    assert nt.tolist() == [int(x) for s, c in zip(sel, (1, 2, 3)) for x in data['nt%d' % c][s]]
    for name in ('dt', 't0', 'xi1', 'xi2', 'xi3', 'w11', 'w22', 'w33', 'w23', 'w31', 'w12'):
        assert np.fromfile(str(tmp_path / ('source-%s.bin' % name)), 'f4').size == n, name
    xi1 = np.fromfile(str(tmp_path / 'source-xi1.bin'), 'f4')
    assert np.array_equal(xi1[:sel[0].sum()], (data['lon'][sel[0]].astype(np.float64) / 100.0).astype('f4'))
    R = srf.slip_vectors(data['stk'], data['dip'], data['rake'])
    w22 = np.fromfile(str(tmp_path / 'source-w22.bin'), 'f4')
    ref = np.concatenate([(data['area'] * R[2][1] * R[c][1])[s] for c, s in zip((0, 1, 2), sel)])
    assert np.allclose(w22, ref, rtol=1e-6)
    hist = np.fromfile(str(tmp_path / 'source-history.bin'), 'f4')
    assert hist.size == int(nt.sum())
    first = data['sv1'][:5].cumsum() * data['dt'][0]
    assert np.allclose(hist[:5], first, rtol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize('fused', [True, False], ids=['fused', 'staged'])
def test_srf_finite_source_parity(fused, tmp_path, oracle_bins, gpu_lib):
    """A potency finite source from write_sord (sord/kinematic_source.f90)
    through both solvers: every output bit for bit."""
    shape = (20, 18, 16)
    prm = {
        'delta': [100.0, 100.0, 100.0, 0.004], 'shape': list(shape) + [30],
        'bc1': ['pml'] * 3, 'bc2': ['pml'] * 3, 'npml': 4, 'source': 'potency', 'itstats': 5, 'itio': 10,
    }
    sc.all_outputs(prm, fields='n', step=5)
    a, b = str(tmp_path / 'oracle'), str(tmp_path / 'gpu')

    def inputs(path):
        os.makedirs(path, exist_ok=True)
        prm['nsource'] = srf.write_sord(os.path.join(path, 'source-'), synthetic_rupture(shape),
                                        delta=(100.0, 100.0, 100.0))
    inputs(a)
    sc.stage(prm, a)
    inputs(b)
    sc.stage(prm, b)
    sc.run_oracle(a, oracle_bins['f32'])
    sc.run_gpu(b, fused=fused)
    res = sc.compare(a, b)
    assert res
    assert np.abs(np.fromfile(os.path.join(a, 'vx.bin'), '<f4')).max() > 0
    bad = {f: r for f, (r, exact) in res.items() if r > 0.0}
    assert not bad, bad
