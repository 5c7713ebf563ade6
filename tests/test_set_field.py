"""sord_set_field (include/sordgpu.h): overwriting state between steps.
Writing back what sord_get_field read leaves every output bit-identical to
an uninterrupted run (the fused step's double buffers are the ones
written); a changed state changes the outputs; moduli written from another
material give that material's run; bad names and sizes, and moduli on a run
with a fault, are SORD_E_PARAM."""
import os

import numpy as np
import pytest

import sordcases as sc


@pytest.mark.gpu
@pytest.mark.parametrize('name', ['interior', 'free'])
def test_set_field_roundtrip_is_transparent(name, tmp_path, gpu_lib):
    from coseis_b200 import _lib
    prm = sc.CASES[name]()
    nt = prm['shape'][3]
    dirs = [str(tmp_path / t) for t in ('whole', 'split', 'changed')]
    for d in dirs:
        sc.stage(prm, d)
    a = _lib.Solver(dirs[0], open(os.path.join(dirs[0], 'sord.in')).read())
    a.run()
    a.close()
    for d, change in ((dirs[1], False), (dirs[2], True)):
        s = _lib.Solver(d, open(os.path.join(d, 'sord.in')).read())
        try:
            s.step(nt // 2)
            for f in ('vx', 'vy', 'vz', 'ux', 'uy', 'uz', 'lam', 'mu', 'yy'):
                x = s.field(f)
                if change and f == 'vx':
                    x = x + np.float32(1e-3) * np.abs(x).max()
                s.set_field(f, x)
                assert np.array_equal(s.field(f), x), f
            s.run()
        finally:
            s.close()
    same = sc.compare(dirs[0], dirs[1])
    assert same and all(exact for rel, exact in same.values()), {f: r for f, (r, e) in same.items() if not e}
    diff = sc.compare(dirs[0], dirs[2])
    assert any(not exact for rel, exact in diff.values())


@pytest.mark.gpu
def test_set_field_errors(tmp_path, gpu_lib):
    from coseis_b200 import _lib
    prm = sc.case_explosion(n=15, nt=2, npml=3)
    d = str(tmp_path)
    sc.stage(prm, d)
    s = _lib.Solver(d, open(os.path.join(d, 'sord.in')).read())
    try:
        x = s.field('vx')
        for bad in (('ax', x), ('vc', x[:-1, :-1, :-1]), ('vx', x[:-1])):
            with pytest.raises(_lib.SordError) as e:
                s.set_field(*bad)
            assert e.value.code == _lib.SORD_E_PARAM
    finally:
        s.close()


@pytest.mark.gpu
def test_set_field_moduli_take_effect(tmp_path, gpu_lib, oracle_bins):
    """Setting lam, mu and yy before the first step to the moduli of a model
    with a different vs gives, bit for bit, the oracle's run of that model
    (vpml fixed, so the PML does not depend on vs)."""
    from coseis_b200 import _lib

    def prm(vs):
        p = sc.case_explosion(n=19, nt=12, npml=4)
        p['vs'] = [vs]
        p['vpml'] = 3000.0
        return p

    other, mine, ref = (str(tmp_path / t) for t in ('other', 'mine', 'ref'))
    sc.stage(prm(3000.0), other)
    sc.stage(prm(3464.0), mine)
    sc.stage(prm(3000.0), ref)
    sc.run_oracle(ref, oracle_bins['f32'])
    a = _lib.Solver(other, open(os.path.join(other, 'sord.in')).read())
    try:
        moduli = {f: a.field(f) for f in ('lam', 'mu', 'yy')}
    finally:
        a.close()
    s = _lib.Solver(mine, open(os.path.join(mine, 'sord.in')).read())
    try:
        assert not np.array_equal(s.field('mu'), moduli['mu'])
        for f, x in moduli.items():
            s.set_field(f, x)
        s.run()
    finally:
        s.close()
    res = sc.compare(ref, mine)
    skip = ('stats-e', 'stats-moment', 'stats-mw')
    bad = {f: r for f, (r, exact) in res.items() if not exact and not f.startswith(skip)}
    assert res and not bad, bad


@pytest.mark.gpu
def test_set_field_moduli_refused_with_fault(tmp_path, gpu_lib):
    from coseis_b200 import _lib
    prm = sc.CASES['rupture']()
    d = str(tmp_path)
    sc.stage(prm, d, inputs=sc.INPUTS.get('rupture'))
    s = _lib.Solver(d, open(os.path.join(d, 'sord.in')).read())
    try:
        s.set_field('vx', s.field('vx'))
        for f in ('lam', 'mu', 'yy'):
            with pytest.raises(_lib.SordError) as e:
                s.set_field(f, s.field(f))
            assert e.value.code == _lib.SORD_E_PARAM
    finally:
        s.close()
