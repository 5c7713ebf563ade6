"""Ensemble entry point (sord_run_ensemble, include/sordgpu.h).

Several rupture scenarios of the batched-ensemble workload (bench.py
rupture_scenario: seeded friction, normal stress and a random initial shear
stress read from a fault-plane '=<' file) are run concurrently on one GPU,
each on its own handle and stream.  Every output must equal the oracle's
(bit-exact except the FP64 energy sums, as in the parity tests) and the
outputs of the same scenarios run one at a time."""
import ctypes
import os
import sys

import numpy as np
import pytest

import sordcases as sc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

LOOSE = ('stats-efric.bin', 'stats-estrain.bin', 'stats-moment.bin', 'stats-mw.bin')
TOL_LOOSE = 1e-4
SHAPES = [(40, 36, 32), (48, 32, 36), (36, 40, 40), (56, 36, 32), (44, 44, 34)]
NT = 40


def _check(res):
    bad = {f: rel for f, (rel, exact) in res.items() if rel > (TOL_LOOSE if f in LOOSE else 0.0)}
    assert not bad, bad


def test_ensemble_bad_arguments():
    from coseis_b200 import _lib
    lib = _lib.load()
    st = (ctypes.c_int * 1)()
    assert lib.sord_run_ensemble(None, 1, 0, 1, st) == _lib.SORD_E_PARAM
    arr = (ctypes.c_char_p * 1)(b'.')
    assert lib.sord_run_ensemble(arr, 1, 0, 0, st) == _lib.SORD_E_PARAM
    assert lib.sord_run_ensemble(arr, -1, 0, 1, st) == _lib.SORD_E_PARAM
    assert _lib.run_ensemble([], nthreads=4) == []


def test_ensemble_missing_directory(tmp_path):
    """A scenario without sord.in fails before any device work; the others'
    status and the message name the failing directory."""
    from coseis_b200 import _lib
    missing = [str(tmp_path / 'a'), str(tmp_path / 'b')]
    with pytest.raises(_lib.SordError) as e:
        _lib.run_ensemble(missing, nthreads=2)
    assert e.value.code == _lib.SORD_E_IO
    assert 'sord.in' in str(e.value)


@pytest.mark.gpu
def test_ensemble_matches_oracle_and_serial(tmp_path, oracle_bins, gpu_lib):
    import bench
    from coseis_b200 import _lib
    idx = list(range(len(SHAPES)))
    ens, ser, ora = [], [], []
    for i, shp in zip(idx, SHAPES):
        for root, out in (('ens', ens), ('ser', ser), ('ora', ora)):
            out += bench.stage_scenarios([i], str(tmp_path / root), nt=NT, shape=shp)
    for d in ora:
        sc.run_oracle(d, oracle_bins['f32'])
    st = _lib.run_ensemble(ens, nthreads=3)
    assert st == [0] * len(ens)
    for d in ser:
        _lib.run_directory(d)
    for a, b, c in zip(ora, ens, ser):
        assert np.fromfile(os.path.join(a, 'trup.bin'), '<f4').min() < 1e8, 'no rupture'
        _check(sc.compare(a, b))
        _check(sc.compare(c, b))


def test_front_end_run_ensemble_stages_every_case(tmp_path):
    """coseis_b200.sord.run_ensemble stages each parameter dict in its own
    directory before the single library call; without a device that call
    fails with the CUDA error, with the directories staged."""
    from coseis_b200 import _lib, sord
    cases = [sc.case_explosion(n=15, nt=2, npml=3), sc.case_pml(n=14, nt=2)]
    dirs = [str(tmp_path / 'a'), str(tmp_path / 'b')]
    try:
        metas = sord.run_ensemble(cases, dirs, nthreads=2)
    except _lib.SordError as e:
        assert e.code == _lib.SORD_E_CUDA
    else:
        assert len(metas) == 2
    for d in dirs:
        assert os.path.exists(os.path.join(d, 'sord.in'))
        assert os.path.exists(os.path.join(d, 'meta.json'))
    with pytest.raises(ValueError):
        sord.run_ensemble(cases, dirs[:1])
