"""The cst.sord-compatible front end (coseis_b200/sord.py) against the
reference front end's output, and its validation errors (CPU only).

tests/golden/frontend.json holds, for three parameter sets, the sord.in
text and metadata produced by the reference's cst/sord.py:prepare and the
sord.in serialisation of cst/sord.py:538-544 (make_golden.py)."""
import copy
import json
import os

import pytest

from coseis_b200 import sord

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
CASES = json.load(open(os.path.join(GOLDEN, 'frontend.json')))


def _stage(args, d):
    cwd = os.getcwd()
    os.chdir(d)
    try:
        return sord.stage(copy.deepcopy(args))
    finally:
        os.chdir(cwd)


@pytest.mark.parametrize('name', sorted(CASES))
def test_sord_in_matches_reference(name, tmp_path):
    c = CASES[name]
    job, meta = _stage(c['args'], str(tmp_path))
    assert open(str(tmp_path / 'sord.in')).read() == c['sord_in']
    for k in ('indices', 'shapes', 'deltas'):
        assert meta[k] == c['meta'][k], k


def test_staged_files(tmp_path):
    c = CASES['explosion']
    job, meta = _stage(c['args'], str(tmp_path))
    for f in ('sord.in', 'parameters.json', 'sord.json', 'meta.json', 'job.json'):
        assert os.path.exists(str(tmp_path / f)), f
    m = json.load(open(str(tmp_path / 'meta.json')))
    assert m['dtype'].endswith('f4')
    assert job['nproc'] == 1


def test_defaults_not_mutated(tmp_path):
    before = copy.deepcopy(sord.parameters)
    _stage({'shape': [11, 11, 11, 2], 'faultnormal': '+z', 'hypocenter': [5.0, 5.0, 0.5],
            'bc1': ['pml', 'pml', 'pml'], 'npml': 2}, str(tmp_path))
    assert sord.parameters == before


def test_expand_slices():
    assert sord.expand_slices([10, 5], []) == [[0, 10, 1], [0, 5, 1]]
    assert sord.expand_slices([10, 5], [[], 3]) == [[0, 10, 1], [3, 4, 1]]
    assert sord.expand_slices([10, 5], [[2, -1, 3], -1]) == [[2, 9, 3], [4, 5, 1]]
    with pytest.raises(Exception):
        sord.expand_slices([10, 5], [1])


@pytest.mark.parametrize('args,msg', [
    ({'shape': [8, 8, 8, 2], 'bc1': ['pml'] * 3, 'bc2': ['pml'] * 3, 'npml': 4}, 'too small for PML'),
    ({'shape': [8, 8, 8, 2], 'vm2': [([], '=', 1.0)]}, 'ouput only'),
    ({'shape': [8, 8, 8, 2], 'mus': [0.6]}, 'only for ruptures'),
    ({'shape': [8, 8, 8, 2], 'vx': [([], '?', 1.0)]}, 'bad i/o operation'),
    ({'shape': [8, 8, 8, 2], 'vx': [([], '=>', 'a.bin'), ([1, 1, 1, []], '=>', 'a.bin')]}, 'duplicate filename'),
])
def test_prepare_errors(args, msg, tmp_path):
    """cst/sord.py:328-329, 391, 396-399: the same exceptions and messages."""
    with pytest.raises(Exception) as e:
        _stage(args, str(tmp_path))
    assert msg in str(e.value)


def test_bad_source_asserts(tmp_path):
    """cst/sord.py:299-300 asserts on source and faultnormal."""
    with pytest.raises(AssertionError):
        _stage({'source': 'dipole'}, str(tmp_path))
    with pytest.raises(AssertionError):
        _stage({'faultnormal': 'z'}, str(tmp_path))


def test_fieldnames_match_reference_tags():
    """Every field of the reference table, with its tags (cst/sord.py:59-163)."""
    for name in ('rho', 'vp', 'vs', 'gam', 'x', 'y', 'z', 'vx', 'ux', 'ax', 'fx', 'pxx', 'mxx', 'wxx',
                 'vm2', 'um2', 'am2', 'wm2', 'mus', 'mud', 'dc', 'tn', 'ts', 'svm', 'sux', 'trup'):
        assert name in sord.fieldnames, name
    assert sord.fieldnames['vx'][0] == 'n~<'
    assert sord.fieldnames['rho'][0] == 'c<'
    assert sord.fieldnames['trup'][0] == 'f~'
    assert sord.boundary_conditions == {'free': 0, 'rigid': 3, '+node': 1, '+cell': 2, '-node': -1,
                                        '-cell': -2, 'pml': 10}
