"""The output loader kept for users of the solver, coseis_b200.bin2npy
(cst/bin2npy.py: .bin files back to arrays with the shapes of meta.json)."""
import json
import os

import numpy as np

from coseis_b200 import bin2npy, sord



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
