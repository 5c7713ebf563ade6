"""SORD output files (.bin) to NumPy arrays, as cst/bin2npy.py.

The files are flat, native-endian, j fastest and time slowest; ``load``
returns them indexed [j, k, l, t] (cst/bin2npy.py:10-27).  Metadata
(``dtype``, ``shape`` or per-file ``shapes``, as in a staged ``meta.json``)
come from keyword arguments or from ``.json`` names in the list.
"""
import json
import os
import sys

import numpy as np


def _shape_of(meta, name):
    shapes = meta.get('shapes', {})
    for key in (name, os.path.basename(name)):
        if key in shapes:
            return shapes[key]
    return meta['shape']


def load(filenames, **metadata):
    """Arrays of the .bin files in `filenames`; .json entries update the
    metadata for the files after them."""
    meta = {'dtype': 'f', 'shape': []}
    meta.update(metadata)
    out = []
    for f in filenames:
        if f.endswith('.json'):
            meta.update(json.load(open(f)))
            continue
        x = np.fromfile(f, meta['dtype'])
        shape = _shape_of(meta, f)
        if shape:
            x = x.reshape(shape[::-1]).T
        out.append(x)
    return out


def convert(args, force=False, **metadata):
    """Write name.npy beside each name.bin (cst/bin2npy.py:30-57); '-' reads
    metadata JSON from standard input, '--force' overwrites."""
    meta = {'dtype': 'f', 'shape': []}
    meta.update(metadata)
    for a in args:
        if a == '-':
            meta.update(json.load(sys.stdin))
            continue
        if a == '--force':
            force = True
            continue
        if a.endswith('.json'):
            meta.update(json.load(open(a)))
            continue
        f = (a[:-4] if a.endswith('.bin') else a) + '.npy'
        if not force and os.path.exists(f):
            continue
        x = np.fromfile(a, meta['dtype'])
        shape = _shape_of(meta, a)
        if shape:
            x = x.reshape(shape[::-1]).T
        print('%s: %s %s' % (f, meta['dtype'], x.shape))
        np.save(f, x)


if __name__ == '__main__':
    convert(sys.argv[1:])
