"""The wave226 workload at its full size (768 x 768 x 384 nodes, terrain
mesh, layered random medium read from '=<' files, moment-tensor source, 64
surface receivers) for its full 1000 steps: fast arithmetic against
reference order (bit-identical to the FP32 oracle on every smaller case).

The FP64 oracle cannot run this size in a test (about 5 hours on 16
threads), so this bounds how far the fast-arithmetic kernels drift from the
reference's own FP32 operation order over a long run on the curvilinear
mesh: relative L2 of the final velocity and displacement volumes and of
the receiver traces, each at most 1e-4.  Both runs hold about 23 GB of
device memory, one after the other; the compared volumes about 11 GB of
host memory.
"""
import glob
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NT = 1000


def _rel(a, b):
    num = sum(float(np.sum((x.astype(np.float64) - y.astype(np.float64)) ** 2)) for x, y in zip(a, b))
    den = sum(float(np.sum(y.astype(np.float64) ** 2)) for y in b)
    return float(np.sqrt(num / den)) if den > 0 else float(np.sqrt(num))


def _run(work, inputs, mode):
    import bench
    from coseis_b200 import _lib
    old = os.environ.get('SORD_ARITHMETIC')
    os.environ['SORD_ARITHMETIC'] = mode
    try:
        text = bench.stage_in(bench.wave_prm(bench.SHAPE, NT), work, inputs)
        s = _lib.Solver(work, text)
        try:
            s.set_arithmetic(mode)
            s.step(NT)
            out = {q: [s.field(q + c) for c in 'xyz'] for q in 'vu'}
        finally:
            s.close()
    finally:
        if old is None:
            del os.environ['SORD_ARITHMETIC']
        else:
            os.environ['SORD_ARITHMETIC'] = old
    return out


def test_wave226_full_fast_vs_reference_order(tmp_path, gpu_lib):
    import bench
    inputs = str(tmp_path / 'inputs')
    bench.make_inputs(bench.SHAPE, inputs)
    ref = _run(str(tmp_path / 'ref'), inputs, 'reference')
    fast = _run(str(tmp_path / 'fast'), inputs, 'fast')
    errs = {q: _rel(fast[q], ref[q]) for q in 'vu'}
    del ref, fast
    recs = sorted(os.path.basename(f) for f in glob.glob(str(tmp_path / 'ref' / 'r*-v*.bin')))
    assert len(recs) == 192
    a = [np.fromfile(str(tmp_path / 'fast' / f), '<f4') for f in recs]
    b = [np.fromfile(str(tmp_path / 'ref' / f), '<f4') for f in recs]
    assert all(x.size == NT for x in b)
    errs['receivers'] = _rel(a, b)
    print('wave226 768x768x384 x %d steps, fast vs reference order:' % NT, errs)
    assert max(errs.values()) <= 1e-4, errs
