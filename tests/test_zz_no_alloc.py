"""The allocation-free statistics reduction (sord_vector_max_noalloc).

Some callers cannot allocate device memory at the point where they need a
reduction (a frozen or exhausted memory pool, an allocation-free section of a
host framework).  For them the library exports one entry point whose scratch
space is a file-scope device array instead of memory it allocates.  This
test drives it through the C ABI on fields produced by a solver run and
checks it against the maxima the solver itself reports through sord_stats
(exact: a maximum of FP32 values has no rounding), on two calls in a row.
It lives in its own file that pytest collects last.
"""
import math

import numpy as np
import pytest

import sordcases as sc

pytestmark = pytest.mark.gpu


def test_vector_max_noalloc_matches_solver_stats(tmp_path, gpu_lib):
    import torch
    from coseis_b200 import _lib

    prm = sc.case_explosion(n=21, nt=10, npml=4)  # statistics every 5 steps
    run = str(tmp_path / 'run')
    sc.stage(prm, run)
    s = _lib.Solver(run, open(run + '/sord.in').read())
    try:
        s.step(5)
        stats = s.stats()
        nn, it, _ = s.info()
        assert it == 5
        dev = {}
        for name in ('vx', 'vy', 'vz', 'ux', 'uy', 'uz'):
            a = np.ascontiguousarray(s.field(name).T)  # (l, k, j): j fastest in memory
            dev[name] = torch.from_numpy(a).cuda()
        out = torch.full((2,), -1.0, dtype=torch.float32, device='cuda')
        torch.cuda.synchronize()
        # two calls in a row: |v|^2 max into out[0], then |u|^2 max into out[1]
        _lib.vector_max_noalloc(dev['vx'].data_ptr(), dev['vy'].data_ptr(), dev['vz'].data_ptr(),
                                nn, [1, 1, 1], nn, out.data_ptr())
        _lib.vector_max_noalloc(dev['ux'].data_ptr(), dev['uy'].data_ptr(), dev['uz'].data_ptr(),
                                nn, [1, 1, 1], nn, out.data_ptr() + 4)
        torch.cuda.synchronize()
        got = out.cpu().numpy().astype(np.float64)
    finally:
        s.close()
    # sord_stats reports sqrt of the FP32 maxima (vmax, umax at index 1, 2)
    assert stats[1] > 0 and stats[2] > 0
    assert math.sqrt(got[0]) == stats[1]
    assert math.sqrt(got[1]) == stats[2]


def _max_sq(f, i1, i2):
    """FP32 max of (x^2 + y^2) + z^2 over the 1-based region, in the
    kernel's order of operations."""
    sl = tuple(slice(a - 1, b) for a, b in zip(i1, i2))
    x, y, z = (np.asarray(c[sl], dtype=np.float32) for c in f)
    return np.float32((x * x + y * y) + z * z).max() if x.size else None


def test_vector_max_noalloc_sub_regions(gpu_lib):
    """Offset sub-regions, a region of two elements and NaN handling,
    exactly against numpy on the same FP32 values."""
    import torch
    from coseis_b200 import _lib

    nn = [13, 11, 9]
    rng = np.random.default_rng(7)
    f = [rng.standard_normal(nn).astype(np.float32) for _ in range(3)]

    def run(fields, i1, i2):
        dev = [torch.from_numpy(np.ascontiguousarray(a.T)).cuda() for a in fields]
        out = torch.full((1,), -1.0, dtype=torch.float32, device='cuda')
        _lib.vector_max_noalloc(dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(), nn, i1, i2,
                                out.data_ptr())
        torch.cuda.synchronize()
        return np.float32(out.cpu().numpy()[0])

    for i1, i2 in (([2, 3, 4], [nn[0] - 1, nn[1] - 2, nn[2] - 1]), ([5, 7, 3], [5, 7, 4]),
                   ([1, 1, 1], [1, 1, 1]), ([13, 2, 1], [13, 11, 9])):
        got = run(f, i1, i2)
        assert got == _max_sq(f, i1, i2), (i1, i2)
    # a NaN inside the region wins; one outside it is not read
    g = [a.copy() for a in f]
    g[1][6, 8, 4] = np.nan
    assert np.isnan(run(g, [2, 3, 4], [12, 9, 8]))
    assert run(g, [2, 3, 6], [12, 9, 8]) == _max_sq(g, [2, 3, 6], [12, 9, 8])


def test_vector_max_noalloc_rejects_bad_regions(gpu_lib):
    import torch
    from coseis_b200 import _lib

    w = torch.zeros(8, dtype=torch.float32, device='cuda')
    out = torch.zeros(1, dtype=torch.float32, device='cuda')
    p = w.data_ptr()
    with pytest.raises(_lib.SordError) as e:
        _lib.vector_max_noalloc(p, p, p, [2, 2, 2], [1, 1, 1], [3, 2, 2], out.data_ptr())
    assert e.value.code == -1
    with pytest.raises(_lib.SordError):
        _lib.vector_max_noalloc(p, p, p, [2048, 2048, 1024], [1, 1, 1], [2048, 2048, 1024], out.data_ptr())
