"""Runs split along l into parts (sord_create_part, coseis_b200.parallel).

The reference splits a run over MPI processes by nproc3 (sord/setup.f90:33-84)
and gives the same outputs for any split (cst/tests/sord_mpi.py runs one
configuration as 1 and as several processes and compares every output).
Here the same configuration runs whole and as 2 or 3 parts:

* CPU: the plane split of setup.f90 (part_planes), the neighbour pairs of an
  exchange, LocalParts and DistExchange (host transport, gloo, world size 2)
  moving halo planes and reducing, and staging with nproc3.
* GPU: the parts (all on device 0, one host thread each) write outputs
  bit-identical to the whole run in reference order (the reference's own
  split test case among them), and in fast arithmetic
  equal to it within 1e-6 relative (bit-identical when the split puts no
  cell into another kernel's arithmetic); the terrain workload with '=<'
  inputs read at per-part offsets; the rejected configurations.
"""
import json
import os
import threading

import numpy as np
import pytest

import sordcases as sc
from coseis_b200 import parallel


def _nl3_restated(nn, p):
    # sord/setup.f90:33-38 line by line: planes per part, then the parts it gives
    nl3 = (nn - 1) // p + 1
    nl3 = max(nl3, 1)
    nproc = (nn - 1) // nl3 + 1
    return nl3, nproc


@pytest.mark.parametrize('nn,p', [(61, 2), (10, 3), (10, 4), (5, 4), (1, 3), (32, 2), (28, 3), (192, 7)])
def test_part_planes(nn, p):
    parts = parallel.part_planes(nn, p)
    nl3, nproc = _nl3_restated(nn, p)
    assert len(parts) == nproc
    covered = [i for a, b in parts for i in range(a, b + 1)]
    assert covered == list(range(1, nn + 1))
    for ip, (a, b) in enumerate(parts):
        # nnoff = nl3 * ip3 - nhalo: the first plane of part ip is nl3 * ip + 1
        assert a == nl3 * ip + 1
        assert b - a + 1 == min(nl3, nn - nl3 * ip)


def test_part_planes_known():
    assert parallel.part_planes(10, 4) == [(1, 3), (4, 6), (7, 9), (10, 10)]
    assert parallel.part_planes(5, 4) == [(1, 2), (3, 4), (5, 5)]


def test_halo_pairs():
    assert parallel.halo_pairs(1) == []
    assert parallel.halo_pairs(3) == [(0, 'hi', 1, 'lo'), (1, 'lo', 0, 'hi'), (1, 'hi', 2, 'lo'), (2, 'lo', 1, 'hi')]


def _buffers(nparts, n):
    """Per part: send_lo, recv_lo, send_hi, recv_hi as numpy arrays (None
    where the part has no neighbour); send planes hold part-specific values."""
    out = []
    for p in range(nparts):
        lo, hi = p > 0, p < nparts - 1
        b = {
            'send_lo': np.full(n, 100.0 * p + 1, np.float32) if lo else None,
            'recv_lo': np.zeros(n, np.float32) if lo else None,
            'send_hi': np.full(n, 100.0 * p + 2, np.float32) if hi else None,
            'recv_hi': np.zeros(n, np.float32) if hi else None,
        }
        if lo:
            b['send_lo'][::7] = -p
        out.append(b)
    return out


def _ptr(a):
    return a.ctypes.data if a is not None else None


def _check_received(bufs):
    for p, b in enumerate(bufs):
        if b['recv_lo'] is not None:
            np.testing.assert_array_equal(b['recv_lo'], bufs[p - 1]['send_hi'])
        if b['recv_hi'] is not None:
            np.testing.assert_array_equal(b['recv_hi'], bufs[p + 1]['send_lo'])


def test_local_parts_host():
    nparts, n = 3, 1000
    bufs = _buffers(nparts, n)
    ex = parallel.LocalParts(nparts, copy=parallel.host_copy, timeout=30.0)
    red = [None] * nparts

    def work(p):
        b = bufs[p]
        rc = ex.halo(p, _ptr(b['send_lo']), _ptr(b['recv_lo']), _ptr(b['send_hi']), _ptr(b['recv_hi']), n)
        assert rc == 0
        vals = [float(p), -float(p), 2.5]
        ex.reduce(p, vals, 3, 0)
        s = [float(p), 1.0]
        ex.reduce(p, s, 2, 1)
        red[p] = (vals, s)
    th = [threading.Thread(target=work, args=(p,)) for p in range(nparts)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    _check_received(bufs)
    for vals, s in red:
        assert vals == [2.0, 0.0, 2.5]
        assert s == [3.0, 3.0]


def test_local_parts_abort():
    """A failing part aborts the exchange: the others leave their next wait."""
    import threading as th_
    ex = parallel.LocalParts(2, copy=parallel.host_copy, timeout=30.0)
    err = []

    def waiter():
        try:
            ex.reduce(0, [1.0], 1, 0)
        except th_.BrokenBarrierError as e:
            err.append(e)
    t = th_.Thread(target=waiter)
    t.start()
    ex.abort()
    t.join(10)
    assert not t.is_alive() and err


def _dist_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    import datetime
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        n = 513
        bufs = _buffers(world, n)
        b = bufs[rank]
        ex = parallel.DistExchange(transport='host', copy=parallel.host_copy)
        ex.halo(rank, _ptr(b['send_lo']), _ptr(b['recv_lo']), _ptr(b['send_hi']), _ptr(b['recv_hi']), n)
        mx = [float(rank), 10.0 - rank]
        ex.reduce(rank, mx, 2, 0)
        sm = [float(rank + 1)]
        ex.reduce(rank, sm, 1, 1)
        got = {k: (None if v is None else v.tolist()) for k, v in b.items() if k.startswith('recv')}
        q.put((rank, got, mx, sm))
    finally:
        dist.destroy_process_group()


def test_dist_exchange_gloo():
    """DistExchange with the host transport over gloo, world size 2."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        port = s.getsockname()[1]
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    procs = [ctx.Process(target=_dist_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r, got, mx, sm = q.get(timeout=120)
        res[r] = (got, mx, sm)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    want = _buffers(2, 513)
    assert res[0][0]['recv_hi'] == want[1]['send_lo'].tolist()
    assert res[1][0]['recv_lo'] == want[0]['send_hi'].tolist()
    assert res[0][0]['recv_lo'] is None and res[1][0]['recv_hi'] is None
    for r in (0, 1):
        assert res[r][1] == [1.0, 10.0]
        assert res[r][2] == [3.0]


def test_stage_nproc3(tmp_path):
    from coseis_b200 import sord
    prm = sc.case_explosion(n=31, nt=4)
    prm['nproc3'] = [1, 1, 3]
    cwd = os.getcwd()
    os.chdir(str(tmp_path))
    try:
        job, meta = sord.stage(prm)
        assert job['nproc'] == 3
        assert json.load(open('sord.json'))['nproc3'] == [1, 1, 3]
        prm['nproc3'] = [2, 1, 1]
        with pytest.raises(Exception, match='split l only'):
            sord.stage(prm)
    finally:
        os.chdir(cwd)


# ---------------------------------------------------------------- GPU


def _run(path, nparts, arithmetic):
    env = {'SORD_FUSED': '1', 'SORD_ARITHMETIC': arithmetic}
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        if nparts == 1:
            from coseis_b200 import _lib
            _lib.run_directory(path)
        else:
            parallel.run_local(path, nparts)
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


def _split_vs_whole(tmp_path, prm, nparts, arithmetic, inputs=None):
    whole, split = str(tmp_path / 'whole'), str(tmp_path / ('split%d' % nparts))
    sc.stage(dict(prm), whole, inputs=inputs)
    p = dict(prm)
    p['nproc3'] = [1, 1, nparts]
    sc.stage(p, split, inputs=inputs)
    assert json.load(open(os.path.join(split, 'sord.json')))['nproc3'] == [1, 1, nparts]
    _run(whole, 1, arithmetic)
    _run(split, nparts, arithmetic)
    return sc.compare(whole, split)


def _explosion():
    prm = sc.case_explosion(n=31, nt=40, npml=6)
    # a snapshot plane across every part and a volume output at the last step
    prm['vz'] = list(prm.get('vz', [])) + [([15, [], [], [None, None, 10]], '=>', 'snapx-vz.bin'),
                                           ([[], [], [], -1], '=>', 'vol-vz.bin')]
    return prm


@pytest.mark.gpu
@pytest.mark.parametrize('nparts', [2, 3])
def test_split_explosion_reference_order(tmp_path, gpu_lib, nparts):
    res = _split_vs_whole(tmp_path, _explosion(), nparts, 'reference')
    bad = {f: r for f, (r, exact) in res.items() if not exact}
    assert res and not bad, bad


@pytest.mark.gpu
@pytest.mark.parametrize('nparts', [2, 3])
def test_split_interior_reference_order(tmp_path, gpu_lib, nparts):
    """Interior tiles and PML slabs in every part (72 x 40 x 28, free top)."""
    res = _split_vs_whole(tmp_path, sc.case_interior(), nparts, 'reference')
    bad = {f: r for f, (r, exact) in res.items() if not exact}
    assert res and not bad, bad


@pytest.mark.gpu
@pytest.mark.parametrize('nparts', [2, 3])
def test_split_interior_fast(tmp_path, gpu_lib, nparts):
    res = _split_vs_whole(tmp_path, sc.case_interior(), nparts, 'fast')
    bad = {f: r for f, (r, exact) in res.items() if r > 1e-6}
    assert res and not bad, bad
    print('fast, %d parts:' % nparts, {f: r for f, (r, exact) in res.items() if not exact})


@pytest.mark.gpu
def test_split_wave_inputs(tmp_path, gpu_lib):
    """The terrain workload: '=<' inputs of rho, vp, vs and z read at each
    part's offset in the shared files; 2 parts of 16 planes."""
    res = _split_vs_whole(tmp_path, sc.case_interior_wave(), 2, 'reference', inputs=sc.interior_wave_inputs)
    bad = {f: r for f, (r, exact) in res.items() if not exact}
    assert res and not bad, bad
    res = _split_vs_whole(tmp_path / 'fast', sc.case_interior_wave(), 2, 'fast', inputs=sc.interior_wave_inputs)
    bad = {f: r for f, (r, exact) in res.items() if r > 1e-6}
    assert res and not bad, bad


@pytest.mark.gpu
def test_split_mpi_case(tmp_path, gpu_lib):
    """cst/tests/sord_mpi.py:12-71 split along l: 5 x 4 x 2 nodes, every
    node and cell field written, a potency point source; two parts of one
    plane each give outputs identical to the whole run."""
    res = _split_vs_whole(tmp_path, sc.case_mpi(), 2, 'reference')
    bad = {f: r for f, (r, exact) in res.items() if not exact}
    assert len(res) > 30 and not bad, bad


@pytest.mark.gpu
def test_split_pml_all_fields(tmp_path, gpu_lib):
    """PML on every face and every node and cell field written each step
    (stress outputs: the separate-kernel step with the force-halo exchange)."""
    res = _split_vs_whole(tmp_path, sc.case_pml(), 2, 'reference')
    bad = {f: r for f, (r, exact) in res.items() if not exact}
    assert len(res) > 30 and not bad, bad


@pytest.mark.gpu
def test_split_rejected(tmp_path, gpu_lib):
    from coseis_b200 import _lib
    # a fault
    prm = sc.case_fault_x()
    prm['nproc3'] = [1, 1, 2]
    d = str(tmp_path / 'fault')
    sc.stage(prm, d)
    with pytest.raises(_lib.SordError, match='fault'):
        parallel.run_local(d, 2)
    # parts thinner than the PML (6 planes + 1): 4 parts of 7, 7, 7 and 4 planes
    prm = sc.case_explosion(n=25, nt=4, npml=6)
    prm['nproc3'] = [1, 1, 4]
    d = str(tmp_path / 'thin')
    sc.stage(prm, d)
    with pytest.raises(_lib.SordError, match='PML'):
        parallel.run_local(d, 4)
    # a whole-run handle on a split sord.in
    prm['nproc3'] = [1, 1, 2]
    d = str(tmp_path / 'whole')
    sc.stage(prm, d)
    with pytest.raises(_lib.SordError, match='sord_create_part'):
        _lib.run_directory(d)
