"""Multi-process host logic of bench.py on CPU (gloo, world size 2).

With N GPUs the bench splits the mesh into N slabs of l planes, one per
rank (strong scaling).  What the ranks share on the host: the scratch
directory that rank 0 creates (outputs of all parts go into shared files),
the timing reduction (the job takes the slowest rank's device time), the
launch count (summed) and the rule that only rank 0 reports."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r'''
import datetime, json, os, sys
sys.path.insert(0, sys.argv[1])
import torch.distributed as dist
import bench
dist.init_process_group('gloo', timeout=datetime.timedelta(seconds=60))
r = dist.get_rank()
ms = [120.0, 180.0][r]
m = bench.reduce_max(dist, ms)
n = bench.reduce_sum(dist, [7, 5][r])
d = bench.shared_workdir(dist, r, 'bench_ranks_')
v = bench.job_rate(1000.0, 10, m)
print(json.dumps({'rank': r, 'max': m, 'sum': n, 'dir': d, 'value': v}))
dist.barrier()
if r == 0:
    os.rmdir(d)
dist.destroy_process_group()
'''


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_gloo_ranks(tmp_path):
    script = str(tmp_path / 'w.py')
    open(script, 'w').write(WORKER)
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE='2', LOCAL_RANK=str(r),
                   MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, script, ROOT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=120)
        assert p.returncode == 0, e[-2000:]
        outs.append(json.loads(o.strip().splitlines()[-1]))
    assert outs[0]['dir'] == outs[1]['dir']
    for o in outs:
        assert o['max'] == 180.0
        assert o['sum'] == 12.0
        # the whole mesh advanced 10 steps in the slowest rank's time
        assert o['value'] == pytest.approx(1000.0 * 10 / 0.180)


def test_split_prm():
    sys.path.insert(0, ROOT)
    import bench
    prm = bench.wave_prm((40, 36, 30), 4, nrec=2)
    assert 'nproc3' not in bench.split_prm(prm, 1)
    p = bench.split_prm(prm, 4)
    assert p['nproc3'] == [1, 1, 4] and 'nproc3' not in prm


def test_reference_arm_other_ranks_do_nothing(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv('RANK', '1')
    monkeypatch.setenv('WORLD_SIZE', '2')

    class A:
        cpu_shape = [8, 8, 8]
        steps = 1
        warmup = 0
    called = []
    monkeypatch.setattr(bench, 'cpu_sample', lambda *a, **k: called.append(1))
    bench.run_reference(A())
    assert not called
    assert capsys.readouterr().out == ''


def test_job_rate_is_whole_mesh():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.job_rate(226492416, 100, 3680.0) == pytest.approx(226492416 * 100 / 3.68)
