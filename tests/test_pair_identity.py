"""Packed f32x2 evaluation (two IEEE-rounded lanes per instruction) of the
stencil templates is bit-identical to the scalar evaluation (GPU)."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')


@pytest.mark.gpu
def test_f32x2_templates_bit_identical(tmp_path):
    exe = str(tmp_path / 'pair')
    subprocess.check_call([NVCC, '-std=c++17', '-O3', '-gencode', 'arch=compute_100a,code=sm_100a', '-fmad=false',
                           '-prec-div=true', '-prec-sqrt=true', '-o', exe, os.path.join(HERE, 'pair_identity.cu')])
    out = subprocess.run([exe, '200000'], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    n, bad, nc, cn, st, hg = map(int, out.stdout.split())
    assert n == 200000
    assert bad == 0, 'mismatches: diff_nc %d, diff_cn %d, stencil %d, hourglass %d' % (nc, cn, st, hg)
