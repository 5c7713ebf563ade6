"""The fused step kernel evaluates each cell's divergence brackets once and
shares them among the cell's eight corner nodes; this pins that evaluation
to the per-node diff_cn brackets (sord/diff_cn_op.f90:19-70) bit for bit."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def test_cell_cn_brackets_match_diff_cn(tmp_path):
    exe = str(tmp_path / 'ident')
    subprocess.check_call(['g++', '-std=c++17', '-O2', '-ffp-contract=off', '-o', exe,
                           os.path.join(HERE, 'stencil_identity.cpp')])
    out = subprocess.run([exe, '20000'], capture_output=True, text=True)
    tot, bad = map(int, out.stdout.split())
    assert tot == 20000 * 24
    assert bad == 0, out.stdout
