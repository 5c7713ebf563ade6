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


def test_fast_brackets_match_reference_forms(tmp_path):
    """The fast-arithmetic interior kernel (sord_set_arithmetic mode 1) uses
    closed-form terrain brackets and the negated gradient brackets as
    divergence brackets: both equal the reference's forms to rounding."""
    exe = str(tmp_path / 'fast')
    subprocess.check_call(['g++', '-std=c++17', '-O2', '-ffp-contract=off', '-o', exe,
                           os.path.join(HERE, 'fast_brackets.cpp')])
    out = subprocess.run([exe, '20000'], capture_output=True, text=True, check=True)
    eterr, ecn = map(float, out.stdout.split())
    # FP32 closed form against the double reference form: a few ulp
    assert eterr < 1e-6, eterr
    # the identity holds in exact arithmetic; double rounding only
    assert ecn < 1e-12, ecn


def test_time_function_rates(tmp_path):
    """The time derivatives behind the adjoint's delay gradient match central
    differences of every smooth source time function."""
    exe = str(tmp_path / 'rate')
    subprocess.check_call(['g++', '-std=c++17', '-O2', '-ffp-contract=off', '-o', exe,
                           os.path.join(HERE, 'timefn_rate.cpp')])
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    assert out[-2] == 'worst' and float(out[-1]) < 1e-6, out
