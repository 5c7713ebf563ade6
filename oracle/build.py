"""Build recipe for the oracle (test infrastructure; see sord_oracle.cpp).

Produces oracle/_build/sord_oracle_f32 and sord_oracle_f64 with g++,
OpenMP, and -ffp-contract=off so that no multiply-add is contracted.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, '_build')


def build(force=False, quiet=True):
    os.makedirs(OUT, exist_ok=True)
    src = os.path.join(HERE, 'sord_oracle.cpp')
    outs = {}
    for tag, real in (('f32', 'float'), ('f64', 'double')):
        exe = os.path.join(OUT, 'sord_oracle_' + tag)
        outs[tag] = exe
        if not force and os.path.exists(exe) and os.path.getmtime(exe) >= os.path.getmtime(src):
            continue
        cmd = ['g++', '-std=c++17', '-O2', '-fopenmp', '-ffp-contract=off',
               '-fno-fast-math', '-DSORD_REAL=' + real, src, '-o', exe]
        if not quiet:
            print(' '.join(cmd))
        subprocess.check_call(cmd)
    return outs


if __name__ == '__main__':
    build(force='--force' in sys.argv, quiet=False)
