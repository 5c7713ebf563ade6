"""Build libsordgpu.so in-tree with nvcc for sm_100a.

-fmad=false keeps every multiply and add separately rounded so that the
kernels follow the FP32 operation order of the Fortran solver exactly;
division and square root stay IEEE (no fast-math).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, 'csrc')
LIB = os.path.join(HERE, 'libsordgpu.so')
SOURCES = ['api.cu', 'kernels.cu', 'fused.cu', 'setup.cu', 'fault.cu', 'fieldio.cu', 'util.cu', 'noalloc.cu', 'adjoint.cu']
HEADERS = ['sord.cuh', 'stencil.cuh', 'inject.cuh', 'timefn.h', 'slab.cuh']
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
FLAGS = [
    '-std=c++17', '-O3', '-lineinfo',
    '-gencode', 'arch=compute_100a,code=sm_100a',
    '-fmad=false', '-prec-div=true', '-prec-sqrt=true',
    '-Xcompiler', '-fPIC,-ffp-contract=off,-fno-fast-math',
    '-shared', '-cudart', 'shared',
]


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(SRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, '..', 'include', 'sordgpu.h'))
    deps.append(__file__)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    if not force and not stale():
        return LIB
    cmd = [NVCC] + FLAGS + list(extra) + [os.path.join(SRC, f) for f in SOURCES] + ['-o', LIB]
    if verbose:
        print(' '.join(cmd))
    subprocess.check_call(cmd)
    return LIB


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose=True,
          extra=['-Xptxas', '-v'] if '--ptxas' in sys.argv else [])
