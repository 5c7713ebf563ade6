"""The C ABI library on a machine without a GPU: it loads, exports every
symbol include/sordgpu.h declares, and fails loudly (an error code, no CPU
fallback) when there is no device.  No compute is launched by the tests
not marked gpu."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, 'include', 'sordgpu.h')


def header_symbols():
    text = open(HEADER).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(sord_\w+)\s*\(', text)))


@pytest.fixture(scope='module')
def lib():
    from coseis_b200 import build as cb
    cb.build()
    from coseis_b200 import _lib
    return _lib.load()


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_exports_every_header_symbol(lib):
    from coseis_b200 import _lib
    syms = header_symbols()
    assert len(syms) >= 15
    assert sorted(_lib.SYMBOLS) == syms
    for s in syms:
        assert hasattr(lib, s), s
    out = subprocess.run(['nm', '-D', '--defined-only', _lib.LIBPATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r' T (sord_\w+)$', out, flags=re.M))
    assert exported == set(syms)


def test_built_for_sm100a(lib):
    from coseis_b200 import build as cb
    assert 'arch=compute_100a,code=sm_100a' in cb.FLAGS
    assert '-fmad=false' in cb.FLAGS


def test_error_strings(lib):
    names = {0: b'SORD_OK', -1: b'SORD_E_PARAM', -2: b'SORD_E_CFL', -3: b'SORD_E_NEGVOL',
             -4: b'SORD_E_NANINF', -5: b'SORD_E_IO', -6: b'SORD_E_CUDA', -7: b'SORD_E_STATE',
             -8: b'SORD_E_NOMEM'}
    for code, name in names.items():
        assert lib.sord_error_string(code) == name


def test_null_arguments(lib):
    assert lib.sord_step(None, 1) == -1
    assert lib.sord_run(None) == -1
    h = ctypes.c_void_p()
    assert lib.sord_create(None, None, 0, ctypes.byref(h)) == -1


def test_bad_deck_is_param_error(lib, tmp_path):
    h = ctypes.c_void_p()
    rc = lib.sord_create(str(tmp_path).encode(), b'1 2 3\n', 0, ctypes.byref(h))
    assert rc in (-1, -6)
    assert lib.sord_last_error(None)


@pytest.mark.skipif(_has_gpu(), reason='checks the no-device path')
def test_no_device_fails_loudly(tmp_path):
    """Staged deck, no GPU: the solver returns SORD_E_CUDA; nothing runs on the CPU."""
    from coseis_b200 import _lib, sord
    cwd = os.getcwd()
    os.chdir(str(tmp_path))
    try:
        sord.stage({'shape': [9, 9, 9, 2]})
    finally:
        os.chdir(cwd)
    with pytest.raises(_lib.SordError) as e:
        _lib.run_directory(str(tmp_path))
    assert e.value.code == -6
    assert not [f for f in os.listdir(str(tmp_path)) if f.startswith('stats-')]


def test_trim_memory_without_device(lib):
    """sord_trim_memory names the missing device instead of doing anything on the CPU."""
    import torch
    from coseis_b200 import _lib
    if torch.cuda.is_available():
        pytest.skip('a device is present')
    assert lib.sord_trim_memory(0) == _lib.SORD_E_CUDA
    assert b'no CUDA device 0' in lib.sord_last_error(None)
    assert lib.sord_trim_memory(-1) == _lib.SORD_E_CUDA


@pytest.mark.gpu
def test_trim_memory_after_destroy(tmp_path, gpu_lib):
    """Handles on one device one after another: each destroy starts the
    return of the pool's memory on a helper thread; sord_trim_memory and the
    next create wait for it, and the runs are unaffected."""
    from coseis_b200 import _lib, sord
    for i in range(3):
        d = str(tmp_path / str(i))
        os.makedirs(d)
        cwd = os.getcwd()
        os.chdir(d)
        try:
            sord.stage({'shape': [21, 21, 21, 4], 'npml': 4, 'bc1': ['pml'] * 3, 'bc2': ['pml'] * 3,
                        'mxx': [([10, 10, 10, []], '.', 1e16, 'brune', 0.1)],
                        'vx': [([[], 10, [], -1], '=>', 'vx.bin')]})
        finally:
            os.chdir(cwd)
        _lib.run_directory(d)
        if i == 1:
            _lib.trim_memory(0)
        assert np.abs(np.fromfile(os.path.join(d, 'vx.bin'), '<f4')).max() > 0
    _lib.trim_memory(0)


def test_noalloc_argument_checks(lib):
    """sord_vector_max_noalloc validates before touching the device."""
    from coseis_b200 import _lib
    fake = 1 << 20
    with pytest.raises(_lib.SordError) as e:
        _lib.vector_max_noalloc(fake, fake, fake, [4, 4, 4], [0, 1, 1], [4, 4, 4], fake)
    assert e.value.code == -1
    with pytest.raises(_lib.SordError):
        _lib.vector_max_noalloc(fake, fake, fake, [2048, 2048, 1024], [1, 1, 1], [2048, 2048, 1024], fake)
    with pytest.raises(_lib.SordError):
        _lib.vector_max_noalloc(None, fake, fake, [4, 4, 4], [1, 1, 1], [4, 4, 4], fake)


def test_product_never_uses_the_oracle():
    """Nothing in the package imports, loads or runs the oracle."""
    pkg = os.path.join(ROOT, 'coseis_b200')
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith(('.py', '.cu', '.cuh', '.h', '.cpp')):
                text = open(os.path.join(dirpath, f)).read()
                hit = re.search(r'import\s+oracle|from\s+oracle|sord_oracle|oracle/_build|oracle\.build', text)
                assert not hit, os.path.join(dirpath, f)
