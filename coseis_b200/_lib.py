"""ctypes binding of libsordgpu.so (include/sordgpu.h).

There is no CPU implementation behind this module: if the shared library is
missing or no CUDA device is present, every entry point raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, 'libsordgpu.so')

# every symbol declared in include/sordgpu.h
SYMBOLS = [
    'sord_create', 'sord_step', 'sord_run', 'sord_run_directory',
    'sord_get_field', 'sord_info', 'sord_stats', 'sord_last_step_ms',
    'sord_kernel_launches', 'sord_set_profiling', 'sord_kernel_times',
    'sord_last_error', 'sord_error_string', 'sord_destroy',
    'sord_vector_max_noalloc', 'sord_run_ensemble', 'sord_adjoint_forward', 'sord_adjoint_backward',
    'sord_set_arithmetic', 'sord_get_arithmetic', 'sord_trim_memory', 'sord_adjoint_source_gradients',
    'sord_adjoint_forward_binomial', 'sord_adjoint_binomial_cost',
    'sord_set_field', 'sord_create_part',
]

# callbacks of a partitioned run (include/sordgpu.h: sord_halo_fn, sord_reduce_fn)
HALO_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong)
REDUCE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                             ctypes.c_int)

# return codes (enum in include/sordgpu.h)
SORD_OK, SORD_E_PARAM, SORD_E_CFL, SORD_E_NEGVOL, SORD_E_NANINF = 0, -1, -2, -3, -4
SORD_E_IO, SORD_E_CUDA, SORD_E_STATE, SORD_E_NOMEM = -5, -6, -7, -8

# sord_set_arithmetic modes
ARITHMETIC = {'reference': 0, 'fast': 1}

_lib = None


class SordError(RuntimeError):
    """Error returned by the solver; ``code`` is the SORD_E_* value."""
    def __init__(self, code, msg):
        RuntimeError.__init__(self, msg)
        self.code = code


def load():
    """Load libsordgpu.so (raises OSError if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise OSError('libsordgpu.so not built: run coseis_b200/build.py')
    lib = ctypes.CDLL(LIBPATH)
    P = ctypes.c_void_p
    lib.sord_create.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(P)]
    lib.sord_create.restype = ctypes.c_int
    lib.sord_create_part.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, HALO_FN, REDUCE_FN,
                                     P, ctypes.POINTER(P)]
    lib.sord_create_part.restype = ctypes.c_int
    lib.sord_step.argtypes = [P, ctypes.c_int]
    lib.sord_step.restype = ctypes.c_int
    lib.sord_run.argtypes = [P]
    lib.sord_run.restype = ctypes.c_int
    lib.sord_run_directory.argtypes = [ctypes.c_char_p, ctypes.c_int]
    lib.sord_run_directory.restype = ctypes.c_int
    lib.sord_get_field.argtypes = [P, ctypes.c_char_p, ctypes.POINTER(ctypes.c_float), ctypes.c_size_t]
    lib.sord_get_field.restype = ctypes.c_int
    lib.sord_set_field.argtypes = [P, ctypes.c_char_p, ctypes.POINTER(ctypes.c_float), ctypes.c_size_t]
    lib.sord_set_field.restype = ctypes.c_int
    lib.sord_info.argtypes = [P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    lib.sord_info.restype = ctypes.c_int
    lib.sord_stats.argtypes = [P, ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    lib.sord_stats.restype = ctypes.c_int
    lib.sord_last_step_ms.argtypes = [P]
    lib.sord_last_step_ms.restype = ctypes.c_double
    lib.sord_kernel_launches.argtypes = [P]
    lib.sord_kernel_launches.restype = ctypes.c_longlong
    lib.sord_set_profiling.argtypes = [P, ctypes.c_int]
    lib.sord_set_profiling.restype = ctypes.c_int
    lib.sord_trim_memory.argtypes = [ctypes.c_int]
    lib.sord_trim_memory.restype = ctypes.c_int
    lib.sord_set_arithmetic.argtypes = [P, ctypes.c_int]
    lib.sord_set_arithmetic.restype = ctypes.c_int
    lib.sord_get_arithmetic.argtypes = [P]
    lib.sord_get_arithmetic.restype = ctypes.c_int
    lib.sord_kernel_times.argtypes = [P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]
    lib.sord_kernel_times.restype = ctypes.c_int
    lib.sord_last_error.argtypes = [P]
    lib.sord_last_error.restype = ctypes.c_char_p
    lib.sord_error_string.argtypes = [ctypes.c_int]
    lib.sord_error_string.restype = ctypes.c_char_p
    lib.sord_destroy.argtypes = [P]
    lib.sord_destroy.restype = None
    IP = ctypes.POINTER(ctypes.c_int)
    lib.sord_run_ensemble.argtypes = [ctypes.POINTER(ctypes.c_char_p), ctypes.c_int, ctypes.c_int, ctypes.c_int, IP]
    lib.sord_run_ensemble.restype = ctypes.c_int
    lib.sord_adjoint_forward.argtypes = [P, ctypes.c_int]
    lib.sord_adjoint_forward.restype = ctypes.c_int
    lib.sord_adjoint_forward_binomial.argtypes = [P, ctypes.c_int]
    lib.sord_adjoint_forward_binomial.restype = ctypes.c_int
    lib.sord_adjoint_binomial_cost.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]
    lib.sord_adjoint_binomial_cost.restype = ctypes.c_int
    FP = ctypes.POINTER(ctypes.c_float)
    lib.sord_adjoint_backward.argtypes = [P, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(FP), IP,
                                          FP, FP, FP, FP, ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    lib.sord_adjoint_backward.restype = ctypes.c_int
    DP = ctypes.POINTER(ctypes.c_double)
    lib.sord_adjoint_source_gradients.argtypes = [P, DP, DP, ctypes.c_int]
    lib.sord_adjoint_source_gradients.restype = ctypes.c_int
    lib.sord_vector_max_noalloc.argtypes = [P, P, P, IP, IP, IP, P, P]
    lib.sord_vector_max_noalloc.restype = ctypes.c_int
    _lib = lib
    return lib


def vector_max_noalloc(w0, w1, w2, nm, i1, i2, out, stream=None):
    """Max of w0^2 + w1^2 + w2^2 over [i1, i2] of device fields (raw device
    pointers as ints, j fastest, extents nm) into the device float ``out``,
    without allocating device memory (include/sordgpu.h)."""
    lib = load()
    a = (ctypes.c_int * 3)(*nm)
    b = (ctypes.c_int * 3)(*i1)
    c = (ctypes.c_int * 3)(*i2)
    _check(lib.sord_vector_max_noalloc(w0, w1, w2, a, b, c, out, stream))


def _check(rc, handle=None):
    if rc != 0:
        lib = load()
        msg = lib.sord_last_error(handle).decode(errors='replace')
        name = lib.sord_error_string(rc).decode()
        raise SordError(rc, '%s: %s' % (name, msg))


def run_ensemble(paths, device=0, nthreads=8):
    """Run many staged directories, `nthreads` concurrently (include/sordgpu.h);
    returns the list of per-scenario return codes, raises on the first failure."""
    lib = load()
    n = len(paths)
    arr = (ctypes.c_char_p * max(n, 1))(*[os.fsencode(p) for p in paths])
    st = (ctypes.c_int * max(n, 1))()
    _check(lib.sord_run_ensemble(arr, n, device, nthreads, st))
    return list(st)[:n]


def binomial_cost(nt, snapshots):
    """Forward steps the binomial checkpointing schedule takes for nt steps
    with `snapshots` kept states (the chain of states that the forward run
    keeps included)."""
    n = ctypes.c_longlong(0)
    _check(load().sord_adjoint_binomial_cost(nt, snapshots, ctypes.byref(n)))
    return n.value


def trim_memory(device=0):
    """Wait for the device memory of destroyed handles to go back to the
    driver (it is returned on a helper thread)."""
    _check(load().sord_trim_memory(device))


def run_directory(path, device=0):
    """Run the staged ``sord.in`` in ``path`` (the whole of ``sord.x``)."""
    lib = load()
    _check(lib.sord_run_directory(os.fsencode(path), device))


class Solver(object):
    """One simulation handle: ``Solver(workdir, text)`` runs the setup;
    ``step(n)`` advances n time steps; ``close()`` frees the device memory."""

    def __init__(self, workdir, sord_in_text, device=0, part=None, exchange=None):
        """part, exchange: part `part` of a run split along l by the sord.in
        parameter nproc3 (sord_create_part); `exchange` provides
        halo(part, send_lo, recv_lo, send_hi, recv_hi, n) and
        reduce(part, vals, op) (coseis_b200.parallel)."""
        lib = load()
        h = ctypes.c_void_p()
        if part is None:
            _check(lib.sord_create(os.fsencode(workdir), sord_in_text.encode(), device, ctypes.byref(h)))
        else:
            def halo(ctx, prt, slo, rlo, shi, rhi, n):
                try:
                    return exchange.halo(prt, slo, rlo, shi, rhi, n)
                except Exception:  # noqa: BLE001 -- reported to the solver as a failed exchange
                    import traceback
                    traceback.print_exc()
                    return 1

            def reduce(ctx, prt, vals, n, op):
                try:
                    return exchange.reduce(prt, vals, n, op)
                except Exception:  # noqa: BLE001
                    import traceback
                    traceback.print_exc()
                    return 1
            # the C callbacks must live as long as the handle
            self._cb = (HALO_FN(halo), REDUCE_FN(reduce))
            _check(lib.sord_create_part(os.fsencode(workdir), sord_in_text.encode(), device, part, self._cb[0],
                                        self._cb[1], None, ctypes.byref(h)))
        self._h = h

    def step(self, n=1):
        _check(load().sord_step(self._h, n), self._h)

    def adjoint_forward(self, segment):
        """Whole forward run keeping a checkpoint every `segment` steps."""
        _check(load().sord_adjoint_forward(self._h, segment), self._h)

    def adjoint_forward_binomial(self, snapshots):
        """Whole forward run for a backward pass with binomial checkpointing
        (at most `snapshots` kept states)."""
        _check(load().sord_adjoint_forward_binomial(self._h, snapshots), self._h)

    def adjoint_backward(self, dtraces, nmoment):
        """dtraces: {receiver file name: dL/d(samples)}.  Returns a dict of
        numpy arrays: lam, mu, yy (real cells, shape (nx-1, ny-1, nz-1),
        index [j, k, l]), mr (nodes, (nx, ny, nz)), moment (nmoment), and
        for each moment op position (nmoment, 3; per metre) and delay
        (nmoment; per second of delay of its time function)."""
        import numpy as np
        nn, it, nt = self.info()
        files = list(dtraces)
        arrs = [np.ascontiguousarray(dtraces[f], dtype=np.float32).ravel() for f in files]
        n = len(files)
        FP = ctypes.POINTER(ctypes.c_float)
        fa = (ctypes.c_char_p * max(n, 1))(*[f.encode() for f in files])
        ta = (FP * max(n, 1))(*[a.ctypes.data_as(FP) for a in arrs])
        na = (ctypes.c_int * max(n, 1))(*[a.size for a in arrs])
        nc = [max(x - 1, 1) for x in nn]
        out = {k: np.zeros(nc[::-1], np.float32) for k in ('lam', 'mu', 'yy')}
        out['mr'] = np.zeros(nn[::-1], np.float32)
        gm = np.zeros(max(nmoment, 1), np.float64)
        ptr = lambda a: a.ctypes.data_as(FP)
        _check(load().sord_adjoint_backward(self._h, n, fa, ta, na, ptr(out['lam']), ptr(out['mu']), ptr(out['yy']),
                                            ptr(out['mr']), gm.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                            nmoment), self._h)
        res = {k: v.T for k, v in out.items()}
        res['moment'] = gm[:nmoment]
        gx = np.zeros(3 * max(nmoment, 1), np.float64)
        gt = np.zeros(max(nmoment, 1), np.float64)
        DP = ctypes.POINTER(ctypes.c_double)
        _check(load().sord_adjoint_source_gradients(self._h, gx.ctypes.data_as(DP), gt.ctypes.data_as(DP), nmoment),
               self._h)
        res['position'] = gx[:3 * nmoment].reshape(nmoment, 3)  # dL/dx of each moment op (per metre)
        res['delay'] = gt[:nmoment]                             # dL/dt0 of each moment op (per second)
        return res

    def run(self):
        _check(load().sord_run(self._h), self._h)

    def info(self):
        nn = (ctypes.c_int * 3)()
        it = ctypes.c_int()
        nt = ctypes.c_int()
        _check(load().sord_info(self._h, nn, ctypes.byref(it), ctypes.byref(nt)), self._h)
        return list(nn), it.value, nt.value

    def field(self, name):
        import numpy as np
        nn, _, _ = self.info()
        cell = name in ('lam', 'mu', 'yy', 'vc')
        shape = [n - 1 if cell else n for n in nn]
        out = np.empty(shape[::-1], dtype=np.float32)
        ptr = out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        _check(load().sord_get_field(self._h, name.encode(), ptr, out.size), self._h)
        return out.T

    def set_field(self, name, a):
        """Overwrite field `name` (vx vy vz ux uy uz lam mu yy) with the array
        `a` of shape (nx, ny, nz) (cells: one less per axis), index [j, k, l]."""
        import numpy as np
        a = np.ascontiguousarray(np.asarray(a, dtype=np.float32).T)
        ptr = a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        _check(load().sord_set_field(self._h, name.encode(), ptr, a.size), self._h)

    def stats(self):
        out = (ctypes.c_double * 16)()
        n = load().sord_stats(self._h, out, 16)
        return list(out)[:n]

    def last_step_ms(self):
        return load().sord_last_step_ms(self._h)

    def set_arithmetic(self, mode):
        """'reference' (bit-identical to the reference's FP32 arithmetic) or
        'fast' (fused multiply-adds and fewer operations in the interior step
        kernel; equal in exact arithmetic)."""
        _check(load().sord_set_arithmetic(self._h, ARITHMETIC[mode]), self._h)

    def arithmetic(self):
        return {v: k for k, v in ARITHMETIC.items()}[load().sord_get_arithmetic(self._h)]

    def set_profiling(self, on=True):
        _check(load().sord_set_profiling(self._h, 1 if on else 0), self._h)

    def kernel_times(self):
        """{class: (ms, launches)} for time, stress, accel, mass, fault, io,
        other and step (the fused whole-step kernel)."""
        ms = (ctypes.c_double * 8)()
        cnt = (ctypes.c_longlong * 8)()
        n = load().sord_kernel_times(self._h, ms, cnt, 8)
        if n < 0:
            _check(n, self._h)
        names = ['time', 'stress', 'accel', 'mass', 'fault', 'io', 'other', 'step']
        return {names[i]: (ms[i], cnt[i]) for i in range(n)}

    def kernel_launches(self):
        return load().sord_kernel_launches(self._h)

    def close(self):
        if getattr(self, '_h', None):
            load().sord_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
