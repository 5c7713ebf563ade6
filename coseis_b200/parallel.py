"""Runs split along l into parts, one handle per part (sord_create_part).

The reference decomposes a run over MPI processes by the sord.in parameter
nproc3 (sord/setup.f90:33-84, process_mpi.f90): every process holds its
block with one halo plane per side, swaps halos at setup and, every step,
the force halo (acceleration.f90:232), and reduces statistics.  Here a run
staged with nproc3 = [1, 1, P] is split into P slabs of l planes; each part
is a handle of the CUDA solver and the communication goes through an
exchange object with two methods:

  halo(part, send_lo, recv_lo, send_hi, recv_hi, n)  fill the part's halo
      planes: recv_lo from part - 1's send_hi, recv_hi from part + 1's
      send_lo (n floats of device memory each, 0 where there is no
      neighbour); return 0
  reduce(part, vals, n, op)  all-reduce n doubles in place (op 0 max,
      1 sum); return 0

LocalParts runs all parts in one process (a host thread per part, device
copies between the parts' buffers; the parts may share a device);
DistExchange runs one part per torch.distributed rank, over NCCL from device
memory or over any backend through host copies.
"""
import ctypes
import threading

cudaMemcpyDefault = 4


def part_planes(nn, nparts):
    """Node planes (1-based, inclusive) of each part of an l axis of nn nodes
    split by nproc3 = nparts: sord/setup.f90:33-38 (nl3 = (nn - 1) / P + 1
    planes per part; the parts that this leaves; the last takes the rest)."""
    nl3 = max((nn - 1) // nparts + 1, 1)
    nproc = (nn - 1) // nl3 + 1
    return [(p * nl3 + 1, min((p + 1) * nl3, nn)) for p in range(nproc)]


def halo_pairs(nparts):
    """The halo copies of one exchange: (receiving part, its side, sending
    part, the sender's side) -- part p's plane below it comes from the top
    core plane of part p - 1, its plane above from the bottom core plane of
    part p + 1."""
    out = []
    for p in range(nparts):
        if p > 0:
            out.append((p, 'lo', p - 1, 'hi'))
        if p < nparts - 1:
            out.append((p, 'hi', p + 1, 'lo'))
    return out


def _cudart():
    # libsordgpu.so links the shared CUDA runtime; it is already loaded
    for name in ('libcudart.so.12', 'libcudart.so'):
        try:
            lib = ctypes.CDLL(name)
            lib.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
            lib.cudaMemcpy.restype = ctypes.c_int
            lib.cudaDeviceSynchronize.restype = ctypes.c_int
            lib.cudaGetDeviceCount.argtypes = [ctypes.POINTER(ctypes.c_int)]
            lib.cudaGetDeviceCount.restype = ctypes.c_int
            return lib
        except OSError:
            continue
    raise OSError('CUDA runtime library not found')


def device_count():
    """Visible CUDA devices (at least 1: the solver reports a missing one)."""
    from coseis_b200 import _lib
    _lib.load()
    n = ctypes.c_int(0)
    if _cudart().cudaGetDeviceCount(ctypes.byref(n)):
        return 1
    return max(n.value, 1)


def device_copy(dst, src, nbytes):
    """Copy between device (or host) pointers, then wait for it."""
    rt = _cudart()
    rc = rt.cudaMemcpy(dst, src, nbytes, cudaMemcpyDefault)
    if rc == 0:
        rc = rt.cudaDeviceSynchronize()
    if rc:
        raise RuntimeError('cudaMemcpy failed (%d)' % rc)


def host_copy(dst, src, nbytes):
    ctypes.memmove(dst, src, nbytes)


class LocalParts(object):
    """All parts of a run in one process: part p's halo planes are copied
    from its neighbours' send buffers once every part has posted them (a
    barrier on each side of the copies).  `copy` moves nbytes between two
    pointers (device_copy for the solver's device buffers)."""

    def __init__(self, nparts, copy=device_copy, timeout=600.0):
        self.nparts = nparts
        self.copy = copy
        self.barrier = threading.Barrier(nparts, timeout=timeout)
        self.posted = [None] * nparts
        self.vals = [None] * nparts

    def halo(self, part, send_lo, recv_lo, send_hi, recv_hi, n):
        self.posted[part] = (send_lo, send_hi)
        self.barrier.wait()
        nbytes = 4 * n
        if recv_lo:
            self.copy(recv_lo, self.posted[part - 1][1], nbytes)
        if recv_hi:
            self.copy(recv_hi, self.posted[part + 1][0], nbytes)
        self.barrier.wait()
        return 0

    def reduce(self, part, vals, n, op):
        self.vals[part] = [vals[i] for i in range(n)]
        self.barrier.wait()
        cols = list(zip(*self.vals))
        res = [max(c) if op == 0 else sum(c) for c in cols]
        self.barrier.wait()
        for i in range(n):
            vals[i] = res[i]
        return 0

    def abort(self):
        self.barrier.abort()


def run_local(workdir, nparts, devices=(0,), arithmetic=None):
    """Run the run staged in `workdir` (its sord.in with nproc3 = [1, 1,
    nparts]) to completion as nparts parts in this process, part p on
    devices[p % len(devices)]; the outputs are those of the whole run."""
    from coseis_b200 import _lib
    import os
    text = open(os.path.join(workdir, 'sord.in')).read()
    ex = LocalParts(nparts)
    first = []
    lock = threading.Lock()

    def work(p):
        s = None
        try:
            s = _lib.Solver(workdir, text, device=devices[p % len(devices)], part=p, exchange=ex)
            if arithmetic:
                s.set_arithmetic(arithmetic)
            s.run()
        except BaseException as e:  # noqa: BLE001 -- the first failure is raised below
            with lock:
                first.append(e)
            ex.abort()  # the other parts stop at their next exchange
        finally:
            if s is not None:
                s.close()
    th = [threading.Thread(target=work, args=(p,)) for p in range(nparts)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    if first:
        raise first[0]


class _DeviceArray(object):
    """A raw device pointer seen as a float32 array by torch."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {'shape': (n,), 'typestr': '<f4', 'data': (ptr, False), 'version': 2}


class DistExchange(object):
    """One part per torch.distributed rank (part = rank).  transport 'device'
    sends the solver's device buffers themselves (NCCL); 'host' copies them
    to host memory first with `copy` (device_copy for device buffers,
    host_copy where the buffers are host memory) and sends CPU tensors
    (gloo).  Every rank takes the same exchanges in the same order."""

    def __init__(self, transport='device', copy=device_copy, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.transport = transport
        self.copy = copy

    def _tensor(self, ptr, n, host):
        import torch
        if self.transport == 'device':
            return torch.as_tensor(_DeviceArray(ptr, n), device='cuda')
        t = torch.empty(n, dtype=torch.float32)
        if not host:
            self.copy(t.data_ptr(), ptr, 4 * n)
        return t

    def halo(self, part, send_lo, recv_lo, send_hi, recv_hi, n):
        dist = self.dist
        ops, recv = [], []
        for send, rcv, peer in ((send_lo, recv_lo, part - 1), (send_hi, recv_hi, part + 1)):
            if send:
                ops.append(dist.P2POp(dist.isend, self._tensor(send, n, False), peer, group=self.group))
            if rcv:
                t = self._tensor(rcv, n, True)
                ops.append(dist.P2POp(dist.irecv, t, peer, group=self.group))
                recv.append((rcv, t))
        if ops and self.transport == 'device':
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        elif ops:
            reqs = [op.op(op.tensor, op.peer, group=self.group) for op in ops]
            for r in reqs:
                r.wait()
        if self.transport == 'device':
            import torch
            torch.cuda.synchronize()
        else:
            for ptr, t in recv:
                self.copy(ptr, t.data_ptr(), 4 * n)
        return 0

    def reduce(self, part, vals, n, op):
        import torch
        dist = self.dist
        dev = 'cuda' if self.transport == 'device' else 'cpu'
        t = torch.tensor([vals[i] for i in range(n)], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX if op == 0 else dist.ReduceOp.SUM, group=self.group)
        t = t.cpu()
        for i in range(n):
            vals[i] = float(t[i])
        return 0


def run_dist(workdir, device, transport='device', arithmetic=None):
    """This rank's part of the run staged in `workdir` (nproc3 = [1, 1,
    world size]), run to completion; every rank calls it."""
    import os
    import torch.distributed as dist
    from coseis_b200 import _lib
    text = open(os.path.join(workdir, 'sord.in')).read()
    s = _lib.Solver(workdir, text, device=device, part=dist.get_rank(), exchange=DistExchange(transport))
    try:
        if arithmetic:
            s.set_arithmetic(arithmetic)
        s.run()
    finally:
        s.close()
