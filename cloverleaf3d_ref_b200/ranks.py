"""A decomposed run with one brick per rank (the reference's MPI model,
clover.f90) over torch.distributed.

Every rank holds one brick of clover_decompose's grid (chunk id = rank + 1)
and runs the library's brick driver on it; the driver calls back into
DistTransport for what MPI carries in the reference: the halo messages of each
axis phase of clover_exchange (clover.f90:474-713) to and from the neighbour
ranks, clover_min of the timestep (timestep.f90) and clover_sum of the field
summary (field_summary.f90). With the gloo backend the messages are host
(pinned) buffers; with NCCL they are device buffers.
"""
import ctypes

import numpy as np

from . import CloverError, FIELD_IDS, field_shape, lib

_DP = ctypes.POINTER(ctypes.c_double)
_EXCHANGE = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _DP, _DP,
                             ctypes.c_longlong, ctypes.c_int, _DP, _DP, ctypes.c_longlong)
_MIN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, _DP)
_SUM = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, _DP, ctypes.c_int)


class TransportStruct(ctypes.Structure):
    """clover_transport (include/clover_b200.h)."""
    _fields_ = [("ctx", ctypes.c_void_p), ("host_staged", ctypes.c_int),
                ("exchange", _EXCHANGE), ("min", _MIN), ("sum", _SUM)]


class _CudaBuffer:
    """A device buffer of n doubles as a __cuda_array_interface__ object."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8",
                                         "data": (ptr, False), "version": 3, "strides": None}


class DistTransport:
    """The callbacks of clover_transport over a torch.distributed group.

    A chunk id c is rank c - 1. Each axis phase posts, for every existing
    neighbour, one send of this rank's message and one receive of the
    neighbour's, as one batch, and waits for them; the reductions are
    all-reduces (MIN, SUM)."""

    def __init__(self, dist, group=None):
        import torch
        self.torch = torch
        self.dist = dist
        self.group = group
        backend = dist.get_backend(group)
        self.on_device = backend == "nccl"
        self.failures = []
        self.s = TransportStruct(None, 0 if self.on_device else 1, _EXCHANGE(self._exchange),
                                 _MIN(self._min), _SUM(self._sum))

    def _view(self, p, n):
        addr = ctypes.cast(p, ctypes.c_void_p).value
        if self.on_device:
            return self.torch.as_tensor(_CudaBuffer(addr, int(n)), device="cuda")
        return self.torch.from_numpy(np.ctypeslib.as_array(p, shape=(int(n),)))

    def _exchange(self, ctx, axis, lo, s_lo, r_lo, n_lo, hi, s_hi, r_hi, n_hi):
        try:
            ops = []
            for nb, s, r, n in ((lo, s_lo, r_lo, n_lo), (hi, s_hi, r_hi, n_hi)):
                if nb < 0 or n <= 0:
                    continue
                ops.append(self.dist.P2POp(self.dist.isend, self._view(s, n), nb - 1, self.group))
                ops.append(self.dist.P2POp(self.dist.irecv, self._view(r, n), nb - 1, self.group))
            if ops:
                for w in self.dist.batch_isend_irecv(ops):
                    w.wait()
                if self.on_device:
                    self.torch.cuda.synchronize()
            return 0
        except Exception as e:  # reported by the driver's failure status
            self.failures.append(repr(e))
            return 1

    def _reduce(self, p, n, op):
        dev = "cuda" if self.on_device else "cpu"
        t = self.torch.tensor([p[i] for i in range(n)], dtype=self.torch.float64, device=dev)
        self.dist.all_reduce(t, op=op, group=self.group)
        for i, v in enumerate(t.cpu().tolist()):
            p[i] = v

    def _min(self, ctx, p):
        try:
            self._reduce(p, 1, self.dist.ReduceOp.MIN)
            return 0
        except Exception as e:
            self.failures.append(repr(e))
            return 1

    def _sum(self, ctx, p, n):
        try:
            self._reduce(p, n, self.dist.ReduceOp.SUM)
            return 0
        except Exception as e:
            self.failures.append(repr(e))
            return 1


class RankBricks:
    """This rank's brick of a deck decomposed over the ranks of `dist`'s
    default group (clover_decompose with world-size chunks), on the current
    CUDA device. ``run``, ``dt_history`` and ``summaries`` are the whole
    deck's (every rank holds the same); ``field`` is this brick's own array
    in its reference layout, ``extent`` its global cell range."""

    def __init__(self, deck, dist):
        L = lib()
        L.clover_gpu_clear_status()
        self.deck = deck
        self.rank = dist.get_rank()
        self.world = dist.get_world_size()
        self.transport = DistTransport(dist)
        self.h = L.clover_bricks_create_rank(ctypes.byref(deck.s), self.world, self.rank,
                                             ctypes.byref(self.transport.s))
        if not self.h:
            raise CloverError("brick start failed on rank %d: %s %s" % (
                self.rank, L.clover_gpu_error_string().decode(), self.transport.failures))
        e = np.zeros(6, dtype=np.int32)
        nb = np.zeros(6, dtype=np.int32)
        L.clover_bricks_extent(self.h, 0, e.ctypes.data, nb.ctypes.data)
        self.extent = tuple(int(v) for v in e)
        self.neighbours = tuple(int(v) for v in nb)

    def run(self, max_steps=2 ** 30):
        n = lib().clover_bricks_run(self.h, max_steps)
        st = lib().clover_gpu_status()
        if n < 0 or st & ~0x4:
            raise CloverError("rank %d: %s %s" % (self.rank, lib().clover_gpu_error_string().decode(),
                                                 self.transport.failures))
        return n

    def dt_history(self, cap=1 << 20):
        out = np.zeros(cap)
        n = lib().clover_bricks_dt_history(self.h, out.ctypes.data, cap)
        return out[:n]

    def summaries(self, cap=100000):
        out = np.zeros((cap, 5))
        st = np.zeros(cap, dtype=np.int32)
        n = lib().clover_bricks_summaries(self.h, out.ctypes.data, st.ctypes.data, cap)
        return out[:n], st[:n]

    def field(self, name):
        e = self.extent
        a = np.zeros(field_shape(name, e[1] - e[0] + 1, e[3] - e[2] + 1, e[5] - e[4] + 1),
                     order="F")
        if lib().clover_bricks_read_field(self.h, 0, FIELD_IDS[name], a.ctypes.data, a.size) != 0:
            raise CloverError("read_field failed")
        return a

    def close(self):
        if self.h:
            lib().clover_bricks_destroy(self.h)
            self.h = None
