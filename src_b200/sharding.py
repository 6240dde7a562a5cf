"""One bunch sharded over ranks: exchange callbacks for scgpu_set_exchange.

The reference distributes a bunch's particles over MPI ranks; the bounds
(get_bounds, PartBunchBase.hpp:1178-1219), the moment sums (calcMoments,
:2185-2259) and the scattered charge (IPPL's distributed rho field) are
reduced across them.  Here each rank holds a shard in its own context and
the library hands the partial results to an exchange callback: a minimum
over doubles (bounds) or a sum of 64-bit integers (the deposit's fixed-point
node sums, exact momentum and moment sums as 32-bit chunks).  Every combined
value is exact, so the shards evolve bitwise as the whole bunch on one GPU.

* ``TorchExchange``: torch.distributed.  With the NCCL backend the buffer is
  reduced in place on the device, on the library's stream; with gloo it goes
  through host memory.
* ``HostExchange``: ranks as threads of one process (one context each),
  combined in host memory -- a single-node fallback and the test harness.
"""
from __future__ import annotations

import threading

import numpy as np

from .scgpu import EXCHANGE_FN

SUM_U64 = 0
MIN_F64 = 1


class _DeviceView:
    """A device buffer as a torch tensor (no copy) through the CUDA array interface."""

    def __init__(self, ptr, count, op):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": "<f8" if op == MIN_F64 else "<i8",
                                         "data": (int(ptr), False), "version": 3, "strides": None}


def _tensor(ptr, count, op):
    import torch
    return torch.as_tensor(_DeviceView(ptr, count, op), device="cuda")


def combine(arrays, op):
    """The exchange's arithmetic on host arrays: elementwise minimum of
    doubles, or the sum of 64-bit integers modulo 2^64."""
    if op == MIN_F64:
        return np.minimum.reduce([np.asarray(a, dtype=np.float64) for a in arrays])
    out = np.zeros_like(np.asarray(arrays[0], dtype=np.uint64))
    for a in arrays:
        out = out + np.asarray(a, dtype=np.uint64)  # wraps modulo 2^64
    return out


class HostExchange:
    """nranks shards driven by nranks host threads of this process."""

    def __init__(self, nranks):
        self.nranks = nranks
        # a rank that never arrives breaks the barrier after the timeout: the
        # callbacks then fail and the library reports SCGPU_ERR_EXCHANGE
        self._barrier = threading.Barrier(nranks, timeout=300)
        self._slots = [None] * nranks
        self._result = None
        self._callbacks = [EXCHANGE_FN(self._make(r)) for r in range(nranks)]

    def callback(self, rank):
        return self._callbacks[rank]

    def _make(self, rank):
        def fn(ptr, count, op, stream, user):
            try:
                import torch
                torch.cuda.ExternalStream(stream).synchronize()
                t = _tensor(ptr, count, op)
                host = t.cpu().numpy()
                self._slots[rank] = host.view(np.uint64) if op == SUM_U64 else host
                if self._barrier.wait() == 0:
                    self._result = combine(self._slots, op)
                self._barrier.wait()
                t.copy_(torch.from_numpy(self._result.view(np.int64) if op == SUM_U64 else self._result))
                torch.cuda.current_stream().synchronize()
                self._barrier.wait()
                return 0
            except Exception:  # noqa: BLE001 -- a failing rank breaks the barrier for the others
                self._barrier.abort()
                return 1
        return fn


class TorchExchange:
    """The ranks of a torch.distributed process group (one shard per rank)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.backend = dist.get_backend(group)
        self._cb = EXCHANGE_FN(self._fn)

    def callback(self):
        return self._cb

    @property
    def capturable(self):
        return False

    def combine_host(self, a, op):
        """Combine a host array over the group (the gloo path's arithmetic)."""
        import torch
        t = torch.from_numpy(np.ascontiguousarray(a).view(np.int64) if op == SUM_U64 else np.ascontiguousarray(a))
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN if op == MIN_F64 else self.dist.ReduceOp.SUM,
                             group=self.group)
        return t.numpy().view(np.uint64) if op == SUM_U64 else t.numpy()

    def _fn(self, ptr, count, op, stream, user):
        try:
            import torch
            ext = torch.cuda.ExternalStream(stream)
            t = _tensor(ptr, count, op)
            if self.backend == "nccl":
                with torch.cuda.stream(ext):
                    self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN if op == MIN_F64 else self.dist.ReduceOp.SUM,
                                         group=self.group)
                return 0
            ext.synchronize()
            host = t.cpu().numpy()
            res = self.combine_host(host.view(np.uint64) if op == SUM_U64 else host, op)
            t.copy_(torch.from_numpy(res.view(np.int64) if op == SUM_U64 else res))
            torch.cuda.current_stream().synchronize()
            return 0
        except Exception:
            return 1


def attach(ctx, callback, total_particles, capturable=False):
    """scgpu_set_exchange on a Context (before its upload)."""
    from . import scgpu
    rc = scgpu.lib().scgpu_set_exchange(ctx.h, callback, None, int(total_particles), 1 if capturable else 0)
    ctx._check(rc, "set_exchange")
    ctx._exchange = callback  # keep the ctypes callback alive with the context
