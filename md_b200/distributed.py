"""The collective behind a split evaluation (mdf_params.rank / nranks).

A context with nranks > 1 computes its share of the pair, bonded,
exclusion/1-4 and PME spread/gather work and sums the int64 charge grid and
the int64 force/energy accumulators over the ranks through a callback
(mdf_set_allreduce).  `torch_allreduce` builds that callback on a
torch.distributed process group: NCCL for one GPU per rank, gloo where the
ranks share a GPU or run on the CPU.  Sums of two's-complement int64 are
exact and order-independent, so every rank ends with the same forces, bit
for bit, as one context computing everything.
"""
from __future__ import annotations

import ctypes as C

import numpy as np


class _DeviceInt64:
    """A CUDA buffer of int64 seen through __cuda_array_interface__ (no copy)."""

    def __init__(self, ptr, count):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": "<i8", "data": (int(ptr), False),
                                         "version": 3, "strides": None, "stream": None}


def torch_allreduce(group=None, host=False):
    """fn(ptr, count, stream, user) -> int for Engine.set_allreduce: an in-place
    int64 sum over `group` (default: the world), queued after the work already
    on `stream` and visible to the work queued after it.  host=True treats
    `ptr` as host memory (the CPU path of the tests)."""
    import torch
    import torch.distributed as dist

    def fn(ptr, count, stream, user):
        try:
            if host:
                buf = np.ctypeslib.as_array(C.cast(C.c_void_p(ptr), C.POINTER(C.c_int64)), shape=(int(count),))
                dist.all_reduce(torch.from_numpy(buf), op=dist.ReduceOp.SUM, group=group)
                return 0
            t = torch.as_tensor(_DeviceInt64(ptr, count), device="cuda")
            with torch.cuda.stream(torch.cuda.ExternalStream(int(stream or 0), device=t.device)):
                dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
            return 0
        except Exception:   # reported to the library as a failed collective
            return 1
    return fn
