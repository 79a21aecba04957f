"""The collectives behind a split evaluation (mdf_params.rank / nranks).

A context with nranks > 1 computes its share of the pair, bonded,
exclusion/1-4 and PME spread/gather work and sums the int64 charge grid and
the int64 force/energy accumulators over the ranks through a callback
(mdf_set_allreduce).  `torch_allreduce` builds that callback on a
torch.distributed process group: NCCL for one GPU per rank, gloo where the
ranks share a GPU or run on the CPU.  Sums of two's-complement int64 are
exact and order-independent, so every rank ends with the same forces, bit
for bit, as one context computing everything.

`torch_collectives` builds the reduce-scatter, all-gather and all-to-all of
mdf_set_collectives (the x-slab distributed reciprocal space and the
reduce-scatter force return) on the same kind of group.  With gloo the
buffers are staged through host memory; with NCCL the collectives run on the
device, ordered on the library's stream.
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


class _DeviceBytes:
    """A CUDA buffer of `n` bytes (as uint8) or int64 words seen through __cuda_array_interface__."""

    def __init__(self, ptr, n, typestr="|u1"):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None, "stream": None}


def torch_collectives(group=None):
    """(reduce_scatter, allgather, alltoall) callbacks for Engine.set_collectives
    on `group` (default: the world)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    nccl = dist.get_backend(group) == "nccl"

    def run(stream, fn):
        s = torch.cuda.ExternalStream(int(stream or 0))
        with torch.cuda.stream(s):
            fn()
            if not nccl:
                s.synchronize()

    def reduce_scatter(send, recv, count, stream, user):
        try:
            src = torch.as_tensor(_DeviceBytes(send, world * count, "<i8"), device="cuda")
            dst = torch.as_tensor(_DeviceBytes(recv, count, "<i8"), device="cuda")

            def go():
                if nccl:
                    dist.reduce_scatter_tensor(dst, src, op=dist.ReduceOp.SUM, group=group)
                else:
                    h = src.cpu()
                    out = torch.empty(count, dtype=torch.int64)
                    dist.reduce_scatter_tensor(out, h, op=dist.ReduceOp.SUM, group=group)
                    dst.copy_(out)
            run(stream, go)
            return 0
        except Exception:
            return 1

    def allgather(send, recv, nbytes, stream, user):
        try:
            src = torch.as_tensor(_DeviceBytes(send, nbytes), device="cuda")
            dst = torch.as_tensor(_DeviceBytes(recv, world * nbytes), device="cuda")

            def go():
                if nccl:
                    dist.all_gather_into_tensor(dst, src, group=group)
                else:
                    out = torch.empty(world * nbytes, dtype=torch.uint8)
                    dist.all_gather_into_tensor(out, src.cpu(), group=group)
                    dst.copy_(out)
            run(stream, go)
            return 0
        except Exception:
            return 1

    def alltoall(send, recv, nbytes, stream, user):
        try:
            src = torch.as_tensor(_DeviceBytes(send, world * nbytes), device="cuda")
            dst = torch.as_tensor(_DeviceBytes(recv, world * nbytes), device="cuda")

            def go():
                if nccl:
                    dist.all_to_all_single(dst, src, group=group)
                else:
                    out = torch.empty(world * nbytes, dtype=torch.uint8)
                    dist.all_to_all_single(out, src.cpu(), group=group)
                    dst.copy_(out)
            run(stream, go)
            return 0
        except Exception:
            return 1

    return reduce_scatter, allgather, alltoall
