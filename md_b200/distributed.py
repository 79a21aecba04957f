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
reduce-scatter force return) on the same kind of group, and `torch_alltoallv`
the all-to-all with per-rank sizes of mdf_set_halo_exchange (grid planes to
and from the spatial neighbours only).  With gloo the buffers are staged
through host memory; with NCCL the collectives run on the device, ordered on
the library's stream.
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


def torch_alltoallv(group=None, host=False):
    """fn(send, send_bytes, recv, recv_bytes, stream, user) -> int for
    Engine.set_halo_exchange on `group` (default: the world): send_bytes[k]
    bytes of `send` go to rank k and recv_bytes[k] bytes from rank k land in
    `recv`, both packed in rank order (torch.distributed.all_to_all_single with
    split sizes).  host=True treats the buffers as host memory (the CPU path
    of the tests)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    nccl = dist.get_backend(group) == "nccl"

    def fn(send, send_bytes, recv, recv_bytes, stream, user):
        try:
            ins = [int(send_bytes[k]) for k in range(world)]
            outs = [int(recv_bytes[k]) for k in range(world)]
            ni, no = sum(ins), sum(outs)
            if host:
                src = torch.from_numpy(np.ctypeslib.as_array(C.cast(C.c_void_p(send), C.POINTER(C.c_uint8)),
                                                             shape=(max(ni, 1),))[:ni])
                dst = torch.from_numpy(np.ctypeslib.as_array(C.cast(C.c_void_p(recv), C.POINTER(C.c_uint8)),
                                                             shape=(max(no, 1),))[:no])
                dist.all_to_all_single(dst, src, outs, ins, group=group)
                return 0
            src = torch.as_tensor(_DeviceBytes(send, ni), device="cuda")
            dst = torch.as_tensor(_DeviceBytes(recv, no), device="cuda")
            s = torch.cuda.ExternalStream(int(stream or 0))
            with torch.cuda.stream(s):
                if nccl:
                    dist.all_to_all_single(dst, src, outs, ins, group=group)
                else:
                    out = torch.empty(no, dtype=torch.uint8)
                    dist.all_to_all_single(out, src.cpu(), outs, ins, group=group)
                    dst.copy_(out)
                    s.synchronize()
            return 0
        except Exception:   # reported to the library as a failed collective
            return 1
    return fn
