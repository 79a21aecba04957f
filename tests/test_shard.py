"""Sharding of the batched workload over ranks: the greedy partition covers
every system once, balances the estimated cost, and is the same on every rank;
the max-over-ranks timing reduction works over a 2-rank gloo group on CPU."""
import os

import pytest

from md_b200 import shard, synth


def _costs(n=256):
    dims = synth._batch_dims(n, 1003)
    out = []
    for L, nres in dims:
        nat = 3 * max(10, int(0.1 * L ** 3 / 3.0) - nres * 10 // 3) + 10 * nres
        g = synth.smooth_grid_size(L, 1.0)
        out.append(shard.system_cost(nat, (g, g, g)))
    return out


@pytest.mark.parametrize("nranks", [1, 2, 4, 8])
def test_partition_covers_and_balances(nranks):
    c = _costs()
    parts = shard.partition(c, nranks)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(c)))
    assert shard.imbalance(c, parts) < 1.02
    assert parts == shard.partition(list(c), nranks)     # deterministic


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    parts = shard.partition(_costs(), world)
    mine = parts[rank]
    # every rank's view of the partition, gathered: they must agree
    views = [None] * world
    dist.all_gather_object(views, parts)
    t = shard.max_over_ranks(1.0 + rank)
    q.put((rank, len(mine), all(v == parts for v in views), t))
    dist.destroy_process_group()


def test_two_rank_gloo_partition_and_max():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert res[0][1] + res[1][1] == 256
    assert all(r[2] for r in res)
    assert all(r[3] == 2.0 for r in res)
