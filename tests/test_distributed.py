"""The split evaluation (mdf_params.rank / nranks, mdf_set_allreduce).

CPU (gloo, 2 ranks): the collective callback of md_b200.distributed, called
through a C function pointer as the library calls it, sums int64 buffers in
place across the ranks, two's-complement wrap-around included.

GPU (gloo, 2 and 3 ranks sharing cuda:0; the collectives run on the host,
no kernel waits on another rank): every rank ends with forces identical bit
for bit to one context evaluating everything - with the all-reduce form and
with the slab-distributed reciprocal space and reduce-scatter force return - mixed and FP64, on the first
evaluation after a list build (pair counting on) and the next; energies agree
to 1e-12 relative + 1e-8 (per-block FP64 sums are rounded to the 2^-32
fixed point before they are added, and the blocks differ) and the pair count
is exact.  Contexts with
nranks > 1 refuse to evaluate without a collective, and the entry points
that do not support the split say so.
"""
import ctypes as C
import os
import socket

import numpy as np
import pytest

from md_b200 import abi


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(worker, world, *args, timeout=300):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=worker, args=(r, world, port, q) + args) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=timeout) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return [res[r] for r in range(world)]


def _init(rank, world, port):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    return dist


def _cb_worker(rank, world, port, q):
    from md_b200 import distributed
    dist = _init(rank, world, port)
    fn = abi.MDF_ALLREDUCE_FN(distributed.torch_allreduce(host=True))
    buf = np.array([rank + 1, -(rank + 1) * 1000, 2 ** 62, 7], dtype=np.int64)
    rc = fn(buf.ctypes.data, 4, None, None)   # as the library would call it
    q.put((rank, (rc, buf.tolist())))
    dist.destroy_process_group()


def _a2av_worker(rank, world, port, q):
    from md_b200 import distributed
    dist = _init(rank, world, port)
    fn = abi.MDF_ALLTOALLV_FN(distributed.torch_alltoallv(host=True))
    # rank r sends k + r bytes of value 16 r + k to rank k (none to itself when k + r == 0)
    send_n = [k + rank for k in range(world)]
    recv_n = [rank + k for k in range(world)]
    send = np.concatenate([np.full(send_n[k], 16 * rank + k, np.uint8) for k in range(world)] + [np.zeros(1, np.uint8)])
    recv = np.full(sum(recv_n) + 1, 255, np.uint8)
    sb = (C.c_int64 * world)(*send_n)
    rb = (C.c_int64 * world)(*recv_n)
    rc = fn(send.ctypes.data, sb, recv.ctypes.data, rb, None, None)   # as the library would call it
    q.put((rank, (rc, recv[:-1].tolist(), int(recv[-1]))))
    dist.destroy_process_group()


def test_alltoallv_callback_three_rank_gloo_cpu():
    """The halo exchange's all-to-all with per-rank sizes (zero-size blocks
    included) through the C function pointer, 3 gloo ranks on the CPU."""
    world = 3
    res = _run(_a2av_worker, world)
    for r, (rc, got, tail) in enumerate(res):
        assert rc == 0
        want = []
        for k in range(world):
            want += [16 * k + r] * (r + k)
        assert got == want
        assert tail == 255   # nothing past the received bytes


def test_allreduce_callback_two_rank_gloo_cpu():
    res = _run(_cb_worker, 2)
    wrap = -2 ** 63   # 2^62 + 2^62 wraps like an int64 accumulator
    for rc, vals in res:
        assert rc == 0
        assert vals == [3, -3000, wrap, 14]


def _eval_worker(rank, world, port, q, cfg, prec, slab=False, halo=False):
    from md_b200 import distributed, engine, synth
    from tests import helpers as H
    dist = _init(rank, world, port)
    s = H.system(cfg)
    flat = H.flat(s, abi.MDF_SEM_PHYSICAL, engine.cmap_coefficients)
    eng = engine.Engine(flat, s.box, semantics=abi.MDF_SEM_PHYSICAL, precision=prec, ewald_tol=1e-5,
                        grid=synth.GRIDS[cfg], rank=rank, nranks=world)
    eng.set_allreduce(distributed.torch_allreduce())
    if slab:
        eng.set_collectives(*distributed.torch_collectives())
    if halo:
        eng.set_halo_exchange(distributed.torch_alltoallv())
    eng.set_positions(s.coords)
    eng.build_pairlist()
    out = []
    for _ in range(2):
        E, F = eng.compute()
        out.append((E, F, eng.pairlist_info()["pairs_in_cutoff"]))
    eng.close()
    q.put((rank, out))
    dist.destroy_process_group()


def _single(cfg, prec):
    from md_b200 import engine, synth
    from tests import helpers as H
    s = H.system(cfg)
    flat = H.flat(s, abi.MDF_SEM_PHYSICAL, engine.cmap_coefficients)
    eng = engine.Engine(flat, s.box, semantics=abi.MDF_SEM_PHYSICAL, precision=prec, ewald_tol=1e-5,
                        grid=synth.GRIDS[cfg])
    eng.set_positions(s.coords)
    eng.build_pairlist()
    out = []
    for _ in range(2):
        E, F = eng.compute()
        out.append((E, F, eng.pairlist_info()["pairs_in_cutoff"]))
    eng.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("cfg,world,prec", [("small", 2, abi.MDF_PREC_MIXED), ("small", 3, abi.MDF_PREC_FP64),
                                            ("c0", 2, abi.MDF_PREC_MIXED)])
def test_split_evaluation_matches_one_context(cfg, world, prec):
    res = _run(_eval_worker, world, cfg, prec)
    ref = _single(cfg, prec)
    for out in res:
        for (E, F, npair), (E0, F0, np0) in zip(out, ref):
            assert np.array_equal(F, F0)
            assert npair == np0
            for k in abi.E_NAMES + ["total"]:
                assert abs(E[k] - E0[k]) <= 1e-12 * abs(E0[k]) + 1e-8, (k, E[k], E0[k])


@pytest.mark.gpu
@pytest.mark.parametrize("cfg,world,prec", [("small", 2, abi.MDF_PREC_MIXED), ("small", 3, abi.MDF_PREC_FP64),
                                            ("c0", 2, abi.MDF_PREC_MIXED), ("c0", 3, abi.MDF_PREC_MIXED)])
def test_slab_pme_and_force_scatter_match_one_context(cfg, world, prec):
    """With mdf_set_collectives the reciprocal space is distributed as x-slabs
    (reduce-scatter of the charge grid, all-to-all transposes around the x
    pass, all-gather of the potential) and the forces return by reduce-scatter
    and all-gather: forces still equal one context's bit for bit, energies to
    1e-12 relative + 1e-8 (3 ranks: grids whose planes do not divide evenly)."""
    res = _run(_eval_worker, world, cfg, prec, True)
    ref = _single(cfg, prec)
    for out in res:
        for (E, F, npair), (E0, F0, np0) in zip(out, ref):
            assert np.array_equal(F, F0)
            assert npair == np0
            for k in abi.E_NAMES + ["total"]:
                assert abs(E[k] - E0[k]) <= 1e-12 * abs(E0[k]) + 1e-8, (k, E[k], E0[k])


@pytest.mark.gpu
@pytest.mark.parametrize("cfg,world,prec", [("small", 2, abi.MDF_PREC_MIXED), ("small", 3, abi.MDF_PREC_FP64),
                                            ("c0", 2, abi.MDF_PREC_MIXED), ("c0", 3, abi.MDF_PREC_MIXED),
                                            ("c0", 4, abi.MDF_PREC_FP64)])
def test_halo_exchange_matches_one_context(cfg, world, prec):
    """With mdf_set_halo_exchange the charge grid and the potential cross
    between the ranks as halo planes around each rank's band (all-to-all with
    per-rank sizes) instead of the whole-grid reduce-scatter and all-gather:
    forces still equal one context's bit for bit."""
    res = _run(_eval_worker, world, cfg, prec, True, True)
    ref = _single(cfg, prec)
    for out in res:
        for (E, F, npair), (E0, F0, np0) in zip(out, ref):
            assert np.array_equal(F, F0)
            assert npair == np0
            for k in abi.E_NAMES + ["total"]:
                assert abs(E[k] - E0[k]) <= 1e-12 * abs(E0[k]) + 1e-8, (k, E[k], E0[k])


@pytest.mark.gpu
def test_halo_exchange_at_960k_atoms():
    """The band decomposition at c4 scale (960,000 atoms, 49 x-columns, PME
    216^3; 4 ranks, bands of 6-7 columns, 7-12 halo planes each): forces equal
    one context's bit for bit."""
    world, cfg, prec = 4, "c4", abi.MDF_PREC_MIXED
    res = _run(_eval_worker, world, cfg, prec, True, True)
    ref = _single(cfg, prec)
    for out in res:
        for (E, F, npair), (E0, F0, np0) in zip(out, ref):
            assert np.array_equal(F, F0)
            assert npair == np0
            assert abs(E["total"] - E0["total"]) <= 1e-12 * abs(E0["total"]) + 1e-8


def _stale_worker(rank, world, port, q, cfg, shift):
    from md_b200 import distributed, engine, synth
    from tests import helpers as H
    dist = _init(rank, world, port)
    try:
        s = H.system(cfg)
        flat = H.flat(s, abi.MDF_SEM_PHYSICAL, engine.cmap_coefficients)
        eng = engine.Engine(flat, s.box, semantics=abi.MDF_SEM_PHYSICAL, precision=abi.MDF_PREC_MIXED,
                            ewald_tol=1e-5, grid=synth.GRIDS[cfg], rank=rank, nranks=world)
        eng.set_allreduce(distributed.torch_allreduce())
        eng.set_collectives(*distributed.torch_collectives())
        eng.set_halo_exchange(distributed.torch_alltoallv())
        eng.set_positions(s.coords)
        eng.build_pairlist()
        eng.compute()
        x = s.coords.copy()
        x[:, 0] += shift   # the whole system moves: every atom leaves its band
        eng.set_positions(x)
        status = 0
        try:
            eng.compute()
        except engine.MDFError as e:
            status = e.status
        eng.build_pairlist()   # every rank: the list and the bands follow the atoms
        E, F = eng.compute()
        eng.close()
        q.put((rank, (status, F)))
    except Exception as e:   # reported, not left to the queue's timeout
        q.put((rank, ("error", repr(e))))
    dist.destroy_process_group()


@pytest.mark.gpu
def test_halo_exchange_reports_atoms_outside_their_band():
    """Atoms moved out of their rank's band since the list build (here the
    whole system, by half a box in x: the same physics, no atom within half
    the skin of its old band) are reported - MDF_ERR_STATE on the ranks that
    own them - instead of being spread into planes nobody receives; after a
    list rebuild the split evaluation equals one context again."""
    from md_b200 import engine, synth
    from tests import helpers as H
    world, cfg = 2, "c0"
    s = H.system(cfg)
    shift = 0.5 * s.box[0]
    res = _run(_stale_worker, world, cfg, shift)
    for st, F in res:
        assert st != "error", F
    assert all(st == abi.MDF_ERR_STATE for st, _ in res)
    flat = H.flat(s, abi.MDF_SEM_PHYSICAL, engine.cmap_coefficients)
    eng = engine.Engine(flat, s.box, semantics=abi.MDF_SEM_PHYSICAL, precision=abi.MDF_PREC_MIXED, ewald_tol=1e-5,
                        grid=synth.GRIDS[cfg])
    x = s.coords.copy()
    x[:, 0] += shift
    eng.set_positions(x)
    eng.build_pairlist()
    _, F0 = eng.compute()
    eng.close()
    for _, F in res:
        assert np.array_equal(F, F0)


@pytest.mark.gpu
def test_split_context_needs_a_collective_and_refuses_the_rest():
    from md_b200 import engine, synth
    from tests import helpers as H
    s = H.system("tiny")
    flat = H.flat(s, abi.MDF_SEM_PHYSICAL, engine.cmap_coefficients)
    eng = engine.Engine(flat, s.box, semantics=abi.MDF_SEM_PHYSICAL, precision=abi.MDF_PREC_MIXED,
                        grid=synth.GRIDS["tiny"], rank=1, nranks=2)
    eng.set_positions(s.coords)
    with pytest.raises(engine.MDFError) as ei:
        eng.compute()
    assert ei.value.status == abi.MDF_ERR_STATE
    with pytest.raises(engine.MDFError) as ei:
        eng.md_init(s.mass)
    assert ei.value.status == abi.MDF_ERR_UNSUPPORTED
    with pytest.raises(engine.MDFError) as ei:
        eng.minimize(max_iter=1, method="lbfgs")
    assert ei.value.status == abi.MDF_ERR_UNSUPPORTED
    eng.close()
    for rank, nranks, sem in ((2, 2, abi.MDF_SEM_PHYSICAL), (0, 2, abi.MDF_SEM_REFERENCE)):
        with pytest.raises(engine.MDFError):
            engine.Engine(flat, s.box, semantics=sem, precision=abi.MDF_PREC_FP64, grid=synth.GRIDS["tiny"],
                          rank=rank, nranks=nranks)


def _bench_worker(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    dist = _init(rank, world, port)
    out = bench.split_bench(0, world, rank, cfg="small", steps=3, warmup=1)
    q.put((rank, out))
    dist.destroy_process_group()


@pytest.mark.gpu
def test_bench_split_line_runs():
    """bench.py's split measurement (run at N > 1 with NCCL under torchrun)
    end to end with 2 gloo ranks on one GPU and a small workload."""
    res = _run(_bench_worker, 2)
    assert res[0]["n_ranks"] == 2 and res[0]["evals_per_s"] > 0 and res[0]["speedup"] > 0
    assert "speedup" not in res[1]
