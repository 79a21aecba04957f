"""Batched evaluation (mdf_batch_*): uneven independent systems in one CUDA
graph launch, one kernel launch per evaluation step for all systems, must give
exactly the single-system results (same kernel bodies on the same data,
fixed-point sums) across graph replays and position updates.  After
autotuning, the batch equals single systems run with the chosen launch shape
(pruning and the pair layout set the order of the FP32 sums of each i
cluster's forces; warps per block, the warp schedule and FFT lines change no
bit of the forces); energies, summed in FP64 per warp before their
fixed-point conversion, may move in the last bits (1e-12 relative + 1e-8
absolute).  The FP64 and mixed batches match the oracle."""
import numpy as np
import pytest

from md_b200 import abi, engine, synth
from oracle import oracle as O
from tests import helpers as H

pytestmark = pytest.mark.gpu
PHYS, FP64, MIXED = abi.MDF_SEM_PHYSICAL, abi.MDF_PREC_FP64, abi.MDF_PREC_MIXED
TERMS = ["bond", "angle", "dihedral", "ub", "improper", "cmap", "vdw", "vdw14", "ee_direct", "ee14", "ee_excl",
         "ee_self", "ee_recip", "total"]
KW = dict(cutoff=9.0, skin=2.0, switch_radius=8.0, ewald_tol=1e-5)

_SYS = None


def systems():
    global _SYS
    if _SYS is None:
        _SYS = synth.make_batch(n_systems=5, seed=77)
    return _SYS


def _flats(ss):
    return [H.flat(s, PHYS, engine.cmap_coefficients) for s in ss]


def _singles(ss, flats, prec, coords=None, **shape):
    out = []
    for k, (s, f) in enumerate(zip(ss, flats)):
        eng = engine.Engine(f, s.box, semantics=PHYS, precision=prec, grid=s.meta["grid"], **KW, **shape)
        eng.set_positions(s.coords)
        eng.build_pairlist()
        if coords is not None:
            eng.set_positions(coords[k])
        out.append(eng.compute())
        eng.close()
    return out


def _same(res, ref, etol=0.0):
    for (E, F), (E1, F1) in zip(res, ref):
        assert np.array_equal(F, F1)
        for t in TERMS:
            # etol > 0: rounding of the per-block FP64 sums (relative) and their
            # fixed-point conversion (2^-32 per block, absolute)
            assert abs(E[t] - E1[t]) <= etol * abs(E1[t]) + (1e-8 if etol else 0.0), (t, E[t], E1[t])


@pytest.mark.parametrize("layout", [0, 1])
@pytest.mark.parametrize("prec", [MIXED, FP64])
def test_batch_equals_single_systems(prec, layout):
    ss = systems()
    flats = _flats(ss)
    b = engine.Batch(flats, [s.box for s in ss], [s.meta["grid"] for s in ss], precision=prec, pair_layout=layout,
                     **KW)
    b.set_positions([s.coords for s in ss])
    res = b.compute()
    ref = _singles(ss, flats, prec, pair_layout=layout)
    _same(res, ref)
    _same(b.compute(), ref)           # a graph replay
    info = b.info()
    # one launch per kernel for all systems: ~17 kernels whatever the batch size
    assert info["n_systems"] == len(ss) and 0 < info["graph_kernels"] <= 20
    b.close()


def test_batch_pinned_host_buffers_in_place():
    """Positions written into the batch's pinned buffer and forces read from
    its pinned force buffer give the same results as the copying calls."""
    ss = systems()
    flats = _flats(ss)
    b = engine.Batch(flats, [s.box for s in ss], [s.meta["grid"] for s in ss], precision=MIXED, **KW)
    pos, frc = b.host_buffers()
    pos[:] = np.concatenate([s.coords for s in ss])
    b.set_positions(pos)
    res = b.compute(copy_forces=False)
    ref = _singles(ss, flats, MIXED)
    _same(res, ref, 1e-12)
    assert np.shares_memory(res[0][1], frc)
    rng = np.random.default_rng(4)
    pos += rng.uniform(-0.1, 0.1, pos.shape)          # new frame written in place
    moved = [pos[b.offsets[k]:b.offsets[k + 1]].copy() for k in range(len(ss))]
    b.set_positions(pos)
    _same(b.compute(copy_forces=False), _singles(ss, flats, MIXED, coords=moved), 1e-12)
    b.close()


def test_batch_autotune_keeps_results_and_follows_positions():
    ss = systems()
    flats = _flats(ss)
    b = engine.Batch(flats, [s.box for s in ss], [s.meta["grid"] for s in ss], precision=MIXED, **KW)
    b.set_positions([s.coords for s in ss])
    rep = b.autotune(reps=2)
    assert rep["n_tried"] == 72 and rep["best_ms"] > 0
    assert rep["pair_schedule"] in (0, 1) and rep["pair_layout"] in (0, 1)
    assert rep["pair_warps"] in (2, 4, 8) and rep["fft_lines"] in (2, 4, 8, 16) and rep["prune_every"] in (0, 1)
    shape = dict(prune_every=rep["prune_every"], pair_layout=rep["pair_layout"])
    _same(b.compute(), _singles(ss, flats, MIXED, **shape), 1e-12)
    # moved positions (within the skin): the graph uploads them at every launch
    rng = np.random.default_rng(3)
    moved = [s.coords + rng.uniform(-0.2, 0.2, s.coords.shape) for s in ss]
    b.set_positions(moved)
    _same(b.compute(), _singles(ss, flats, MIXED, coords=moved, **shape), 1e-12)
    b.close()


def test_fp64_batch_matches_oracle():
    ss = systems()[:2]
    flats = _flats(ss)
    b = engine.Batch(flats, [s.box for s in ss], [s.meta["grid"] for s in ss], precision=FP64, **KW)
    b.set_positions([s.coords for s in ss])
    res = b.compute()
    for (E, F), s, f in zip(res, ss, flats):
        p = O.make_params(PHYS, s.box, s.meta["grid"], H.alpha_for(1e-5, 9.0), H.KC, cutoff=9.0, switch=8.0)
        e2, f2, _, _, _ = O.evaluate(f, p, s.coords)
        assert H.frel(F, f2) < 1e-9
        for t in TERMS[:-1]:
            assert abs(E[t] - e2[abi.E_INDEX[t]]) <= 1e-9 * max(1.0, abs(e2[abi.E_INDEX[t]])), t
    b.close()


@pytest.mark.parametrize("layout", [0, 1])
def test_mixed_batch_matches_oracle_every_system(layout):
    """The mixed-precision batch (the c3 workload's precision) against the FP64
    oracle on every member: forces <= 1e-5 rms relative (the mixed-path
    target), total energy 1e-6 relative, each system with its own box and
    PME grid; whole-entry and half-entry pair kernels."""
    ss = systems()
    flats = _flats(ss)
    b = engine.Batch(flats, [s.box for s in ss], [s.meta["grid"] for s in ss], precision=MIXED, pair_layout=layout,
                     **KW)
    b.set_positions([s.coords for s in ss])
    res = b.compute()
    for (E, F), s, f in zip(res, ss, flats):
        p = O.make_params(PHYS, s.box, s.meta["grid"], H.alpha_for(1e-5, 9.0), H.KC, cutoff=9.0, switch=8.0)
        e2, f2, _, _, _ = O.evaluate(f, p, s.coords)
        assert H.frel(F, f2) <= 1e-5, (s.name, H.frel(F, f2))
        tot2 = sum(e2[abi.E_INDEX[t]] for t in TERMS[:-1])
        assert H.rel(E["total"], tot2) < 1e-6, (s.name, E["total"], tot2)
    b.close()


def test_batch_submit_collect_pipelined_equals_compute():
    """Pipelined batches (mdf_batch_submit / mdf_batch_collect, two in flight,
    copies on their own streams) give the plain batch's forces and energies
    bit for bit, frame by frame; a fresh batch's first submission builds its
    lists from the submitted positions."""
    ss = systems()
    flats = _flats(ss)
    rng = np.random.default_rng(21)
    frames = [np.concatenate([s.coords + rng.uniform(-0.1, 0.1, s.coords.shape) for s in ss]) for _ in range(4)]
    b = engine.Batch(flats, [s.box for s in ss], [s.meta["grid"] for s in ss], precision=MIXED, **KW)
    b.set_positions(frames[0])
    b.build_pairlists()
    ref = []
    for x in frames:
        b.set_positions(x)
        res = b.compute()
        ref.append((np.concatenate([f for _, f in res]), [e for e, _ in res]))
    outs = [np.zeros_like(x) for x in frames]
    got = []
    b.submit(frames[0].ctypes.data, outs[0].ctypes.data)
    for k in range(1, len(frames)):
        b.submit(frames[k].ctypes.data, outs[k].ctypes.data)
        got.append(b.collect())
    got.append(b.collect())
    for k in range(len(frames)):
        assert np.array_equal(outs[k].reshape(-1, 3), ref[k][0]), k
        for e, e_ref in zip(got[k], ref[k][1]):
            assert e["total"] == e_ref["total"] and e["ee_recip"] == e_ref["ee_recip"], k
    # a third submission without a collect is refused
    b.submit(frames[0].ctypes.data, outs[0].ctypes.data)
    b.submit(frames[1].ctypes.data, outs[1].ctypes.data)
    with pytest.raises(engine.MDFError):
        b.submit(frames[2].ctypes.data, outs[2].ctypes.data)
    b.collect(); b.collect()
    b.close()
    # fresh batch: the first submission builds the lists
    b2 = engine.Batch(flats, [s.box for s in ss], [s.meta["grid"] for s in ss], precision=MIXED, **KW)
    out = np.zeros_like(frames[0])
    b2.submit(frames[0].ctypes.data, out.ctypes.data)
    e = b2.collect()
    b2.close()
    b3 = engine.Batch(flats, [s.box for s in ss], [s.meta["grid"] for s in ss], precision=MIXED, **KW)
    b3.set_positions(frames[0])
    res = b3.compute()
    b3.close()
    assert np.array_equal(out.reshape(-1, 3), np.concatenate([f for _, f in res]))
    assert all(x["total"] == r[0]["total"] for x, r in zip(e, res))


def test_self_pruning_batch_equals_single_systems():
    """Self-pruning systems (prune_every < 0) in a batch: the captured prune
    kernels decide on the device, frame by frame, exactly as single contexts
    in the same mode do (forces bit for bit over frames that move by up to
    0.05 A against a 0.3 A margin), and within the mixed bound of the oracle."""
    ss = systems()[:3]
    flats = _flats(ss)
    kw = dict(KW, prune_every=-1, prune_margin=0.3)
    b = engine.Batch(flats, [s.box for s in ss], [s.meta["grid"] for s in ss], precision=MIXED, **kw)
    rng = np.random.default_rng(8)
    frames = [[s.coords for s in ss]]
    for _ in range(4):
        frames.append([x + rng.uniform(-0.03, 0.03, x.shape) for x in frames[-1]])
    b.set_positions(frames[0])
    got = []
    for fr in frames:
        b.set_positions(fr)
        got.append(b.compute())
    b.close()
    for k, (s, f) in enumerate(zip(ss, flats)):
        eng = engine.Engine(f, s.box, semantics=PHYS, precision=MIXED, grid=s.meta["grid"], **kw)
        eng.set_positions(frames[0][k])
        eng.build_pairlist()
        for n, fr in enumerate(frames):
            eng.set_positions(fr[k])
            E, F = eng.compute()
            assert np.array_equal(F, got[n][k][1]), (k, n)
        eng.close()
    p = O.make_params(PHYS, ss[0].box, ss[0].meta["grid"], H.alpha_for(1e-5, 9.0), H.KC, cutoff=9.0, switch=8.0)
    e2, f2, _, _, _ = O.evaluate(flats[0], p, frames[-1][0])
    assert H.frel(got[-1][0][1], f2) <= 1e-5


@pytest.mark.parametrize("prec", [MIXED, FP64])
def test_batch_with_a_large_lj_table_equals_single_systems(prec):
    """One member with 60 LJ types (its pair table does not fit the pair
    kernels' shared memory): the whole batch reads the tables from global
    memory and still equals the single systems bit for bit."""
    ss = systems()[:3]
    flats = _flats(ss)
    flats[1] = H.many_types(flats[1])
    b = engine.Batch(flats, [s.box for s in ss], [s.meta["grid"] for s in ss], precision=prec, **KW)
    b.set_positions([s.coords for s in ss])
    res = b.compute()
    _same(res, _singles(ss, flats, prec))
    b.close()
