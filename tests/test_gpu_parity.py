"""GPU parity: libmdf (through its C ABI) against the oracles.

Tolerances:
  REFERENCE, FP64 vs the unmodified reference (golden O1 fixtures):
      energies 1e-9 relative, forces 1e-9 rms relative (spec: 1e-6 / 1e-5);
      the reference's PME-chain forces 1e-8 (the GPU charge grid is int64
      fixed point at 2^-40).
  PHYSICAL, FP64 vs O2: energies 1e-9 relative, forces 1e-9 rms relative.
  PHYSICAL, MIXED vs O2: forces <= 1e-5 rms relative (the target), total
      energy 1e-6 relative.
"""
import math

import numpy as np
import pytest

from md_b200 import abi, engine, synth
from oracle import oracle as O
from tests import helpers as H

pytestmark = pytest.mark.gpu
REF, PHYS = abi.MDF_SEM_REFERENCE, abi.MDF_SEM_PHYSICAL
FP64, MIXED = abi.MDF_PREC_FP64, abi.MDF_PREC_MIXED
E_REF_TERMS = ["bond", "angle", "dihedral", "ub", "improper", "cmap", "vdw", "ee", "ee_pairlist", "ee_cutoff",
               "ee_direct", "ee_self"]
E_PHYS_TERMS = ["bond", "angle", "dihedral", "ub", "improper", "cmap", "vdw", "vdw14", "ee_direct", "ee14",
                "ee_excl", "ee_self", "ee_recip"]


def make_engine(s, sem, prec, grid, tol=1e-5, **kw):
    flat = H.flat(s, sem, engine.cmap_coefficients)
    eng = engine.Engine(flat, s.box, semantics=sem, precision=prec, ewald_tol=tol, grid=grid, **kw)
    eng.set_positions(s.coords)
    eng.build_pairlist()
    return eng, flat


@pytest.mark.parametrize("case", ["tiny", "tiny_sentinel", "small", "c0", "c1"])
def test_reference_fp64_matches_reference_cpu(case):
    g = H.golden(case)
    m = g["meta"]
    s = H.system(m["config"], m["sentinels"])
    eng, _ = make_engine(s, REF, FP64, m["grid"])
    E, F = eng.compute(pme_reference=True)
    for k in E_REF_TERMS:
        assert H.rel(E[k], g["energies"][k]) < 1e-9, (k, E[k], g["energies"][k])
    H.check_forces_vs_golden(F, g, 1e-9, "forces")
    H.check_forces_vs_golden(eng.pme_forces(), g, 1e-8, "forces_pme")
    eng.close()


@pytest.mark.parametrize("cfg", ["tiny", "small", "c0", "c1"])
def test_physical_fp64_matches_o2(cfg):
    """The FP64 GPU path (the denominator of the mixed/FP64 ratio) against O2,
    up to the 100k-atom workload the ratio is quoted on."""
    s = H.system(cfg)
    grid = synth.GRIDS[cfg]
    eng, flat = make_engine(s, PHYS, FP64, grid)
    E, F = eng.compute()
    e2, f2, vir2, _, np2 = H.o2_physical(cfg, flat)
    for k in E_PHYS_TERMS:
        ref = e2[abi.E_INDEX[k]]
        assert abs(E[k] - ref) <= 1e-9 * max(abs(ref), 1.0), (k, E[k], ref)
    assert H.frel(F, f2) < 1e-9
    assert np.allclose(E["virial"].ravel(), vir2, rtol=1e-9, atol=1e-7)
    assert eng.pairlist_info()["pairs_in_cutoff"] == np2
    eng.close()


@pytest.mark.parametrize("cfg", ["small", "c0", "c1"])
def test_mixed_precision_force_error_below_1e5(cfg):
    s = H.system(cfg)
    grid = synth.GRIDS[cfg]
    eng, flat = make_engine(s, PHYS, MIXED, grid)
    E, F = eng.compute()
    e2, f2, _, _, _ = H.o2_physical(cfg, flat)
    err = H.frel(F, f2)
    assert err <= 1e-5, err
    tot2 = sum(e2[abi.E_INDEX[k]] for k in E_PHYS_TERMS)
    assert H.rel(E["total"], tot2) < 1e-6
    eng.close()


@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_bit_reproducible(prec):
    s = H.system("small")
    eng, _ = make_engine(s, PHYS, prec, (32, 32, 32))
    E1, F1 = eng.compute()
    E2, F2 = eng.compute()
    assert np.array_equal(F1, F2)
    assert all(E1[k] == E2[k] for k in E_PHYS_TERMS)
    # a fresh context (fresh pairlist build) gives the same bits too
    eng2, _ = make_engine(s, PHYS, prec, (32, 32, 32))
    E3, F3 = eng2.compute()
    assert np.array_equal(F1, F3)
    eng.close(); eng2.close()


def test_periodic_images_of_positions_give_identical_results():
    """Whole-box shifts of individual molecules change nothing (min image)."""
    s = H.system("small")
    eng, flat = make_engine(s, PHYS, FP64, (32, 32, 32))
    E1, F1 = eng.compute()
    x = s.coords.copy()
    nchain = s.meta["n_chain"]
    # shift every water molecule by a random whole-box vector
    rng = np.random.default_rng(3)
    for w in range(nchain, s.natoms, 3):
        x[w:w + 3] += rng.integers(-2, 3, 3) * s.box
    eng.set_positions(x)
    eng.build_pairlist()
    E2, F2 = eng.compute()
    assert H.frel(F2, F1) < 1e-10
    assert H.rel(E2["total"], E1["total"]) < 1e-10
    eng.close()


def test_list_reuse_within_skin_matches_rebuild():
    s = H.system("small")
    eng, flat = make_engine(s, PHYS, FP64, (32, 32, 32))
    rng = np.random.default_rng(5)
    x = s.coords + rng.uniform(-0.4, 0.4, s.coords.shape)   # < skin/2
    eng.set_positions(x)
    E1, F1 = eng.compute()           # old list
    eng.build_pairlist()
    E2, F2 = eng.compute()           # new list
    assert H.frel(F1, F2) < 1e-10
    assert H.rel(E1["total"], E2["total"]) < 1e-10
    eng.close()


def test_force_shifted_lj_and_noncubic_box():
    s = synth.make_system("nc", (31.0, 27.5, 36.0), 900, 6, seed=77)
    grid = (32, 27, 36)
    flat = H.flat(s, PHYS, engine.cmap_coefficients)
    eng = engine.Engine(flat, s.box, semantics=PHYS, precision=FP64, ewald_tol=1e-5, grid=grid, switch_radius=0.0)
    eng.set_positions(s.coords)
    E, F = eng.compute()
    p = O.make_params(PHYS, s.box, grid, H.alpha_for(1e-5), H.KC, switch=0.0)
    e2, f2, _, _, _ = O.evaluate(flat, p, s.coords)
    assert H.frel(F, f2) < 1e-9
    for k in E_PHYS_TERMS:
        ref = e2[abi.E_INDEX[k]]
        assert abs(E[k] - ref) <= 1e-9 * max(abs(ref), 1.0), k
    eng.close()


def test_smallest_box_two_cutoffs():
    """Box edge exactly twice the cutoff: several images per cluster pair."""
    s = synth.make_system("b20", 20.0, 250, 2, seed=8)
    flat = H.flat(s, PHYS, engine.cmap_coefficients)
    eng = engine.Engine(flat, s.box, semantics=PHYS, precision=FP64, ewald_tol=1e-5, grid=(20, 20, 20))
    eng.set_positions(s.coords)
    E, F = eng.compute()
    p = O.make_params(PHYS, s.box, (20, 20, 20), H.alpha_for(1e-5), H.KC)
    e2, f2, _, _, np2 = O.evaluate(flat, p, s.coords)
    assert H.frel(F, f2) < 1e-9
    assert eng.pairlist_info()["pairs_in_cutoff"] == np2
    eng.close()


def test_pure_water_no_bonded_chain():
    s = synth.make_system("w", 24.0, 460, 0, seed=9)
    eng, flat = make_engine(s, PHYS, MIXED, (24, 24, 24))
    E, F = eng.compute()
    p = O.make_params(PHYS, s.box, (24, 24, 24), H.alpha_for(1e-5), H.KC)
    e2, f2, _, _, _ = O.evaluate(flat, p, s.coords)
    assert H.frel(F, f2) < 1e-5
    eng.close()


def test_nacl_madelung_on_gpu():
    x, q, box = H.nacl_crystal(4, 5.64)
    flat = H.simple_flat(q)
    eng = engine.Engine(flat, box, semantics=PHYS, precision=FP64, ewald_alpha=0.42, grid=(64, 64, 64),
                        switch_radius=0.0)
    eng.set_positions(x)
    E, F = eng.compute()
    etot = E["ee_direct"] + E["ee_recip"] + E["ee_self"]
    M = -etot / (len(q) / 2) * (5.64 / 2) / H.KC
    assert abs(M - H.MADELUNG_NACL) < 2e-6
    assert np.abs(F).max() < 1e-6          # perfect lattice: no net force
    eng.close()


@pytest.mark.parametrize("prec", [MIXED, FP64])
def test_many_lj_types_table_in_global_memory(prec):
    """60 LJ types: the 61 x 61 pair table exceeds the shared-memory budget
    of the pair kernels (40 KB FP32, 96 KB FP64), so they read it from global
    memory (the other form of their body); both precisions against O2."""
    s = H.system("small")
    flat = H.many_types(H.flat(s, PHYS, engine.cmap_coefficients))
    grid = synth.GRIDS["small"]
    eng = engine.Engine(flat, s.box, semantics=PHYS, precision=prec, ewald_tol=1e-5, grid=grid)
    eng.set_positions(s.coords)
    eng.build_pairlist()
    E, F = eng.compute()
    p = O.make_params(PHYS, s.box, grid, H.alpha_for(1e-5), H.KC)
    e2, f2, _, _, np2 = O.evaluate(flat, p, s.coords)
    if prec == FP64:
        assert H.frel(F, f2) < 1e-9
        for k in ("vdw", "vdw14", "ee_direct"):
            ref = e2[abi.E_INDEX[k]]
            assert abs(E[k] - ref) <= 1e-9 * max(abs(ref), 1.0), (k, E[k], ref)
    else:
        assert H.frel(F, f2) < 1e-5
        ref = e2[abi.E_INDEX["vdw"]]
        assert abs(E["vdw"] - ref) <= 1e-5 * max(abs(ref), 1.0), (E["vdw"], ref)
    # FP32 distances may put a pair within an ulp of the cutoff on the other side
    slack = 0 if prec == FP64 else 2
    assert abs(eng.pairlist_info()["pairs_in_cutoff"] - np2) <= slack
    eng.close()


@pytest.mark.parametrize("tol", [0.5, 0.9])
def test_ewald_tolerance_without_splitting_rejected(tol):
    # sqrt(-ln(2 tol)) has no positive value for tol >= 0.5
    s = H.system("tiny")
    flat = H.flat(s, PHYS, engine.cmap_coefficients)
    with pytest.raises(engine.MDFError) as e:
        engine.Engine(flat, s.box, semantics=PHYS, precision=MIXED, ewald_tol=tol, grid=(24, 24, 24))
    assert e.value.status == 1


def test_nonfinite_position_reported_not_faulted():
    s = H.system("tiny")
    eng, _ = make_engine(s, PHYS, MIXED, (24, 24, 24))
    x = s.coords.copy()
    x[5, 1] = np.nan
    eng.set_positions(x)
    with pytest.raises(engine.MDFError) as e:
        eng.compute()
    assert e.value.status == 4
    # the context stays usable
    eng.set_positions(s.coords)
    E, F = eng.compute()
    assert np.isfinite(F).all()
    eng.close()


@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_pruned_list_matches_unpruned(prec):
    """Pruning only drops cluster pairs without an atom pair inside the
    cutoff: the pruned evaluation equals the unpruned one up to the order in
    which the pair kernel sums (entries move between lanes)."""
    s = H.system("small")
    flat = H.flat(s, PHYS, engine.cmap_coefficients)
    out = []
    for every in (0, 1):
        eng = engine.Engine(flat, s.box, semantics=PHYS, precision=prec, ewald_tol=1e-5, grid=(32, 32, 32),
                            prune_every=every)
        eng.set_positions(s.coords)
        out.append(eng.compute())
        info = eng.pairlist_info()
        if every:
            assert 0 < info["cluster_pairs_pruned"] < info["cluster_pairs"]
        eng.close()
    (E0, F0), (E1, F1) = out
    tol = 1e-12 if prec == FP64 else 1e-6
    assert H.frel(F1, F0) < tol
    assert all(abs(E0[k] - E1[k]) <= tol * max(1.0, abs(E0[k])) for k in E_PHYS_TERMS)


def test_prune_interval_with_margin_tracks_moving_atoms():
    """Prune every 4 evaluations with a 1 A margin while atoms drift by up to
    0.1 A per evaluation: forces equal an exact (per-evaluation) prune."""
    s = H.system("small")
    flat = H.flat(s, PHYS, engine.cmap_coefficients)
    a = engine.Engine(flat, s.box, semantics=PHYS, precision=FP64, ewald_tol=1e-5, grid=(32, 32, 32),
                      prune_every=4, prune_margin=1.0)
    b = engine.Engine(flat, s.box, semantics=PHYS, precision=FP64, ewald_tol=1e-5, grid=(32, 32, 32))
    rng = np.random.default_rng(11)
    x = s.coords.copy()
    for step in range(9):
        a.set_positions(x)
        b.set_positions(x)
        Ea, Fa = a.compute()
        Eb, Fb = b.compute()
        assert H.frel(Fa, Fb) < 1e-12, step
        x = x + rng.uniform(-0.1, 0.1, x.shape)
    a.close(); b.close()


@pytest.mark.parametrize("layout", [0, 1])
@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_self_pruning_tracks_moving_atoms(prec, layout):
    """prune_every < 0: the pack kernel measures the largest displacement
    since the last prune and the prune kernel re-prunes only beyond
    prune_margin / 2.  Atoms drift up to 0.05 A per evaluation against a
    0.3 A margin, so the lists are reused for some evaluations and re-pruned
    on the device for others: forces equal an exact prune at every evaluation
    (FP64 to 1e-12; mixed to the order of the FP32 sums) and the reported list
    holds at least the exact prune's entries."""
    s = H.system("small")
    flat = H.flat(s, PHYS, engine.cmap_coefficients)
    kw = dict(semantics=PHYS, precision=prec, ewald_tol=1e-5, grid=(32, 32, 32), pair_layout=layout)
    a = engine.Engine(flat, s.box, prune_every=-1, prune_margin=0.3, **kw)
    b = engine.Engine(flat, s.box, prune_every=1, **kw)
    rng = np.random.default_rng(12)
    x = s.coords.copy()
    a.set_positions(x); a.build_pairlist()
    b.set_positions(x); b.build_pairlist()
    tol = 1e-12 if prec == FP64 else 1e-6
    for step in range(12):
        a.set_positions(x)
        b.set_positions(x)
        Ea, Fa = a.compute()
        Eb, Fb = b.compute()
        assert H.frel(Fa, Fb) < tol, step
        assert abs(Ea["total"] - Eb["total"]) <= tol * abs(Eb["total"]) + 1e-8, step
        assert a.pairlist_info()["cluster_pairs_pruned"] >= b.pairlist_info()["cluster_pairs_pruned"]
        x = x + rng.uniform(-0.03, 0.03, x.shape)
    a.close(); b.close()


@pytest.mark.parametrize("prec", [FP64, MIXED])
@pytest.mark.parametrize("n,charged", [(1, True), (2, True), (2, False), (9, True), (17, False)])
def test_few_atoms_match_o2(n, charged, prec):
    """Ragged sizes: one atom (a lone cluster, only self and net-charge
    reciprocal terms), one pair, one full cluster plus one, two clusters
    plus one; charged and neutral LJ-only atoms (the PME chain on an empty
    charge grid)."""
    rng = np.random.default_rng(100 + n)
    box = np.full(3, 24.0)
    x = rng.uniform(0.0, 24.0, (n, 3))
    while n > 1 and min(np.linalg.norm(((x[i] - x[j] + 12) % 24) - 12) for i in range(n)
                        for j in range(i)) < 2.5:
        x = rng.uniform(0.0, 24.0, (n, 3))
    q = rng.normal(0.0, 0.5, n) if charged else np.zeros(n)
    flat = H.simple_flat(q, lj_a=[6.0e5], lj_b=[600.0])
    eng = engine.Engine(flat, box, semantics=PHYS, precision=prec, ewald_tol=1e-5, grid=(24, 24, 24))
    eng.set_positions(x)
    E, F = eng.compute()
    p = O.make_params(PHYS, box, (24, 24, 24), H.alpha_for(1e-5), H.KC)
    e2, f2, _, _, np2 = O.evaluate(flat, p, x)
    # mixed: largest component error against the largest force, with a floor
    # of 1e-5 kcal/mol/A (FP32 grid noise; a lone charge feels only the
    # ~4e-3 discretisation force of the mesh)
    tol, floor = (1e-9, 1e-9) if prec == FP64 else (5e-5, 1e-5)
    scale = max(np.abs(f2).max(), 1e-12)
    assert np.abs(F - f2).max() <= tol * scale + floor, (np.abs(F - f2).max(), scale)
    for k in ("vdw", "ee_direct", "ee_self", "ee_recip"):
        ref = e2[abi.E_INDEX[k]]
        assert abs(E[k] - ref) <= tol * max(abs(ref), 1.0), (k, E[k], ref)
    assert eng.pairlist_info()["pairs_in_cutoff"] == np2
    eng.close()


@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_autotune_keeps_forces_and_reports(prec):
    """mdf_autotune tries 72 launch shapes and keeps the fastest."""
    s = H.system("small")
    eng, _ = make_engine(s, PHYS, prec, synth.GRIDS["small"])
    E0, F0 = eng.compute()
    rep = eng.autotune(reps=2)
    assert rep["n_tried"] == 72 and rep["best_ms"] > 0 and rep["best_ms"] <= rep["default_ms"]
    assert rep["pair_schedule"] in (0, 1) and rep["pair_layout"] in (0, 1)
    assert rep["pair_warps"] in (2, 4, 8) and rep["fft_lines"] in (2, 4, 8, 16) and rep["prune_every"] in (0, 1)
    E1, F1 = eng.compute()
    # the launch shape changes only the order of FP32 sums (MIXED); a fresh
    # context with the chosen shape reproduces the tuned one bit for bit
    tol = 1e-10 if prec == FP64 else 1e-6
    assert H.frel(F1, F0) < tol
    assert abs(E1["total"] - E0["total"]) <= tol * abs(E0["total"]) + 1e-8
    flat = H.flat(s, PHYS, engine.cmap_coefficients)
    eng2 = engine.Engine(flat, s.box, semantics=PHYS, precision=prec, ewald_tol=1e-5, grid=synth.GRIDS["small"],
                         prune_every=rep["prune_every"], pair_warps=rep["pair_warps"], fft_lines=rep["fft_lines"],
                         pair_schedule=rep["pair_schedule"], pair_layout=rep["pair_layout"])
    eng2.set_positions(s.coords)
    eng2.build_pairlist()
    E2, F2 = eng2.compute()
    assert np.array_equal(F1, F2)
    assert E1["total"] == E2["total"]
    eng.close(); eng2.close()


@pytest.mark.parametrize("prec", [FP64, MIXED])
@pytest.mark.parametrize("cfg", ["small", "c1"])
@pytest.mark.parametrize("schedule", [0, 1])
def test_half_layout_matches_o2(cfg, prec, schedule):
    """The half-entry (4 x 8) pair kernel: the same pairs as the whole-entry
    kernel (pairs_in_cutoff equal), forces against O2 at the precision's
    bound, and equal to the whole-entry evaluation up to FP32 sum order."""
    s = H.system(cfg)
    grid = synth.GRIDS[cfg]
    flat = H.flat(s, PHYS, engine.cmap_coefficients)
    out = []
    for layout in (0, 1):
        eng = engine.Engine(flat, s.box, semantics=PHYS, precision=prec, ewald_tol=1e-5, grid=grid,
                            pair_layout=layout, pair_schedule=schedule)
        eng.set_positions(s.coords)
        eng.build_pairlist()
        E, F = eng.compute()
        E2, F2 = eng.compute()
        assert np.array_equal(F, F2)
        out.append((E, F, eng.pairlist_info()["pairs_in_cutoff"]))
        eng.close()
    (E0, F0, n0), (E1, F1, n1) = out
    e2, f2, _, _, np2 = H.o2_physical(cfg, flat)
    if prec == FP64:
        assert n0 == n1 == np2
    else:
        # FP32 pair vectors (~1e-6 A) decide the pairs at r = rc: the
        # synthetic lattices put a few pairs exactly on the cutoff
        assert abs(n0 - np2) <= 4 and abs(n1 - np2) <= 4, (n0, n1, np2)
    if prec == FP64:
        assert H.frel(F1, f2) < 1e-9
        assert H.frel(F1, F0) < 1e-10   # FP64 sums of each i atom's force in another order
        for k in E_PHYS_TERMS:
            ref = e2[abi.E_INDEX[k]]
            assert abs(E1[k] - ref) <= 1e-9 * max(abs(ref), 1.0), (k, E1[k], ref)
    else:
        assert H.frel(F1, f2) <= 1e-5
        assert H.frel(F1, F0) < 1e-6
        tot2 = sum(e2[abi.E_INDEX[k]] for k in E_PHYS_TERMS)
        assert H.rel(E1["total"], tot2) < 1e-6


@pytest.mark.parametrize("case", ["tiny", "tiny_sentinel", "small"])
def test_reference_mixed_matches_reference_cpu(case):
    """REFERENCE semantics in mixed precision (FP32 pair arithmetic, the
    reference's order-5 PME chain in FP32) against the unmodified reference:
    forces to 1e-5 rms relative, every continuous energy term to 1e-5
    relative (absolute floor 1e-4 kcal/mol for terms near zero).  The plain
    Coulomb sums truncated at r = rc ("ee", "ee_pairlist") jump by k q q / rc
    when a pair crosses the cutoff, and FP32 rounding of r^2 moves pairs that
    lie within ~1e-6 A of it across: those two are held to 1e-3."""
    g = H.golden(case)
    m = g["meta"]
    s = H.system(m["config"], m["sentinels"])
    eng, _ = make_engine(s, REF, MIXED, m["grid"])
    E, F = eng.compute()
    for k in E_REF_TERMS:
        ref = g["energies"][k]
        tol = 1e-3 if k in ("ee", "ee_pairlist") else 1e-5
        assert abs(E[k] - ref) <= tol * abs(ref) + 1e-4, (k, E[k], ref)
    H.check_forces_vs_golden(F, g, 1e-5, "forces")
    eng.close()


@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_box_change_equals_fresh_context(prec):
    """mdf_set_box with scaled positions gives the forces a context created
    at the new box gives, bit for bit (PME tables, shifts and list rebuilt)."""
    s = H.system("small")
    grid = synth.GRIDS["small"]
    eng, flat = make_engine(s, PHYS, prec, grid)
    eng.compute()
    f = 1.03
    box2, x2 = np.asarray(s.box) * f, s.coords * f
    eng.set_box(box2)
    eng.set_positions(x2)
    E1, F1 = eng.compute()
    e2 = engine.Engine(flat, box2, semantics=PHYS, precision=prec, ewald_tol=1e-5, grid=grid)
    e2.set_positions(x2)
    E2, F2 = e2.compute()
    assert np.array_equal(F1, F2)
    assert abs(E1["total"] - E2["total"]) <= 1e-12 * abs(E2["total"]) + 1e-8
    eng.close(); e2.close()


def test_c4_960k_atoms_fp64_and_mixed_match_o2():
    """The dynamics workload (215 A box, 320,000 flexible waters, 960,000 atoms,
    PME 216^3) at its starting positions: the FP64 GPU path against O2 at
    1e-9, the mixed path against O2 at <= 1e-5 rms relative force error and
    a total energy within 1e-6 of the summed term magnitudes, and mixed
    against FP64 on the GPU."""
    s = H.system("c4")
    grid = synth.GRIDS["c4"]
    e64, flat = make_engine(s, PHYS, FP64, grid)
    E64, F64 = e64.compute()
    e64.close()
    emx, _ = make_engine(s, PHYS, MIXED, grid)
    Emx, Fmx = emx.compute()
    emx.close()
    e2, f2, _, _, _ = H.o2_physical("c4", flat)
    assert H.frel(F64, f2) < 1e-9, H.frel(F64, f2)
    for k in E_PHYS_TERMS:
        ref = e2[abi.E_INDEX[k]]
        assert abs(E64[k] - ref) <= 1e-9 * max(abs(ref), 1.0), (k, E64[k], ref)
    assert H.frel(Fmx, f2) <= 1e-5, H.frel(Fmx, f2)
    assert H.frel(Fmx, F64) <= 1e-5, H.frel(Fmx, F64)
    # the lattice start's total (-3.6e4) is a sum of terms a hundred times
    # larger that nearly cancel: the bound is relative to their magnitudes
    tot2 = sum(e2[abi.E_INDEX[k]] for k in E_PHYS_TERMS)
    scale = sum(abs(e2[abi.E_INDEX[k]]) for k in E_PHYS_TERMS)
    assert abs(Emx["total"] - tot2) <= 1e-6 * scale, (Emx["total"], tot2, scale)


@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_pipelined_submit_collect_equals_compute(prec):
    """mdf_submit / mdf_collect with two evaluations in flight (positions in and
    forces out on the copy stream) give mdf_compute's forces and energies bit
    for bit, each evaluation at its own positions."""
    import torch
    s = H.system("small")
    eng, flat = make_engine(s, PHYS, prec, (32, 32, 32))
    rng = np.random.default_rng(11)
    frames = [s.coords + rng.uniform(-0.05, 0.05, s.coords.shape) for _ in range(5)]
    ref = []
    for x in frames:
        eng.set_positions(x)
        ref.append(eng.compute())
    xs = [torch.from_numpy(np.ascontiguousarray(x.reshape(-1))).pin_memory() for x in frames]
    fs = [torch.empty(3 * s.natoms, dtype=torch.float64).pin_memory() for _ in frames]
    out = []
    eng.submit(xs[0].data_ptr(), fs[0].data_ptr())
    for k in range(1, len(frames)):
        eng.submit(xs[k].data_ptr(), fs[k].data_ptr())
        out.append(eng.collect())
    out.append(eng.collect())
    for k, (E, F) in enumerate(ref):
        assert np.array_equal(fs[k].numpy().reshape(-1, 3), F), k
        assert all(out[k][t] == E[t] for t in E_PHYS_TERMS), k
    with pytest.raises(engine.MDFError):
        eng.collect()                 # nothing in flight
    eng.close()
