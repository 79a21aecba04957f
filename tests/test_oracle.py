"""The oracles themselves: O2 (FP64 restatement) pinned against the
unmodified reference (O1 golden fixtures), plus physics known-answer tests
for the PHYSICAL semantics.  CPU only."""
import math
import os

import numpy as np
import pytest

from md_b200 import abi
from oracle import oracle as O
from tests import helpers as H

REF, PHYS = abi.MDF_SEM_REFERENCE, abi.MDF_SEM_PHYSICAL
E_REF_TERMS = ["bond", "angle", "dihedral", "ub", "improper", "cmap", "vdw", "ee", "ee_pairlist", "ee_cutoff",
               "ee_direct", "ee_self"]


def test_fft_ref_matches_numpy():
    import ctypes as C
    lib = C.CDLL(O.LIB)
    lib.fft_ref_r2c_3d.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]
    lib.fft_ref_c2r_3d.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]
    rng = np.random.default_rng(0)
    for shape in [(6, 10, 8), (12, 9, 15), (5, 7, 11)]:
        x = rng.normal(size=shape)
        out = np.zeros(shape[:2] + (shape[2] // 2 + 1,), dtype=np.complex128)
        lib.fft_ref_r2c_3d(x.ctypes.data, out.ctypes.data, *shape)
        assert np.abs(out - np.fft.rfftn(x)).max() < 1e-10
        back = np.zeros(shape)
        lib.fft_ref_c2r_3d(out.ctypes.data, back.ctypes.data, *shape)
        assert np.abs(back / np.prod(shape) - x).max() < 1e-12


@pytest.mark.parametrize("case", ["tiny", "tiny_sentinel", "small"])
def test_golden_inputs_regenerate(case):
    g = H.golden(case)
    s = H.system(g["meta"]["config"], g["meta"]["sentinels"])
    assert H.files_sha(s) == [g["meta"]["sha_prmtop"], g["meta"]["sha_rst7"]]


@pytest.mark.parametrize("case", ["tiny", "tiny_sentinel", "small", "c0"])
def test_o2_reference_matches_o1(case):
    """O2 in REFERENCE semantics reproduces the unmodified reference's numbers."""
    g = H.golden(case)
    m = g["meta"]
    s = H.system(m["config"], m["sentinels"])
    flat = H.flat(s, REF)
    p = O.make_params(REF, s.box, m["grid"], m["alpha"], H.KC)
    e, f, _, fp, _ = O.evaluate(flat, p, s.coords, pme_ref=True)
    for k in E_REF_TERMS:
        assert H.rel(e[abi.E_INDEX[k]], g["energies"][k]) < 1e-12, (k, e[abi.E_INDEX[k]], g["energies"][k])
    H.check_forces_vs_golden(f, g, 1e-12, "forces")
    H.check_forces_vs_golden(fp, g, 1e-12, "forces_pme")


def test_sentinels_make_semantics_agree_on_term_sets():
    """With a zero-constant tuple appended to every list the reference's
    loaders truncate, REFERENCE and PHYSICAL flattenings hold the same terms."""
    s = H.system("tiny", True)
    a, b = H.flat(s, REF), H.flat(s, PHYS)
    for name in ["bond_atoms", "angle_atoms", "dihedral_atoms", "ub_atoms", "cmap_atoms", "improper_atoms"]:
        ra, rb = getattr(a, name), getattr(b, name)
        w = {"bond_atoms": 2, "ub_atoms": 2, "angle_atoms": 3, "dihedral_atoms": 4, "improper_atoms": 4,
             "cmap_atoms": 5}[name]
        real_a = ra.reshape(-1, w)
        real_b = rb.reshape(-1, w)
        if name == "improper_atoms":
            assert np.array_equal(real_a, real_b)
        else:
            # PHYSICAL has exactly the sentinel rows more
            assert len(real_b) >= len(real_a)


def _fd_check(flat, p, x, atoms, h=1e-5):
    e, f, _, _, _ = O.evaluate(flat, p, x)
    worst = 0.0
    for a in atoms:
        for k in range(3):
            xp, xm = x.copy(), x.copy()
            xp[a, k] += h
            xm[a, k] -= h
            ep = O.evaluate(flat, p, xp, want_forces=False)[0].sum()
            em = O.evaluate(flat, p, xm, want_forces=False)[0].sum()
            fd = -(ep - em) / (2 * h)
            worst = max(worst, abs(fd - f[a, k]) / (1 + abs(fd)))
    return worst


def test_o2_physical_forces_are_minus_gradient():
    s = H.system("tiny")
    flat = H.flat(s, PHYS)
    p = O.make_params(PHYS, s.box, (24, 24, 24), H.alpha_for(1e-5), H.KC)
    atoms = list(range(0, 30, 2)) + [100, 400, 845]
    assert _fd_check(flat, p, s.coords.copy(), atoms) < 1e-6


def test_reference_torsion_forces_are_not_minus_gradient():
    """Documents the reference's torsion-force formulas (src/System/BondedForces.cpp:193-239):
    with bonded terms alone, REFERENCE forces on the chain differ from -dE/dx
    while PHYSICAL forces match it."""
    s = H.system("tiny")
    flat = H.flat(s, REF)
    flat.charge = np.zeros_like(flat.charge)
    flat.nb_index = np.zeros_like(flat.nb_index)
    flat._struct = None
    p_ref = O.make_params(REF, s.box, (24, 24, 24), H.alpha_for(1e-5), H.KC, allpairs=False)
    p_phys = O.make_params(PHYS, s.box, (24, 24, 24), H.alpha_for(1e-5), H.KC, recip=False)
    atoms = list(range(0, 30, 3))
    assert _fd_check(flat, p_phys, s.coords.copy(), atoms) < 1e-6
    assert _fd_check(flat, p_ref, s.coords.copy(), atoms) > 1e-2


def test_pme_converges_to_exact_ewald():
    s = H.system("tiny")
    flat = H.flat(s, PHYS)
    alpha = H.alpha_for(1e-5)
    e_ex, f_ex = O.ewald_recip_exact(s.q, s.coords, s.box, alpha, H.KC, 14)
    errs = []
    for K in (24, 48):
        p = O.make_params(PHYS, s.box, (K, K, K), alpha, H.KC)
        e, f, _ = O.pme_recip(flat, p, s.coords)
        errs.append((H.rel(e, e_ex), H.frel(f, f_ex)))
    assert errs[0][0] < 3e-3 and errs[1][0] < 1e-4
    assert errs[1][1] < 3e-4
    assert errs[1][0] < errs[0][0] / 10          # order-4 convergence


def test_madelung_constant_nacl():
    """Known answer: rock salt Madelung constant 1.747565 from direct + reciprocal + self."""
    x, q, box = H.nacl_crystal(4, 5.64)
    flat = H.simple_flat(q)
    alpha = 0.42          # erfc(alpha rc) ~ 3e-9: real-space truncation below the tolerance
    p = O.make_params(PHYS, box, (64, 64, 64), alpha, H.KC, switch=0.0)
    e, _, _, _, _ = O.evaluate(flat, p, x, want_forces=False)
    etot = e[abi.E_INDEX["ee_direct"]] + e[abi.E_INDEX["ee_recip"]] + e[abi.E_INDEX["ee_self"]]
    r0 = 5.64 / 2
    M = -etot / (len(q) / 2) * r0 / H.KC
    assert abs(M - H.MADELUNG_NACL) < 2e-6, M
    # exact reciprocal sum: tighter
    er, _ = O.ewald_recip_exact(q, x, box, alpha, H.KC, 18)
    etot2 = e[abi.E_INDEX["ee_direct"]] + er + e[abi.E_INDEX["ee_self"]]
    M2 = -etot2 / (len(q) / 2) * r0 / H.KC
    assert abs(M2 - H.MADELUNG_NACL) < 1e-7, M2


def test_virial_is_minus_box_strain_derivative():
    s = H.system("tiny")
    flat = H.flat(s, PHYS)
    alpha = 0.33

    def erec(eps, d):
        box = s.box.copy(); x = s.coords.copy()
        box[d] *= 1 + eps; x[:, d] *= 1 + eps
        return O.pme_recip(flat, O.make_params(PHYS, box, (32, 32, 32), alpha, H.KC), x)[0]
    _, _, vir = O.pme_recip(flat, O.make_params(PHYS, s.box, (32, 32, 32), alpha, H.KC), s.coords)
    for d in range(3):
        h = 1e-5
        dE = (erec(h, d) - erec(-h, d)) / (2 * h)
        assert abs(vir[4 * d] + dE) < 1e-6 * max(1.0, abs(dE))


@pytest.mark.skipif(not os.path.exists(O.O1), reason="O1 harness not built")
def test_o1_harness_reproduces_golden():
    """The compiled reference still gives the committed numbers (tiny)."""
    g = H.golden("tiny")
    res = O.run_o1(os.path.join(g["dir"], "tiny.prmtop"), os.path.join(g["dir"], "tiny.rst7"), g["meta"]["grid"])
    for k in E_REF_TERMS:
        assert res["energies"][k] == g["energies"][k]
    assert np.array_equal(res["forces"], g["forces"])
