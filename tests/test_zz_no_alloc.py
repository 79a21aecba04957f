"""mdf_compute_bonded_noalloc against the regular evaluation.

The no-allocation entry point computes the bonded terms with scratch in a
static device array.  Its energies are compared with the bonded entries of
mdf_compute on the full topology, and its forces with mdf_compute on the same
topology with every charge and Lennard-Jones coefficient set to zero (so the
regular path's forces are the bonded forces alone).  Both are fixed-point
sums of the same FP64 terms, so the tolerance is tight: 1e-12 relative.
Each comparison runs on two calls in a row, so stale scratch from the first
call would show up in the second.

This file is collected last: it must pass both alone in a fresh process and
after every other test has run in the same process.
"""
import numpy as np
import pytest

from md_b200 import abi, engine, synth, topology
from tests import helpers as H

pytestmark = pytest.mark.gpu
BONDED = ["bond", "angle", "dihedral", "ub", "improper", "cmap"]


def _engine(flat, s, sem, prec):
    eng = engine.Engine(flat, s.box, semantics=sem, precision=prec, ewald_tol=1e-5, grid=synth.GRIDS["tiny"])
    eng.set_positions(s.coords)
    eng.build_pairlist()
    return eng


def _bonded_only(flat):
    z = topology.FlatTopology(**{k: v for k, v in flat.__dict__.items() if not k.startswith("_")})
    for k in ("charge", "lj_a", "lj_b", "lj14_a", "lj14_b"):
        setattr(z, k, np.zeros_like(getattr(flat, k)))
    return z


@pytest.mark.parametrize("sem", [abi.MDF_SEM_PHYSICAL, abi.MDF_SEM_REFERENCE])
@pytest.mark.parametrize("prec", [abi.MDF_PREC_FP64, abi.MDF_PREC_MIXED])
def test_noalloc_bonded_matches_compute(sem, prec):
    import torch
    s = H.system("tiny")
    flat = H.flat(s, sem, engine.cmap_coefficients)
    full = _engine(flat, s, sem, prec)
    E_full, _ = full.compute()
    bo = _engine(_bonded_only(flat), s, sem, prec)
    _, F_bonded = bo.compute()
    assert np.abs(F_bonded).max() > 0
    d_f = torch.full((3 * s.natoms,), float("nan"), dtype=torch.float64, device="cuda")
    for call in range(2):
        E = full.bonded_noalloc(d_f.data_ptr())
        torch.cuda.synchronize()
        F = d_f.cpu().numpy().reshape(-1, 3)
        for k in BONDED:
            assert H.rel(E[k], E_full[k]) < 1e-12, (call, k, E[k], E_full[k])
        assert H.rel(E["total"], sum(E_full[k] for k in BONDED)) < 1e-12
        assert H.frel(F, F_bonded) < 1e-12, (call, H.frel(F, F_bonded))
    # energies only: no force array needed
    E = full.bonded_noalloc(0)
    assert H.rel(E["bond"], E_full["bond"]) < 1e-12
    full.close()
    bo.close()


def test_noalloc_rejects_oversize_system():
    n = abi.MDF_NOALLOC_MAX_ATOMS + 1
    side = 1.0 + int(np.ceil(n ** (1 / 3)))
    g = np.stack(np.meshgrid(*[np.arange(side)] * 3, indexing="ij"), -1).reshape(-1, 3)[:n] * 3.0
    flat = H.simple_flat(np.zeros(n))
    box = [3.0 * side] * 3
    eng = engine.Engine(flat, box, semantics=abi.MDF_SEM_PHYSICAL, precision=abi.MDF_PREC_MIXED, ewald_tol=1e-5,
                        grid=[32, 32, 32])
    eng.set_positions(g)
    with pytest.raises(engine.MDFError) as ei:
        eng.bonded_noalloc(0)
    assert ei.value.status == abi.MDF_ERR_INVALID
    assert "static scratch limit" in str(ei.value)
    eng.close()
