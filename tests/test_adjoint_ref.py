"""The FP64 PyTorch reference used for mdf_backward agrees with the oracle's
PHYSICAL energies and forces (so its autograd gradients are the gradients of
the same function the engine computes)."""
import numpy as np
import pytest

from md_b200 import abi, synth, topology
from oracle import oracle as O
from tests import helpers as H
from tests.adjoint_ref import NonbondedRef

PHYS = abi.MDF_SEM_PHYSICAL
TERMS = ["vdw", "vdw14", "ee_direct", "ee14", "ee_excl", "ee_self", "ee_recip"]


def _bonded_only(flat):
    z = topology.FlatTopology(**{k: v for k, v in flat.__dict__.items() if not k.startswith("_")})
    for k in ("charge", "lj_a", "lj_b", "lj14_a", "lj14_b"):
        setattr(z, k, np.zeros_like(getattr(flat, k)))
    return z


def test_torch_reference_matches_oracle_energies_and_forces():
    torch = pytest.importorskip("torch")
    s = H.system("tiny")
    grid = synth.GRIDS["tiny"]
    flat = H.flat(s, PHYS)
    alpha = H.alpha_for(1e-5)
    p = O.make_params(PHYS, s.box, grid, alpha, H.KC)
    e2, f2, _, _, _ = O.evaluate(flat, p, s.coords)
    _, fb, _, _, _ = O.evaluate(_bonded_only(flat), p, s.coords)
    ref = NonbondedRef(flat, s.box, grid, alpha, H.KC)
    q = torch.tensor(flat.charge)
    A, B = torch.tensor(flat.lj_a), torch.tensor(flat.lj_b)
    x = torch.tensor(s.coords)
    E = ref.energy(q, A, B, x)
    for k in TERMS:
        assert H.rel(float(E[k]), e2[abi.E_INDEX[k]]) < 1e-10, (k, float(E[k]), e2[abi.E_INDEX[k]])
    F, _ = ref.forces(q, A, B, x)
    assert H.frel(F.detach().numpy(), f2 - fb) < 1e-10
