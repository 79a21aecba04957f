"""mdf_backward: the adjoint of the PHYSICAL forces and energy with respect to
charges and the LJ A/B table.

Loss (the c2 workload): L = mean over atoms of |F - F_target|^2 + 1e-3 E_total,
F_target = forces + N(0, 0.5^2) noise (seeded).
  * FP64 engine vs the FP64 PyTorch reference gradient (double backward of
    tests/adjoint_ref.py, pinned to the oracle): 1e-8 relative (norm of the
    difference over the norm) for dL/dq, dL/dA and dL/dB on `tiny`.
  * mixed engine vs the same reference: 1e-5 relative.
  * central finite differences of the FP64 engine's loss on 64 seeded
    parameters of the c0 system (charges, and A/B entries of the chain types;
    step 1e-4 relative to the parameter): 1e-5 relative per parameter, or
    1e-7 of the largest derivative of that kind for near-zero derivatives.
  * the torch.autograd.Function wrapper returns the same gradients.
"""
import numpy as np
import pytest

from md_b200 import abi, engine, synth
from tests import helpers as H

pytestmark = pytest.mark.gpu
PHYS, FP64, MIXED = abi.MDF_SEM_PHYSICAL, abi.MDF_PREC_FP64, abi.MDF_PREC_MIXED


def _setup(cfg, prec):
    s = H.system(cfg)
    grid = synth.GRIDS[cfg]
    flat = H.flat(s, PHYS, engine.cmap_coefficients)
    eng = engine.Engine(flat, s.box, semantics=PHYS, precision=prec, ewald_tol=1e-5, grid=grid)
    eng.set_positions(s.coords)
    eng.build_pairlist()
    return s, grid, flat, eng


def _loss_grads(F, E, Ft):
    n = F.shape[0]
    L = float(((F - Ft) ** 2).sum() / n + 1e-3 * E["total"])
    return L, 2.0 * (F - Ft) / n, 1e-3


def _target(F, seed=5):
    return F + np.random.default_rng(seed).normal(0.0, 0.5, F.shape)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("prec,tol", [(FP64, 1e-8), (MIXED, 1e-5)])
def test_adjoint_matches_fp64_reference_gradient(prec, tol):
    from tests.adjoint_ref import NonbondedRef
    s, grid, flat, eng = _setup("tiny", prec)
    E, F = eng.compute()
    Ft = _target(F)
    _, gF, gE = _loss_grads(F, E, Ft)
    dq, dA, dB = eng.backward(gF, gE)
    ref = NonbondedRef(flat, s.box, grid, H.alpha_for(1e-5), H.KC)
    rq, rA, rB = ref.vjp(flat.charge, flat.lj_a, flat.lj_b, s.coords, gF, gE)
    assert _rel(dq, rq) < tol, _rel(dq, rq)
    assert _rel(dA, rA) < tol, _rel(dA, rA)
    assert _rel(dB, rB) < tol, _rel(dB, rB)
    eng.close()


def test_adjoint_matches_central_differences_c0():
    s, grid, flat, eng = _setup("c0", FP64)
    q0, A0, B0 = flat.charge.copy(), flat.lj_a.copy(), flat.lj_b.copy()
    E, F = eng.compute()
    Ft = _target(F)

    def loss(q, A, B):
        eng.set_parameters(q, A, B)
        E_, F_ = eng.compute()
        return _loss_grads(F_, E_, Ft)[0]

    L0, gF, gE = _loss_grads(F, E, Ft)
    eng.set_parameters(q0, A0, B0)
    dq, dA, dB = eng.backward(gF, gE)
    rng = np.random.default_rng(7)
    # charges of random atoms; A/B entries used by some type pair (nonzero coefficient)
    used = np.flatnonzero(A0 != 0)
    picks = [("q", int(i)) for i in rng.choice(flat.natoms, 32, replace=False)]
    picks += [("A", int(i)) for i in rng.choice(used, 16, replace=False)]
    picks += [("B", int(i)) for i in rng.choice(used, 16, replace=False)]
    bad = []
    for kind, i in picks:
        base = {"q": q0, "A": A0, "B": B0}[kind]
        h = 1e-4 * abs(base[i])
        args_p = [q0.copy(), A0.copy(), B0.copy()]
        args_m = [q0.copy(), A0.copy(), B0.copy()]
        k = {"q": 0, "A": 1, "B": 2}[kind]
        args_p[k][i] += h
        args_m[k][i] -= h
        fd = (loss(*args_p) - loss(*args_m)) / (2 * h)
        g = {"q": dq, "A": dA, "B": dB}[kind]
        an = g[i]
        if not (abs(fd - an) <= 1e-5 * abs(fd) or abs(fd - an) <= 1e-7 * np.abs(g).max()):
            bad.append((kind, i, fd, an))
    eng.set_parameters(q0, A0, B0)
    eng.close()
    assert not bad, bad


def test_autograd_function_wraps_backward():
    torch = pytest.importorskip("torch")
    from md_b200.autograd import MDForces
    s, grid, flat, eng = _setup("tiny", FP64)
    q = torch.tensor(flat.charge, requires_grad=True)
    A = torch.tensor(flat.lj_a, requires_grad=True)
    B = torch.tensor(flat.lj_b, requires_grad=True)
    F, E = MDForces.apply(q, A, B, eng)
    Ft = torch.from_numpy(_target(F.detach().numpy()))
    L = ((F - Ft) ** 2).sum() / F.shape[0] + 1e-3 * E
    L.backward()
    _, gF, gE = _loss_grads(F.detach().numpy(), {"total": float(E.detach())}, Ft.numpy())
    dq, dA, dB = eng.backward(gF, gE)
    assert np.allclose(q.grad.numpy(), dq, rtol=1e-12, atol=0)
    assert np.allclose(A.grad.numpy(), dA, rtol=1e-12, atol=0)
    assert np.allclose(B.grad.numpy(), dB, rtol=1e-12, atol=0)
    eng.close()


def test_backward_rejects_reference_semantics():
    s = H.system("tiny")
    flat = H.flat(s, abi.MDF_SEM_REFERENCE, engine.cmap_coefficients)
    eng = engine.Engine(flat, s.box, semantics=abi.MDF_SEM_REFERENCE, precision=FP64, ewald_tol=1e-5,
                        grid=synth.GRIDS["tiny"])
    eng.set_positions(s.coords)
    with pytest.raises(engine.MDFError) as ei:
        eng.backward(np.zeros((s.natoms, 3)), 1.0)
    assert ei.value.status == 9
    eng.close()
