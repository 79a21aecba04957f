"""L-BFGS minimiser (mdf_minimize_lbfgs).

  * known minimum: distorted flexible waters with bonded terms only (no
    charges, no LJ) relax to their equilibrium geometry, E -> 0, max |F| to
    1e-6, every O-H at r0 and every H-O-H at theta0 (FP64, 1e-6);
  * on a clashing synthetic start it lowers energy and the largest force
    further than steepest descent does in the same number of iterations, and
    the reported energy and force agree with a fresh evaluation at the final
    positions;
  * bit-reproducible: two runs end on identical positions;
  * bad history lengths are rejected.
"""
import math

import numpy as np
import pytest

from md_b200 import abi, engine, synth
from tests import helpers as H

pytestmark = pytest.mark.gpu
PHYS, FP64, MIXED = abi.MDF_SEM_PHYSICAL, abi.MDF_PREC_FP64, abi.MDF_PREC_MIXED

R0, T0 = 0.9572, math.radians(104.52)


def _waters(nw=8, box=30.0, seed=5):
    """nw flexible waters on a coarse lattice, bonds stretched and angles bent
    at random; bonded terms only."""
    rng = np.random.default_rng(seed)
    pos, bonds, angles = [], [], []
    side = int(math.ceil(nw ** (1 / 3)))
    for w in range(nw):
        o = (np.array([w % side, (w // side) % side, w // (side * side)]) + 0.5) * (box / side)
        r1, r2 = R0 * rng.uniform(0.9, 1.15, 2)
        th = T0 * rng.uniform(0.85, 1.1)
        u = rng.normal(size=3); u /= np.linalg.norm(u)
        v = rng.normal(size=3); v -= u * (u @ v); v /= np.linalg.norm(v)
        h1 = o + r1 * u
        h2 = o + r2 * (math.cos(th) * u + math.sin(th) * v)
        b = 3 * w
        pos += [o, h1, h2]
        bonds += [b, b + 1, b, b + 2]
        angles += [b + 1, b, b + 2]
    f = H.simple_flat(np.zeros(3 * nw))
    f.bond_atoms = np.asarray(bonds, np.int32)
    f.bond_k = np.full(2 * nw, 450.0)
    f.bond_r0 = np.full(2 * nw, R0)
    f.angle_atoms = np.asarray(angles, np.int32)
    f.angle_k = np.full(nw, 55.0)
    f.angle_theta0 = np.full(nw, T0)
    return f, np.array(pos), np.full(3, box)


def test_lbfgs_reaches_the_known_minimum():
    f, x0, box = _waters()
    eng = engine.Engine(f, box, semantics=PHYS, precision=FP64, ewald_tol=1e-5, grid=(32, 32, 32))
    eng.set_positions(x0)
    r = eng.minimize(max_iter=500, fmax_tol=1e-6, max_step=0.1, method="lbfgs")
    assert r["fmax_final"] <= 1e-6, r
    assert abs(r["e_final"]) < 1e-9, r
    assert r["evaluations"] >= r["iterations"] + 1
    x, _ = eng.md_state(velocities=False)
    for w in range(len(x) // 3):
        o, h1, h2 = x[3 * w], x[3 * w + 1], x[3 * w + 2]
        a, b = h1 - o, h2 - o
        assert abs(np.linalg.norm(a) - R0) < 1e-6 and abs(np.linalg.norm(b) - R0) < 1e-6
        th = math.acos(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))
        assert abs(th - T0) < 1e-6
    eng.close()


def _engine(s, prec, coords=None):
    flat = H.flat(s, PHYS, engine.cmap_coefficients)
    eng = engine.Engine(flat, s.box, semantics=PHYS, precision=prec, ewald_tol=1e-5, grid=synth.GRIDS[s.name])
    eng.set_positions(s.coords if coords is None else coords)
    eng.build_pairlist()
    return eng


@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_lbfgs_beats_steepest_descent_and_reports_truthfully(prec):
    s = H.system("tiny")
    res = {}
    for method in ("sd", "lbfgs"):
        eng = _engine(s, prec)
        res[method] = eng.minimize(max_iter=60, fmax_tol=1e-3, max_step=0.1, method=method)
        if method == "lbfgs":
            x, _ = eng.md_state(velocities=False)
        eng.close()
    sd, lb = res["sd"], res["lbfgs"]
    assert lb["e_final"] < lb["e_initial"]
    assert lb["e_final"] < sd["e_final"], res
    assert lb["fmax_final"] < sd["fmax_final"], res
    e2 = _engine(s, prec, coords=x)
    E, F = e2.compute()
    assert abs(E["total"] - lb["e_final"]) < 1e-6 * abs(lb["e_final"]) + 1e-6
    assert np.abs(F).max() <= lb["fmax_final"] * (1 + 1e-5) + 1e-6
    e2.close()


def test_lbfgs_is_reproducible():
    s = H.system("tiny")
    xs = []
    for _ in range(2):
        eng = _engine(s, MIXED)
        eng.minimize(max_iter=40, fmax_tol=1e-3, method="lbfgs", history=5)
        xs.append(eng.md_state(velocities=False)[0])
        eng.close()
    assert np.array_equal(xs[0], xs[1])


@pytest.mark.parametrize("history", [-1, 65])
def test_bad_history_rejected(history):
    s = H.system("tiny")
    eng = _engine(s, MIXED)
    with pytest.raises(engine.MDFError) as ei:
        eng.minimize(max_iter=5, method="lbfgs", history=history)
    assert ei.value.status == abi.MDF_ERR_INVALID
    eng.close()
