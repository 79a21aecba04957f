"""Minimiser and velocity-Verlet dynamics (mdf_minimize, mdf_md_*).

  * one step equals velocity Verlet written out on the host with the
    engine's own forces (FP64: positions 1e-12 A, velocities 1e-10 relative);
  * time reversal: N steps, velocities negated, N steps back to the start
    (FP64, 1e-8 A);
  * the steepest-descent minimiser lowers the energy and the largest force;
  * NVE energy conservation after a short minimisation: over 100 fs at
    0.25 fs the total energy's spread stays below 1e-3 of the kinetic energy
    (FP64 and mixed) and the two paths' drifts agree to 1e-3 of it; halving
    the step cuts the FP64 spread by more than 2.5x (the O(dt^2) error of
    velocity Verlet: what is left is integration error, not a force that
    disagrees with the energy);
  * the rebuild schedule (every 10 steps) and the displacement trigger;
  * the rst7 writer round-trips positions and velocities.
"""
import numpy as np
import pytest

from md_b200 import abi, engine, synth
from tests import helpers as H

pytestmark = pytest.mark.gpu
PHYS, FP64, MIXED = abi.MDF_SEM_PHYSICAL, abi.MDF_PREC_FP64, abi.MDF_PREC_MIXED
ACC = 418.4


def _engine(s, prec, coords=None, **kw):
    flat = H.flat(s, PHYS, engine.cmap_coefficients)
    eng = engine.Engine(flat, s.box, semantics=PHYS, precision=prec, ewald_tol=1e-5, grid=synth.GRIDS[s.name], **kw)
    eng.set_positions(s.coords if coords is None else coords)
    eng.build_pairlist()
    return eng


def _v0(s, seed=3, T=300.0):
    rng = np.random.default_rng(seed)
    sd = np.sqrt(0.0019872041 * T * ACC / s.mass)[:, None]
    v = rng.normal(size=(s.natoms, 3)) * sd
    return v - (s.mass[:, None] * v).sum(0) / s.mass.sum()


def test_one_step_is_velocity_verlet():
    s = H.system("tiny")
    dt = 0.0005
    eng = _engine(s, FP64)
    _, F0 = eng.compute()
    v0 = _v0(s)
    eng.md_init(s.mass, v0)
    eng.md_run(1, dt, chunk=1)
    x1, v1 = eng.md_state()
    a0 = F0 * ACC / s.mass[:, None]
    vh = v0 + 0.5 * dt * a0
    xh = s.coords + dt * vh
    e2 = _engine(s, FP64, coords=xh)
    _, F1 = e2.compute()
    vh1 = vh + 0.5 * dt * F1 * ACC / s.mass[:, None]
    assert np.abs(x1 - xh).max() < 1e-12
    assert H.frel(v1, vh1) < 1e-10
    eng.close(); e2.close()


@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_self_pruning_dynamics_matches_pruning_every_step(prec):
    """Dynamics in graph-captured chunks with device-decided pruning
    (prune_every < 0, 0.2 A margin) follows the trajectory of pruning at
    every step: 80 steps of 0.25 fs from a minimised start, positions to
    1e-9 A (FP64) / 1e-4 A (mixed: FP32 sums in another order, amplified
    over the trajectory)."""
    s = H.system("small")
    e0 = _engine(s, FP64)
    e0.minimize(max_iter=300, fmax_tol=5.0)
    x0, _ = e0.md_state(velocities=False)
    e0.close()
    out = []
    for kw in (dict(prune_every=-1, prune_margin=0.2), dict(prune_every=1)):
        eng = _engine(s, prec, coords=x0, **kw)
        eng.md_init(s.mass, _v0(s))
        eng.md_run(80, 0.00025, chunk=10)
        out.append(eng.md_state()[0])
        eng.close()
    tol = 1e-9 if prec == FP64 else 1e-4
    assert np.abs(out[0] - out[1]).max() < tol


def test_time_reversal():
    s = H.system("tiny")
    eng = _engine(s, FP64)
    eng.md_init(s.mass, _v0(s))
    eng.md_run(40, 0.0005, chunk=10)
    x, v = eng.md_state()
    eng.md_init(s.mass, -v)
    eng.md_run(40, 0.0005, chunk=10)
    xb, _ = eng.md_state()
    assert np.abs(xb - s.coords).max() < 1e-8
    eng.close()


def test_minimiser_lowers_energy_and_forces():
    s = H.system("tiny")
    eng = _engine(s, MIXED)
    r = eng.minimize(max_iter=100, fmax_tol=1.0)
    assert r["iterations"] > 0
    assert r["e_final"] < r["e_initial"]
    x, _ = eng.md_state(velocities=False)
    e2 = _engine(s, MIXED, coords=x)
    E, F = e2.compute()
    assert abs(E["total"] - r["e_final"]) < 1e-6 * abs(r["e_final"]) + 1e-6
    # a fresh list changes the FP32 rounding of the mixed forces (~1e-6)
    assert np.abs(F).max() <= r["fmax_final"] * (1 + 1e-5) + 1e-6
    eng.close(); e2.close()


def test_nve_energy_conservation_fp64_and_mixed():
    s = H.system("small")
    out = {}
    for prec, dt, n in ((FP64, 0.00025, 400), (MIXED, 0.00025, 400), (FP64, 0.000125, 800)):
        eng = _engine(s, prec)
        eng.minimize(max_iter=300, fmax_tol=5.0)
        eng.md_init(s.mass, _v0(s))
        rep, samp = eng.md_run(n, dt, chunk=10)
        assert rep["steps"] == n and len(samp) == n // 10
        tot = samp[:, 1] + samp[:, 2]
        ke = samp[:, 2].mean()
        out[(prec, dt)] = (tot[-1] - tot[0], tot.std(), ke)
        eng.close()
    d64, s64, ke = out[(FP64, 0.00025)]
    dmx, smx, _ = out[(MIXED, 0.00025)]
    assert s64 < 1e-3 * ke and smx < 1e-3 * ke, out
    assert abs(dmx - d64) < 1e-3 * ke, out
    assert out[(FP64, 0.000125)][1] * 2.5 < s64, out


def test_rebuild_schedule_and_trigger():
    s = H.system("tiny")
    eng = _engine(s, MIXED)
    eng.minimize(max_iter=300, fmax_tol=5.0)
    eng.md_init(s.mass, temperature=300.0, seed=9)
    rep, _ = eng.md_run(50, 0.0005, chunk=10, rebuild_every=10)
    assert rep["rebuilds"] == 4
    rep, _ = eng.md_run(100, 0.0005, chunk=10, rebuild_every=0)
    assert rep["rebuilds"] < 10          # fewer than one per chunk: the trigger, not a schedule
    eng.close()


def test_rst7_writer_round_trip(tmp_path):
    s = H.system("tiny")
    eng = _engine(s, FP64)
    eng.md_init(s.mass, temperature=300.0, seed=2)
    eng.md_run(10, 0.0005)
    x, v = eng.md_state()
    p = tmp_path / "out.rst7"
    eng.write_rst7(p, "test", 0.005)
    lines = p.read_text().splitlines()
    n = int(lines[1][:6])
    assert n == s.natoms and abs(float(lines[1][6:]) - 0.005) < 1e-12
    vals = np.array([float(t[i:i + 12]) for t in lines[2:] for i in range(0, len(t), 12)])
    xr, vr, box = vals[:3 * n], vals[3 * n:6 * n], vals[6 * n:]
    assert np.abs(xr - x.reshape(-1)).max() < 1e-6
    assert np.abs(vr * 20.455 - v.reshape(-1)).max() < 1e-5
    assert np.allclose(box, list(s.box) + [90.0, 90.0, 90.0])
    eng.close()
