"""The shared-memory tile spread and gather (PHYSICAL PME) against the per-atom
kernels with global atomics (mdf_params.pme_tile = -1).

The charge grid is an int64 fixed-point sum, so every tile height gives the
same grid bit for bit; the gather evaluates each atom's stencil in the same
order as the per-atom kernel, so forces agree to the last bits (checked to
1e-13 of the largest force).  Grids that are not multiples of the tile
(30 x 36 x 28 with 8-line tiles) exercise the partial edge tiles.  An atom
moved past the tile kernels' reach without a list rebuild is an error, not a
dropped charge."""
import numpy as np
import pytest

from md_b200 import abi, engine
from tests import helpers as H

pytestmark = pytest.mark.gpu

PHYS, MIXED, FP64 = abi.MDF_SEM_PHYSICAL, abi.MDF_PREC_MIXED, abi.MDF_PREC_FP64


def _run(s, prec, grid, tile, coords=None):
    flat = H.flat(s, PHYS, engine.cmap_coefficients)
    eng = engine.Engine(flat, s.box, semantics=PHYS, precision=prec, ewald_tol=1e-5, grid=grid, pme_tile=tile)
    eng.set_positions(s.coords)
    eng.build_pairlist()
    if coords is not None:
        eng.set_positions(coords)
    E, F = eng.compute()
    Q, P = eng.pme_grids()
    eng.close()
    return E, F, Q, P


@pytest.mark.parametrize("cfg,grid", [("small", (32, 32, 32)), ("small", (30, 36, 28)), ("c0", (72, 72, 72))])
@pytest.mark.parametrize("prec", [MIXED, FP64])
def test_tiles_match_per_atom_kernels(cfg, grid, prec):
    s = H.system(cfg)
    rng = np.random.default_rng(11)
    moved = s.coords + rng.uniform(-0.3, 0.3, s.coords.shape)   # within half the skin of the build
    E0, F0, Q0, P0 = _run(s, prec, grid, -1, moved)
    for tile in (0, 1, 2, 8):
        E, F, Q, P = _run(s, prec, grid, tile, moved)
        assert np.array_equal(Q, Q0), tile
        assert np.array_equal(P, P0), tile
        assert np.abs(F - F0).max() <= 1e-13 * np.abs(F0).max(), tile
        assert abs(E["ee"] - E0["ee"]) <= 1e-12 * abs(E0["ee"]), tile


def test_stale_list_is_an_error():
    s = H.system("small")
    flat = H.flat(s, PHYS, engine.cmap_coefficients)
    eng = engine.Engine(flat, s.box, semantics=PHYS, precision=MIXED, ewald_tol=1e-5, grid=(32, 32, 32))
    eng.set_positions(s.coords)
    eng.build_pairlist()
    x = s.coords.copy()
    i = int(np.flatnonzero(np.abs(flat.charge) > 0.1)[0])
    x[i, 0] += 0.5 * s.box[0]   # half a box away from its list column (more than half the skin + 1 A)
    eng.set_positions(x)
    with pytest.raises(engine.MDFError) as ei:
        eng.compute()
    assert ei.value.status == abi.MDF_ERR_STATE
    eng.build_pairlist()   # a rebuild clears it
    eng.compute()
    eng.close()


def test_bad_tile_rejected():
    s = H.system("tiny")
    flat = H.flat(s, PHYS, engine.cmap_coefficients)
    with pytest.raises(engine.MDFError):
        engine.Engine(flat, s.box, semantics=PHYS, precision=MIXED, grid=(24, 24, 24), pme_tile=9)
