"""The hand-written PME FFT chain against cuFFT (through torch.fft on the GPU):
the potential grid C*Q the engine gathers from equals
N * irfftn(c(m) * rfftn(Q)) computed with cuFFT on the engine's own charge
grid Q, c(m) the smooth-PME influence function.  FP64 to 1e-12, mixed (FP32
FFT) to 1e-5, relative L2."""
import numpy as np
import pytest

from md_b200 import abi, engine, synth
from tests import helpers as H

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cfg", ["small", "c0"])
@pytest.mark.parametrize("prec,tol", [(abi.MDF_PREC_FP64, 1e-12), (abi.MDF_PREC_MIXED, 1e-5)])
def test_fft_chain_matches_cufft(cfg, prec, tol):
    import torch
    s = H.system(cfg)
    grid = synth.GRIDS[cfg]
    flat = H.flat(s, abi.MDF_SEM_PHYSICAL, engine.cmap_coefficients)
    eng = engine.Engine(flat, s.box, semantics=abi.MDF_SEM_PHYSICAL, precision=prec, ewald_tol=1e-5, grid=grid)
    eng.set_positions(s.coords)
    eng.compute()
    Q, P = eng.pme_grids()
    eng.close()
    # the influence function only (NonbondedRef builds it; its pair tables are not used)
    c = _influence(s.box, grid, H.alpha_for(1e-5), H.KC)
    q = torch.tensor(Q, device="cuda")
    S = torch.fft.rfftn(q)
    Pr = torch.fft.irfftn(S * torch.tensor(c[:, :, :grid[2] // 2 + 1], device="cuda"), s=tuple(grid))
    Pr = Pr.cpu().numpy() * (grid[0] * grid[1] * grid[2])
    assert H.frel(P, Pr) < tol, H.frel(P, Pr)


def _influence(box, grid, alpha, kc):
    import math
    from tests.adjoint_ref import _bmod
    Kx, Ky, Kz = grid
    V = box[0] * box[1] * box[2]
    mx = np.fft.fftfreq(Kx, 1.0 / Kx) / box[0]
    my = np.fft.fftfreq(Ky, 1.0 / Ky) / box[1]
    mz = np.fft.fftfreq(Kz, 1.0 / Kz) / box[2]
    MX, MY, MZ = np.meshgrid(mx, my, mz, indexing="ij")
    m2 = MX ** 2 + MY ** 2 + MZ ** 2
    m2[0, 0, 0] = 1.0
    c = (kc / (math.pi * V)) * np.exp(-math.pi ** 2 * m2 / alpha ** 2) / m2
    c = c * _bmod(Kx)[:, None, None] * _bmod(Ky)[None, :, None] * _bmod(Kz)[None, None, :]
    c[0, 0, 0] = 0.0
    return c
