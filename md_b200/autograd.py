"""torch.autograd.Function around mdf_compute / mdf_backward.

    F, E = MDForces.apply(q, lj_a, lj_b, engine)

q: per-atom charges [N] (internal unit), lj_a / lj_b: the LJ table [n_ljpair]
(NONBONDED_PARM_INDEX - 1 order), all float64 CPU tensors; engine: an
md_b200.engine.Engine in PHYSICAL semantics with positions and pairlist set.
Returns forces [N, 3] and the total energy (0-d), float64.  backward calls
the engine's adjoint (mdf_backward) at the same parameters; positions are
constants.
"""
from __future__ import annotations

import numpy as np
import torch


class MDForces(torch.autograd.Function):
    @staticmethod
    def forward(ctx, q, lj_a, lj_b, engine):
        qn = q.detach().cpu().numpy().astype(np.float64)
        an = lj_a.detach().cpu().numpy().astype(np.float64)
        bn = lj_b.detach().cpu().numpy().astype(np.float64)
        engine.set_parameters(qn, an, bn)
        E, F = engine.compute()
        ctx.engine = engine
        ctx.params = (qn, an, bn)
        return torch.from_numpy(F), torch.tensor(E["total"], dtype=torch.float64)

    @staticmethod
    def backward(ctx, gF, gE):
        eng = ctx.engine
        eng.set_parameters(*ctx.params)
        gFn = None if gF is None else gF.detach().cpu().numpy().astype(np.float64)
        gEn = 0.0 if gE is None else float(gE)
        dq, dA, dB = eng.backward(gFn, gEn)
        return torch.from_numpy(dq), torch.from_numpy(dA), torch.from_numpy(dB), None
