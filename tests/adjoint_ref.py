"""FP64 PyTorch restatement of the PHYSICAL nonbonded energy, used as the
reference gradient for mdf_backward.  TEST INFRASTRUCTURE ONLY.

E(q, A, B; x) = LJ (switched, r <= rc, non-excluded pairs)
              + k q q erfc(alpha r)/r (r <= rc, non-excluded)
              - k q q erf(alpha r)/r (excluded pairs, no cutoff)
              + k q q/(scee r) + (A14/r^12 - B14/r^6)/scnb (1-4 pairs)
              - k alpha/sqrt(pi) sum q^2 - k pi Q^2/(2 V alpha^2)
              + smooth PME order 4 (Essmann et al. 1995) on the given grid,
the definitions of the oracle's PHYSICAL mode (oracle/mdf_oracle.c).  Pairs
are enumerated densely (minimum image), so this is for systems of a few
thousand atoms.  Forces come from autograd; the reference gradient of a loss
L(F, E) is the gradient of gE E + v . F (v = dL/dF) with respect to
(q, A, B), by double backward.
"""
from __future__ import annotations

import math

import numpy as np
import torch

DT = torch.float64


def _bmod(K, order=4):
    """1/|b(m)|^2 per grid index, zeros bridged (Essmann et al. eq. 4.4)."""
    def card(n, x):
        if x <= 0 or x >= n:
            return 0.0
        if n == 2:
            return 1.0 - abs(x - 1.0)
        return (x * card(n - 1, x) + (n - x) * card(n - 1, x - 1.0)) / (n - 1)
    b = np.zeros(K)
    for m in range(K):
        sr = si = 0.0
        for k in range(order - 1):
            v = card(order, k + 1.0)
            a = 2 * math.pi * m * k / K
            sr += v * math.cos(a)
            si += v * math.sin(a)
        b[m] = sr * sr + si * si
    for m in range(K):
        if b[m] < 1e-7:
            b[m] = 0.5 * (b[(m - 1) % K] + b[(m + 1) % K])
    return 1.0 / b


class NonbondedRef:
    def __init__(self, flat, box, grid, alpha, kc, cutoff=10.0, switch=9.0):
        self.N = flat.natoms
        self.box = torch.tensor(box, dtype=DT)
        self.K = tuple(int(k) for k in grid)
        self.alpha, self.kc, self.rc, self.rsw = float(alpha), float(kc), float(cutoff), float(switch)
        nt = flat.ntypes
        nbi = np.asarray(flat.nb_index).reshape(nt, nt)
        types = np.asarray(flat.type)
        i, j = np.triu_indices(self.N, 1)
        excl = set()
        ex = np.asarray(flat.excl_pairs).reshape(-1, 2)
        for a, b in ex:
            excl.add((min(a, b), max(a, b)))
        keep = np.ones(len(i), bool)
        if excl:
            key = i.astype(np.int64) * self.N + j
            exk = np.array([a * self.N + b for a, b in excl], np.int64)
            keep = ~np.isin(key, exk)
        self.pi = torch.from_numpy(i[keep])
        self.pj = torch.from_numpy(j[keep])
        nb = nbi[types[i[keep]], types[j[keep]]]
        self.pnb = torch.from_numpy(nb.astype(np.int64) - 1)     # -1: no LJ
        self.ex = torch.from_numpy(ex.astype(np.int64)) if len(ex) else torch.zeros((0, 2), dtype=torch.int64)
        p14 = np.asarray(flat.pairs14).reshape(-1, 2)
        self.p14 = torch.from_numpy(p14.astype(np.int64))
        self.scee = torch.from_numpy(np.asarray(flat.scee14, float))
        self.scnb = torch.from_numpy(np.asarray(flat.scnb14, float))
        nb14 = nbi[types[p14[:, 0]], types[p14[:, 1]]] if len(p14) else np.zeros(0, int)
        self.p14nb = torch.from_numpy(nb14.astype(np.int64) - 1)
        self.A14 = torch.from_numpy(np.asarray(flat.lj14_a, float))
        self.B14 = torch.from_numpy(np.asarray(flat.lj14_b, float))
        # PME influence function on the full grid
        Kx, Ky, Kz = self.K
        L = box
        V = float(L[0] * L[1] * L[2])
        self.V = V
        mx = np.fft.fftfreq(Kx, 1.0 / Kx) / L[0]
        my = np.fft.fftfreq(Ky, 1.0 / Ky) / L[1]
        mz = np.fft.fftfreq(Kz, 1.0 / Kz) / L[2]
        MX, MY, MZ = np.meshgrid(mx, my, mz, indexing="ij")
        m2 = MX ** 2 + MY ** 2 + MZ ** 2
        m2[0, 0, 0] = 1.0
        bx, by, bz = _bmod(Kx), _bmod(Ky), _bmod(Kz)
        c = (self.kc / (math.pi * V)) * np.exp(-math.pi ** 2 * m2 / self.alpha ** 2) / m2
        c = c * bx[:, None, None] * by[None, :, None] * bz[None, None, :]
        c[0, 0, 0] = 0.0
        self.infl = torch.from_numpy(c)

    def _mic(self, d):
        return d - self.box * torch.round(d / self.box)

    def energy(self, q, A, B, x):
        """Nonbonded energy terms (dict of scalars) at positions x [N, 3]."""
        kc, al, rc = self.kc, self.alpha, self.rc
        out = {}
        d = self._mic(x[self.pi] - x[self.pj])
        r2 = (d * d).sum(-1)
        inc = r2 <= rc * rc
        d, r2 = d[inc], r2[inc]
        pi, pj, pnb = self.pi[inc], self.pj[inc], self.pnb[inc]
        r = torch.sqrt(r2)
        out["ee_direct"] = (kc * q[pi] * q[pj] * torch.erfc(al * r) / r).sum()
        lj = pnb >= 0
        rl, r2l, k = r[lj], r2[lj], pnb[lj]
        i6 = 1.0 / r2l ** 3
        U = A[k] * i6 * i6 - B[k] * i6
        x_ = torch.clamp((rl - self.rsw) / (rc - self.rsw), min=0.0)
        S = 1 - 10 * x_ ** 3 + 15 * x_ ** 4 - 6 * x_ ** 5
        out["vdw"] = (U * S).sum()
        # excluded pairs
        if len(self.ex):
            de = self._mic(x[self.ex[:, 0]] - x[self.ex[:, 1]])
            re = torch.sqrt((de * de).sum(-1))
            out["ee_excl"] = (-kc * q[self.ex[:, 0]] * q[self.ex[:, 1]] * torch.erf(al * re) / re).sum()
        else:
            out["ee_excl"] = torch.zeros((), dtype=DT)
        # 1-4 pairs
        if len(self.p14):
            d4 = self._mic(x[self.p14[:, 0]] - x[self.p14[:, 1]])
            r4 = torch.sqrt((d4 * d4).sum(-1))
            out["ee14"] = (kc * q[self.p14[:, 0]] * q[self.p14[:, 1]] / (self.scee * r4)).sum()
            k4 = self.p14nb
            ok = k4 >= 0
            i6 = 1.0 / r4[ok] ** 6
            out["vdw14"] = ((self.A14[k4[ok]] * i6 * i6 - self.B14[k4[ok]] * i6) / self.scnb[ok]).sum()
        else:
            out["ee14"] = torch.zeros((), dtype=DT)
            out["vdw14"] = torch.zeros((), dtype=DT)
        out["ee_self"] = -kc * al / math.sqrt(math.pi) * (q * q).sum()
        Q = q.sum()
        out["ee_recip"] = self._pme(q, x) - kc * math.pi * Q * Q / (2 * self.V * al * al)
        return out

    def _pme(self, q, x):
        Kx, Ky, Kz = self.K
        K = torch.tensor(self.K, dtype=DT)
        xw = x - self.box * torch.floor(x / self.box)
        u = xw * (K / self.box)
        base = torch.floor(u.detach())
        w = u - base
        base = base.long()
        th = torch.stack([(1 - w) ** 3 / 6, (3 * w ** 3 - 6 * w ** 2 + 4) / 6,
                          (-3 * w ** 3 + 3 * w ** 2 + 3 * w + 1) / 6, w ** 3 / 6], dim=-1)   # [N, 3, 4]
        off = torch.arange(4) - 1
        ix = (base[:, 0, None] + off) % Kx
        iy = (base[:, 1, None] + off) % Ky
        iz = (base[:, 2, None] + off) % Kz
        wgt = q[:, None, None, None] * th[:, 0, :, None, None] * th[:, 1, None, :, None] * th[:, 2, None, None, :]
        idx = (ix[:, :, None, None] * Ky + iy[:, None, :, None]) * Kz + iz[:, None, None, :]
        Qg = torch.zeros(Kx * Ky * Kz, dtype=DT).index_add(0, idx.reshape(-1), wgt.reshape(-1))
        S = torch.fft.fftn(Qg.reshape(Kx, Ky, Kz))
        return 0.5 * (self.infl * (S.real ** 2 + S.imag ** 2)).sum()

    def total(self, q, A, B, x):
        return sum(self.energy(q, A, B, x).values())

    def forces(self, q, A, B, x):
        """Nonbonded forces [N, 3] (autograd, graph kept for double backward)."""
        x = x.detach().requires_grad_(True)
        E = self.total(q, A, B, x)
        (g,) = torch.autograd.grad(E, x, create_graph=True)
        return -g, E

    def vjp(self, q0, A0, B0, x, v, gE):
        """Gradient of gE E + v . F with respect to (q, A, B)."""
        q = torch.as_tensor(q0, dtype=DT).clone().requires_grad_(True)
        A = torch.as_tensor(A0, dtype=DT).clone().requires_grad_(True)
        B = torch.as_tensor(B0, dtype=DT).clone().requires_grad_(True)
        xt = torch.as_tensor(x, dtype=DT)
        F, E = self.forces(q, A, B, xt)
        phi = gE * E + (torch.as_tensor(v, dtype=DT).reshape(-1, 3) * F).sum()
        dq, dA, dB = torch.autograd.grad(phi, (q, A, B), allow_unused=True)
        z = lambda t, n: torch.zeros(n, dtype=DT) if t is None else t
        return (z(dq, len(q0)).numpy(), z(dA, len(A0)).numpy(), z(dB, len(B0)).numpy())
