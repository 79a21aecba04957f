"""Shared helpers for the test suite (golden fixtures, systems, comparisons)."""
import hashlib
import json
import math
import os
import tempfile

import numpy as np

from md_b200 import abi, synth, topology

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
KC = synth.KC

_SYS_CACHE = {}
_O2_CACHE = {}


def alpha_for(tol, cutoff=10.0):
    # src/System/PBC.cpp:88-91
    return math.sqrt(-math.log(2 * tol)) / cutoff


def golden(case):
    d = os.path.join(GOLDEN, case)
    with open(os.path.join(d, "meta.json")) as f:
        meta = json.load(f)
    with open(os.path.join(d, "energies.json")) as f:
        en = json.load(f)
    out = dict(meta=meta, energies=en, dir=d)
    if os.path.exists(os.path.join(d, "forces.npy")):
        out["forces"] = np.load(os.path.join(d, "forces.npy"))
        out["forces_pme"] = np.load(os.path.join(d, "forces_pme.npy"))
    else:
        z = np.load(os.path.join(d, "forces_digest.npz"))
        out["digest"] = {k: z[k] for k in z.files}
    return out


def system(cfg, sentinels=False):
    key = (cfg, sentinels)
    if key not in _SYS_CACHE:
        _SYS_CACHE[key] = synth.make_config(cfg, sentinels=sentinels)
    return _SYS_CACHE[key]


def o2_physical(cfg, flat_phys):
    """O2 PHYSICAL evaluation of a named workload at its grid, Ewald tol 1e-5
    (cached: several tests compare against the same oracle result)."""
    if cfg not in _O2_CACHE:
        from oracle import oracle as O
        s = system(cfg)
        p = O.make_params(abi.MDF_SEM_PHYSICAL, s.box, synth.GRIDS[cfg], alpha_for(1e-5), KC)
        _O2_CACHE[cfg] = O.evaluate(flat_phys, p, s.coords)
    return _O2_CACHE[cfg]


def files_sha(sysm):
    tmp = tempfile.mkdtemp(prefix="sha_")
    p, r = synth.write_files(sysm, tmp, stem="x")
    out = []
    for path in (p, r):
        with open(path, "rb") as f:
            out.append(hashlib.sha256(f.read()).hexdigest())
    import shutil
    shutil.rmtree(tmp, ignore_errors=True)
    return out


def flat(sysm, semantics, cmap_fn=None):
    if cmap_fn is None:
        from oracle import oracle as O
        cmap_fn = O.cmap_coeff
    return topology.flatten(sysm, semantics, cmap_fn)


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def frel(f, g):
    return float(np.linalg.norm(np.asarray(f) - np.asarray(g)) / max(np.linalg.norm(g), 1e-300))


def check_forces_vs_golden(F, g, tol, key="forces"):
    """Full-force or digest comparison against an O1 fixture."""
    if key in g:
        assert frel(F, g[key]) < tol, (key, frel(F, g[key]))
    else:
        dg = g["digest"]
        sub = F[dg["idx"]]
        ref = dg[key]
        assert frel(sub, ref) < tol, (key, frel(sub, ref))
        nrm = dg["norm" if key == "forces" else "norm_pme"]
        assert rel(np.linalg.norm(F), float(nrm)) < tol


def simple_flat(charges, ntypes=1, types=None, lj_a=None, lj_b=None, excl_pairs=None):
    """A topology with charges and LJ only (no bonded terms)."""
    n = len(charges)
    types = np.zeros(n, np.int32) if types is None else np.asarray(types, np.int32)
    npair = ntypes * (ntypes + 1) // 2
    nb = np.zeros(ntypes * ntypes, np.int32)
    for i in range(ntypes):
        for j in range(ntypes):
            hi, lo = max(i, j) + 1, min(i, j) + 1
            nb[i * ntypes + j] = hi * (hi - 1) // 2 + lo
    la = np.zeros(npair) if lj_a is None else np.asarray(lj_a, float)
    lb = np.zeros(npair) if lj_b is None else np.asarray(lj_b, float)
    z2 = np.zeros(0, np.int32)
    zf = np.zeros(0)
    ex = z2 if excl_pairs is None else np.asarray(excl_pairs, np.int32).reshape(-1)
    return topology.FlatTopology(
        charge=np.ascontiguousarray(charges, dtype=np.float64), type=types, ntypes=ntypes, nb_index=nb,
        lj_a=la, lj_b=lb, lj14_a=la.copy(), lj14_b=lb.copy(),
        bond_atoms=z2, bond_k=zf, bond_r0=zf, ub_atoms=z2, ub_k=zf, ub_r0=zf,
        angle_atoms=z2, angle_k=zf, angle_theta0=zf, dihedral_atoms=z2, dihedral_k=zf, dihedral_n=zf,
        dihedral_phase=zf, improper_atoms=z2, improper_k=zf, improper_phase=zf,
        cmap_atoms=z2, cmap_set=z2, cmap_nsets=0, cmap_res=24, cmap_coeff=zf,
        excl_pairs=ex, pairs14=z2, scee14=zf, scnb14=zf)


def nacl_crystal(ncell=4, a=5.64):
    """Rock-salt lattice: ncell^3 conventional cells, charges +-1."""
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    pos, q = [], []
    for i in range(ncell):
        for j in range(ncell):
            for k in range(ncell):
                o = np.array([i, j, k], float)
                for b in base:
                    pos.append((o + b) * a); q.append(1.0)
                    pos.append((o + b + np.array([0.5, 0, 0])) * a); q.append(-1.0)
    return np.array(pos) + 0.25 * a, np.array(q), np.full(3, ncell * a)


MADELUNG_NACL = 1.747564594633


def many_types(flat, ntypes=60, seed=5):
    """A copy of a flat topology with `ntypes` LJ types (atom i gets type
    i mod ntypes; per-type well depths and radii seeded, Lorentz-Berthelot
    pairs A = eps R^12, B = 2 eps R^6): a pair table too large for the pair
    kernels' shared memory (more than 51 types in FP32, 55 in FP64)."""
    from md_b200 import topology
    rng = np.random.default_rng(seed)
    eps = rng.uniform(0.05, 0.3, ntypes)
    rhalf = rng.uniform(0.6, 1.0, ntypes)
    nb = np.zeros((ntypes, ntypes), np.int32)
    a, b = [], []
    for i in range(ntypes):
        for j in range(i, ntypes):
            e, r = np.sqrt(eps[i] * eps[j]), rhalf[i] + rhalf[j]
            a.append(e * r ** 12)
            b.append(2.0 * e * r ** 6)
            nb[i, j] = nb[j, i] = len(a)   # 1-based
    arrays = dict(flat.__dict__)
    arrays.pop("_struct", None)
    arrays.update(type=(np.arange(flat.natoms) % ntypes).astype(np.int32), ntypes=ntypes,
                  nb_index=np.ascontiguousarray(nb.ravel()), lj_a=np.array(a), lj_b=np.array(b),
                  lj14_a=0.5 * np.array(a), lj14_b=0.5 * np.array(b))
    return topology.FlatTopology(**arrays)
