"""Seeded synthetic Amber/CHARMM-style systems and their prmtop/rst7 files.

The reference code (prateekbansal97/MD) reads a CHARMM-flavoured Amber
``prmtop`` plus an ``rst7`` (``src/AmberTopology/AmberTopology.cpp:86-101``).
No topology ships with it, so every workload here is generated: flexible
3-site waters on a jittered lattice plus one synthetic polymer chain carrying
every bonded term the reference evaluates (bond, angle, Urey-Bradley, cosine
dihedral, CHARMM improper, CMAP).

The written files honour the reference parser's quirks:

* first line ``%VERSION``; ``%FLAG NAME`` lines carry no trailing blanks
  (``src/util/IO.cpp:55-66`` takes everything after the first space);
* numeric fields are whitespace separated (``src/util/IO.cpp:109-136``);
  ``ATOM_NAME``/``RESIDUE_LABEL`` are fixed 4-character fields
  (``src/AmberTopology/TopologyParser.cpp:25-42``);
* bond/angle/dihedral atom entries are 3*index, dihedral flags are carried by
  the sign of the 3rd (exclude 1-4) and 4th (improper) entry
  (``src/AmberTopology/CreateBondedFromParsed.cpp:176-216``);
* exactly 5 CMAP parameter sets of 24x24
  (``src/AmberTopology/CreateNonBondedFromParsed.cpp:67-72``);
* the rst7 holds coordinates then the 6 box numbers, no velocities
  (``src/AmberTopology/AmberTopology.cpp:392-444``).

Every floating value is formatted to text and parsed back before it is
returned, so the arrays handed to the GPU engine are bit-identical to what a
parser of the written files obtains.  Charges are stored by the reference as
``prmtop_charge / 18.2206899283247`` computed in ``long double``
(``src/AmberTopology/TopologyParser.cpp:44-56``); ``q`` reproduces that.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

# Square root of the Coulomb constant used by the reference, in its own units
# (src/AmberTopology/TopologyParser.cpp:52, src/NonBonded/CoulombicEE.cpp:12).
SQRT_KC_STR = "18.2206899283247"
SQRT_KC = float(SQRT_KC_STR)
KC = float(np.longdouble(SQRT_KC_STR) * np.longdouble(SQRT_KC_STR))

WATER_R_OH = 0.9572
WATER_THETA = math.radians(104.52)
WATER_K_BOND = 450.0
WATER_K_ANGLE = 55.0
WATER_O_SIGMA, WATER_O_EPS = 3.1507, 0.1521
CMAP_RES = 24
N_CMAP_SETS = 5


def _fmt_e(v):
    return "%16.8E" % v


def _rt(vals, fmt="%16.8E"):
    """Round-trip values through their text form (what a parser will read)."""
    a = np.asarray(vals, dtype=np.float64)
    return np.array([float(fmt % x) for x in a.ravel()], dtype=np.float64).reshape(a.shape)


def _rt_coord(a):
    a = np.asarray(a, dtype=np.float64)
    return np.array([float("%12.7f" % x) for x in a.ravel()]).reshape(a.shape)


def charge_to_internal(prmtop_charge):
    """prmtop charge -> the reference's internal charge (long double divide)."""
    c = np.asarray(prmtop_charge, dtype=np.float64)
    ld = np.array([np.longdouble("%16.8E" % x) for x in c], dtype=np.longdouble)
    return (ld / np.longdouble(SQRT_KC_STR)).astype(np.float64)


@dataclass
class SynthSystem:
    """A generated system in prmtop terms (0-based atom indices)."""
    name: str
    box: np.ndarray                    # (3,) Angstrom, orthorhombic
    coords: np.ndarray                 # (N,3) unwrapped, molecules whole
    atom_names: list
    charge_prmtop: np.ndarray          # (N,) prmtop units (e * 18.22...)
    q: np.ndarray                      # (N,) reference internal units
    mass: np.ndarray
    atomic_number: np.ndarray
    type_index: np.ndarray             # (N,) 1-based atom type
    ntypes: int
    nb_parm_index: np.ndarray          # (ntypes*ntypes,) 1-based into lj tables
    lj_a: np.ndarray
    lj_b: np.ndarray
    lj14_a: np.ndarray
    lj14_b: np.ndarray
    bond_k: np.ndarray
    bond_r0: np.ndarray
    bonds_h: np.ndarray                # (M,3) i, j, type(0-based)
    bonds_noh: np.ndarray
    angle_k: np.ndarray
    angle_t0: np.ndarray
    angles_h: np.ndarray               # (M,4) i, j, k, type
    angles_noh: np.ndarray
    dih_k: np.ndarray
    dih_n: np.ndarray
    dih_phase: np.ndarray
    scee: np.ndarray
    scnb: np.ndarray
    dihedrals_h: np.ndarray            # (M,7) i,j,k,l,type,exclude14,improper
    dihedrals_noh: np.ndarray
    ub_k: np.ndarray
    ub_r0: np.ndarray
    ub: np.ndarray                     # (M,3) i, j, type
    imp_k: np.ndarray
    imp_phase: np.ndarray
    impropers: np.ndarray              # (M,5) i,j,k,l,type
    cmap_res: np.ndarray               # (5,)
    cmap_grids: np.ndarray             # (5, res*res) row-major [phi][psi]
    cmaps: np.ndarray                  # (M,6) a,b,c,d,e,set(1-based)
    excluded: list                     # per atom: sorted partners j>i (0-based)
    residue_labels: list
    residue_pointer: np.ndarray        # 1-based first atom of each residue
    meta: dict = field(default_factory=dict)

    @property
    def natoms(self):
        return int(self.coords.shape[0])


# --------------------------------------------------------------------------
# geometry helpers

def _rand_rot(rng, n):
    """n random rotation matrices (uniform quaternions)."""
    u1, u2, u3 = rng.random((3, n))
    q = np.stack([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2),
                  np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                  np.sqrt(u1) * np.sin(2 * np.pi * u3),
                  np.sqrt(u1) * np.cos(2 * np.pi * u3)], axis=1)
    x, y, z, w = q.T
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z); R[:, 0, 1] = 2 * (x * y - z * w); R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w); R[:, 1, 1] = 1 - 2 * (x * x + z * z); R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w); R[:, 2, 1] = 2 * (y * z + x * w); R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


class _Hash:
    """Periodic spatial hash for incremental overlap tests."""

    def __init__(self, box, cell):
        self.box = np.asarray(box, float)
        self.n = np.maximum(1, (self.box // cell).astype(int))
        self.cell = self.box / self.n
        self.d = {}
        self.pts = []

    def key(self, p):
        w = p - self.box * np.floor(p / self.box)
        return tuple(np.minimum((w / self.cell).astype(int), self.n - 1))

    def add(self, p, tag):
        self.d.setdefault(self.key(p), []).append(len(self.pts))
        self.pts.append((np.array(p, float), tag))

    def near(self, p, r):
        k = self.key(p)
        out = []
        rng = [range(-1, 2) if self.n[d] > 2 else range(self.n[d]) for d in range(3)]
        seen = set()
        for dx in rng[0]:
            for dy in rng[1]:
                for dz in rng[2]:
                    if self.n[0] > 2:
                        kk0 = (k[0] + dx) % self.n[0]
                    else:
                        kk0 = dx
                    kk1 = (k[1] + dy) % self.n[1] if self.n[1] > 2 else dy
                    kk2 = (k[2] + dz) % self.n[2] if self.n[2] > 2 else dz
                    kk = (kk0, kk1, kk2)
                    if kk in seen:
                        continue
                    seen.add(kk)
                    for idx in self.d.get(kk, ()):
                        q, tag = self.pts[idx]
                        dd = p - q
                        dd -= self.box * np.round(dd / self.box)
                        if dd @ dd < r * r:
                            out.append(tag)
        return out


def _chain_clear(pos, box, dmin):
    """No two chain atoms more than three bonds apart closer than dmin (min image)."""
    from scipy.spatial import cKDTree
    w = pos - box * np.floor(pos / box)
    w = np.minimum(w, np.nextafter(box, 0))
    pairs = cKDTree(w, boxsize=box).query_pairs(dmin, output_type="ndarray")
    return not np.any(np.abs(pairs[:, 0] - pairs[:, 1]) > 3) if len(pairs) else True


def _place_next(a, b, c, r, theta, phi):
    """Position d with |cd|=r, angle(b,c,d)=theta, dihedral(a,b,c,d)=phi."""
    bc = c - b
    bc /= np.linalg.norm(bc)
    n = np.cross(b - a, bc)
    nn = np.linalg.norm(n)
    if nn < 1e-8:
        n = np.cross(bc, [1.0, 0.0, 0.0])
        if np.linalg.norm(n) < 1e-8:
            n = np.cross(bc, [0.0, 1.0, 0.0])
        nn = np.linalg.norm(n)
    n /= nn
    m = np.cross(n, bc)
    d2 = np.array([-r * math.cos(theta), r * math.sin(theta) * math.cos(phi), r * math.sin(theta) * math.sin(phi)])
    return c + d2[0] * bc + d2[1] * m + d2[2] * n


# --------------------------------------------------------------------------

def make_system(name, box, n_waters, n_residues, seed, atoms_per_residue=10,
                n_chain_types=40, sentinels=False, water_first=False, min_contact=0.0):
    """Build one seeded system.

    box: cubic edge (float) or 3-tuple.  ``sentinels`` appends a zero-force-
    constant tuple to every term list the reference's loaders truncate
    (``src/AmberTopology/CreateBondedFromParsed.cpp:11,74,100,126,152,178,220,262``),
    so that reference-semantics and physical-semantics term sets coincide.
    ``min_contact`` > 0 rejects chain positions closer than that to any earlier
    chain atom more than three bonds away (used by the batch systems, whose
    small boxes crowd the walk).
    """
    rng = np.random.default_rng(seed)
    box = np.array([box] * 3 if np.isscalar(box) else box, dtype=np.float64)
    n_chain = n_residues * atoms_per_residue if n_residues > 0 else 0

    # ---------------- chain (self avoiding walk, periodic min-image checks)
    chain_types_sigma = rng.uniform(2.5, 4.0, n_chain_types)
    chain_types_eps = rng.uniform(0.02, 0.2, n_chain_types)
    n_bond_types_chain = 12
    bond_k_c = rng.uniform(200.0, 500.0, n_bond_types_chain)
    bond_r0_c = rng.uniform(1.0, 1.6, n_bond_types_chain)
    n_angle_types_chain = 12
    angle_k_c = rng.uniform(30.0, 100.0, n_angle_types_chain)
    angle_t0_c = np.radians(rng.uniform(100.0, 120.0, n_angle_types_chain))

    chain_pos = np.zeros((n_chain, 3))
    chain_bond_type = rng.integers(0, n_bond_types_chain, max(n_chain - 1, 0))
    chain_angle_type = rng.integers(0, n_angle_types_chain, max(n_chain - 2, 0))
    for _retry in range(50 if min_contact > 0 else 1):
        walk_ok = True
        if n_chain > 0:
            hsh = _Hash(box, 3.0)
            center = box / 2.0
            start = center + rng.uniform(-1, 1, 3)
            chain_pos[0] = start
            hsh.add(chain_pos[0], 0)
            for i in range(1, n_chain):
                r = bond_r0_c[chain_bond_type[i - 1]] * (1.0 + rng.normal(0, 0.02))
                best, best_score = None, -1e9
                fallback = None
                for attempt in range(400 if min_contact > 0 else 60):
                    if i == 1:
                        v = rng.normal(size=3); v /= np.linalg.norm(v)
                        cand = chain_pos[0] + r * v
                    else:
                        th = angle_t0_c[chain_angle_type[i - 2]] + rng.normal(0, 0.03)
                        ph = rng.uniform(-math.pi, math.pi)
                        a = chain_pos[i - 3] if i >= 3 else chain_pos[i - 2] + np.array([0.3, 0.7, 0.1])
                        cand = _place_next(a, chain_pos[i - 2], chain_pos[i - 1], r, th, ph)
                    if np.any(np.abs(cand - center) > 0.62 * box):
                        fallback = cand
                        continue
                    if min_contact > 0 and [t for t in hsh.near(cand, min_contact) if t < i - 3]:
                        continue
                    near = [t for t in hsh.near(cand, 2.7) if t < i - 3]
                    if not near:
                        best = cand
                        break
                    score = -len(near)
                    if score > best_score or best is None:
                        best, best_score = cand, score
                if best is None:
                    best = fallback
                if best is None:        # crowded: start the walk again
                    walk_ok = False
                    break
                chain_pos[i] = best
                hsh.add(best, i)
        if walk_ok and (min_contact <= 0 or n_chain == 0 or _chain_clear(chain_pos, box, min_contact)):
            break
    else:
        raise RuntimeError("chain walk found no clash-free path for %s" % name)

    # ---------------- waters on a jittered lattice
    nl = int(math.ceil(n_waters ** (1.0 / 3.0) - 1e-9)) if n_waters > 0 else 0
    if n_waters > 0:
        while nl ** 3 < n_waters:
            nl += 1
        a = box / nl
        sites = np.stack(np.meshgrid(np.arange(nl), np.arange(nl), np.arange(nl), indexing="ij"), -1).reshape(-1, 3)
        pick = rng.choice(sites.shape[0], size=n_waters, replace=False)
        pick.sort()
        O = (sites[pick] + 0.5) * a + rng.uniform(-0.2, 0.2, (n_waters, 3))
        R = _rand_rot(rng, n_waters)
        h1 = np.array([WATER_R_OH, 0.0, 0.0])
        h2 = np.array([WATER_R_OH * math.cos(WATER_THETA), WATER_R_OH * math.sin(WATER_THETA), 0.0])
        H1 = O + np.einsum("nij,j->ni", R, h1) + rng.normal(0, 0.01, (n_waters, 3))
        H2 = O + np.einsum("nij,j->ni", R, h2) + rng.normal(0, 0.01, (n_waters, 3))
        keep = np.ones(n_waters, bool)
        if n_chain > 0:
            from scipy.spatial import cKDTree
            wrapped_c = chain_pos - box * np.floor(chain_pos / box)
            tree = cKDTree(wrapped_c, boxsize=box)
            for arr in (O, H1, H2):
                w = arr - box * np.floor(arr / box)
                w = np.minimum(w, np.nextafter(box, 0))
                d, _ = tree.query(w, k=1)
                keep &= d > 2.5
        O, H1, H2 = O[keep], H1[keep], H2[keep]
    else:
        O = H1 = H2 = np.zeros((0, 3))
    nw = O.shape[0]

    # ---------------- atom ordering: chain first (Amber convention) unless water_first
    water_pos = np.stack([O, H1, H2], axis=1).reshape(-1, 3)
    if water_first:
        coords = np.concatenate([water_pos, chain_pos])
        w0, c0 = 0, 3 * nw
    else:
        coords = np.concatenate([chain_pos, water_pos])
        c0, w0 = 0, n_chain
    N = coords.shape[0]
    coords = _rt_coord(coords)

    # ---------------- types / LJ tables (Lorentz-Berthelot)
    ntypes = n_chain_types + 2
    sig = np.concatenate([chain_types_sigma, [WATER_O_SIGMA, 0.0]])
    eps = np.concatenate([chain_types_eps, [WATER_O_EPS, 0.0]])
    tO, tH = n_chain_types + 1, n_chain_types + 2       # 1-based
    type_index = np.zeros(N, np.int64)
    chain_atom_types = rng.integers(1, n_chain_types + 1, n_chain)
    type_index[c0:c0 + n_chain] = chain_atom_types
    type_index[w0:w0 + 3 * nw:3] = tO
    type_index[w0 + 1:w0 + 3 * nw:3] = tH
    type_index[w0 + 2:w0 + 3 * nw:3] = tH
    npair = ntypes * (ntypes + 1) // 2
    lj_a = np.zeros(npair); lj_b = np.zeros(npair)
    nb_idx = np.zeros(ntypes * ntypes, np.int64)
    for i in range(1, ntypes + 1):
        for j in range(1, ntypes + 1):
            hi, lo = max(i, j), min(i, j)
            ico = hi * (hi - 1) // 2 + lo
            nb_idx[(i - 1) * ntypes + (j - 1)] = ico
            if i >= j:
                s = 0.5 * (sig[i - 1] + sig[j - 1])
                e = math.sqrt(eps[i - 1] * eps[j - 1])
                if sig[i - 1] == 0.0 or sig[j - 1] == 0.0:
                    e = 0.0
                lj_a[ico - 1] = 4 * e * s ** 12
                lj_b[ico - 1] = 4 * e * s ** 6
    lj_a, lj_b = _rt(lj_a), _rt(lj_b)
    lj14_a, lj14_b = lj_a.copy(), lj_b.copy()

    # ---------------- charges
    charge_e = np.zeros(N)
    if n_chain > 0:
        cq = rng.normal(0, 0.3, n_chain)
        cq -= cq.mean()
        charge_e[c0:c0 + n_chain] = cq
    charge_e[w0:w0 + 3 * nw:3] = -0.834
    charge_e[w0 + 1:w0 + 3 * nw:3] = 0.417
    charge_e[w0 + 2:w0 + 3 * nw:3] = 0.417
    charge_prmtop = _rt(charge_e * SQRT_KC)
    q = charge_to_internal(charge_prmtop)

    mass = np.zeros(N); atomic_number = np.zeros(N, np.int64)
    mass[c0:c0 + n_chain] = 12.011; atomic_number[c0:c0 + n_chain] = 6
    mass[w0:w0 + 3 * nw:3] = 15.999; atomic_number[w0:w0 + 3 * nw:3] = 8
    mass[w0 + 1:w0 + 3 * nw:3] = 1.008; atomic_number[w0 + 1:w0 + 3 * nw:3] = 1
    mass[w0 + 2:w0 + 3 * nw:3] = 1.008; atomic_number[w0 + 2:w0 + 3 * nw:3] = 1
    names = ["C%-3d" % (i % 1000) if False else ("C" + str(i % 10)) for i in range(n_chain)]
    atom_names = [None] * N
    for i in range(n_chain):
        atom_names[c0 + i] = names[i]
    for w in range(nw):
        atom_names[w0 + 3 * w] = "OH2"; atom_names[w0 + 3 * w + 1] = "H1"; atom_names[w0 + 3 * w + 2] = "H2"

    # ---------------- bonded tables
    # bond types: 0 = water O-H, 1.. chain
    bond_k = _rt(np.concatenate([[WATER_K_BOND], bond_k_c]))
    bond_r0 = _rt(np.concatenate([[WATER_R_OH], bond_r0_c]))
    angle_k = _rt(np.concatenate([[WATER_K_ANGLE], angle_k_c]))
    angle_t0 = _rt(np.concatenate([[WATER_THETA], angle_t0_c]))
    bonds_h = []
    angles_h = []
    for w in range(nw):
        o = w0 + 3 * w
        bonds_h.append((o, o + 1, 0)); bonds_h.append((o, o + 2, 0))
        angles_h.append((o + 1, o, o + 2, 0))
    bonds_noh = [(c0 + i, c0 + i + 1, 1 + int(chain_bond_type[i])) for i in range(n_chain - 1)]
    angles_noh = [(c0 + i, c0 + i + 1, c0 + i + 2, 1 + int(chain_angle_type[i])) for i in range(n_chain - 2)]

    n_dih_types = 24
    dih_k = _rt(rng.uniform(0.1, 2.0, n_dih_types))
    dih_n = _rt(rng.integers(1, 4, n_dih_types).astype(float))
    dih_phase = _rt(rng.choice([0.0, math.pi], n_dih_types))
    scee = _rt(np.full(n_dih_types, 1.2))
    scnb = _rt(np.full(n_dih_types, 2.0))
    dihedrals = []  # (i,j,k,l,type,excl14,improper)
    for i in range(n_chain - 3):
        t = int(rng.integers(0, n_dih_types))
        dihedrals.append((c0 + i, c0 + i + 1, c0 + i + 2, c0 + i + 3, t, 0, 0))
        if rng.random() < 0.3:  # second Fourier term on the same quadruplet
            t2 = int(rng.integers(0, n_dih_types))
            dihedrals.append((c0 + i, c0 + i + 1, c0 + i + 2, c0 + i + 3, t2, 1, 0))
    for i in range(1, n_chain - 3, 9):  # Amber-style improper carried by the dihedral list
        t = int(rng.integers(0, n_dih_types))
        dihedrals.append((c0 + i, c0 + i + 1, c0 + i + 2, c0 + i + 3, t, 1, 1))
    # split between the "with H" and "without H" lists
    dih_h = [d for k, d in enumerate(dihedrals) if k % 3 == 0]
    dih_noh = [d for k, d in enumerate(dihedrals) if k % 3 != 0]

    n_ub_types = 8
    ub_k = _rt(rng.uniform(5.0, 50.0, n_ub_types))
    ub_r0 = _rt(rng.uniform(2.0, 2.6, n_ub_types))
    ub = [(c0 + i, c0 + i + 2, int(rng.integers(0, n_ub_types))) for i in range(0, n_chain - 2, 2)]

    n_imp_types = 6
    imp_k = _rt(rng.uniform(10.0, 100.0, n_imp_types))
    imp_phase = _rt(np.array([0.0, 0.0, 0.0, 0.0, 2.8, -2.8][:n_imp_types]))
    impropers = [(c0 + i, c0 + i + 1, c0 + i + 2, c0 + i + 3, int(rng.integers(0, n_imp_types)))
                 for i in range(0, n_chain - 3, 4)]

    # CMAP: 5 sets of smooth periodic 24x24 grids (low Fourier modes)
    res = CMAP_RES
    ang = -math.pi + 2 * math.pi * np.arange(res) / res
    P, S = np.meshgrid(ang, ang, indexing="ij")
    grids = np.zeros((N_CMAP_SETS, res * res))
    for s in range(N_CMAP_SETS):
        g = np.zeros((res, res))
        for m1 in range(0, 3):
            for m2 in range(0, 3):
                amp = rng.normal(0, 1.0)
                p1, p2 = rng.uniform(0, 2 * math.pi, 2)
                g += amp * np.cos(m1 * P + p1) * np.cos(m2 * S + p2)
        g *= 2.0 / max(1e-9, np.abs(g).max())
        grids[s] = _rt(g.ravel(), "%16.8E")
    cmaps = [(c0 + i, c0 + i + 1, c0 + i + 2, c0 + i + 3, c0 + i + 4, int(rng.integers(1, N_CMAP_SETS + 1)))
             for i in range(0, n_chain - 4, atoms_per_residue // 2 if atoms_per_residue >= 2 else 1)]

    if sentinels:
        # one zero-constant tuple per truncated list; parameters get a dedicated zero type
        bond_k = np.concatenate([bond_k, [0.0]]); bond_r0 = np.concatenate([bond_r0, [1.0]])
        zb = len(bond_k) - 1
        angle_k = np.concatenate([angle_k, [0.0]]); angle_t0 = np.concatenate([angle_t0, [1.9]])
        za = len(angle_k) - 1
        dih_k = np.concatenate([dih_k, [0.0]]); dih_n = np.concatenate([dih_n, [1.0]])
        dih_phase = np.concatenate([dih_phase, [0.0]]); scee = np.concatenate([scee, [1.2]])
        scnb = np.concatenate([scnb, [2.0]])
        zd = len(dih_k) - 1
        ub_k = np.concatenate([ub_k, [0.0]]); ub_r0 = np.concatenate([ub_r0, [2.0]])
        zu = len(ub_k) - 1
        # sentinel atoms: 1,2,3,4 (never atom 0 in a signed slot)
        a1, a2, a3, a4, a5 = 1, 2, 3, 4, 5
        bonds_h.append((a1, a2, zb)); bonds_noh.append((a1, a2, zb))
        angles_h.append((a1, a2, a3, za)); angles_noh.append((a1, a2, a3, za))
        dih_h.append((a1, a2, a3, a4, zd, 1, 0)); dih_noh.append((a1, a2, a3, a4, zd, 1, 0))
        ub.append((a1, a3, zu))
        grids = np.concatenate([grids, np.zeros((0, res * res))])
        cmaps.append((a1, a2, a3, a4, a5, 0))   # set 0 is remapped below to a zero grid

    cmap_res = np.full(N_CMAP_SETS, res, np.int64)
    if sentinels:
        # a zero CMAP term needs a zero grid: make set 5 the zero set, remap users
        cmaps = [c if c[5] != 5 else c[:5] + (4,) for c in cmaps]
        cmaps = [c if c[5] != 0 else c[:5] + (5,) for c in cmaps]
        grids[4] = 0.0

    # ---------------- exclusions (1-2, 1-3, 1-4 over bonds/angles/dihedrals), j>i only
    excl = [set() for _ in range(N)]

    def _ex(i, j):
        if i == j:
            return
        a, b = min(i, j), max(i, j)
        excl[a].add(b)
    for (i, j, t) in bonds_h + bonds_noh:
        _ex(i, j)
    for (i, j, k, t) in angles_h + angles_noh:
        _ex(i, j); _ex(j, k); _ex(i, k)
    for (i, j, k, l, t, e14, imp) in dih_h + dih_noh:
        _ex(i, j); _ex(j, k); _ex(k, l); _ex(i, k); _ex(j, l); _ex(i, l)
    excluded = [sorted(s) for s in excl]

    # residues: chain residues of atoms_per_residue, waters one residue each
    labels, ptr = [], []
    order = [("chain", c0, n_chain), ("water", w0, 3 * nw)]
    if water_first:
        order = order[::-1]
    for kind, s0, cnt in order:
        if kind == "chain":
            for r in range(0, cnt, atoms_per_residue):
                labels.append("RES"); ptr.append(s0 + r + 1)
        else:
            for r in range(0, cnt, 3):
                labels.append("TIP3"); ptr.append(s0 + r + 1)

    def arr(x, w):
        return np.array(x, dtype=np.int64).reshape(-1, w)

    return SynthSystem(
        name=name, box=_rt(box, "%12.7f"), coords=coords, atom_names=atom_names,
        charge_prmtop=charge_prmtop, q=q, mass=_rt(mass), atomic_number=atomic_number,
        type_index=type_index, ntypes=ntypes, nb_parm_index=nb_idx,
        lj_a=lj_a, lj_b=lj_b, lj14_a=lj14_a, lj14_b=lj14_b,
        bond_k=bond_k, bond_r0=bond_r0, bonds_h=arr(bonds_h, 3), bonds_noh=arr(bonds_noh, 3),
        angle_k=angle_k, angle_t0=angle_t0, angles_h=arr(angles_h, 4), angles_noh=arr(angles_noh, 4),
        dih_k=dih_k, dih_n=dih_n, dih_phase=dih_phase, scee=scee, scnb=scnb,
        dihedrals_h=arr(dih_h, 7), dihedrals_noh=arr(dih_noh, 7),
        ub_k=ub_k, ub_r0=ub_r0, ub=arr(ub, 3),
        imp_k=imp_k, imp_phase=imp_phase, impropers=arr(impropers, 5),
        cmap_res=cmap_res, cmap_grids=grids, cmaps=arr(cmaps, 6),
        excluded=excluded, residue_labels=labels, residue_pointer=np.array(ptr, np.int64),
        meta=dict(seed=seed, n_waters=nw, n_chain=n_chain, sentinels=sentinels))


# --------------------------------------------------------------------------
# named workloads

CONFIGS = {
    # small cases the oracle finishes in well under a second
    "tiny": dict(box=22.0, n_waters=300, n_residues=3, seed=11),
    "small": dict(box=30.0, n_waters=800, n_residues=8, seed=12),
    # 66 A cube, about 9,000 waters (after removing those overlapping the
    # chain) + a 120-residue chain: about 28k atoms
    "c0": dict(box=66.0, n_waters=10050, n_residues=120, seed=1000),
    # 100 A cube, about 32,000 waters (after overlap removal) + a 400-residue
    # chain: about 100k atoms
    "c1": dict(box=100.0, n_waters=35300, n_residues=400, seed=1001),
    # 215 A cube of about 320,000 waters (about 960k atoms)
    "c4": dict(box=215.0, n_waters=320000, n_residues=0, seed=1004),
}

# PME grids used with each named workload
GRIDS = {"tiny": (24, 24, 24), "small": (32, 32, 32), "c0": (72, 72, 72),
         "c1": (100, 100, 100), "c4": (216, 216, 216)}


def make_config(name, sentinels=False, **over):
    kw = dict(CONFIGS[name]); kw.update(over)
    return make_system(name, sentinels=sentinels, **kw)


def smooth_grid_size(L, spacing=1.0):
    """Smallest 2^a 3^b 5^c >= L/spacing."""
    n = int(math.ceil(L / spacing - 1e-9))
    while True:
        m = n
        for p in (2, 3, 5):
            while m % p == 0:
                m //= p
        if m == 1:
            return n
        n += 1


def _batch_dims(n_systems, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_systems):
        L = float(rng.uniform(25.0, 40.0))
        nres = int(rng.integers(10, 31))
        out.append((L, nres))
    return out


def make_batch_member(k, n_systems=256, seed=1003):
    """System k of make_batch(n_systems, seed), built on its own."""
    L, nres = _batch_dims(n_systems, seed)[k]
    # water count for roughly 0.1 atoms / A^3 minus the chain share
    nw = max(10, int(0.1 * L ** 3 / 3.0) - nres * 10 // 3)
    sysm = make_system("batch%03d" % k, L, nw, nres, seed * 1000 + k, min_contact=2.0)
    g = smooth_grid_size(sysm.box[0], 1.0)
    sysm.meta["grid"] = (g, g, g)
    return sysm


def make_batch(n_systems=256, seed=1003):
    """Uneven independent systems: edge U(25,40) A, 10-30-residue chain."""
    return [make_batch_member(k, n_systems, seed) for k in range(n_systems)]


# --------------------------------------------------------------------------
# writers

def _write_section(f, flag, fmt, values, per_line, conv):
    f.write("%%FLAG %s\n" % flag)
    f.write("%%FORMAT(%s)\n" % fmt)
    vals = list(values)
    if not vals:
        f.write("\n")
        return
    for s in range(0, len(vals), per_line):
        f.write("".join(conv(v) for v in vals[s:s + per_line]) + "\n")


def _ifmt(v):
    return "%8d" % v


def write_prmtop(sysm: SynthSystem, path):
    N = sysm.natoms
    bonds_h, bonds_noh = sysm.bonds_h, sysm.bonds_noh
    ang_h, ang_noh = sysm.angles_h, sysm.angles_noh
    dh, dnh = sysm.dihedrals_h, sysm.dihedrals_noh
    nexcl = [max(1, len(e)) for e in sysm.excluded]
    excl_flat = []
    for e in sysm.excluded:
        excl_flat.extend([j + 1 for j in e] if e else [0])
    npair = len(sysm.lj_a)
    pointers = [N, sysm.ntypes, len(bonds_h), len(bonds_noh), len(ang_h), len(ang_noh), len(dh), len(dnh),
                0, 0, len(excl_flat), len(sysm.residue_labels), len(bonds_noh), len(ang_noh), len(dnh),
                len(sysm.bond_k), len(sysm.angle_k), len(sysm.dih_k), 1, 0, 0, 0, 0, 0, 0, 0, 0,
                1, 10, 0, 0]

    def dih_entries(d):
        out = []
        for (i, j, k, l, t, e14, imp) in d:
            kk = -3 * k if e14 else 3 * k
            ll = -3 * l if imp else 3 * l
            out += [3 * i, 3 * j, kk, ll, t + 1]
        return out

    with open(path, "w") as f:
        f.write("%VERSION  VERSION_STAMP = V0001.000  DATE = 12/03/26  00:00:00\n")
        f.write("%FLAG TITLE\n%FORMAT(20a4)\n" + sysm.name[:80] + "\n")
        _write_section(f, "POINTERS", "10I8", pointers, 10, _ifmt)
        _write_section(f, "ATOM_NAME", "20a4", sysm.atom_names, 20, lambda s: "%-4s" % s[:4])
        _write_section(f, "CHARGE", "5E16.8", sysm.charge_prmtop, 5, _fmt_e)
        _write_section(f, "ATOMIC_NUMBER", "10I8", sysm.atomic_number, 10, _ifmt)
        _write_section(f, "MASS", "5E16.8", sysm.mass, 5, _fmt_e)
        _write_section(f, "ATOM_TYPE_INDEX", "10I8", sysm.type_index, 10, _ifmt)
        _write_section(f, "NUMBER_EXCLUDED_ATOMS", "10I8", nexcl, 10, _ifmt)
        _write_section(f, "NONBONDED_PARM_INDEX", "10I8", sysm.nb_parm_index, 10, _ifmt)
        _write_section(f, "RESIDUE_LABEL", "20a4", sysm.residue_labels, 20, lambda s: "%-4s" % s[:4])
        _write_section(f, "RESIDUE_POINTER", "10I8", sysm.residue_pointer, 10, _ifmt)
        _write_section(f, "BOND_FORCE_CONSTANT", "5E16.8", sysm.bond_k, 5, _fmt_e)
        _write_section(f, "BOND_EQUIL_VALUE", "5E16.8", sysm.bond_r0, 5, _fmt_e)
        _write_section(f, "ANGLE_FORCE_CONSTANT", "5E16.8", sysm.angle_k, 5, _fmt_e)
        _write_section(f, "ANGLE_EQUIL_VALUE", "5E16.8", sysm.angle_t0, 5, _fmt_e)
        _write_section(f, "CHARMM_UREY_BRADLEY_COUNT", "2I8", [len(sysm.ub), len(sysm.ub_k)], 2, _ifmt)
        _write_section(f, "CHARMM_UREY_BRADLEY", "10I8",
                       [v for (i, j, t) in sysm.ub for v in (i + 1, j + 1, t + 1)], 10, _ifmt)
        _write_section(f, "CHARMM_UREY_BRADLEY_FORCE_CONSTANT", "5E16.8", sysm.ub_k, 5, _fmt_e)
        _write_section(f, "CHARMM_UREY_BRADLEY_EQUIL_VALUE", "5E16.8", sysm.ub_r0, 5, _fmt_e)
        _write_section(f, "DIHEDRAL_FORCE_CONSTANT", "5E16.8", sysm.dih_k, 5, _fmt_e)
        _write_section(f, "DIHEDRAL_PERIODICITY", "5E16.8", sysm.dih_n, 5, _fmt_e)
        _write_section(f, "DIHEDRAL_PHASE", "5E16.8", sysm.dih_phase, 5, _fmt_e)
        _write_section(f, "SCEE_SCALE_FACTOR", "5E16.8", sysm.scee, 5, _fmt_e)
        _write_section(f, "SCNB_SCALE_FACTOR", "5E16.8", sysm.scnb, 5, _fmt_e)
        _write_section(f, "CHARMM_NUM_IMPROPERS", "10I8", [len(sysm.impropers)], 10, _ifmt)
        _write_section(f, "CHARMM_IMPROPERS", "10I8",
                       [v for r in sysm.impropers for v in (r[0] + 1, r[1] + 1, r[2] + 1, r[3] + 1, r[4] + 1)],
                       10, _ifmt)
        _write_section(f, "CHARMM_NUM_IMPR_TYPES", "I8", [len(sysm.imp_k)], 1, _ifmt)
        _write_section(f, "CHARMM_IMPROPER_FORCE_CONSTANT", "5E16.8", sysm.imp_k, 5, _fmt_e)
        _write_section(f, "CHARMM_IMPROPER_PHASE", "5E16.8", sysm.imp_phase, 5, _fmt_e)
        _write_section(f, "LENNARD_JONES_ACOEF", "5E16.8", sysm.lj_a, 5, _fmt_e)
        _write_section(f, "LENNARD_JONES_BCOEF", "5E16.8", sysm.lj_b, 5, _fmt_e)
        _write_section(f, "LENNARD_JONES_14_ACOEF", "5E16.8", sysm.lj14_a, 5, _fmt_e)
        _write_section(f, "LENNARD_JONES_14_BCOEF", "5E16.8", sysm.lj14_b, 5, _fmt_e)
        _write_section(f, "BONDS_INC_HYDROGEN", "10I8",
                       [v for (i, j, t) in bonds_h for v in (3 * i, 3 * j, t + 1)], 10, _ifmt)
        _write_section(f, "BONDS_WITHOUT_HYDROGEN", "10I8",
                       [v for (i, j, t) in bonds_noh for v in (3 * i, 3 * j, t + 1)], 10, _ifmt)
        _write_section(f, "ANGLES_INC_HYDROGEN", "10I8",
                       [v for (i, j, k, t) in ang_h for v in (3 * i, 3 * j, 3 * k, t + 1)], 10, _ifmt)
        _write_section(f, "ANGLES_WITHOUT_HYDROGEN", "10I8",
                       [v for (i, j, k, t) in ang_noh for v in (3 * i, 3 * j, 3 * k, t + 1)], 10, _ifmt)
        _write_section(f, "DIHEDRALS_INC_HYDROGEN", "10I8", dih_entries(dh), 10, _ifmt)
        _write_section(f, "DIHEDRALS_WITHOUT_HYDROGEN", "10I8", dih_entries(dnh), 10, _ifmt)
        _write_section(f, "EXCLUDED_ATOMS_LIST", "10I8", excl_flat, 10, _ifmt)
        _write_section(f, "BOX_DIMENSIONS", "5E16.8", [90.0] + list(sysm.box), 5, _fmt_e)
        _write_section(f, "CHARMM_CMAP_COUNT", "2I8", [len(sysm.cmaps), N_CMAP_SETS], 2, _ifmt)
        _write_section(f, "CHARMM_CMAP_RESOLUTION", "20I4", sysm.cmap_res, 20, lambda v: "%4d" % v)
        for s in range(N_CMAP_SETS):
            _write_section(f, "CHARMM_CMAP_PARAMETER_%02d" % (s + 1), "8(F9.5)", sysm.cmap_grids[s], 8,
                           lambda v: " " + _fmt_e(v))
        _write_section(f, "CHARMM_CMAP_INDEX", "6I8",
                       [v for r in sysm.cmaps for v in (r[0] + 1, r[1] + 1, r[2] + 1, r[3] + 1, r[4] + 1, r[5])],
                       6, _ifmt)


def write_rst7(sysm: SynthSystem, path):
    c = sysm.coords.ravel()
    with open(path, "w") as f:
        f.write(sysm.name[:80] + "\n")
        f.write("%6d\n" % sysm.natoms)
        for s in range(0, len(c), 6):
            f.write("".join("%12.7f" % v for v in c[s:s + 6]) + "\n")
        b = list(sysm.box) + [90.0, 90.0, 90.0]
        f.write("".join("%12.7f" % v for v in b) + "\n")


def write_files(sysm: SynthSystem, directory, stem=None):
    os.makedirs(directory, exist_ok=True)
    stem = stem or sysm.name
    p, r = os.path.join(directory, stem + ".prmtop"), os.path.join(directory, stem + ".rst7")
    write_prmtop(sysm, p)
    write_rst7(sysm, r)
    return p, r
