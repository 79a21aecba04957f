"""Flatten a parsed Amber/CHARMM topology into the mdf_topology C struct.

This is the host-side post-processing the reference performs after parsing
(src/AmberTopology/CreateBondedFromParsed.cpp, CreateNonBondedFromParsed.cpp),
with the semantics switch:

REFERENCE (as the reference runs)
  * the loaders for bonds, angles, dihedrals, Urey-Bradley and CMAP stop one
    tuple early (loop bounds ``i + w < size`` with step ``w``,
    CreateBondedFromParsed.cpp:11,74,100,126,152,178,220,262); impropers keep
    every tuple (:41);
  * exclusion lists stay empty (the push goes into a copy,
    CreateNonBondedFromParsed.cpp:33-36), so no pair is excluded and no pair is
    ever flagged 1-4.
PHYSICAL
  * every tuple;
  * the prmtop EXCLUDED_ATOMS_LIST plus the 1-4 set from proper dihedrals
    without the exclude-1-4 flag (CreateNonBondedFromParsed.cpp:124-169); SCEE
    (and SCNB) per 1-4 pair is the largest over the dihedrals that generate it
    (the reference's rule at :151-160).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi


class FlatTopology:
    """numpy arrays backing one mdf_topology; keeps them alive for ctypes."""

    def __init__(self, **arrays):
        self.__dict__.update(arrays)
        self._struct = None

    @property
    def natoms(self):
        return int(self.charge.shape[0])

    def struct(self):
        if self._struct is not None:
            return self._struct
        t = abi.mdf_topology()

        def dp(a):
            return a.ctypes.data_as(C.POINTER(C.c_double))

        def ip(a):
            return a.ctypes.data_as(C.POINTER(C.c_int32))
        t.natoms = self.natoms
        t.charge = dp(self.charge); t.type = ip(self.type); t.ntypes = self.ntypes
        t.nb_index = ip(self.nb_index); t.n_ljpair = len(self.lj_a)
        t.lj_a = dp(self.lj_a); t.lj_b = dp(self.lj_b); t.lj14_a = dp(self.lj14_a); t.lj14_b = dp(self.lj14_b)
        t.n_bonds = len(self.bond_k); t.bond_atoms = ip(self.bond_atoms); t.bond_k = dp(self.bond_k)
        t.bond_r0 = dp(self.bond_r0)
        t.n_ub = len(self.ub_k); t.ub_atoms = ip(self.ub_atoms); t.ub_k = dp(self.ub_k); t.ub_r0 = dp(self.ub_r0)
        t.n_angles = len(self.angle_k); t.angle_atoms = ip(self.angle_atoms); t.angle_k = dp(self.angle_k)
        t.angle_theta0 = dp(self.angle_theta0)
        t.n_dihedrals = len(self.dihedral_k); t.dihedral_atoms = ip(self.dihedral_atoms)
        t.dihedral_k = dp(self.dihedral_k); t.dihedral_n = dp(self.dihedral_n)
        t.dihedral_phase = dp(self.dihedral_phase)
        t.n_impropers = len(self.improper_k); t.improper_atoms = ip(self.improper_atoms)
        t.improper_k = dp(self.improper_k); t.improper_phase = dp(self.improper_phase)
        t.n_cmaps = len(self.cmap_set); t.cmap_atoms = ip(self.cmap_atoms); t.cmap_set = ip(self.cmap_set)
        t.cmap_nsets = self.cmap_nsets; t.cmap_res = self.cmap_res; t.cmap_coeff = dp(self.cmap_coeff)
        t.n_excl = len(self.excl_pairs) // 2; t.excl_pairs = ip(self.excl_pairs)
        t.n_pairs14 = len(self.scee14); t.pairs14 = ip(self.pairs14)
        t.scee14 = dp(self.scee14); t.scnb14 = dp(self.scnb14)
        self._struct = t
        return t


def _i32(a, w=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.int32))
    return a.reshape(-1) if w is None else a.reshape(-1)


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64)).reshape(-1)


def flatten(sysm, semantics, cmap_coeff_fn):
    """SynthSystem (or any object with the same prmtop fields) -> FlatTopology.

    cmap_coeff_fn(nsets, res, grids[nsets, res*res]) -> coeff[nsets*res*res*16]
    builds the REFERENCE CMAP table (the reference's 16x16-matrix patches).
    PHYSICAL semantics always use the C1 spline table of
    mdf_cmap_coefficients_spline instead: the reference's patches do not meet
    along the cell edges, so their energy jumps as a torsion crosses a grid
    line and dynamics cannot conserve energy.
    """
    ref = semantics == abi.MDF_SEM_REFERENCE

    def trunc(a):
        # REFERENCE: drop the last tuple (loop bound i + w < size)
        return a[:-1] if (ref and len(a) > 0) else a

    bonds = np.concatenate([trunc(sysm.bonds_h), trunc(sysm.bonds_noh)]).reshape(-1, 3)
    angles = np.concatenate([trunc(sysm.angles_h), trunc(sysm.angles_noh)]).reshape(-1, 4)
    dihs = np.concatenate([trunc(sysm.dihedrals_h), trunc(sysm.dihedrals_noh)]).reshape(-1, 7)
    ub = trunc(sysm.ub).reshape(-1, 3)
    cm = trunc(sysm.cmaps).reshape(-1, 6)
    imp = sysm.impropers.reshape(-1, 5)

    res = int(sysm.cmap_res[0]) if len(sysm.cmap_res) else 24
    nsets = int(sysm.cmap_grids.shape[0])
    grids = np.ascontiguousarray(sysm.cmap_grids, dtype=np.float64)
    if ref:
        coeff = _f64(cmap_coeff_fn(nsets, res, grids))
    else:
        from . import engine
        coeff = _f64(engine.cmap_coefficients_spline(nsets, res, grids))

    if ref:
        excl = np.zeros(0, np.int32)
        p14 = np.zeros(0, np.int32)
        scee = np.zeros(0)
        scnb = np.zeros(0)
    else:
        N = sysm.natoms
        ex = set()
        for i, js in enumerate(sysm.excluded):
            for j in js:
                ex.add((min(i, j), max(i, j)))
        near = set()
        for (i, j, t) in bonds:
            near.add((min(i, j), max(i, j)))
        for (i, j, k, t) in angles:
            near.add((min(i, k), max(i, k)))
        pairs14 = {}
        for (i, j, k, l, t, e14, impf) in dihs:
            if impf or e14:
                continue
            key = (min(i, l), max(i, l))
            if key in near:
                continue
            sc, sn = float(sysm.scee[t]), float(sysm.scnb[t])
            if key in pairs14:
                ps, pn = pairs14[key]
                pairs14[key] = (max(ps, sc), max(pn, sn))
            else:
                pairs14[key] = (sc, sn)
        for key in pairs14:
            ex.add(key)
        exl = sorted(ex)
        excl = _i32(np.array(exl, dtype=np.int64).reshape(-1, 2))
        keys = sorted(pairs14)
        p14 = _i32(np.array(keys, dtype=np.int64).reshape(-1, 2))
        scee = _f64([pairs14[k][0] for k in keys])
        scnb = _f64([pairs14[k][1] for k in keys])

    return FlatTopology(
        charge=_f64(sysm.q), type=_i32(np.asarray(sysm.type_index) - 1), ntypes=int(sysm.ntypes),
        nb_index=_i32(sysm.nb_parm_index),
        lj_a=_f64(sysm.lj_a), lj_b=_f64(sysm.lj_b), lj14_a=_f64(sysm.lj14_a), lj14_b=_f64(sysm.lj14_b),
        bond_atoms=_i32(bonds[:, :2]), bond_k=_f64(sysm.bond_k[bonds[:, 2]]), bond_r0=_f64(sysm.bond_r0[bonds[:, 2]]),
        ub_atoms=_i32(ub[:, :2]), ub_k=_f64(sysm.ub_k[ub[:, 2]]), ub_r0=_f64(sysm.ub_r0[ub[:, 2]]),
        angle_atoms=_i32(angles[:, :3]), angle_k=_f64(sysm.angle_k[angles[:, 3]]),
        angle_theta0=_f64(sysm.angle_t0[angles[:, 3]]),
        dihedral_atoms=_i32(dihs[:, :4]), dihedral_k=_f64(sysm.dih_k[dihs[:, 4]]),
        dihedral_n=_f64(sysm.dih_n[dihs[:, 4]]), dihedral_phase=_f64(sysm.dih_phase[dihs[:, 4]]),
        improper_atoms=_i32(imp[:, :4]), improper_k=_f64(sysm.imp_k[imp[:, 4]]),
        improper_phase=_f64(sysm.imp_phase[imp[:, 4]]),
        cmap_atoms=_i32(cm[:, :5]), cmap_set=_i32(cm[:, 5] - 1), cmap_nsets=nsets, cmap_res=res,
        cmap_coeff=coeff,
        excl_pairs=excl, pairs14=p14, scee14=scee, scnb14=scnb,
    )
