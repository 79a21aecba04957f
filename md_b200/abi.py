"""ctypes mirror of include/mdf.h (the C ABI of libmdf.so)."""
import ctypes as C

MDF_SEM_REFERENCE, MDF_SEM_PHYSICAL = 0, 1
MDF_PREC_FP64, MDF_PREC_MIXED = 0, 1

STATUS = {0: "MDF_OK", 1: "MDF_ERR_INVALID", 2: "MDF_ERR_CUDA", 3: "MDF_ERR_CAPACITY",
          4: "MDF_ERR_NONFINITE", 5: "MDF_ERR_OVERFLOW", 6: "MDF_ERR_TIMEOUT", 7: "MDF_ERR_STATE",
          8: "MDF_ERR_NOMEM", 9: "MDF_ERR_UNSUPPORTED"}

E_NAMES = ["bond", "angle", "dihedral", "ub", "improper", "cmap", "vdw", "vdw14", "ee", "ee_pairlist",
           "ee_cutoff", "ee_direct", "ee14", "ee_excl", "ee_self", "ee_recip"]
E_INDEX = {n: i for i, n in enumerate(E_NAMES)}
MDF_E_COUNT = len(E_NAMES)

MDF_OK, MDF_ERR_INVALID, MDF_ERR_CUDA, MDF_ERR_CAPACITY = 0, 1, 2, 3
MDF_ERR_NONFINITE, MDF_ERR_OVERFLOW, MDF_ERR_TIMEOUT, MDF_ERR_STATE = 4, 5, 6, 7
MDF_ERR_NOMEM, MDF_ERR_UNSUPPORTED = 8, 9
MDF_NOALLOC_MAX_ATOMS = 131072   # include/mdf.h: scratch limit of mdf_compute_bonded_noalloc
MDF_COMPUTE_ENERGY = 1
MDF_COMPUTE_FORCES = 2
MDF_COMPUTE_PME_REFERENCE = 4

# int (*)(uint64_t *d_buf, int64_t count, void *stream, void *user): the sum over ranks (mdf_set_allreduce)
MDF_ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p)
# (send, recv, count or bytes, stream, user) -> int: reduce-scatter, all-gather, all-to-all
MDF_REDUCE_SCATTER_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p)
MDF_ALLGATHER_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p)
MDF_ALLTOALL_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p)
# mdf_alltoallv_bytes(send, send_bytes[nranks], recv, recv_bytes[nranks], stream, user)
MDF_ALLTOALLV_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_int64), C.c_void_p, C.POINTER(C.c_int64),
                               C.c_void_p, C.c_void_p)

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class mdf_energies(C.Structure):
    _fields_ = [("e", C.c_double * MDF_E_COUNT), ("total", C.c_double), ("virial", C.c_double * 9)]

    def as_dict(self):
        d = {n: self.e[i] for i, n in enumerate(E_NAMES)}
        d["total"] = self.total
        return d


class mdf_topology(C.Structure):
    _fields_ = [
        ("natoms", C.c_int32), ("charge", _dp), ("type", _ip), ("ntypes", C.c_int32), ("nb_index", _ip),
        ("n_ljpair", C.c_int32), ("lj_a", _dp), ("lj_b", _dp), ("lj14_a", _dp), ("lj14_b", _dp),
        ("n_bonds", C.c_int32), ("bond_atoms", _ip), ("bond_k", _dp), ("bond_r0", _dp),
        ("n_ub", C.c_int32), ("ub_atoms", _ip), ("ub_k", _dp), ("ub_r0", _dp),
        ("n_angles", C.c_int32), ("angle_atoms", _ip), ("angle_k", _dp), ("angle_theta0", _dp),
        ("n_dihedrals", C.c_int32), ("dihedral_atoms", _ip),
        ("dihedral_k", _dp), ("dihedral_n", _dp), ("dihedral_phase", _dp),
        ("n_impropers", C.c_int32), ("improper_atoms", _ip), ("improper_k", _dp), ("improper_phase", _dp),
        ("n_cmaps", C.c_int32), ("cmap_atoms", _ip), ("cmap_set", _ip),
        ("cmap_nsets", C.c_int32), ("cmap_res", C.c_int32), ("cmap_coeff", _dp),
        ("n_excl", C.c_int32), ("excl_pairs", _ip),
        ("n_pairs14", C.c_int32), ("pairs14", _ip), ("scee14", _dp), ("scnb14", _dp),
    ]


class mdf_params(C.Structure):
    _fields_ = [
        ("semantics", C.c_int32), ("precision", C.c_int32), ("box", C.c_double * 3),
        ("cutoff", C.c_double), ("skin", C.c_double), ("switch_radius", C.c_double),
        ("ewald_tol", C.c_double), ("ewald_alpha", C.c_double), ("grid", C.c_int32 * 3),
        ("pme_order", C.c_int32), ("coulomb_const", C.c_double), ("device", C.c_int32),
        ("prune_every", C.c_int32), ("prune_margin", C.c_double), ("pair_warps", C.c_int32),
        ("fft_lines", C.c_int32), ("rank", C.c_int32), ("nranks", C.c_int32), ("pair_schedule", C.c_int32),
        ("pair_layout", C.c_int32),
    ]


class mdf_tune_report(C.Structure):
    _fields_ = [("pair_warps", C.c_int32), ("fft_lines", C.c_int32), ("prune_every", C.c_int32),
                ("n_tried", C.c_int32), ("best_ms", C.c_double), ("default_ms", C.c_double),
                ("pair_schedule", C.c_int32), ("pair_layout", C.c_int32)]


class mdf_md_report(C.Structure):
    _fields_ = [("steps", C.c_int64), ("rebuilds", C.c_int64), ("samples", C.c_int64), ("wall_s", C.c_double),
                ("pe_first", C.c_double), ("ke_first", C.c_double), ("pe_last", C.c_double),
                ("ke_last", C.c_double), ("rebuild_s", C.c_double), ("record_s", C.c_double), ("wait_s", C.c_double)]


class mdf_min_report(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("rebuilds", C.c_int32), ("e_initial", C.c_double),
                ("e_final", C.c_double), ("fmax_final", C.c_double), ("evaluations", C.c_int32),
                ("reserved", C.c_int32)]

