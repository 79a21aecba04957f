"""Python binding of libmdf (ctypes over include/mdf.h).

This is plumbing for tests, the benchmark and Python users; the product is
the C ABI.  There is no CPU fallback: without the built library or without a
CUDA device every call raises MDFError.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

_LIB = None
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libmdf.so")

EXPORTS = [
    "mdf_params_default", "mdf_create", "mdf_destroy", "mdf_last_error", "mdf_status_string",
    "mdf_set_positions", "mdf_set_positions_device", "mdf_set_box", "mdf_build_pairlist", "mdf_compute",
    "mdf_compute_async", "mdf_fetch", "mdf_submit", "mdf_collect", "mdf_forces_device", "mdf_get_pme_forces", "mdf_set_stream",
    "mdf_pairlist_info", "mdf_enable_timing", "mdf_kernel_times", "mdf_cmap_coefficients",
    "mdf_kernel_launches", "mdf_probe_fma_tflops", "mdf_probe_l2_reductions", "mdf_compute_bonded_noalloc", "mdf_set_parameters",
    "mdf_backward", "mdf_batch_create", "mdf_batch_destroy", "mdf_batch_last_error", "mdf_batch_info",
    "mdf_batch_set_positions", "mdf_batch_host_buffers", "mdf_batch_build_pairlists", "mdf_batch_compute", "mdf_batch_launch",
    "mdf_batch_fetch", "mdf_batch_submit", "mdf_batch_collect", "mdf_batch_autotune", "mdf_cmap_coefficients_spline",
    "mdf_pme_grids", "mdf_set_allreduce", "mdf_set_collectives", "mdf_set_halo_exchange", "mdf_autotune", "mdf_minimize", "mdf_minimize_lbfgs", "mdf_md_init", "mdf_md_run", "mdf_md_state", "mdf_md_write_rst7",
]


class MDFError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s: %s" % (abi.STATUS.get(status, status), message))
        self.status = status


def library(path=None):
    """Load libmdf.so (building it first if the sources are present and it is missing)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = path or LIB_PATH
    if not os.path.exists(path):
        from . import build as _build
        _build.build()
    lib = C.CDLL(path)
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int32)
    lib.mdf_params_default.argtypes = [C.POINTER(abi.mdf_params)]
    lib.mdf_params_default.restype = None
    lib.mdf_create.argtypes = [C.POINTER(abi.mdf_topology), C.POINTER(abi.mdf_params), C.POINTER(C.c_void_p)]
    lib.mdf_destroy.argtypes = [C.c_void_p]
    lib.mdf_destroy.restype = None
    lib.mdf_last_error.argtypes = [C.c_void_p]
    lib.mdf_last_error.restype = C.c_char_p
    lib.mdf_status_string.argtypes = [C.c_int]
    lib.mdf_status_string.restype = C.c_char_p
    lib.mdf_set_positions.argtypes = [C.c_void_p, dp]
    lib.mdf_set_positions_device.argtypes = [C.c_void_p, C.c_void_p]
    lib.mdf_set_box.argtypes = [C.c_void_p, dp]
    lib.mdf_build_pairlist.argtypes = [C.c_void_p]
    lib.mdf_compute.argtypes = [C.c_void_p, C.c_uint32, dp, C.POINTER(abi.mdf_energies)]
    lib.mdf_compute_async.argtypes = [C.c_void_p, C.c_uint32]
    lib.mdf_fetch.argtypes = [C.c_void_p, dp, C.POINTER(abi.mdf_energies)]
    lib.mdf_submit.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
    lib.mdf_collect.argtypes = [C.c_void_p, C.POINTER(abi.mdf_energies)]
    lib.mdf_forces_device.argtypes = [C.c_void_p, C.c_void_p]
    lib.mdf_get_pme_forces.argtypes = [C.c_void_p, dp]
    lib.mdf_pme_grids.argtypes = [C.c_void_p, C.POINTER(C.c_int32), dp, dp]
    lib.mdf_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    lib.mdf_pairlist_info.argtypes = [C.c_void_p] + [C.POINTER(C.c_int64)] * 4
    lib.mdf_enable_timing.argtypes = [C.c_void_p, C.c_int]
    lib.mdf_kernel_times.argtypes = [C.c_void_p, C.POINTER(C.c_char_p), C.POINTER(C.c_float), C.c_int]
    lib.mdf_cmap_coefficients.argtypes = [C.c_int, C.c_int, dp, dp]
    lib.mdf_cmap_coefficients_spline.argtypes = [C.c_int, C.c_int, dp, dp]
    lib.mdf_kernel_launches.argtypes = [C.c_void_p]
    lib.mdf_kernel_launches.restype = C.c_int64
    lib.mdf_probe_fma_tflops.argtypes = [C.c_int, C.c_int, dp]
    lib.mdf_probe_l2_reductions.argtypes = [C.c_int, C.c_int64, C.c_int, dp]
    lib.mdf_set_parameters.argtypes = [C.c_void_p, dp, dp, dp]
    lib.mdf_backward.argtypes = [C.c_void_p, dp, C.c_double, dp, dp, dp]
    lib.mdf_minimize.argtypes = [C.c_void_p, C.c_int32, C.c_double, C.c_double, C.POINTER(abi.mdf_min_report)]
    lib.mdf_autotune.argtypes = [C.c_void_p, C.c_int, C.POINTER(abi.mdf_tune_report)]
    lib.mdf_set_allreduce.argtypes = [C.c_void_p, abi.MDF_ALLREDUCE_FN, C.c_void_p]
    lib.mdf_set_collectives.argtypes = [C.c_void_p, abi.MDF_REDUCE_SCATTER_FN, abi.MDF_ALLGATHER_FN,
                                        abi.MDF_ALLTOALL_FN, C.c_void_p]
    lib.mdf_set_halo_exchange.argtypes = [C.c_void_p, abi.MDF_ALLTOALLV_FN, C.c_void_p]
    lib.mdf_minimize_lbfgs.argtypes = [C.c_void_p, C.c_int32, C.c_double, C.c_double, C.c_int32,
                                       C.POINTER(abi.mdf_min_report)]
    lib.mdf_md_init.argtypes = [C.c_void_p, dp, dp, C.c_double, C.c_uint64]
    lib.mdf_md_run.argtypes = [C.c_void_p, C.c_int64, C.c_double, C.c_int32, C.c_int32, dp, C.c_int64,
                               C.POINTER(abi.mdf_md_report)]
    lib.mdf_md_state.argtypes = [C.c_void_p, dp, dp]
    lib.mdf_md_write_rst7.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p, C.c_double]
    vp = C.c_void_p
    lib.mdf_batch_create.argtypes = [C.c_int, C.POINTER(C.POINTER(abi.mdf_topology)), C.POINTER(abi.mdf_params),
                                     C.POINTER(vp)]
    lib.mdf_batch_destroy.argtypes = [vp]
    lib.mdf_batch_destroy.restype = None
    lib.mdf_batch_last_error.argtypes = [vp]
    lib.mdf_batch_last_error.restype = C.c_char_p
    lib.mdf_batch_info.argtypes = [vp] + [C.POINTER(C.c_int64)] * 3
    lib.mdf_batch_set_positions.argtypes = [vp, dp]
    lib.mdf_batch_host_buffers.argtypes = [vp, C.POINTER(dp), C.POINTER(dp)]
    lib.mdf_batch_build_pairlists.argtypes = [vp]
    lib.mdf_batch_compute.argtypes = [vp, C.c_uint32, dp, C.POINTER(abi.mdf_energies)]
    lib.mdf_batch_launch.argtypes = [vp, C.c_uint32, vp]
    lib.mdf_batch_fetch.argtypes = [vp, C.c_uint32, dp, C.POINTER(abi.mdf_energies)]
    lib.mdf_batch_submit.argtypes = [vp, C.c_uint32, dp, dp]
    lib.mdf_batch_collect.argtypes = [vp, C.POINTER(abi.mdf_energies)]
    lib.mdf_batch_autotune.argtypes = [vp, C.c_int, C.POINTER(abi.mdf_tune_report)]
    lib.mdf_compute_bonded_noalloc.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.POINTER(abi.mdf_energies)]
    _LIB = lib
    return lib


def cmap_coefficients_spline(nsets, res, grids):
    """C1 periodic-spline bicubic CMAP table (PHYSICAL semantics), host only."""
    g = np.ascontiguousarray(grids, dtype=np.float64)
    out = np.zeros(nsets * res * res * 16)
    rc = library().mdf_cmap_coefficients_spline(nsets, res, g.ctypes.data_as(C.POINTER(C.c_double)),
                                                out.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise MDFError(rc, "mdf_cmap_coefficients_spline")
    return out


def cmap_coefficients(nsets, res, grids):
    """Bicubic CMAP coefficient table through the C ABI (host only, no GPU)."""
    g = np.ascontiguousarray(grids, dtype=np.float64)
    out = np.zeros(nsets * res * res * 16)
    rc = library().mdf_cmap_coefficients(nsets, res, g.ctypes.data_as(C.POINTER(C.c_double)),
                                         out.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise MDFError(rc, "mdf_cmap_coefficients")
    return out


def probe_fma_tflops(device=0, precision=abi.MDF_PREC_MIXED):
    """Measured CUDA-core FMA throughput (TFLOP/s) of the device."""
    v = C.c_double(0)
    rc = library().mdf_probe_fma_tflops(device, precision, C.byref(v))
    if rc != 0:
        raise MDFError(rc, "mdf_probe_fma_tflops")
    return v.value


def probe_l2_reductions(device=0, words=10077696, pattern=0):
    """Measured int64 reductions per second into an L2-resident buffer of
    `words` 64-bit words (default: the 216^3 PME grid); pattern 0 = the charge
    spread's 32-byte rows, 1 = 256-byte warp runs."""
    v = C.c_double(0)
    rc = library().mdf_probe_l2_reductions(device, int(words), int(pattern), C.byref(v))
    if rc != 0:
        raise MDFError(rc, "mdf_probe_l2_reductions")
    return v.value


def default_params():
    p = abi.mdf_params()
    library().mdf_params_default(C.byref(p))
    return p


class Engine:
    """One libmdf context (one system on one GPU)."""

    def __init__(self, flat, box, semantics=abi.MDF_SEM_PHYSICAL, precision=abi.MDF_PREC_MIXED, cutoff=10.0,
                 skin=2.0, switch_radius=9.0, ewald_tol=1e-5, ewald_alpha=0.0, grid=(0, 0, 0), pme_order=4,
                 device=0, prune_every=1, prune_margin=0.0, rank=0, nranks=1, pair_warps=0, fft_lines=0,
                 pair_schedule=0, pair_layout=0):
        self.lib = library()
        self.flat = flat
        self.natoms = flat.natoms
        self.n_ljpair = int(len(flat.lj_a))
        p = default_params()
        p.semantics, p.precision = int(semantics), int(precision)
        for k in range(3):
            p.box[k] = float(box[k])
            p.grid[k] = int(grid[k])
        p.cutoff, p.skin, p.switch_radius = float(cutoff), float(skin), float(switch_radius)
        p.ewald_tol, p.ewald_alpha, p.pme_order, p.device = float(ewald_tol), float(ewald_alpha), int(pme_order), int(device)
        p.prune_every, p.prune_margin = int(prune_every), float(prune_margin)
        p.rank, p.nranks = int(rank), int(nranks)
        p.pair_warps, p.fft_lines = int(pair_warps), int(fft_lines)
        p.pair_schedule, p.pair_layout = int(pair_schedule), int(pair_layout)
        self.params = p
        h = C.c_void_p()
        rc = self.lib.mdf_create(C.byref(flat.struct()), C.byref(p), C.byref(h))
        if rc != 0:
            raise MDFError(rc, self.lib.mdf_last_error(None).decode())
        self.h = h
        self._f = np.zeros((self.natoms, 3))

    def _check(self, rc, what):
        if rc != 0:
            raise MDFError(rc, "%s: %s" % (what, self.lib.mdf_last_error(self.h).decode()))

    def close(self):
        if getattr(self, "h", None):
            self.lib.mdf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_positions(self, xyz):
        x = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1)
        if x.size != 3 * self.natoms:
            raise ValueError("expected %d coordinates" % (3 * self.natoms))
        self._check(self.lib.mdf_set_positions(self.h, x.ctypes.data_as(C.POINTER(C.c_double))), "set_positions")

    def set_positions_ptr(self, host_ptr):
        """Host positions from a raw pointer (e.g. pinned memory)."""
        self._check(self.lib.mdf_set_positions(self.h, C.cast(C.c_void_p(host_ptr), C.POINTER(C.c_double))),
                    "set_positions")

    def compute_into(self, forces_ptr, energy=True):
        """mdf_compute writing forces to a raw host pointer; returns energies."""
        flags = abi.MDF_COMPUTE_FORCES | (abi.MDF_COMPUTE_ENERGY if energy else 0)
        e = abi.mdf_energies()
        self._check(self.lib.mdf_compute(self.h, flags, C.cast(C.c_void_p(forces_ptr), C.POINTER(C.c_double)),
                                         C.byref(e)), "compute")
        return e

    def submit(self, xyz_ptr, forces_ptr, energy=True):
        """mdf_submit: positions from and forces to raw host pointers (pinned for
        overlap); returns at once, mdf_collect finishes the oldest."""
        flags = abi.MDF_COMPUTE_FORCES | (abi.MDF_COMPUTE_ENERGY if energy else 0)
        self._check(self.lib.mdf_submit(self.h, flags, C.c_void_p(xyz_ptr), C.c_void_p(forces_ptr or None)), "submit")

    def collect(self):
        """mdf_collect: waits for the oldest submitted evaluation; its energies."""
        e = abi.mdf_energies()
        self._check(self.lib.mdf_collect(self.h, C.byref(e)), "collect")
        return e.as_dict()

    def launches(self):
        return int(self.lib.mdf_kernel_launches(self.h))

    def set_positions_device(self, ptr):
        self._check(self.lib.mdf_set_positions_device(self.h, C.c_void_p(ptr)), "set_positions_device")

    def autotune(self, reps=5):
        """mdf_autotune: the fastest launch shapes for this context (kept)."""
        r = abi.mdf_tune_report()
        self._check(self.lib.mdf_autotune(self.h, int(reps), C.byref(r)), "autotune")
        return dict(pair_warps=r.pair_warps, fft_lines=r.fft_lines, prune_every=r.prune_every,
                    pair_schedule=r.pair_schedule, pair_layout=r.pair_layout, n_tried=r.n_tried,
                    best_ms=r.best_ms, default_ms=r.default_ms)

    def set_allreduce(self, fn):
        """The sum over ranks for a split context (nranks > 1): fn(ptr, count,
        stream, user) -> 0, summing `count` int64 at device pointer `ptr` in place,
        ordered on the CUDA stream handle `stream` (md_b200.distributed builds
        one from a torch.distributed group)."""
        self._allreduce_cb = abi.MDF_ALLREDUCE_FN(fn)   # kept alive with the engine
        self._check(self.lib.mdf_set_allreduce(self.h, self._allreduce_cb, None), "set_allreduce")

    def set_collectives(self, reduce_scatter, allgather, alltoall):
        """The distributed reciprocal space and force return of a split context
        (mdf_set_collectives): three callbacks (md_b200.distributed builds them
        from a torch.distributed group); None for all three goes back to the
        all-reduce form."""
        if reduce_scatter is None:
            self._coll_cb = None
            self._check(self.lib.mdf_set_collectives(self.h, abi.MDF_REDUCE_SCATTER_FN(), abi.MDF_ALLGATHER_FN(),
                                                     abi.MDF_ALLTOALL_FN(), None), "set_collectives")
            return
        self._coll_cb = (abi.MDF_REDUCE_SCATTER_FN(reduce_scatter), abi.MDF_ALLGATHER_FN(allgather),
                         abi.MDF_ALLTOALL_FN(alltoall))   # kept alive with the engine
        self._check(self.lib.mdf_set_collectives(self.h, *self._coll_cb, None), "set_collectives")

    def set_halo_exchange(self, alltoallv):
        """Exchange only halo planes of the PME grids between the ranks of a
        split context (mdf_set_halo_exchange): an all-to-all with per-rank
        sizes (md_b200.distributed.torch_alltoallv); None goes back to the
        whole-grid reduce-scatter and all-gather."""
        if alltoallv is None:
            self._a2av_cb = None
            self._check(self.lib.mdf_set_halo_exchange(self.h, abi.MDF_ALLTOALLV_FN(), None), "set_halo_exchange")
            return
        self._a2av_cb = abi.MDF_ALLTOALLV_FN(alltoallv)   # kept alive with the engine
        self._check(self.lib.mdf_set_halo_exchange(self.h, self._a2av_cb, None), "set_halo_exchange")

    def set_box(self, box):
        b = np.ascontiguousarray(box, dtype=np.float64)
        self._check(self.lib.mdf_set_box(self.h, b.ctypes.data_as(C.POINTER(C.c_double))), "set_box")

    def set_stream(self, stream_ptr):
        self._check(self.lib.mdf_set_stream(self.h, C.c_void_p(stream_ptr)), "set_stream")

    def build_pairlist(self):
        self._check(self.lib.mdf_build_pairlist(self.h), "build_pairlist")

    def compute(self, energy=True, forces=True, pme_reference=False):
        flags = (abi.MDF_COMPUTE_ENERGY if energy else 0) | (abi.MDF_COMPUTE_FORCES if forces else 0)
        if pme_reference:
            flags |= abi.MDF_COMPUTE_PME_REFERENCE
        e = abi.mdf_energies()
        f = np.zeros((self.natoms, 3)) if forces else None
        fp = f.ctypes.data_as(C.POINTER(C.c_double)) if forces else None
        self._check(self.lib.mdf_compute(self.h, flags, fp, C.byref(e)), "compute")
        out = e.as_dict() if energy else None
        if energy:
            out["virial"] = np.array(e.virial[:]).reshape(3, 3)
        return out, f

    def compute_async(self, energy=True, pme_reference=False):
        flags = abi.MDF_COMPUTE_FORCES | (abi.MDF_COMPUTE_ENERGY if energy else 0)
        if pme_reference:
            flags |= abi.MDF_COMPUTE_PME_REFERENCE
        self._check(self.lib.mdf_compute_async(self.h, flags), "compute_async")

    def fetch(self, forces=True, energy=True):
        e = abi.mdf_energies()
        f = np.zeros((self.natoms, 3)) if forces else None
        fp = f.ctypes.data_as(C.POINTER(C.c_double)) if forces else None
        self._check(self.lib.mdf_fetch(self.h, fp, C.byref(e) if energy else None), "fetch")
        return (e.as_dict() if energy else None), f

    def forces_device(self, ptr):
        self._check(self.lib.mdf_forces_device(self.h, C.c_void_p(ptr)), "forces_device")

    def set_parameters(self, charge=None, lj_a=None, lj_b=None):
        """Replace charges and/or the LJ A/B table (None keeps the current values)."""
        def p(a):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float64)
            self._keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_double))
        self._keep = []
        self._check(self.lib.mdf_set_parameters(self.h, p(charge), p(lj_a), p(lj_b)), "set_parameters")

    def backward(self, dL_dF, dL_dE):
        """dL/dq [N], dL/dA [n_ljpair], dL/dB [n_ljpair] for dL/dF [N, 3] and dL/dE."""
        g = None if dL_dF is None else np.ascontiguousarray(dL_dF, dtype=np.float64).reshape(-1)
        dq = np.zeros(self.natoms)
        dA = np.zeros(self.n_ljpair)
        dB = np.zeros(self.n_ljpair)
        dp_ = C.POINTER(C.c_double)
        self._check(self.lib.mdf_backward(self.h, None if g is None else g.ctypes.data_as(dp_), float(dL_dE),
                                          dq.ctypes.data_as(dp_), dA.ctypes.data_as(dp_), dB.ctypes.data_as(dp_)),
                    "backward")
        return dq, dA, dB

    def minimize(self, max_iter=200, fmax_tol=10.0, max_step=0.1, method="sd", history=8):
        """Minimise from the current positions: method "sd" (steepest descent,
        mdf_minimize) or "lbfgs" (mdf_minimize_lbfgs with `history` pairs);
        returns the report dict."""
        r = abi.mdf_min_report()
        if method == "lbfgs":
            rc = self.lib.mdf_minimize_lbfgs(self.h, int(max_iter), float(fmax_tol), float(max_step), int(history),
                                             C.byref(r))
        elif method == "sd":
            rc = self.lib.mdf_minimize(self.h, int(max_iter), float(fmax_tol), float(max_step), C.byref(r))
        else:
            raise ValueError("method must be 'sd' or 'lbfgs'")
        self._check(rc, "minimize")
        return {k: getattr(r, k) for k, _ in abi.mdf_min_report._fields_ if k != "reserved"}

    def md_init(self, masses, velocities=None, temperature=300.0, seed=1):
        """Start dynamics: masses [N] amu, velocities [N, 3] A/ps or Maxwell at temperature."""
        m = np.ascontiguousarray(masses, dtype=np.float64)
        v = None if velocities is None else np.ascontiguousarray(velocities, dtype=np.float64).reshape(-1)
        dp_ = C.POINTER(C.c_double)
        self._check(self.lib.mdf_md_init(self.h, m.ctypes.data_as(dp_), None if v is None else v.ctypes.data_as(dp_),
                                         float(temperature), int(seed)), "md_init")

    def md_run(self, nsteps, dt_ps, chunk=10, rebuild_every=0):
        """Velocity-Verlet steps; returns (report dict, samples [n, 3]: t ps, PE, KE)."""
        ch = max(int(chunk), 1)
        cap = (int(nsteps) + ch - 1) // ch + 1
        samp = np.zeros((cap, 3))
        r = abi.mdf_md_report()
        self._check(self.lib.mdf_md_run(self.h, int(nsteps), float(dt_ps), int(chunk), int(rebuild_every),
                                        samp.ctypes.data_as(C.POINTER(C.c_double)), cap, C.byref(r)), "md_run")
        rep = {k: getattr(r, k) for k, _ in abi.mdf_md_report._fields_}
        return rep, samp[:min(int(r.samples), cap)]

    def md_state(self, velocities=True):
        x = np.zeros((self.natoms, 3))
        v = np.zeros((self.natoms, 3)) if velocities else None
        dp_ = C.POINTER(C.c_double)
        self._check(self.lib.mdf_md_state(self.h, x.ctypes.data_as(dp_), v.ctypes.data_as(dp_) if velocities else None),
                    "md_state")
        return x, v

    def write_rst7(self, path, title="md_b200 restart", time_ps=0.0):
        self._check(self.lib.mdf_md_write_rst7(self.h, str(path).encode(), title.encode(), float(time_ps)),
                    "write_rst7")

    def bonded_noalloc(self, forces_ptr, energy=True):
        """Bonded terms only, with the library's static scratch (no device
        allocation); forces_ptr is a device array [3 natoms] or 0."""
        e = abi.mdf_energies()
        flags = (abi.MDF_COMPUTE_ENERGY if energy else 0) | (abi.MDF_COMPUTE_FORCES if forces_ptr else 0)
        self._check(self.lib.mdf_compute_bonded_noalloc(self.h, flags, C.c_void_p(forces_ptr or None), C.byref(e)),
                    "compute_bonded_noalloc")
        return e.as_dict() if energy else None

    def pme_grids(self):
        """(Q, C*Q) of the last evaluation, each [K0, K1, K2]."""
        k = (C.c_int32 * 3)()
        self._check(self.lib.mdf_pme_grids(self.h, k, None, None), "pme_grids")
        K = tuple(k)
        q = np.zeros(K)
        p = np.zeros(K)
        dp_ = C.POINTER(C.c_double)
        self._check(self.lib.mdf_pme_grids(self.h, k, q.ctypes.data_as(dp_), p.ctypes.data_as(dp_)), "pme_grids")
        return q, p

    def pme_forces(self):
        f = np.zeros((self.natoms, 3))
        self._check(self.lib.mdf_get_pme_forces(self.h, f.ctypes.data_as(C.POINTER(C.c_double))), "pme_forces")
        return f

    def pairlist_info(self):
        a, b, p, c = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        self._check(self.lib.mdf_pairlist_info(self.h, C.byref(a), C.byref(b), C.byref(p), C.byref(c)),
                    "pairlist_info")
        return dict(clusters=a.value, cluster_pairs=b.value, cluster_pairs_pruned=p.value, pairs_in_cutoff=c.value)

    def enable_timing(self, on=True):
        self._check(self.lib.mdf_enable_timing(self.h, 1 if on else 0), "enable_timing")

    def kernel_times(self):
        names = (C.c_char_p * 32)()
        ms = (C.c_float * 32)()
        n = self.lib.mdf_kernel_times(self.h, names, ms, 32)
        return [(names[i].decode(), ms[i]) for i in range(n)]


class Batch:
    """Many independent PHYSICAL systems evaluated by one CUDA graph launch
    (mdf_batch_*).  flats / boxes / grids: one per system."""

    def __init__(self, flats, boxes, grids, precision=abi.MDF_PREC_MIXED, cutoff=9.0, skin=2.0, switch_radius=8.0,
                 ewald_tol=1e-5, device=0, prune_every=1, pair_schedule=0, pair_layout=0, prune_margin=0.0):
        self.lib = library()
        self.flats = list(flats)
        n = len(self.flats)
        self.natoms = [f.natoms for f in self.flats]
        self.offsets = np.concatenate([[0], np.cumsum(self.natoms)])
        tops = (C.POINTER(abi.mdf_topology) * n)(*[C.pointer(f.struct()) for f in self.flats])
        params = (abi.mdf_params * n)()
        for k in range(n):
            p = default_params()
            p.semantics, p.precision = abi.MDF_SEM_PHYSICAL, int(precision)
            for d in range(3):
                p.box[d] = float(boxes[k][d])
                p.grid[d] = int(grids[k][d])
            p.cutoff, p.skin, p.switch_radius = float(cutoff), float(skin), float(switch_radius)
            p.ewald_tol, p.device = float(ewald_tol), int(device)
            p.prune_every, p.prune_margin = int(prune_every), float(prune_margin)
            p.pair_schedule, p.pair_layout = int(pair_schedule), int(pair_layout)
            params[k] = p
        self._tops, self._params = tops, params
        h = C.c_void_p()
        rc = self.lib.mdf_batch_create(n, tops, params, C.byref(h))
        if rc != 0:
            raise MDFError(rc, "batch_create: %s" % self.lib.mdf_last_error(None).decode())
        self.h = h
        self.n = n

    def _check(self, rc, what):
        if rc != 0:
            raise MDFError(rc, "%s: %s" % (what, self.lib.mdf_batch_last_error(self.h).decode()))

    def close(self):
        if getattr(self, "h", None):
            self.lib.mdf_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def host_buffers(self):
        """(positions, forces): numpy [total atoms, 3] views of the batch's pinned
        host buffers (mdf_batch_host_buffers).  Positions written into the first
        and passed to set_positions, and forces read from the second after
        compute(copy_forces=False), move no extra host copy."""
        dp_ = C.POINTER(C.c_double)
        p, f = dp_(), dp_()
        self._check(self.lib.mdf_batch_host_buffers(self.h, C.byref(p), C.byref(f)), "host_buffers")
        n = int(self.offsets[-1])
        return (np.ctypeslib.as_array(p, shape=(n, 3)), np.ctypeslib.as_array(f, shape=(n, 3)))

    def set_positions(self, coords):
        """coords: a list of [n_k, 3] arrays, one per system, or one [total, 3]
        array (the positions view of host_buffers() is used in place)."""
        if isinstance(coords, np.ndarray) and coords.dtype == np.float64 and coords.flags.c_contiguous \
                and coords.size == 3 * int(self.offsets[-1]):
            x = coords
        else:
            x = np.ascontiguousarray(np.concatenate([np.asarray(c, float).reshape(-1) for c in coords]))
        self._check(self.lib.mdf_batch_set_positions(self.h, x.ctypes.data_as(C.POINTER(C.c_double))), "set_positions")

    def build_pairlists(self):
        self._check(self.lib.mdf_batch_build_pairlists(self.h), "build_pairlists")

    def compute(self, energy=True, forces=True, copy_forces=True):
        """Per system: (energies dict or None, forces [n_k, 3] or None).  With
        copy_forces=False the forces are views of the pinned host buffer (valid
        until the next evaluation)."""
        flags = (abi.MDF_COMPUTE_ENERGY if energy else 0) | (abi.MDF_COMPUTE_FORCES if forces else 0)
        if forces and not copy_forces:
            F = self.host_buffers()[1].reshape(-1)
            fptr = None
        else:
            F = np.zeros(3 * int(self.offsets[-1])) if forces else None
            fptr = F.ctypes.data_as(C.POINTER(C.c_double)) if forces else None
        E = (abi.mdf_energies * self.n)() if energy else None
        self._check(self.lib.mdf_batch_compute(self.h, flags, fptr, E), "compute")
        out = []
        for k in range(self.n):
            e = E[k].as_dict() if energy else None
            f = F[3 * self.offsets[k]:3 * self.offsets[k + 1]].reshape(-1, 3) if forces else None
            out.append((e, f))
        return out

    def launch(self, energy=True, stream_ptr=None):
        flags = abi.MDF_COMPUTE_FORCES | (abi.MDF_COMPUTE_ENERGY if energy else 0)
        self._check(self.lib.mdf_batch_launch(self.h, flags, C.c_void_p(stream_ptr) if stream_ptr else None),
                    "launch")

    def fetch_into(self, forces_ptr, energy=True):
        flags = abi.MDF_COMPUTE_FORCES | (abi.MDF_COMPUTE_ENERGY if energy else 0)
        self._check(self.lib.mdf_batch_fetch(self.h, flags, C.cast(forces_ptr, C.POINTER(C.c_double))
                                             if forces_ptr else None, None), "fetch")

    def submit(self, xyz_ptr, forces_ptr, energy=True):
        """Pipelined evaluation (mdf_batch_submit): positions from the pinned
        host buffer at xyz_ptr (all systems, concatenated), forces into the one
        at forces_ptr; at most two in flight, collect() in order."""
        flags = abi.MDF_COMPUTE_FORCES | (abi.MDF_COMPUTE_ENERGY if energy else 0)
        self._check(self.lib.mdf_batch_submit(self.h, flags, C.cast(xyz_ptr, C.POINTER(C.c_double)),
                                              C.cast(forces_ptr, C.POINTER(C.c_double)) if forces_ptr else None),
                    "submit")

    def collect(self, energy=True):
        """Wait for the oldest submitted evaluation; its energies per system."""
        E = (abi.mdf_energies * self.n)() if energy else None
        self._check(self.lib.mdf_batch_collect(self.h, E), "collect")
        return [E[k].as_dict() for k in range(self.n)] if energy else None

    def autotune(self, reps=5):
        r = abi.mdf_tune_report()
        self._check(self.lib.mdf_batch_autotune(self.h, int(reps), C.byref(r)), "autotune")
        return dict(pair_warps=r.pair_warps, fft_lines=r.fft_lines, prune_every=r.prune_every,
                    pair_schedule=r.pair_schedule, pair_layout=r.pair_layout, n_tried=r.n_tried,
                    best_ms=r.best_ms, default_ms=r.default_ms)

    def info(self):
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        self._check(self.lib.mdf_batch_info(self.h, C.byref(a), C.byref(b), C.byref(c)), "info")
        return dict(n_systems=a.value, total_atoms=b.value, graph_kernels=c.value)

