"""Python access to the oracles.  TEST INFRASTRUCTURE ONLY.

O1  the unmodified reference driven by o1_harness (oracle/_ref/o1_harness)
O2  the FP64 C restatement (oracle/_ref/liboracle.so)

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline / reference
arm import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(REF_DIR, "liboracle.so")
O1 = os.path.join(REF_DIR, "o1_harness")
REF_ON_MDF = os.path.join(REF_DIR, "ref_on_mdf")
# reference checkout the O1 recipe compiles: $MD_REFERENCE, else the default location
REFERENCE_SRC = os.environ.get("MD_REFERENCE", "/root/reference")

_lib = None


class oracle_params(C.Structure):
    _fields_ = [("semantics", C.c_int), ("box", C.c_double * 3), ("cutoff", C.c_double),
                ("list_cutoff", C.c_double), ("switch_radius", C.c_double), ("alpha", C.c_double),
                ("kc", C.c_double), ("grid", C.c_int * 3), ("pme_order", C.c_int),
                ("do_allpairs", C.c_int), ("do_recip", C.c_int)]


def build(quiet=True):
    """Compile the oracles (O1 only where the reference sources are present)."""
    targets = ["_ref/liboracle.so"]
    if os.path.isdir(REFERENCE_SRC):
        targets.append("_ref/o1_harness")
        # the reference's own System on libmdf (needs libmdf.so built first)
        if os.path.exists(os.path.join(os.path.dirname(HERE), "md_b200", "libmdf.so")):
            targets.append("_ref/ref_on_mdf")
    out = subprocess.run(["make", "-s", "-j8", "REF=" + REFERENCE_SRC] + targets, cwd=HERE, capture_output=True,
                         text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = C.CDLL(LIB)
        dp = C.POINTER(C.c_double)
        _lib.oracle_eval.argtypes = [C.c_void_p, C.POINTER(oracle_params), dp, dp, dp, dp, dp,
                                     C.POINTER(C.c_long)]
        _lib.oracle_pme_ref_grids.argtypes = [C.c_void_p, C.POINTER(oracle_params), dp, dp, dp]
        _lib.oracle_pme_recip.argtypes = [C.c_void_p, C.POINTER(oracle_params), dp, dp, dp]
        _lib.oracle_pme_recip.restype = C.c_double
        _lib.oracle_ewald_recip_exact.argtypes = [C.c_int, dp, dp, dp, C.c_double, C.c_double, C.c_int, dp]
        _lib.oracle_ewald_recip_exact.restype = C.c_double
        _lib.oracle_cmap_coeff.argtypes = [C.c_int, C.c_int, dp, dp]
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def cmap_coeff(nsets, res, grids):
    out = np.zeros(nsets * res * res * 16)
    g = np.ascontiguousarray(grids, dtype=np.float64)
    lib().oracle_cmap_coeff(nsets, res, _dp(g), _dp(out))
    return out


def make_params(semantics, box, grid, alpha, kc, cutoff=10.0, skin=2.0, switch=9.0, order=4,
                allpairs=True, recip=True):
    p = oracle_params()
    p.semantics = semantics
    for k in range(3):
        p.box[k] = float(box[k]); p.grid[k] = int(grid[k])
    p.cutoff = cutoff; p.list_cutoff = cutoff + skin; p.switch_radius = switch
    p.alpha = alpha; p.kc = kc; p.pme_order = order
    p.do_allpairs = int(allpairs); p.do_recip = int(recip)
    return p


def evaluate(flat, params, x, pme_ref=False, want_forces=True):
    """O2 evaluation -> (energies[16], forces[N,3] or None, virial[9], f_pme_ref or None, npairs)."""
    n = flat.natoms
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    f = np.zeros(3 * n) if want_forces else None
    e = np.zeros(16)
    vir = np.zeros(9)
    fp = np.zeros(3 * n) if pme_ref else None
    npairs = C.c_long(0)
    t = flat.struct()
    rc = lib().oracle_eval(C.byref(t), C.byref(params), _dp(x), _dp(f), _dp(e), _dp(vir), _dp(fp),
                           C.byref(npairs))
    if rc != 0:
        raise RuntimeError("oracle_eval failed")
    return (e, None if f is None else f.reshape(-1, 3), vir, None if fp is None else fp.reshape(-1, 3),
            int(npairs.value))


def pme_ref_grids(flat, params, x):
    K = int(np.prod(list(params.grid)))
    gq, gp = np.zeros(K), np.zeros(K)
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    lib().oracle_pme_ref_grids(C.byref(flat.struct()), C.byref(params), _dp(x), _dp(gq), _dp(gp))
    return gq, gp


def ewald_recip_exact(q, x, box, alpha, kc, kmax):
    q = np.ascontiguousarray(q, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    f = np.zeros_like(x)
    b = np.ascontiguousarray(box, dtype=np.float64)
    e = lib().oracle_ewald_recip_exact(len(q), _dp(q), _dp(x), _dp(b), alpha, kc, kmax, _dp(f))
    return e, f.reshape(-1, 3)


def pme_recip(flat, params, x):
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    f = np.zeros_like(x)
    vir = np.zeros(9)
    e = lib().oracle_pme_recip(C.byref(flat.struct()), C.byref(params), _dp(x), _dp(f), _dp(vir))
    return e, f.reshape(-1, 3), vir


# ------------------------------------------------------------------ O1

def run_o1(prmtop, rst7, grid, tol=1e-5, allpairs=True, dump_grids=False, outdir=None):
    """Run the unmodified reference on a prmtop/rst7 pair; returns a dict."""
    if not os.path.exists(O1):
        raise FileNotFoundError("O1 harness not built (needs the reference sources)")
    own = outdir is None
    outdir = outdir or tempfile.mkdtemp(prefix="o1_")
    cmd = [O1, prmtop, rst7, outdir, "--tol", repr(tol), "--grid"] + [str(g) for g in grid]
    if not allpairs:
        cmd.append("--no-allpairs")
    if dump_grids:
        cmd.append("--dump-grids")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("o1_harness failed: " + r.stderr[-2000:])
    res = read_o1(outdir)
    if own:
        import shutil
        shutil.rmtree(outdir, ignore_errors=True)
    return res


def read_o1(outdir):
    res = {"energies": {}, "info": {}}
    with open(os.path.join(outdir, "energies.txt")) as f:
        for line in f:
            k, v = line.split()
            res["energies"][k] = float(v)
    with open(os.path.join(outdir, "info.txt")) as f:
        for line in f:
            parts = line.split()
            res["info"][parts[0]] = parts[1:] if len(parts) > 2 else parts[1]
    res["forces"] = np.fromfile(os.path.join(outdir, "forces.bin"), dtype=np.float64).reshape(-1, 3)
    res["forces_pme"] = np.fromfile(os.path.join(outdir, "forces_pme.bin"), dtype=np.float64).reshape(-1, 3)
    for g in ("grid_q", "grid_phi"):
        p = os.path.join(outdir, g + ".bin")
        if os.path.exists(p):
            res[g] = np.fromfile(p, dtype=np.float64)
    return res


def run_ref_on_mdf(prmtop, rst7, grid, tol=1e-5, repeat=1, precision="fp64"):
    """The reference's own System with calculate_energies / calculate_forces
    on libmdf (oracle/binding): energies and forces in the O1 harness format."""
    if not os.path.exists(REF_ON_MDF):
        raise FileNotFoundError("ref_on_mdf not built (needs the reference sources and libmdf.so)")
    outdir = tempfile.mkdtemp(prefix="refmdf_")
    cmd = [REF_ON_MDF, prmtop, rst7, outdir, "--tol", repr(tol), "--grid"] + [str(g) for g in grid] + \
          ["--repeat", str(repeat)]
    env = dict(os.environ, MD_MDF_PRECISION=precision)
    r = subprocess.run(cmd, capture_output=True, text=True, env=env)
    if r.returncode != 0:
        raise RuntimeError("ref_on_mdf failed (%d): %s" % (r.returncode, r.stderr[-2000:]))
    res = {"energies": {}}
    with open(os.path.join(outdir, "energies.txt")) as f:
        for line in f:
            k, v = line.split()
            res["energies"][k] = float(v)
    res["forces"] = np.fromfile(os.path.join(outdir, "forces.bin"), dtype=np.float64).reshape(-1, 3)
    import shutil
    shutil.rmtree(outdir, ignore_errors=True)
    return res


def bench_o1(prmtop, rst7, grid, steps, warmup=1, tol=1e-5):
    """Time the reference's evaluation (PME chain + list energies + calculate_forces)."""
    import json
    cmd = [O1, prmtop, rst7, "/tmp", "--tol", repr(tol), "--grid"] + [str(g) for g in grid] + \
          ["--bench", str(steps), "--bench-warmup", str(warmup)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("o1_harness bench failed: " + r.stderr[-2000:])
    for line in r.stdout.splitlines()[::-1]:
        if line.startswith("{"):
            return json.loads(line)
    raise RuntimeError("no JSON from o1_harness")
