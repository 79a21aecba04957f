"""Build libmdf.so in-tree for sm_100a (B200) with nvcc.

    python -m md_b200.build          # build if sources changed
    python -m md_b200.build --force  # rebuild everything
"""
from __future__ import annotations

import glob
import hashlib
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
REPO = os.path.dirname(PKG)
LIB = os.path.join(PKG, "libmdf.so")
HOST = os.path.join(PKG, "host")
CLI = os.path.join(PKG, "mdb200")
BUILD = os.path.join(PKG, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", "-I" + os.path.join(REPO, "include")]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _digest():
    h = hashlib.sha256()
    for p in sources() + sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + sorted(glob.glob(os.path.join(CSRC, "*.hpp"))) + \
            [os.path.join(REPO, "include", "mdf.h")] + \
            sorted(glob.glob(os.path.join(HOST, "*.?pp"))):
        with open(p, "rb") as f:
            h.update(p.encode())
            h.update(f.read())
    h.update(" ".join(ARCH + FLAGS).encode())
    return h.hexdigest()


def build(force=False, verbose=False, jobs=8):
    os.makedirs(BUILD, exist_ok=True)
    stamp = os.path.join(BUILD, "stamp")
    dig = _digest()
    if not force and os.path.exists(LIB) and os.path.exists(stamp) and open(stamp).read() == dig:
        return LIB
    objs, procs = [], []
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        cmd = [NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd = ["g++", "-O3", "-fPIC", "-std=c++17", "-I" + os.path.join(REPO, "include"), "-c", src, "-o", obj]
        procs.append((src, cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        if len(procs) >= jobs:
            _drain(procs, verbose)
    _drain(procs, verbose)
    link = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
    out = subprocess.run(link, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("link failed:\n" + out.stdout + out.stderr)
    build_host()
    with open(stamp, "w") as f:
        f.write(dig)
    return LIB


def build_host():
    """The C++ host (md_b200/host): prmtop/rst7 reader, mdb200::System and the
    mdb200 command line, linked against libmdf.so (rpath to this directory)."""
    srcs = sorted(glob.glob(os.path.join(HOST, "*.cpp")))
    cmd = ["g++", "-O2", "-std=c++17", "-I" + os.path.join(REPO, "include"), "-o", CLI] + srcs + \
          ["-L" + PKG, "-lmdf", "-Wl,-rpath,$ORIGIN", "-L/usr/local/cuda/lib64", "-lcudart"]
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("host build failed:\n" + " ".join(cmd) + "\n" + out.stdout + out.stderr)
    return CLI


def _drain(procs, verbose):
    while procs:
        src, cmd, p = procs.pop(0)
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), out))
        if verbose and out.strip():
            print(out)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
