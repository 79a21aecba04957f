"""The reference's own md::System running on libmdf (the drop-in claim).

oracle/_ref/ref_on_mdf is the unmodified reference compiled with
src/System/System.cpp replaced by oracle/binding/MdfBackend.cpp, the file a
maintainer adds in the reference's ENABLE_CUDA slot: System's private
calculate_energies() and calculate_forces() (include/System/System.h:78-170,
src/System/System.cpp:9-39) call libmdf through include/mdf.h and read only
the reference's own parsed state.  Its energies and forces must equal the
reference's CPU numbers (golden fixtures from the same prmtop/rst7):
1e-9 relative per energy term and 1e-9 rms relative on the forces (FP64),
1e-5 rms relative on the forces in mixed precision.
"""
import os
import tempfile

import numpy as np
import pytest

from md_b200 import synth
from oracle import oracle as O
from tests import helpers as H

pytestmark = pytest.mark.gpu
TERMS = ["bond", "angle", "dihedral", "ub", "improper", "cmap", "vdw", "ee", "ee_pairlist", "ee_cutoff",
         "ee_direct", "ee_self"]


def _inputs(case):
    g = H.golden(case)
    m = g["meta"]
    kept = os.path.join(g["dir"], case + ".prmtop")
    if os.path.exists(kept):
        return g, kept, os.path.join(g["dir"], case + ".rst7")
    s = H.system(m["config"], m["sentinels"])
    d = tempfile.mkdtemp(prefix="bind_")
    prm, rst = synth.write_files(s, d, stem=case)
    assert H.files_sha(s) == [m["sha_prmtop"], m["sha_rst7"]]   # the very files the reference read
    return g, prm, rst


@pytest.mark.parametrize("case", ["tiny", "tiny_sentinel", "small", "c0"])
def test_reference_system_on_libmdf_matches_reference_cpu(case):
    g, prm, rst = _inputs(case)
    r = O.run_ref_on_mdf(prm, rst, g["meta"]["grid"], tol=g["meta"]["tol"], repeat=2)
    for k in TERMS:
        assert H.rel(r["energies"][k], g["energies"][k]) < 1e-9, (k, r["energies"][k], g["energies"][k])
    H.check_forces_vs_golden(r["forces"], g, 1e-9, "forces")


def test_reference_system_on_libmdf_mixed_precision():
    g, prm, rst = _inputs("small")
    r = O.run_ref_on_mdf(prm, rst, g["meta"]["grid"], tol=g["meta"]["tol"], precision="mixed")
    H.check_forces_vs_golden(r["forces"], g, 1e-5, "forces")
    for k in ("bond", "angle", "dihedral", "ub", "improper", "cmap"):
        assert H.rel(r["energies"][k], g["energies"][k]) < 1e-9, k
