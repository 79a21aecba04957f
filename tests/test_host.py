"""The C++ host (md_b200/host): the Amber prmtop/rst7 reader and the
flattening with the REFERENCE/PHYSICAL switch produce exactly the arrays of the
Python host (md_b200/topology.py) on the same files; and the mdb200 command
line, the reference's `./md <prmtop> <coords>` on the GPU, prints the
reference's own energies (golden O1 fixture) for the same files."""
import os
import re
import subprocess

import numpy as np
import pytest

from md_b200 import abi, build, engine, synth
from tests import helpers as H

CLI = build.CLI
ARRAYS = {"charge": np.float64, "type": np.int32, "nb_index": np.int32, "lj_a": np.float64, "lj_b": np.float64,
          "lj14_a": np.float64, "lj14_b": np.float64, "bond_atoms": np.int32, "bond_k": np.float64,
          "bond_r0": np.float64, "ub_atoms": np.int32, "ub_k": np.float64, "ub_r0": np.float64,
          "angle_atoms": np.int32, "angle_k": np.float64, "angle_theta0": np.float64,
          "dihedral_atoms": np.int32, "dihedral_k": np.float64, "dihedral_n": np.float64,
          "dihedral_phase": np.float64, "improper_atoms": np.int32, "improper_k": np.float64,
          "improper_phase": np.float64, "cmap_atoms": np.int32, "cmap_set": np.int32, "cmap_coeff": np.float64,
          "excl_pairs": np.int32, "pairs14": np.int32, "scee14": np.float64, "scnb14": np.float64}


def _files(cfg, sentinels, tmp_path):
    s = H.system(cfg, sentinels)
    return s, synth.write_files(s, str(tmp_path), stem=cfg)


@pytest.mark.parametrize("cfg,sent", [("tiny", False), ("tiny", True), ("small", False)])
@pytest.mark.parametrize("sem", [abi.MDF_SEM_REFERENCE, abi.MDF_SEM_PHYSICAL])
def test_cpp_reader_matches_python_flatten(cfg, sent, sem, tmp_path):
    engine.library()   # builds libmdf.so and the mdb200 command line
    s, (prm, rst) = _files(cfg, sent, tmp_path)
    out = tmp_path / "dump"
    out.mkdir()
    args = [CLI, prm, rst, "--dump-topology", str(out)] + (["--physical"] if sem == abi.MDF_SEM_PHYSICAL else [])
    subprocess.run(args, check=True, capture_output=True)
    flat = H.flat(s, sem, engine.cmap_coefficients)
    for name, dt in ARRAYS.items():
        got = np.fromfile(out / (name + ".bin"), dtype=dt)
        want = np.asarray(getattr(flat, name)).reshape(-1).astype(dt)
        assert got.shape == want.shape, (name, got.shape, want.shape)
        assert np.array_equal(got, want), name


def _energies(text):
    out = {}
    for key, label in (("bond", "Bond:"), ("angle", "Angle:"), ("dihedral", "CosineDihedral:"),
                       ("ub", "Urey-Bradley:"), ("improper", "Impropers:"), ("cmap", "CMAP energy:"),
                       ("vdw", "VDW:"), ("ee", "EE:"), ("ee_pairlist", "EE pairlist:"),
                       ("ee_cutoff", "EE_energy_pairlist_cutoff_"), ("ee_direct", "EE_energy_pairlist_ewald_direct_"),
                       ("ee_self", "EE_energy_pairlist_ewald_self_")):
        m = re.search(r"^" + re.escape(label) + r"\s*(\S+)", text, re.M)
        out[key] = float(m.group(1))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["tiny", "tiny_sentinel"])
def test_cli_prints_the_references_energies(case, tmp_path):
    g = H.golden(case)
    m = g["meta"]
    s, (prm, rst) = _files(m["config"], m["sentinels"], tmp_path)
    fo = tmp_path / "forces.bin"
    grid = [str(k) for k in m["grid"]]
    r = subprocess.run([CLI, prm, rst, "--tol", str(m["tol"]), "--grid"] + grid + ["--forces-out", str(fo)],
                       check=True, capture_output=True, text=True)
    E = _energies(r.stdout)
    for k, v in E.items():
        assert H.rel(v, g["energies"][k]) < 1e-9, (k, v, g["energies"][k])
    F = np.fromfile(fo, dtype=np.float64).reshape(-1, 3)
    H.check_forces_vs_golden(F, g, 1e-9, "forces")


@pytest.mark.gpu
def test_cli_minimise_and_dynamics(tmp_path):
    """The command line's --minimize (L-BFGS) lowers the energy, and --md runs
    velocity Verlet and writes a restart the reader takes back (PHYSICAL,
    mixed)."""
    import re
    s, (prm, rst) = _files("tiny", False, tmp_path)
    out = tmp_path / "out.rst7"
    r = subprocess.run([CLI, prm, rst, "--physical", "--mixed", "--grid", "24", "24", "24", "--minimize", "50",
                        "--md", "100", "0.0005", "--rst7-out", str(out)], check=True, capture_output=True, text=True)
    m = re.search(r"minimised \(L-BFGS\): (\d+) iterations, (\d+) evaluations, E (\S+) -> (\S+),", r.stdout)
    assert m, r.stdout
    assert int(m.group(1)) > 0 and int(m.group(2)) > int(m.group(1))
    assert float(m.group(4)) < float(m.group(3))
    d = re.search(r"dynamics: (\d+) steps", r.stdout)
    assert d and int(d.group(1)) == 100, r.stdout
    lines = out.read_text().splitlines()   # title; atom count + time; fixed 12-column fields
    assert int(lines[1][:6]) == s.natoms
    vals = np.array([float(t[i:i + 12]) for t in lines[2:] for i in range(0, len(t), 12)])
    assert vals.size == 6 * s.natoms + 6 and np.isfinite(vals).all()


def test_cpp_reader_at_960k_atoms(tmp_path):
    """The dynamics workload (320,000 flexible waters, 960,000 atoms) written as
    prmtop/rst7 (~100 MB + 35 MB) and read back by the C++ reader: the same
    PHYSICAL arrays as the Python host, and the read + flatten within a few
    seconds (mdb200 times and prints both; about 1.1 s on one core here)."""
    engine.library()
    s, (prm, rst) = _files("c4", False, tmp_path)
    out = tmp_path / "dump"
    out.mkdir()
    r = subprocess.run([CLI, prm, rst, "--physical", "--dump-topology", str(out)], check=True, capture_output=True,
                       text=True)
    m = re.search(r"read (\d+) atoms in (\S+) s, flattened in (\S+) s", r.stdout)
    assert m and int(m.group(1)) == s.natoms, r.stdout
    assert float(m.group(2)) + float(m.group(3)) < 10.0, r.stdout
    flat = H.flat(s, abi.MDF_SEM_PHYSICAL, engine.cmap_coefficients)
    for name in ("charge", "type", "bond_atoms", "bond_k", "angle_atoms", "angle_theta0", "excl_pairs"):
        got = np.fromfile(out / (name + ".bin"), dtype=ARRAYS[name])
        want = np.asarray(getattr(flat, name)).reshape(-1).astype(ARRAYS[name])
        assert np.array_equal(got, want), name
