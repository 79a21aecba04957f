"""Generate the golden fixtures from the UNMODIFIED reference (O1).

Run in a container that has the reference sources (it builds oracle/_ref/
o1_harness from them):

    python tests/golden/make_golden.py [case ...]   # default: every case

For every case it writes tests/golden/<case>/:
  meta.json          generator config, sha256 of the written prmtop/rst7 text,
                     Ewald alpha, PME grid, the reference's pair-list size
  energies.json      every energy member the reference computes (%.17g)
  forces.npy         calculate_forces() result (small cases) or
  forces_digest.npz  norms and two atom subsets of it (large cases)
  forces_pme.npy     gather_forces_pme() result (the forces the reference
                     computes in init() and then discards)
The tiny cases also keep their prmtop/rst7 so parsers can be checked against
the exact files the reference read.  Inputs of the other cases are
regenerated by md_b200.synth and checked against the recorded hashes.
"""
import hashlib
import json
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from md_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

CASES = [
    # name, config, sentinels, keep input files, full forces
    ("tiny", "tiny", False, True, True),
    ("tiny_sentinel", "tiny", True, True, True),
    ("small", "small", False, False, True),
    ("c0", "c0", False, False, False),
    ("c1", "c1", False, False, False),
]
DIGEST_ATOMS = 256


def sha(path):
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def digest_indices(n):
    rng = np.random.default_rng(12345)
    return np.concatenate([np.arange(min(DIGEST_ATOMS, n)), rng.choice(n, size=min(DIGEST_ATOMS, n), replace=False)])


def main(only=()):
    O.build()
    for name, cfg, sent, keep, full in CASES:
        if only and name not in only:
            continue
        out = os.path.join(HERE, name)
        os.makedirs(out, exist_ok=True)
        s = synth.make_config(cfg, sentinels=sent)
        tmp = tempfile.mkdtemp(prefix="golden_")
        prm, rst = synth.write_files(s, tmp, stem=name)
        grid = synth.GRIDS[cfg]
        res = O.run_o1(prm, rst, grid, tol=1e-5, allpairs=True)
        meta = dict(config=cfg, sentinels=sent, grid=list(grid), tol=1e-5, natoms=s.natoms,
                    sha_prmtop=sha(prm), sha_rst7=sha(rst), alpha=float(res["info"]["alpha"]),
                    reference_pairs=int(res["info"]["pairs"]))
        with open(os.path.join(out, "meta.json"), "w") as f:
            json.dump(meta, f, indent=1)
        with open(os.path.join(out, "energies.json"), "w") as f:
            f.write("{\n" + ",\n".join('  "%s": %.17g' % (k, v) for k, v in res["energies"].items()) + "\n}\n")
        if full:
            np.save(os.path.join(out, "forces.npy"), res["forces"])
            np.save(os.path.join(out, "forces_pme.npy"), res["forces_pme"])
        else:
            idx = digest_indices(s.natoms)
            np.savez_compressed(os.path.join(out, "forces_digest.npz"), idx=idx, forces=res["forces"][idx],
                                forces_pme=res["forces_pme"][idx],
                                norm=np.linalg.norm(res["forces"]), norm_pme=np.linalg.norm(res["forces_pme"]))
        if keep:
            shutil.copy(prm, os.path.join(out, name + ".prmtop"))
            shutil.copy(rst, os.path.join(out, name + ".rst7"))
        shutil.rmtree(tmp, ignore_errors=True)
        print(name, s.natoms, "pairs", meta["reference_pairs"])


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
