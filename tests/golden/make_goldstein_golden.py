"""Generates tests/golden/goldstein_small.npz: seeded wrapped-phase stacks
with the reference's own results for the branch-cut stages that are
compiled here from its sources (oracle/ref_goldstein -> oracle/_ref):
the 8 nearest residues of every residue (shortest_compute_kernel run on the
host) and the branch list of its linker (get_branches_goldstein_compute),
both fed with the oracle's residue table.  The oracle's residue maps, steps
and unwrapped phases are stored beside them.

Run from the repository root after `make -C oracle/ref_goldstein`:
    python tests/golden/make_goldstein_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import cases  # noqa: E402
from oracle import goldstein as g  # noqa: E402

CASES = [((32, 32, 2), 0, 0.6), ((48, 40, 3), 1, 0.9), ((64, 64, 2), 2, 1.2), ((17, 23, 1), 3, 1.5),
         ((40, 40, 1), 5, 3.0), ((24, 24, 2), 6, 2.0)]


def main():
    lib = g.ref_lib()
    if lib is None:
        raise SystemExit("build oracle/_ref first: make -C oracle/ref_goldstein")
    out = {}
    for k, (shape, seed, noise) in enumerate(CASES):
        ph = cases.wrapped_phase(shape, seed, noise)
        uw, it = g.unwrapp2(ph, return_intermediates=True)
        M = it["residue"].shape
        near = g.ref_nearest(lib, it["table"], it["lookup"], it["lookup_z_start"], it["square_size"], 8, M)
        br = g.ref_branches(lib, it["table"], near, it["square_size"], it["lookup"], it["lookup_z_start"], M)
        out.update({f"c{k}_phase": ph, f"c{k}_residue": it["residue"], f"c{k}_table": it["table"],
                    f"c{k}_ref_nearest": near, f"c{k}_ref_branches": br, f"c{k}_step1": it["step1"],
                    f"c{k}_step2": it["step2"], f"c{k}_unwrapped": uw})
    out["n_cases"] = np.int32(len(CASES))
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "goldstein_small.npz"), **out)


if __name__ == "__main__":
    main()
