"""Generates tests/golden/bench_fp64.npz from the oracle in double precision
(test fixture): the transmitted and reflected fields of four illuminations of
the benchmark workload (bench.py: 128^3 seeded multi-sphere phantom, seed 0,
default boundary -> 152^3 padded grid, Bornmax 40) -- normal incidence and one
plane wave on each of the NA 0.3 / 0.6 / 0.9 rings (illuminations 0, 5, 13,
37 of the 49).  The GPU test states each field's error against these FP64
results (tests/test_measured_configs_gpu.py); the 3D fields are too large to
store and are compared with the single-precision oracle at test time.

The double-precision values are stored as complex64 (their rounding, 6e-8,
is far below the errors being measured).

usage: python tests/golden/make_bench_golden.py      (about a minute and a half on 8 cores)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from oracle import cbs  # noqa: E402

SEL = [0, 5, 13, 37]


def main():
    p = bench.workload_params()
    p["return_reflection"] = True
    RI, fields = bench.workload_inputs(p)
    o = cbs.ForwardSolverCBS(p, single=False)
    o.set_RI(RI)
    t, r, _ = o.solve(np.ascontiguousarray(fields[:, :, :, SEL]))
    np.savez_compressed(os.path.join(HERE, "bench_fp64.npz"), sel=np.array(SEL), bornmax=o.Bornmax,
                        trans64=t.astype(np.complex64), ref64=r.astype(np.complex64))


if __name__ == "__main__":
    main()
