"""Generates tests/golden/cbs_small.npz from the oracle (test fixture).

The reference is MATLAB and cannot run here, so these vectors pin the
*oracle* (regression fixture, parity unpinned): the GPU tests compare against
them and the CPU tests check that the oracle still reproduces them.

usage: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

from oracle import cbs  # noqa: E402
import cases  # noqa: E402


def run(single):
    p = cases.small_params(return_reflection=True, return_3D=True)
    s = cbs.ForwardSolverCBS(p, single=single)
    s.set_RI(cases.small_RI())
    fields = cases.circle_fields(p, 3)
    return fields, s.solve(fields), s


def main():
    fields, (t32, r32, f32), s = run(True)
    _, (t64, r64, f64), _ = run(False)
    np.savez_compressed(
        os.path.join(HERE, "cbs_small.npz"),
        fields=fields, RI=cases.small_RI(),
        trans32=t32, ref32=r32, field3d32=f32,
        trans64=t64.astype(np.complex128), ref64=r64.astype(np.complex128),
        bornmax=np.int32(s.Bornmax), eps=np.float32(s.eps_imag))
    print("Bornmax", s.Bornmax, "eps", s.eps_imag, "padded", s.V.shape)


if __name__ == "__main__":
    main()
