"""Generates tests/golden/vector_small.npz from the oracle (test fixture).

Dyadic (vector_simulation) solves of a small seeded phantom: the isotropic
RI, an RI tensor (birefringent with an xy coupling term) and the vector
gradient of BACKWARD_SOLVER_MULTI.get_gradiant_static, in single and double
precision.  The reference is MATLAB and cannot run here, so these vectors pin
the *oracle* (regression fixture, parity unpinned).

usage: python tests/golden/make_vector_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

from oracle import cbs, multi  # noqa: E402
import cases  # noqa: E402

SIZE = [20, 20, 13]


def params():
    p = cases.params(SIZE, [1.5, 1.5, 1.0], return_reflection=True, return_3D=True)
    p["vector_simulation"] = True
    return p


def inputs():
    RI = cases.sphere_phantom(SIZE, [0.1] * 3, cases.NM, seed=21, n_spheres=2, radius_um=(0.3, 0.6))
    f = cases.circle_fields(cases.params(SIZE, [1.5, 1.5, 1.0]), 2)
    fv = np.zeros((SIZE[0], SIZE[1], 2, 2), np.complex64)
    fv[:, :, 0, 0] = f[:, :, 0, 0]
    fv[:, :, 1, 1] = f[:, :, 0, 1]
    T = np.full(RI.shape + (3, 3), cases.NM, np.float64)
    for i in range(3):
        T[:, :, :, i, i] = cases.NM + (RI - cases.NM) * (1 - 0.25 * i)
    T[:, :, :, 0, 1] = T[:, :, :, 1, 0] = cases.NM + (RI - cases.NM) * 0.2
    return RI, T, fv


def compute(single):
    RI, T, fv = inputs()
    p = params()
    out = {}
    o = cbs.ForwardSolverCBS(p, single=single)
    o.set_RI(RI)
    out["iso_trans"], out["iso_ref"], _ = o.solve(fv)
    ot = cbs.ForwardSolverCBS(p, single=single)
    ot.set_RI(T)
    out["ten_trans"], out["ten_ref"], _ = ot.solve(fv)
    RI0 = (RI * 0.7 + cases.NM * 0.3).astype(np.float32)
    out["grad"], out["err"] = multi.get_gradient_static(RI0, fv, out["iso_trans"], o)
    return out


def main():
    RI, T, fv = inputs()
    o32, o64 = compute(True), compute(False)
    np.savez_compressed(os.path.join(HERE, "vector_small.npz"), RI=RI, fields=fv,
                        **{k + "32": np.asarray(v) for k, v in o32.items()},
                        **{k + "64": np.asarray(v) for k, v in o64.items()})


if __name__ == "__main__":
    main()
