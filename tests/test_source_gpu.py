"""odt_solve_source, CudaBorn's legacy action 2 (CUDA_CODE/main.cpp:139-163:
a 3D source in, the 3D field out): driven by the incident fields that the
input stage of odt_solve forms (the refocused input over the RI grid, here
from the single-precision oracle), it must give odt_solve's 3D fields
(relative L2 1e-5 per illumination; the two incident fields differ in the
last places), on a grid with the fused xy-pass and on one without; fields of
the wrong size are rejected."""
import numpy as np
import pytest

import cases
from oracle import cbs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("size,bt", [([64, 64, 16], [6, 6, 6]), ([30, 26, 21], [2, 3, 1.5])])
def test_solve_source_equals_solve(size, bt):
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN

    p = cases.params(size, bt, return_transmission=False, return_3D=True)
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=9, n_spheres=2, radius_um=(0.3, 0.8))
    fields = cases.circle_fields(p, 3)
    s = FORWARD_SOLVER_CONVERGENT_BORN(p)
    try:
        s.set_RI(RI)
        _, _, f3 = s.solve(fields)
        o = cbs.ForwardSolverCBS(p, single=True)
        o.set_RI(RI)
        inp = o.transform_field_3D(cbs.fftc2(fields.astype(np.complex64)))
        src = np.stack([o.refocus_source(inp[:, :, 0, k]) for k in range(3)], axis=-1).astype(np.complex64)
        got = s.solve_source(src)
        assert got.shape == src.shape
        for k in range(3):
            assert cbs.rel_l2(got[..., k], f3[:, :, :, 0, k]) < 1e-5, k
        one = s.solve_source(src[..., 1])
        assert one.shape == src.shape[:3] and cbs.rel_l2(one, got[..., 1]) < 1e-6
        with pytest.raises(ValueError):
            s.solve_source(src[:-1])
    finally:
        s.delete()
