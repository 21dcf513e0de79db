"""Padded grids with lengths outside the radix tiles (a prime factor above
31): the reference pads the RI grid by the boundary width without rounding
(FORWARD_SOLVER_CONVERGENT_BORN.m:129), so any length occurs, and its fftn /
fft2 take any length.  The library runs such axes through Bluestein's
algorithm (csrc/fft_any.cu) and the Born loop unfused (csrc/born_any.cu).

  * RI grid 37 x 20 x 17 -> padded 61 x 44 x 41 (x and z Bluestein), field
    37 x 20 and convolution grid 74 x 40 (x Bluestein in the input / output
    stages);
  * RI grid 20 x 37 x 23 -> padded 44 x 61 x 47 (y and z), field 20 x 37,
    convolution 40 x 74 (y);
both against the single-precision oracle (relative L2 per illumination 2e-5
for the transmitted and 3D fields, 5e-5 reflected: the chirp-z transforms
add a few units of rounding per axis), with and without the phase ramp; and
the gradient of BACKWARD_SOLVER_MULTI on the first grid against the oracle's
(relative L2 5e-5)."""
import numpy as np
import pytest

import cases
from oracle import cbs

pytestmark = pytest.mark.gpu


def worst(a, b):
    return max(cbs.rel_l2(a[..., k], b[..., k]) for k in range(a.shape[-1]))


@pytest.mark.parametrize("size,acyclic", [([37, 20, 17], True), ([20, 37, 23], True), ([37, 20, 17], False)])
def test_bluestein_grid_matches_oracle(size, acyclic):
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN

    p = cases.params(size, [6, 6, 6], return_reflection=True, return_3D=True, acyclic=acyclic)
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=sum(size), n_spheres=2, radius_um=(0.3, 0.7))
    fields = cases.circle_fields(p, 3)
    s = FORWARD_SOLVER_CONVERGENT_BORN(p)
    try:
        assert s.sim_size == [v + 24 for v in size]
        s.set_RI(RI)
        t, r, f = s.solve(fields)
        bm = s.Bornmax
    finally:
        s.delete()
    assert bm >= 4
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    ot, orr, of = o.solve(fields)
    e = (worst(f, of), worst(t, ot), worst(r, orr))
    print("Bluestein grid", size, "acyclic", acyclic, "3D / trans / ref:", e)
    assert e[0] < 2e-5 and e[1] < 2e-5 and e[2] < 5e-5


def test_bluestein_grid_gradient_matches_oracle():
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN
    from oracle import multi

    size = [37, 20, 17]
    p = cases.params(size, [6, 6, 6], return_transmission=True, return_3D=True)
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=5, n_spheres=2, radius_um=(0.3, 0.7))
    fields = cases.circle_fields(p, 2)
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    meas, _, _ = o.solve(fields)
    RI0 = (RI * 0.7 + cases.NM * 0.3).astype(np.float32)   # a misfit that is not zero
    s = FORWARD_SOLVER_CONVERGENT_BORN(p)
    try:
        s.set_RI(RI0)
        s.set_RI_adjoint(RI0)
        g, err = s.gradient(fields, meas)
    finally:
        s.delete()
    go, erro = multi.get_gradient_static(RI0, fields, meas, cbs.ForwardSolverCBS(p, single=True))
    assert cbs.rel_l2(g, go) < 5e-5
    assert abs(err - erro) / erro < 5e-5
