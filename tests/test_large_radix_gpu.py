"""GPU parity of the generic tile kernels for padded lengths whose prime
factors reach 23, 29 and 31 (radix class 3): such lengths arise from odd z
sizes (which the reference's inverse solver requires) with boundary widths
other than the default, e.g. 129 + 2*8 = 145 = 5 * 29.  Grids
(46, 48, 29) = (2*23, 48, 29) and (48, 62, 31) = (48, 2*31, 31) against the
single-precision oracle: relative L2 per illumination 1e-5 for the
transmitted and 3D fields, 3e-5 reflected."""
import numpy as np
import pytest

import cases
from oracle import cbs

pytestmark = pytest.mark.gpu


def worst(a, b):
    return max(cbs.rel_l2(a[..., k], b[..., k]) for k in range(a.shape[-1]))


@pytest.mark.parametrize("size", [[22, 24, 5], [24, 38, 7]])
def test_radix_23_29_31_match_oracle(size):
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN

    p = cases.params(size, [6, 6, 6], return_reflection=True, return_3D=True)
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=sum(size), n_spheres=2, radius_um=(0.1, 0.2))
    fields = cases.circle_fields(p, 2)
    s = FORWARD_SOLVER_CONVERGENT_BORN(p)
    s.set_RI(RI)
    t, r, f = s.solve(fields)
    assert s.sim_size == [v + 24 for v in size]
    s.delete()
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    ot, orr, of = o.solve(fields)
    assert worst(f, of) < 1e-5 and worst(t, ot) < 1e-5 and worst(r, orr) < 3e-5
