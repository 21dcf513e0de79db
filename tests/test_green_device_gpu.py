"""The plane part of truncated_green_plus on the GPU (odt_green_planes,
used by FORWARD_SOLVER_CONVERGENT_BORN unless green_on_device=False) against
the host build (CBSHostSetup, bit-identical to the oracle's single-precision
set-up): the refocusing kernel and the transmission / reflection kernels
within rel-L2 5e-6 (the device applies the centred DFT / crop chains as
single-precision GEMMs, accumulating over the oversized grid's length,
where the host runs FFTs: 1.3e-6 apart on these grids), and a solve within
1e-6 of one on host-built kernels.""" 
import numpy as np
import pytest

import cases
from oracle import cbs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("size", [[32, 30, 21], [40, 40, 21]])
def test_device_green_matches_host(size):
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN
    from inverse_solver_b200.forward import CBSHostSetup

    p = cases.params(size, [6, 6, 6], return_reflection=True, return_3D=True)
    h = CBSHostSetup(p)
    d = FORWARD_SOLVER_CONVERGENT_BORN(p)
    for name in ("refocusing_util", "kernel_trans", "kernel_ref"):
        assert cbs.rel_l2(getattr(d, name), getattr(h, name)) < 5e-6, name
    hp = dict(p, green_on_device=False)
    hs = FORWARD_SOLVER_CONVERGENT_BORN(hp)
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=sum(size), n_spheres=2, radius_um=(0.3, 0.6))
    fields = cases.circle_fields(p, 2)
    d.set_RI(RI)
    hs.set_RI(RI)
    t1, r1, f1 = d.solve(fields)
    t2, r2, f2 = hs.solve(fields)
    assert cbs.rel_l2(t1, t2) < 1e-6 and cbs.rel_l2(f1, f2) < 1e-6 and cbs.rel_l2(r1, r2) < 1e-5
    d.delete()
    hs.delete()
