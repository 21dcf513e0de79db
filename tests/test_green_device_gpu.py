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
        e = cbs.rel_l2(getattr(d, name), getattr(h, name))
        print("device vs host", size, name, e)
        assert e < 5e-6, name
    hp = dict(p, green_on_device=False)
    hs = FORWARD_SOLVER_CONVERGENT_BORN(hp)
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=sum(size), n_spheres=2, radius_um=(0.3, 0.6))
    fields = cases.circle_fields(p, 2)
    d.set_RI(RI)
    hs.set_RI(RI)
    t1, r1, f1 = d.solve(fields)
    t2, r2, f2 = hs.solve(fields)
    print("solve on device vs host kernels", size, cbs.rel_l2(t1, t2), cbs.rel_l2(f1, f2), cbs.rel_l2(r1, r2))
    assert cbs.rel_l2(t1, t2) < 1e-6 and cbs.rel_l2(f1, f2) < 1e-6 and cbs.rel_l2(r1, r2) < 1e-5
    d.delete()
    hs.delete()


@pytest.mark.parametrize("size", [[32, 30, 21], [64, 48, 33]])
def test_tensor_core_gemms_match_simt(size, monkeypatch):
    """The plane GEMMs run on the tensor cores (csrc/tc_gemm.cu: tcgen05
    kind::tf32, every operand split into two TF32 parts, three products per
    K step accumulated in tensor memory per 32-wide K block, the blocks added
    in FP32 registers) by default; ODT_GREEN_GEMM=simt selects the FP32 SIMT
    kernel.  The two agree within rel-L2 2e-6 (measured 5.6e-7 - 7.8e-7) and
    both within 5e-6 of the host build (whose FFT route differs from either by
    5.6e-7 - 8.6e-7)."""
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN
    from inverse_solver_b200.forward import CBSHostSetup

    p = cases.params(size, [6, 6, 6], return_reflection=True, return_3D=True)
    h = CBSHostSetup(p)
    tc = FORWARD_SOLVER_CONVERGENT_BORN(p)
    monkeypatch.setenv("ODT_GREEN_GEMM", "simt")
    sm = FORWARD_SOLVER_CONVERGENT_BORN(p)
    try:
        for name in ("refocusing_util", "kernel_trans", "kernel_ref"):
            a, b, ref = getattr(tc, name), getattr(sm, name), getattr(h, name)
            print("tc vs simt / host", size, name, cbs.rel_l2(a, b), cbs.rel_l2(a, ref), cbs.rel_l2(b, ref))
            assert cbs.rel_l2(a, b) < 2e-6, name
            assert cbs.rel_l2(a, ref) < 5e-6 and cbs.rel_l2(b, ref) < 5e-6, name
    finally:
        tc.delete()
        sm.delete()
