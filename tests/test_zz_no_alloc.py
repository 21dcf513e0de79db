"""odt_born_series_noalloc: the Born-series loop for callers that cannot let
the library allocate GPU memory (a host framework that owns the device
memory pool, or a request loop that must stay out of the driver's allocator).
It runs on a fixed per-device scratch array; here it is called twice in a row
through the C ABI and each result is compared with the field that the
allocating entry point (odt_solve) returns for the same illumination, within
the 1e-5 relative-L2 tolerance of the other GPU tests.  This file is named to
be collected last.
"""
import ctypes as C

import numpy as np
import pytest

import cases
from oracle import cbs

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _small_case():
    p = cases.small_params(return_transmission=False, return_3D=True)
    return p, cases.small_RI()


def _large_radix_case():
    """Padded grid 46 x 48 x 29 (radices 23 and 29)."""
    size = [22, 24, 5]
    p = cases.params(size, [6, 6, 6], return_transmission=False, return_3D=True)
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=sum(size), n_spheres=2, radius_um=(0.1, 0.2))
    return p, RI


@pytest.mark.parametrize("make_case", [_small_case, _large_radix_case], ids=["small", "radix23_29"])
def test_noalloc_born_series_matches_solve_on_two_calls(make_case):
    import torch

    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN, _lib

    p, RI = make_case()
    fields = cases.circle_fields(p, 2)
    s = FORWARD_SOLVER_CONVERGENT_BORN(p)
    s.set_RI(RI)
    _, _, f3 = s.solve(fields)  # allocating entry point

    # incident fields inside the ROI: refocused input (single precision)
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    inp = o.transform_field_3D(cbs.fftc2(fields.astype(np.complex64)))

    dev = torch.device("cuda", 0)

    def on_dev(a, dtype):
        flat = np.ascontiguousarray(np.asarray(a, dtype=dtype).ravel(order="F"))
        return torch.from_numpy(flat).to(dev)

    keep = []
    args = _lib.NoallocBornArgs()
    args.sim_size[:] = s.sim_size
    args.roi[:] = [int(r) for r in s.ROI]
    args.bornmax = int(s.Bornmax)
    args.acyclic = 1
    args.eps_imag = float(s.eps_imag)
    args.green_scale = float(np.float32(4 * np.pi ** 2))
    args.green_offset = float(np.float32((2 * np.pi * s.utility_border.k0_nm) ** 2))
    for i in range(3):
        m = on_dev(s.attenuation_mask1d[i], np.float32)
        r = on_dev(s.ramp1d[i], np.complex64)
        q = on_dev(s.kq2[i], np.float32)
        keep += [m, r, q]
        args.mask[i], args.ramp[i], args.kq2[i] = m.data_ptr(), r.data_ptr(), q.data_ptr()
    V = on_dev(s.V, np.complex64)
    keep.append(V)
    args.V = V.data_ptr()
    args.stream = None
    R = s.expected_RI_size
    lib = _lib.load()
    for k in range(2):  # two calls in a row share the scratch array
        einc = on_dev(o.refocus_source(inp[:, :, 0, k]), np.complex64)
        fout = torch.empty(R[0] * R[1] * R[2], dtype=torch.complex64, device=dev)
        args.einc = einc.data_ptr()
        args.fout = fout.data_ptr()
        _lib.check(lib.odt_born_series_noalloc(C.byref(args)))
        got = fout.cpu().numpy().reshape(R, order="F")
        err = cbs.rel_l2(got, f3[:, :, :, 0, k])
        assert err < TOL, (k, err)
    s.delete()


def test_noalloc_rejects_grids_beyond_the_fixed_scratch():
    from inverse_solver_b200 import _lib

    args = _lib.NoallocBornArgs()
    args.sim_size[:] = [160, 160, 160]
    args.roi[:] = [1, 160, 1, 160, 1, 160]
    args.bornmax = 1
    args.acyclic = 1
    args.eps_imag = 1.0
    one = C.c_float(1.0)
    for i in range(3):
        args.mask[i] = args.ramp[i] = args.kq2[i] = C.addressof(one)
    args.V = args.einc = args.fout = C.addressof(one)
    lib = _lib.load()
    st = lib.odt_born_series_noalloc(C.byref(args))
    assert st == 4
    assert b"fixed array" in lib.odt_last_error()
