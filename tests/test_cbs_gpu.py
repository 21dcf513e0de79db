"""GPU parity of the CBS forward solve (libodt through its C ABI) against the
oracle's single-precision restatement of FORWARD_SOLVER_CONVERGENT_BORN.m.

Tolerances (relative L2):
  * vs the single-precision oracle: 1e-5 for the transmitted and 3D fields;
    the reflected field, ~25x weaker than the transmitted one, 3e-5;
  * vs the double-precision oracle (the reference run in double): 2e-4,
    dominated by the single-precision Green's-function setup the reference
    itself uses.
"""
import os

import numpy as np
import pytest

import cases
from oracle import cbs

pytestmark = pytest.mark.gpu

TOL_T = 1e-5
TOL_3D = 1e-5
TOL_R = 3e-5
TOL_FP64 = 2e-4

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "cbs_small.npz")


def worst(a, b):
    """Largest per-illumination relative L2 error (last axis = illumination)."""
    return max(cbs.rel_l2(a[..., k], b[..., k]) for k in range(a.shape[-1]))


def _solver(p):
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN
    return FORWARD_SOLVER_CONVERGENT_BORN(p)


def test_small_case_matches_golden():
    g = np.load(GOLDEN)
    p = cases.small_params(return_reflection=True, return_3D=True)
    s = _solver(p)
    s.set_RI(g["RI"])
    assert s.Bornmax == int(g["bornmax"])
    t, r, f = s.solve(g["fields"])
    assert worst(t, g["trans32"]) < TOL_T
    assert worst(f, g["field3d32"]) < TOL_3D
    assert worst(r, g["ref32"]) < TOL_R
    assert worst(t, g["trans64"]) < TOL_FP64
    assert worst(r, g["ref64"]) < TOL_FP64
    s.delete()


def test_cfg1_bead_matches_oracle():
    """64^3 bead (RI 1.4607 in 1.3355), 16-voxel boundary, normal incidence,
    default iteration count (28 on the 96^3 padded grid)."""
    p = cases.cfg1_params(return_reflection=True, return_3D=True)
    RI = cases.cfg1_RI()
    inp = cases.normal_field([64, 64])
    s = _solver(p)
    s.set_RI(RI)
    assert s.Bornmax == 28 and s.sim_size == [96, 96, 96]
    t, r, f = s.solve(inp)
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    ot, orr, of = o.solve(inp)
    assert worst(t, ot) < TOL_T
    assert worst(f, of) < TOL_3D
    assert worst(r, orr) < TOL_R
    s.delete()


@pytest.mark.parametrize("iters", [1, 2, 3, 4, 7])
def test_iteration_count_edge_cases(iters):
    """The two interleaved half-series (jj = 1, 2, 3 bookkeeping) for short
    series, including Bornmax < 3."""
    p = cases.small_params(return_reflection=True, return_3D=True, iterations_number=iters)
    RI = cases.small_RI()
    fields = cases.circle_fields(p, 2)
    s = _solver(p)
    s.set_RI(RI)
    t, r, f = s.solve(fields)
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    ot, orr, of = o.solve(fields)
    assert worst(f, of) < TOL_3D
    assert worst(t, ot) < TOL_T
    assert worst(r, orr) < TOL_R
    s.delete()


def test_cyclic_xy_matches_oracle():
    p = cases.params([24, 20, 18], [0, 0, 2], return_reflection=True, return_3D=True)
    RI = cases.small_RI()[:24, :20, :18]
    fields = cases.circle_fields(p, 3)
    s = _solver(p)
    s.set_RI(RI)
    t, r, f = s.solve(fields)
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    ot, orr, of = o.solve(fields)
    assert worst(f, of) < TOL_3D
    assert worst(t, ot) < TOL_T
    assert worst(r, orr) < TOL_R
    s.delete()


def test_radix7_grid_matches_oracle():
    """Padded grid [56, 38, 24] (radices 7x8, 19x2, 3x8)."""
    p = cases.params([48, 30, 20], [2, 2, 1], return_reflection=True, return_3D=True)
    RI = cases.sphere_phantom([48, 30, 20], [0.1] * 3, cases.NM, seed=7, n_spheres=2,
                              radius_um=(0.3, 0.8))
    fields = cases.circle_fields(p, 2)
    s = _solver(p)
    s.set_RI(RI)
    assert s.sim_size == [56, 38, 24]
    t, r, f = s.solve(fields)
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    ot, orr, of = o.solve(fields)
    assert worst(f, of) < TOL_3D
    assert worst(t, ot) < TOL_T
    assert worst(r, orr) < TOL_R
    s.delete()


def test_batch_chunking_is_bit_identical():
    """Illuminations are independent: solving 5 in chunks of 2 or all at once
    gives identical bits."""
    RI = cases.small_RI()
    outs = []
    for mb in (2, 5):
        p = cases.small_params(return_reflection=True, return_3D=True, max_batch=mb)
        s = _solver(p)
        s.set_RI(RI)
        outs.append(s.solve(cases.circle_fields(p, 5)))
        assert s.batch() == mb
        s.delete()
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def test_device_api_matches_host_api():
    import torch

    p = cases.small_params(return_reflection=True, return_3D=True)
    RI = cases.small_RI()
    fields = cases.circle_fields(p, 3)
    s = _solver(p)
    s.set_RI(RI)
    t, r, f = s.solve(fields)
    F = s.field_size
    R = s.expected_RI_size
    fin = torch.from_numpy(np.ascontiguousarray(fields[:, :, 0, :].transpose(2, 1, 0))).cuda()
    dt = torch.empty((3, F[1], F[0]), dtype=torch.complex64, device="cuda")
    dr = torch.empty_like(dt)
    d3 = torch.empty((3, R[2], R[1], R[0]), dtype=torch.complex64, device="cuda")
    s.solve_device(fin, dt, dr, d3)
    torch.cuda.synchronize()
    assert np.array_equal(dt.cpu().numpy().transpose(2, 1, 0), t[:, :, 0, :])
    assert np.array_equal(dr.cpu().numpy().transpose(2, 1, 0), r[:, :, 0, :])
    assert np.array_equal(d3.cpu().numpy().transpose(3, 2, 1, 0), f[:, :, :, 0, :])
    s.delete()


def test_nan_input_is_reported():
    from inverse_solver_b200 import OdtError

    p = cases.small_params()
    s = _solver(p)
    s.set_RI(cases.small_RI())
    x = cases.circle_fields(p, 1)
    x[3, 4, 0, 0] = np.nan
    with pytest.raises(OdtError) as e:
        s.solve(x)
    assert e.value.status == 7
    s.delete()


def test_prime_length_dyadic_solve_is_rejected():
    """Padded lengths with a prime factor above 31 (29 + 2 * 4 = 37 along x
    and y; the dyadic solver needs a square field) run through Bluestein
    transforms for scalar solves (tests/test_any_length_gpu.py); the dyadic
    branch has no such path and is refused with ODT_ERR_UNSUPPORTED, while
    the scalar solver of the same grid is created."""
    from inverse_solver_b200 import OdtError

    p = cases.params([29, 29, 16], [2, 2, 2])
    _solver(p).delete()
    pv = dict(p, vector_simulation=True)
    with pytest.raises(OdtError) as e:
        _solver(pv)
    assert e.value.status == 6 and "dyadic" in str(e.value)


def test_solve_before_set_RI_and_bad_shapes():
    from inverse_solver_b200 import OdtError

    p = cases.small_params()
    s = _solver(p)
    with pytest.raises(OdtError) as e:
        s.solve(cases.circle_fields(p, 1))
    assert e.value.status == 5
    with pytest.raises(ValueError):
        s.set_RI(np.ones((5, 5, 5), np.float32))
    s.delete()
