"""GPU parity of the pipelined Born passes (csrc/born_pipe.cu, the x-pass of
iterations 2 onward and the final pass;
csrc/cols_pipe.cu, the y-FFTs and the z-pass: persistent CTAs, bulk / tiled
asynchronous copies, compile-time 8 x R2 plans), which the library selects
for grid lengths 88, 120, 152, 200, 216 and (x and y) 280.

  * against the single-precision oracle on grids that put each of 88, 120
    and 152 on each axis (relative L2 per illumination 1e-5 for the
    transmitted and 3D fields, 3e-5 reflected);
  * against the library's generic tile kernels (ODT_KERNELS=generic) on the
    benchmark's 152^3 grid with a partial last y-tile and several batches:
    relative L2 <= 1e-6 (the same operations; only the compiler's
    contraction choices may differ)."""
import os

import numpy as np
import pytest

import cases
from oracle import cbs

pytestmark = pytest.mark.gpu


def worst(a, b):
    return max(cbs.rel_l2(a[..., k], b[..., k]) for k in range(a.shape[-1]))


def _solve(p, RI, fields, kernels=None):
    """Solve with ODT_KERNELS=kernels; the fused xy-pass is off (ODT_XY=0) so
    that these tests exercise the separate pipelined x-, y- and z-passes
    (tests/test_xy_gpu.py covers the fused pass)."""
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN

    old = os.environ.get("ODT_KERNELS")
    old_xy = os.environ.get("ODT_XY")
    os.environ["ODT_XY"] = "0"
    if kernels:
        os.environ["ODT_KERNELS"] = kernels
    try:
        s = FORWARD_SOLVER_CONVERGENT_BORN(p)
        s.set_RI(RI)
        out = s.solve(fields)
        info = (s.sim_size, s.Bornmax)
        s.delete()
    finally:
        if old is None:
            os.environ.pop("ODT_KERNELS", None)
        else:
            os.environ["ODT_KERNELS"] = old
        if old_xy is None:
            os.environ.pop("ODT_XY", None)
        else:
            os.environ["ODT_XY"] = old_xy
    return out, info


@pytest.mark.parametrize("size", [[64, 96, 64], [128, 24, 128], [96, 64, 16]])
def test_pipe_passes_match_oracle(size):
    """Padded grids (88, 120, 88), (152, 48, 152), (120, 88, 40)."""
    p = cases.params(size, [6, 6, 6], return_reflection=True, return_3D=True)
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=size[0], n_spheres=3,
                              radius_um=(0.3, 0.8))
    fields = cases.circle_fields(p, 2)
    (t, r, f), (sim, bm) = _solve(p, RI, fields)
    assert sim == [v + 24 for v in size] and bm >= 4
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    ot, orr, of = o.solve(fields)
    assert worst(f, of) < 1e-5
    assert worst(t, ot) < 1e-5
    assert worst(r, orr) < 3e-5


def test_pipe_matches_generic_on_benchmark_grid():
    from inverse_solver_b200.inputs import ring_illumination, sphere_phantom

    size = [128, 128, 128]
    p = cases.params(size, [6, 6, 6], return_3D=True, max_batch=3)
    RI = sphere_phantom(size, [0.1] * 3, cases.NM, seed=0)
    fields = np.ascontiguousarray(ring_illumination(p)[:, :, :, :5])
    (t1, _, f1), (sim, bm) = _solve(p, RI, fields)
    (t2, _, f2), _ = _solve(p, RI, fields, kernels="generic")
    assert sim == [152, 152, 152] and bm >= 30
    assert worst(t1, t2) < 1e-6
    assert worst(f1, f2) < 1e-6


def test_pipe_passes_cyclic_boundary_matches_oracle():
    """acyclic = false (no phase ramp, no Green's-function flips) through the
    pipelined x-, y- and z-passes: padded grid (120, 88, 40)."""
    size = [96, 64, 16]
    p = cases.params(size, [6, 6, 6], return_3D=True, acyclic=False)
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=9, n_spheres=3, radius_um=(0.3, 0.8))
    fields = cases.circle_fields(p, 2)
    (t, _, f), (sim, bm) = _solve(p, RI, fields)
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    ot, _, of = o.solve(fields)
    assert worst(f, of) < 1e-5 and worst(t, ot) < 1e-5


@pytest.mark.parametrize("size", [[176, 24, 16], [24, 192, 16], [24, 24, 192], [192, 24, 16]])
def test_pipe_radix_25_27_match_oracle(size):
    """Padded lengths 200 = 8 x 25 and 216 = 8 x 27 on each axis in turn:
    (200, 48, 40), (48, 216, 40), (48, 48, 216), (216, 48, 40); the x-pass
    uses tiles of 8 lines there."""
    p = cases.params(size, [6, 6, 6], return_3D=True)
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=sum(size), n_spheres=2,
                              radius_um=(0.3, 0.8))
    fields = cases.circle_fields(p, 2)
    (t, _, f), (sim, bm) = _solve(p, RI, fields)
    assert sim == [v + 24 for v in size] and bm >= 4
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    ot, _, of = o.solve(fields)
    assert worst(f, of) < 1e-5 and worst(t, ot) < 1e-5


@pytest.mark.parametrize("size", [[256, 24, 16], [24, 256, 16]])
def test_pipe_radix_35_matches_oracle(size):
    """Padded length 280 = 8 x 35 (the x-y planes of the 256 x 256 x 192
    serving grid; the 35-point butterfly is the 5 x 7 composite) on the x-
    and the y-axis: (280, 48, 40) and (48, 280, 40)."""
    p = cases.params(size, [6, 6, 6], return_3D=True, iterations_number=8)
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=sum(size) + 1, n_spheres=2,
                              radius_um=(0.3, 0.8))
    fields = cases.circle_fields(p, 2)
    (t, _, f), (sim, bm) = _solve(p, RI, fields)
    assert sim == [v + 24 for v in size] and bm == 8
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    ot, _, of = o.solve(fields)
    assert worst(f, of) < 1e-5 and worst(t, ot) < 1e-5


@pytest.mark.parametrize("iters", [1, 2, 3, 4, 5, 6])
def test_pipe_short_series_match_oracle(iters):
    """The pipelined x-pass in iterations 2 and 3 (incident-field source,
    the half-series bookkeeping) and in the final pass (Field(ROI) +
    incident field) after odd and even last iterations, for short series on
    a padded (88, 48, 40) grid."""
    size = [64, 24, 16]
    p = cases.params(size, [6, 6, 6], return_reflection=True, return_3D=True, iterations_number=iters)
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=77, n_spheres=2, radius_um=(0.3, 0.8))
    fields = cases.circle_fields(p, 2)
    (t, r, f), (sim, bm) = _solve(p, RI, fields)
    assert bm == iters
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    ot, orr, of = o.solve(fields)
    assert worst(f, of) < 1e-5 and worst(t, ot) < 1e-5 and worst(r, orr) < 3e-5
