"""GPU parity of the fused xy-pass (csrc/born_xy.cu: the whole x-y plane of
one z and illumination in shared memory -- inverse y- and x-FFT, update,
source, forward x- and y-FFT -- with the spectrum in its permuted order for
the z-pass), which the library selects for scalar solves on square x-y grids
of 8 R points, 11 <= R <= 20 (with the pipelined z-pass where the z length
allows it, else the generic one).

  * against the single-precision oracle on grids covering every R of the
    xy-pass and every z length of the pipelined z-pass (see
    test_fused_xy_matches_oracle), for short series of 1-6 iterations (the first,
    early and final kinds) and without the phase ramp (acyclic = false):
    relative L2 per illumination 1e-5 (transmitted, 3D), 3e-5 (reflected);
  * against the separate pipelined passes (ODT_XY=0) on the benchmark's
    152^3 grid: relative L2 <= 5e-6 (the same arithmetic except the order of
    the x and y transforms' radix passes);
  * the per-kernel timing shows the fused kinds and no separate x- or
    y-passes."""
import os

import numpy as np
import pytest

import cases
from oracle import cbs

pytestmark = pytest.mark.gpu


def worst(a, b):
    return max(cbs.rel_l2(a[..., k], b[..., k]) for k in range(a.shape[-1]))


def _solve(p, RI, fields, xy=True, profile=False):
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN

    old = os.environ.get("ODT_XY")
    os.environ["ODT_XY"] = "1" if xy else "0"
    try:
        s = FORWARD_SOLVER_CONVERGENT_BORN(p)
        s.set_RI(RI)
        if profile:
            s.set_profiling(True)
        out = s.solve(fields)
        kt = s.kernel_times() if profile else None
        info = (s.sim_size, s.Bornmax, kt)
        s.delete()
    finally:
        if old is None:
            os.environ.pop("ODT_XY", None)
        else:
            os.environ["ODT_XY"] = old
    return out, info


# z lengths 8 R2 of the pipelined z-pass
Z_PIPE = {8 * r for r in (11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 25, 27)}


@pytest.mark.parametrize("size", [[64, 64, 16], [96, 96, 64], [128, 128, 16], [72, 72, 72], [104, 104, 40],
                                  [104, 104, 104], [80, 80, 80], [88, 88, 16], [112, 112, 16], [120, 120, 16],
                                  [136, 136, 16], [64, 64, 88], [64, 64, 112], [64, 64, 120], [64, 64, 136]])
def test_fused_xy_matches_oracle(size):
    """Padded x-y planes of 88, 96, 104, 112, 120, 128, 136, 144, 152 and
    160 points (R = 11 ... 20; 12, 14, 16, 18, 20 are the composite even
    butterflies with padded plane rows); z lengths with the generic z-pass
    (40, 64) and the pipelined one (88, 96, 104, 112, 120, 128, 136, 144,
    160)."""
    p = cases.params(size, [6, 6, 6], return_reflection=True, return_3D=True)
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=size[0] + 5, n_spheres=3, radius_um=(0.3, 0.8))
    fields = cases.circle_fields(p, 3)
    (t, r, f), (sim, bm, kt) = _solve(p, RI, fields, profile=True)
    assert sim == [v + 24 for v in size] and bm >= 4
    used = {k for k, (ms, n) in kt.items() if n > 0}
    assert {"born_xy", "born_xy_edge"} <= used
    assert ("born_z_pipe" if sim[2] in Z_PIPE else "born_z") in used
    assert not used & {"born_x", "born_y", "born_x_pipe", "born_y_pipe", "born_x_pipe_edge"}
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    ot, orr, of = o.solve(fields)
    assert worst(f, of) < 1e-5
    assert worst(t, ot) < 1e-5
    assert worst(r, orr) < 3e-5


@pytest.mark.parametrize("iters", [1, 2, 3, 4, 5, 6])
def test_fused_xy_short_series_match_oracle(iters):
    """The first kind (iteration 1), the early kind (iterations 2 and 3) and
    the final pass after odd and even last iterations, on (88, 88, 40)."""
    size = [64, 64, 16]
    p = cases.params(size, [6, 6, 6], return_reflection=True, return_3D=True, iterations_number=iters)
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=78, n_spheres=2, radius_um=(0.3, 0.8))
    fields = cases.circle_fields(p, 2)
    (t, r, f), (sim, bm, _) = _solve(p, RI, fields)
    assert bm == iters
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    ot, orr, of = o.solve(fields)
    assert worst(f, of) < 1e-5 and worst(t, ot) < 1e-5 and worst(r, orr) < 3e-5


def test_fused_xy_cyclic_boundary_matches_oracle():
    size = [96, 96, 16]
    p = cases.params(size, [6, 6, 6], return_3D=True, acyclic=False)
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=19, n_spheres=3, radius_um=(0.3, 0.8))
    fields = cases.circle_fields(p, 2)
    (t, _, f), _ = _solve(p, RI, fields)
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    ot, _, of = o.solve(fields)
    assert worst(f, of) < 1e-5 and worst(t, ot) < 1e-5


def test_fused_xy_matches_separate_passes_on_benchmark_grid():
    from inverse_solver_b200.inputs import ring_illumination, sphere_phantom

    size = [128, 128, 128]
    p = cases.params(size, [6, 6, 6], return_3D=True, max_batch=3)
    RI = sphere_phantom(size, [0.1] * 3, cases.NM, seed=0)
    fields = np.ascontiguousarray(ring_illumination(p)[:, :, :, :5])
    (t1, _, f1), (sim, bm, _) = _solve(p, RI, fields, xy=True)
    (t2, _, f2), _ = _solve(p, RI, fields, xy=False)
    assert sim == [152, 152, 152] and bm >= 30
    assert worst(t1, t2) < 5e-6
    assert worst(f1, f2) < 5e-6
