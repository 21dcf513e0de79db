"""The reduced-precision storage mode of the Born loop (odt_set_field_storage
with ODT_STORAGE_B16: the spectral array T and Field_n stored as 16-bit
block floating point -- 8 values per shared exponent, 15-bit mantissas --
while every operation computes in FP32 and Field, V and the inputs and
outputs stay complex64).

relative L2 <= 1e-4 against the FP64 oracle.
  * config 1 (64^3 bead -> 96^3 padded, 28 iterations, normal incidence):
    3D and transmitted fields against the FP64 oracle;
  * the benchmark grid (128^3 seeded phantom -> 152^3, Bornmax 40): the 3D
    field of the normal-incidence and an NA-0.9 illumination against the FP64
    oracle (the Born loop's own result; the CPU experiment that chose the
    format measured 4.7e-5 / 5.7e-5 there), and the transmitted fields of the
    four fixture illuminations against tests/golden/bench_fp64.npz within the
    bound the FP32 path meets (2e-4: the single-precision Green's function
    set-up dominates the transmitted field's error, up to 1.1e-4 for the
    FP32 reference itself) and within 1e-4 of the FP32 path;
  * on every other plane radix of the fused xy-pass (104, 112, 128, 136, 144
    and 160-point cubes, with the pipelined z-pass on the same radix) the 3D
    field is within 1e-4 of the FP32 path, which is checked against the
    oracle on those radices in test_xy_gpu.py;
  * graph replays of a b16 solve give the same bits as its eager run;
  * a grid the mode does not cover fails with ODT_ERR_UNSUPPORTED."""
import os

import numpy as np
import pytest

import cases
from oracle import cbs

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _solve(p, RI, fields, storage):
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN

    s = FORWARD_SOLVER_CONVERGENT_BORN(dict(p, field_storage=storage))
    try:
        s.set_RI(RI)
        return s.solve(fields), (list(s.sim_size), s.Bornmax)
    finally:
        s.delete()


def test_b16_config1_within_1e4_of_fp64():
    p = cases.cfg1_params(return_3D=True)
    RI = cases.cfg1_RI()
    f = cases.normal_field([64, 64, 64], 1)
    (t, _, f3), (sim, bm) = _solve(p, RI, f, "b16")
    assert sim == [96, 96, 96] and bm == 28
    o = cbs.ForwardSolverCBS(p, single=False)
    o.set_RI(RI)
    ot, _, of = o.solve(f)
    e3, et = cbs.rel_l2(f3, of), cbs.rel_l2(t, ot)
    print("config 1, b16 vs FP64: field3d %.2e trans %.2e" % (e3, et))
    assert e3 < 1e-4 and et < 1e-4


def test_b16_bench_grid_within_1e4_of_fp64():
    import bench

    p = dict(bench.workload_params(), return_3D=True)
    RI, fields = bench.workload_inputs(p)
    sel = [0, 5, 13, 37]
    f4 = np.ascontiguousarray(fields[:, :, :, sel])
    (t16, _, f16), (sim, bm) = _solve(p, RI, f4, "b16")
    (t32, _, _), _ = _solve(p, RI, f4, "complex64")
    assert sim == [152, 152, 152] and bm == 40
    g = np.load(os.path.join(ROOT, "tests", "golden", "bench_fp64.npz"))
    assert list(g["sel"]) == sel
    o = cbs.ForwardSolverCBS(p, single=False)
    o.set_RI(RI)
    _, _, of = o.solve(np.ascontiguousarray(fields[:, :, :, [0, 37]]))
    errs = []
    for j, k in enumerate([0, 3]):   # illuminations 0 and 37
        e3 = cbs.rel_l2(f16[..., k], of[..., j])
        errs.append(e3)
        assert e3 < 1e-4, (sel[k], e3)
    for k in range(4):
        et = cbs.rel_l2(t16[..., k], g["trans64"][..., k])
        assert et < 2e-4, (sel[k], et)
        assert cbs.rel_l2(t16[..., k], t32[..., k]) < 1e-4
    print("bench grid, b16 field3d vs FP64 (illuminations 0, 37):", errs)


@pytest.mark.parametrize("n", [80, 88, 104, 112, 120, 136])
def test_b16_other_radices_within_1e4_of_fp32(n):
    size = [n, n, n]
    p = cases.params(size, [6, 6, 6], return_3D=True)
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=n, n_spheres=3, radius_um=(0.4, 0.9))
    fields = cases.circle_fields(p, 2)
    (t16, _, f16), (sim, _) = _solve(p, RI, fields, "b16")
    (t32, _, f32), _ = _solve(p, RI, fields, "complex64")
    assert sim == [n + 24] * 3
    e3, et = cbs.rel_l2(f16, f32), cbs.rel_l2(t16, t32)
    print("%d^3 padded, b16 vs FP32: field3d %.2e trans %.2e" % (n + 24, e3, et))
    assert e3 < 1e-4 and et < 1e-4


def test_b16_graph_replays_equal_eager():
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN

    size = [64, 64, 64]
    p = cases.params(size, [6, 6, 6], return_3D=True, field_storage="b16")
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=5, n_spheres=3, radius_um=(0.4, 0.9))
    fields = cases.circle_fields(p, 2)
    s = FORWARD_SOLVER_CONVERGENT_BORN(p)
    try:
        s.set_RI(RI)
        outs = [s.solve(fields) for _ in range(3)]   # eager, captured, replayed
    finally:
        s.delete()
    for o in outs[1:]:
        assert np.array_equal(o[0], outs[0][0]) and np.array_equal(o[2], outs[0][2])
    (t32, _, f32), _ = _solve(dict(p, field_storage="complex64"), RI, fields, "complex64")
    assert cbs.rel_l2(outs[0][2], f32) < 1e-4


def test_b16_unsupported_grid_is_rejected():
    from inverse_solver_b200._lib import OdtError

    p = cases.small_params(return_3D=True)
    with pytest.raises(OdtError) as ei:
        _solve(p, cases.small_RI(), cases.circle_fields(p, 1), "b16")
    assert ei.value.status == 6 and "B16" in str(ei.value)
