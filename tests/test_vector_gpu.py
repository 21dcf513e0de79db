"""GPU parity of the dyadic (vector) solver (vector_simulation,
pole_num = 3: polarisation change of basis on the GPU, three field
components per illumination, dyadic Green's function in the z-pass)
against the oracle's single-precision restatement.  Tolerances as for the
scalar solver: relative L2 1e-5 (transmitted, 3D), 3e-5 (reflected); the
single-precision result against the double-precision oracle is stated."""
import numpy as np
import pytest

import cases
from oracle import cbs

pytestmark = pytest.mark.gpu

SIZE = [28, 28, 20]


def vparams(**kw):
    p = cases.params(SIZE, [2, 2, 1.5], **kw)
    p["vector_simulation"] = True
    return p


def _inputs(n):
    f = cases.circle_fields(cases.params(SIZE, [2, 2, 1.5]), n)
    fv = np.zeros((SIZE[0], SIZE[1], 2, n), np.complex64)
    for k in range(n):
        a = k / max(1, n - 1) * np.pi / 2
        fv[:, :, 0, k] = f[:, :, 0, k] * np.float32(np.cos(a))
        fv[:, :, 1, k] = f[:, :, 0, k] * np.float32(np.sin(a))
    return fv


def worst(a, b):
    return max(cbs.rel_l2(a[..., k], b[..., k]) for k in range(a.shape[-1]))


@pytest.mark.parametrize("acyclic", [True, False])
def test_vector_solve_matches_oracle(acyclic):
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN

    p = vparams(return_reflection=True, return_3D=True, acyclic=acyclic)
    RI = cases.sphere_phantom(SIZE, [0.1] * 3, cases.NM, seed=5, n_spheres=2, radius_um=(0.4, 0.8))
    fv = _inputs(3)
    s = FORWARD_SOLVER_CONVERGENT_BORN(p)
    s.set_RI(RI)
    t, r, f3 = s.solve(fv)
    s.delete()
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    ot, orr, of = o.solve(fv)
    assert t.shape == ot.shape == (28, 28, 2, 3) and f3.shape == of.shape == (28, 28, 20, 3, 3)
    assert worst(f3, of) < 1e-5
    assert worst(t, ot) < 1e-5
    assert worst(r, orr) < 3e-5
    o64 = cbs.ForwardSolverCBS(p, single=False)
    o64.set_RI(RI)
    t64, _, f64 = o64.solve(fv)
    e64 = worst(t, t64)
    print("vector GPU vs FP64 oracle: trans %.2e, 3D %.2e" % (e64, worst(f3, f64)))
    assert e64 < 2e-4


def test_vector_batches_are_independent():
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN

    RI = cases.sphere_phantom(SIZE, [0.1] * 3, cases.NM, seed=6, n_spheres=2, radius_um=(0.4, 0.8))
    fv = _inputs(4)
    outs = []
    for mb in (1, 4):
        s = FORWARD_SOLVER_CONVERGENT_BORN(vparams(return_3D=True, max_batch=mb))
        s.set_RI(RI)
        outs.append(s.solve(fv))
        s.delete()
    for a, b in zip(outs[0], outs[1]):
        if a is not None:
            assert np.array_equal(a, b)


def test_dyadic_handle_needs_polarisation_basis():
    import ctypes as C

    from inverse_solver_b200 import _lib

    lib = _lib.load()
    g = _lib.Geometry()
    g.sim_size[:] = [32, 32, 24]
    g.ri_size[:] = [28, 28, 20]
    g.field_size[:] = [28, 28]
    g.conv_size[:] = [56, 56]
    g.pol = 3
    z = np.zeros((56, 56, 20), np.complex64, order="F")
    pu = np.ones((28, 28), np.float32, order="F")
    h = C.c_uint32(0)
    _lib.check(lib.odt_create(C.byref(g), z.ctypes.data, z.ctypes.data, None, pu.ctypes.data,
                              pu.ctypes.data, C.byref(h)))
    try:
        a = _lib.SolveArgs()
        a.fields_in = z.ctypes.data
        a.n_ill = 1
        a.trans = z.ctypes.data
        assert lib.odt_solve(h.value, C.byref(a)) == 5   # not ready
        g.pol = 2
        assert lib.odt_create(C.byref(g), z.ctypes.data, z.ctypes.data, None, pu.ctypes.data,
                              pu.ctypes.data, C.byref(C.c_uint32(0))) == 1
    finally:
        lib.odt_destroy(h.value)


def test_vector_on_pipelined_grid_matches_oracle():
    """Dyadic solve on a padded (88, 88, 40) grid: the x- and y-passes of the
    three components run through the pipelined kernels, the z-pass through
    the dyadic one."""
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN

    size = [64, 64, 16]
    p = cases.params(size, [6, 6, 6], return_3D=True)
    p["vector_simulation"] = True
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=12, n_spheres=2, radius_um=(0.3, 0.8))
    f = cases.circle_fields(cases.params(size, [6, 6, 6]), 2)
    fv = np.zeros((64, 64, 2, 2), np.complex64)
    fv[:, :, 0, 0] = f[:, :, 0, 0]
    fv[:, :, 1, 1] = f[:, :, 0, 1]
    s = FORWARD_SOLVER_CONVERGENT_BORN(p)
    s.set_RI(RI)
    assert s.sim_size == [88, 88, 40]
    t, _, f3 = s.solve(fv)
    s.delete()
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    ot, _, of = o.solve(fv)
    assert worst(f3, of) < 1e-5 and worst(t, ot) < 1e-5
