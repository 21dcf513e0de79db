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


def _gradient_case():
    p = vparams(return_transmission=True, return_reflection=True, return_3D=True)
    RI = cases.sphere_phantom(SIZE, [0.1] * 3, cases.NM, seed=8, n_spheres=2, radius_um=(0.4, 0.8))
    fv = _inputs(3)
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    meas, _, _ = o.solve(fv)
    return p, RI, fv, meas


def test_vector_gradient_matches_oracle():
    """Fused dyadic gradient (odt_gradient on a pol = 3 handle) against the
    oracle's get_gradiant_static on the vector solver: relative L2 1e-5 on
    the gradient, relative 1e-5 on the misfit; host and device entry points
    give the same gradient bits."""
    import torch

    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN
    from oracle import multi

    p, RI, fv, meas = _gradient_case()
    RI0 = (RI * 0.7 + cases.NM * 0.3).astype(np.float32)
    s = FORWARD_SOLVER_CONVERGENT_BORN(p)
    s.set_RI(RI0)
    s.set_RI_adjoint(RI0)
    g, err = s.gradient(fv, meas)
    dev = torch.device("cuda", 0)

    def up(a):
        return torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.complex64).ravel(order="F"))).to(dev)

    gd = torch.empty(int(np.prod(SIZE)), dtype=torch.complex64, device=dev)
    errd = s.gradient_device(up(fv), up(meas), gd)
    gd = gd.cpu().numpy().reshape(SIZE, order="F")
    s.delete()
    o = cbs.ForwardSolverCBS(p, single=True)
    go, erro = multi.get_gradient_static(RI0, fv, meas, o)
    assert g.shape == go.shape == tuple(SIZE)
    assert cbs.rel_l2(g, go) < 1e-5
    assert abs(err - erro) / erro < 1e-5
    # the misfit is a double-precision atomic sum: equal up to its order
    assert np.array_equal(g, gd) and abs(err - errd) <= 1e-12 * err


def test_vector_fista_outer_iteration_matches_oracle():
    """One FISTA outer iteration of BACKWARD_SOLVER_MULTI.solve on the dyadic
    solver through the device-resident loop, against the oracle's
    solve_multi: relative L2 1e-5 on RI - RI_bg (odd z, as the reference
    requires)."""
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN
    from inverse_solver_b200.backward import BACKWARD_SOLVER_MULTI
    from oracle import multi

    size = [28, 28, 19]
    p = cases.params(size, [2, 2, 1.5], return_transmission=True, return_reflection=True, return_3D=True)
    p["vector_simulation"] = True
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=9, n_spheres=2, radius_um=(0.4, 0.8))
    f = cases.circle_fields(cases.params(size, [2, 2, 1.5]), 2)
    fv = np.zeros((size[0], size[1], 2, 2), np.complex64)
    fv[:, :, 0, 0] = f[:, :, 0, 0]
    fv[:, :, 1, 1] = f[:, :, 0, 1]
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    meas, _, _ = o.solve(fv)

    class Blurred:
        def solve(self, input_field, output_field):
            return (RI * 0.5 + cases.NM * 0.5).astype(np.float32)

    bp = BACKWARD_SOLVER_MULTI.get_default_parameters(dict(
        RI_bg=cases.NM, wavelength=cases.LAM, NA=p["NA"], resolution=p["resolution"],
        size=p["size"], forward_solver=FORWARD_SOLVER_CONVERGENT_BORN,
        forward_solver_parameters=p, init_solver=Blurred(), step=0.01, tv_param=0.001,
        inner_itt=10, itter_max=1, use_non_negativity=True, nmin=cases.NM, nmax=1.5))
    b = BACKWARD_SOLVER_MULTI(bp)
    assert b._use_device_loop()
    got = b.solve(fv, meas)
    ref, errs = multi.solve_multi(bp, Blurred().solve(None, None), fv, meas, o)
    assert cbs.rel_l2(got - cases.NM, ref - cases.NM) < 1e-5
    assert np.allclose(b.err_list, errs, rtol=1e-5)
    b.delete()


def _tensor(RI):
    """Birefringent, coupled RI tensor [x, y, z, 3, 3]: the scalar RI scaled
    per axis on the diagonal, a symmetric xy term, zero potential elsewhere."""
    T = np.empty(RI.shape + (3, 3), np.float32)
    T[...] = np.float32(cases.NM)
    for i in range(3):
        T[:, :, :, i, i] = cases.NM + (RI - cases.NM) * (1 - 0.25 * i)
    T[:, :, :, 0, 1] = T[:, :, :, 1, 0] = cases.NM + (RI - cases.NM) * 0.2
    return T


@pytest.mark.parametrize("acyclic", [True, False])
def test_tensor_RI_solve_matches_oracle(acyclic):
    """RI tensor (size(RI,4) > 1) through odt_set_tensor_potential: the
    component-coupling x-step and emitter against the oracle's tensor
    branches; tolerances as for the isotropic dyadic solve."""
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN

    p = vparams(return_reflection=True, return_3D=True, acyclic=acyclic)
    RI = cases.sphere_phantom(SIZE, [0.1] * 3, cases.NM, seed=5, n_spheres=2, radius_um=(0.4, 0.8))
    T = _tensor(RI)
    fv = _inputs(3)
    s = FORWARD_SOLVER_CONVERGENT_BORN(p)
    s.set_RI({"scatt_pott": T})
    t, r, f3 = s.solve(fv)
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(T)
    assert s.Bornmax == o.Bornmax and float(s.eps_imag) == float(o.eps_imag)
    ot, orr, of = o.solve(fv)
    assert worst(f3, of) < 1e-5
    assert worst(t, ot) < 1e-5
    assert worst(r, orr) < 3e-5
    # the scalar potential of the same handle afterwards: the isotropic solve
    s.set_RI(RI)
    t2, _, _ = s.solve(fv)
    s.delete()
    o2 = cbs.ForwardSolverCBS(p, single=True)
    o2.set_RI(RI)
    ot2, _, _ = o2.solve(fv)
    assert worst(t2, ot2) < 1e-5
    o64 = cbs.ForwardSolverCBS(p, single=False)
    o64.set_RI(T)
    t64, _, _ = o64.solve(fv)
    print("tensor GPU vs FP64 oracle: trans %.2e" % worst(t, t64))


def test_tensor_RI_on_pipelined_grid_matches_oracle():
    """Tensor solve on a padded (88, 88, 40) grid: plain x-FFTs around the
    coupling step, pipelined y-passes, dyadic z-pass; graph replays give the
    eager result's bits; odt_gradient refuses a tensor potential."""
    import ctypes as C

    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN, _lib

    size = [64, 64, 16]
    p = cases.params(size, [6, 6, 6], return_3D=True)
    p["vector_simulation"] = True
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=12, n_spheres=2, radius_um=(0.3, 0.8))
    T = _tensor(RI)
    f = cases.circle_fields(cases.params(size, [6, 6, 6]), 2)
    fv = np.zeros((64, 64, 2, 2), np.complex64)
    fv[:, :, 0, 0] = f[:, :, 0, 0]
    fv[:, :, 1, 1] = f[:, :, 0, 1]
    s = FORWARD_SOLVER_CONVERGENT_BORN(p)
    s.set_RI(T)
    assert s.sim_size == [88, 88, 40]
    t, _, f3 = s.solve(fv)
    # second and third solves: captured into a CUDA graph, then replayed
    for _ in range(2):
        t2, _, f32 = s.solve(fv)
        assert np.array_equal(t2, t) and np.array_equal(f32, f3)
    a = _lib.GradientArgs()
    g = np.zeros(size, np.complex64, order="F")
    err = C.c_double(0)
    a.fields_in, a.fields_meas = _lib.ptr(np.asfortranarray(fv)), _lib.ptr(np.asfortranarray(fv))
    a.n_ill = 2
    a.grad = _lib.ptr(g)
    a.err = C.addressof(err)
    a.memory = _lib.ODT_MEM_HOST
    s.set_RI_adjoint(RI)
    assert _lib.load().odt_gradient(s._handle, C.byref(a)) != 0
    s.delete()
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(T)
    ot, _, of = o.solve(fv)
    assert worst(f3, of) < 1e-5 and worst(t, ot) < 1e-5
