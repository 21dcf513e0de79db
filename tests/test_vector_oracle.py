"""Dyadic (vector) branch without a GPU: the polarisation basis of
polarisation_utility (FORWARD_SOLVER.m:131-180) and its 2 <-> 3 component
round trip, the library's host tables against the oracle's, and the oracle's
vector solve (single against double precision; weak-scatterer limit against
the scalar solve)."""
import numpy as np

import cases
from inverse_solver_b200.forward import CBSHostSetup
from inverse_solver_b200.optics import polarisation_basis
from oracle import cbs

SIZE = [28, 28, 20]


def vparams(**kw):
    p = cases.params(SIZE, [2, 2, 1.5], **kw)
    p["vector_simulation"] = True
    return p


def test_basis_is_orthonormal_and_tangent():
    p = vparams()
    R2, P2, E, K = cbs.polarisation_utility(SIZE[:2], p, cbs.Prec(True))
    assert np.allclose(np.sum(R2 * R2, 2), 1, atol=1e-6)
    assert np.allclose(np.sum(P2 * P2, 2), 1, atol=1e-6)
    assert np.allclose(np.sum(R2 * P2, 2), 0, atol=1e-6)
    assert K.sum() > 0 and not K.all()
    e = E[K]
    assert np.allclose(np.sum(e * e, 1), 1, atol=1e-5)
    # the tangent is orthogonal to the perpendicular vector (P2 has no z part)
    assert np.allclose(np.sum(E[:, :, :2] * P2, 2)[K], 0, atol=1e-5)


def test_polarisation_round_trip_is_identity_on_propagating_pixels():
    """transform_field_2D(transform_field_3D(f)) without the pupil factors:
    the 2 -> 3 -> 2 basis change returns f wherever K_mask holds."""
    p = vparams(use_abbe_sine=False)
    p["NA"] = 1.3
    o = cbs.ForwardSolverCBS(p, single=False)
    rng = np.random.default_rng(0)
    f = rng.standard_normal((28, 28, 2, 3)) + 1j * rng.standard_normal((28, 28, 2, 3))
    NA = o.utility["NA_circle"]
    _, _, _, K = cbs.polarisation_utility(SIZE[:2], p, cbs.Prec(False))
    g = o.transform_field_2D(o.transform_field_3D(f))
    m = (NA & K)[:, :, None, None]
    assert np.allclose(g * m, f * m, atol=1e-12)


def test_library_basis_equals_oracle_bitwise():
    p = vparams()
    ref = cbs.polarisation_utility(SIZE[:2], p, cbs.Prec(True))
    got = polarisation_basis(SIZE[:2], p)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)


def test_library_dyadic_tables_equal_oracle():
    p = vparams()
    RI = cases.sphere_phantom(SIZE, [0.1] * 3, cases.NM, seed=5, n_spheres=2, radius_um=(0.4, 0.8))
    h = CBSHostSetup(p)
    h.prepare_potential(RI)
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    for a, b in zip(h.rads1d, o.rads1d):
        assert np.array_equal(a, np.fft.ifftshift(b))
    assert h.green_absorbtion_correction == o.green_absorbtion_correction
    r = o.rads
    assert np.array_equal(r[:, 0, 0, 0], h.rads1d[0])
    assert np.array_equal(r[0, :, 0, 1], h.rads1d[1])
    assert np.array_equal(r[0, 0, :, 2], h.rads1d[2])


def _vector_inputs(n=2):
    f = cases.circle_fields(cases.params(SIZE, [2, 2, 1.5]), n)
    fv = np.zeros((SIZE[0], SIZE[1], 2, n), np.complex64)
    fv[:, :, 0, 0] = f[:, :, 0, 0]                     # x-polarised
    fv[:, :, 0, 1] = f[:, :, 0, 1] * np.float32(0.6)   # mixed polarisation
    fv[:, :, 1, 1] = f[:, :, 0, 1] * np.float32(0.8)
    return fv


def test_vector_oracle_single_vs_double_and_scalar_limit():
    p = vparams(return_reflection=True, return_3D=True)
    RI = cases.sphere_phantom(SIZE, [0.1] * 3, cases.NM, seed=5, n_spheres=2, radius_um=(0.4, 0.8))
    fv = _vector_inputs()
    o32 = cbs.ForwardSolverCBS(p, single=True)
    o32.set_RI(RI)
    t, r, f3 = o32.solve(fv)
    o64 = cbs.ForwardSolverCBS(p, single=False)
    o64.set_RI(RI)
    t64, r64, f364 = o64.solve(fv)
    assert t.shape == (28, 28, 2, 2) and f3.shape == (28, 28, 20, 3, 2)
    assert cbs.rel_l2(t, t64) < 1e-5 and cbs.rel_l2(f3, f364) < 1e-5 and cbs.rel_l2(r, r64) < 1e-4
    # x-polarised input: the x component follows the scalar solve to within the
    # (small) vector coupling of this weak phantom; little cross-polarisation
    ps = cases.params(SIZE, [2, 2, 1.5], return_3D=True)
    os_ = cbs.ForwardSolverCBS(ps, single=True)
    os_.set_RI(RI)
    ts, _, _ = os_.solve(fv[:, :, 0:1, 0:1])
    assert cbs.rel_l2(t[:, :, 0, 0], ts[:, :, 0, 0]) < 0.05
    assert np.linalg.norm(t[:, :, 1, 0]) < 0.05 * np.linalg.norm(t[:, :, 0, 0])


def _vector_gradient_case():
    from oracle import multi

    p = vparams(return_transmission=True, return_reflection=True, return_3D=True)
    RI = cases.sphere_phantom(SIZE, [0.1] * 3, cases.NM, seed=8, n_spheres=1, radius_um=(0.5, 0.7))
    f = cases.circle_fields(cases.params(SIZE, [2, 2, 1.5]), 2)
    fv = np.zeros((SIZE[0], SIZE[1], 2, 2), np.complex64)
    fv[:, :, 0, 0] = f[:, :, 0, 0]
    fv[:, :, 1, 1] = f[:, :, 0, 1]
    return multi, p, RI, fv


def test_vector_gradient_of_a_zero_misfit_is_zero():
    """get_gradiant_static (BACKWARD_SOLVER_MULTI.m:30-54) on the dyadic
    solver: measured fields equal to the model's give err = 0 and a zero
    adjoint source, hence a zero gradient over all three components."""
    multi, p, RI, fv = _vector_gradient_case()
    o = cbs.ForwardSolverCBS(p, single=False)
    o.set_RI(RI)
    meas, _, src3d = o.solve(fv)
    assert src3d.shape == (SIZE[0], SIZE[1], SIZE[2], 3, 2)
    g, err = multi.get_gradient_static(RI, fv, meas, o)
    assert g.shape == tuple(SIZE) and err == 0.0
    assert np.abs(g).max() == 0.0


def test_vector_gradient_is_the_mean_over_components_and_illuminations():
    """The gradient of two illuminations is the mean of the two one-
    illumination gradients (the reference's mean over [pole_num, n_ill]),
    and the misfits add."""
    multi, p, RI, fv = _vector_gradient_case()
    o = cbs.ForwardSolverCBS(p, single=False)
    o.set_RI(RI)
    meas, _, _ = o.solve(fv)
    RI0 = (RI * 0.6 + cases.NM * 0.4).astype(np.float32)
    g, err = multi.get_gradient_static(RI0, fv, meas, o)
    parts = [multi.get_gradient_static(RI0, fv[:, :, :, k:k + 1], meas[:, :, :, k:k + 1], o)
             for k in range(2)]
    assert err > 0 and abs(err - parts[0][1] - parts[1][1]) <= 1e-12 * err
    assert cbs.rel_l2(g, (parts[0][0] + parts[1][0]) / 2) < 1e-12


def _tensor_of(RI, off=None):
    """[x, y, z, 3, 3] RI tensor with RI on the diagonal and `off` (default:
    the background index, i.e. zero potential) off the diagonal."""
    T = np.empty(RI.shape + (3, 3), dtype=np.float64)
    T[...] = cases.NM if off is None else off[..., None, None]
    for i in range(3):
        T[:, :, :, i, i] = RI
    return T


def test_isotropic_tensor_equals_the_isotropic_vector_solve():
    """An RI tensor with the scalar RI on its diagonal and zero potential off
    it (FORWARD_SOLVER_CONVERGENT_BORN.m's size(RI,4) > 1 branches) gives the
    isotropic dyadic solve: same eps_imag and Bornmax, fields equal up to the
    order of the operations."""
    p = vparams(return_reflection=True, return_3D=True)
    RI = cases.sphere_phantom(SIZE, [0.1] * 3, cases.NM, seed=5, n_spheres=2, radius_um=(0.4, 0.8))
    fv = np.zeros((SIZE[0], SIZE[1], 2, 1), np.complex64)
    fv[:, :, 0, 0] = cases.circle_fields(cases.params(SIZE, [2, 2, 1.5]), 1)[:, :, 0, 0]
    for single, tol in ((False, 1e-12), (True, 1e-5)):
        a = cbs.ForwardSolverCBS(p, single=single)
        a.set_RI(RI)
        b = cbs.ForwardSolverCBS(p, single=single)
        b.set_RI({"scatt_pott": _tensor_of(RI)})
        assert b.tensor and a.eps_imag == b.eps_imag and a.Bornmax == b.Bornmax
        ra, rb = a.solve(fv), b.solve(fv)
        for x, y in zip(ra, rb):
            assert cbs.rel_l2(y, x) < tol


def test_anisotropic_tensor_couples_the_components():
    """A birefringent sphere (a lower RI along x) changes the transmitted
    field of an x-polarised input against the isotropic one, and an off-diagonal term
    moves light from an x-polarised input into the y polarisation."""
    p = vparams(return_3D=True)
    RI = cases.sphere_phantom(SIZE, [0.1] * 3, cases.NM, seed=5, n_spheres=1, radius_um=(0.6, 0.8))
    fv = np.zeros((SIZE[0], SIZE[1], 2, 1), np.complex64)
    fv[:, :, 0, 0] = 1
    iso = cbs.ForwardSolverCBS(p, single=False)
    iso.set_RI(_tensor_of(RI))
    ti, _, _ = iso.solve(fv)
    T = _tensor_of(RI)
    T[:, :, :, 0, 0] = cases.NM + (RI - cases.NM) * 0.5
    ani = cbs.ForwardSolverCBS(p, single=False)
    ani.set_RI(T)
    ta, _, _ = ani.solve(fv)
    assert cbs.rel_l2(ta, ti) > 1e-4
    off = np.where(RI > cases.NM, np.float32(cases.NM + 0.01), np.float32(cases.NM)).astype(np.float32)
    T2 = _tensor_of(RI, off=off)
    cpl = cbs.ForwardSolverCBS(p, single=False)
    cpl.set_RI(T2)
    tc, _, _ = cpl.solve(fv)
    assert np.linalg.norm(tc[:, :, 1]) > 10 * np.linalg.norm(ti[:, :, 1]) + 1e-12


def test_tensor_RI_argument_checks():
    import pytest

    p = vparams()
    o = cbs.ForwardSolverCBS(p, single=True)
    RI = np.full(SIZE, cases.NM, np.float32)
    with pytest.raises(ValueError):
        o.set_RI({"scatt_pott": RI})          # struct form needs a tensor
    sp = cases.params(SIZE, [2, 2, 1.5])
    with pytest.raises(ValueError):
        cbs.ForwardSolverCBS(sp, single=True).set_RI(_tensor_of(RI))   # scalar Green's function


def test_oracle_reproduces_the_vector_golden_fixture():
    """tests/golden/vector_small.npz (make_vector_golden.py): isotropic and
    RI-tensor dyadic solves and the vector gradient.  The oracle still gives
    them (regression pin of the oracle), and single against double precision
    stays within 1e-4 (the single-precision error the parity bar allows)."""
    import os
    import sys

    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    sys.path.insert(0, here)
    import make_vector_golden as mvg

    g = np.load(os.path.join(here, "vector_small.npz"))
    for single, sfx, tol in ((True, "32", 1e-6), (False, "64", 1e-12)):
        out = mvg.compute(single)
        for k in ("iso_trans", "iso_ref", "ten_trans", "ten_ref", "grad"):
            assert cbs.rel_l2(out[k], g[k + sfx]) < tol, (k, sfx)
        assert abs(float(out["err"]) - float(g["err" + sfx])) <= tol * float(g["err" + sfx])
    for k in ("iso_trans", "ten_trans", "grad"):
        assert cbs.rel_l2(g[k + "32"], g[k + "64"]) < 1e-4, k
