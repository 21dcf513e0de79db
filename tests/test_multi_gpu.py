"""GPU parity of the inverse-solver pieces (BACKWARD_SOLVER_MULTI.m) against
the oracle's single-precision restatement:
  * TV prox (odt_tv_prox vs TV_FISTA_inner_v2): rel-L2 <= 1e-5
  * fused gradient (odt_gradient vs get_gradiant_static): rel-L2 <= 1e-5 on
    the gradient, relative 1e-5 on the misfit
  * two FISTA outer iterations of BACKWARD_SOLVER_MULTI.solve: rel-L2 <= 1e-5
    on the RI update RI - RI_bg
"""
import numpy as np
import pytest

import cases
from oracle import cbs, multi

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cplx", [False, True])
def test_tv_prox_matches_oracle(cplx):
    from inverse_solver_b200.backward import TV_FISTA_inner_v2

    rng = np.random.default_rng(3)
    x = rng.standard_normal((20, 18, 13)).astype(np.float32) * 0.05
    vim = 0.0
    if cplx:
        x = (x + 1j * 0.03 * rng.standard_normal(x.shape)).astype(np.complex64)
        vim = 0.02
    args = (0.01, -0.04, 0.06, vim, True, False, 50)
    got = TV_FISTA_inner_v2(x, *args)
    ref = multi.tv_fista_inner_v2(x, *args, cbs.Prec(True))
    assert got.dtype == ref.dtype
    assert cbs.rel_l2(got, ref) < 1e-5


def _multi_case(n_ill=3):
    p = cases.small_params(return_transmission=True, return_reflection=True, return_3D=True)
    RI = cases.small_RI()
    fields = cases.circle_fields(p, n_ill)
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    meas, _, _ = o.solve(fields)
    return p, RI, fields, meas


def test_fused_gradient_matches_oracle():
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN

    p, RI, fields, meas = _multi_case()
    # gradient at a perturbed RI so that the misfit is not zero
    RI0 = (RI * 0.7 + cases.NM * 0.3).astype(np.float32)
    s = FORWARD_SOLVER_CONVERGENT_BORN(p)
    s.set_RI(RI0)
    s.set_RI_adjoint(RI0)
    g, err = s.gradient(fields, meas)
    o = cbs.ForwardSolverCBS(p, single=True)
    go, erro = multi.get_gradient_static(RI0, fields, meas, o)
    assert cbs.rel_l2(g, go) < 1e-5
    assert abs(err - erro) / erro < 1e-5
    s.delete()


def test_fista_two_outer_iterations_match_oracle():
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN
    from inverse_solver_b200.backward import BACKWARD_SOLVER_MULTI

    p, RI, fields, meas = _multi_case()

    class Blurred:
        """Initial guess: the phantom pulled 50% towards the background (a
        constant RI_bg guess has zero potential, hence eps_imag = 0, which
        the reference divides by as well)."""

        def solve(self, input_field, output_field):
            return (RI * 0.5 + cases.NM * 0.5).astype(np.float32)

    bp = BACKWARD_SOLVER_MULTI.get_default_parameters(dict(
        RI_bg=cases.NM, wavelength=cases.LAM, NA=p["NA"], resolution=p["resolution"],
        size=p["size"], forward_solver=FORWARD_SOLVER_CONVERGENT_BORN,
        forward_solver_parameters=p, init_solver=Blurred(), step=0.01, tv_param=0.001,
        inner_itt=20, itter_max=2, use_non_negativity=True, nmin=cases.NM, nmax=1.5))
    b = BACKWARD_SOLVER_MULTI(bp)
    got = b.solve(fields, meas)
    o = cbs.ForwardSolverCBS(p, single=True)
    ref, errs = multi.solve_multi(bp, Blurred().solve(None, None), fields, meas, o)
    assert cbs.rel_l2(got - cases.NM, ref - cases.NM) < 1e-5
    assert np.allclose(b.err_list, errs, rtol=1e-5)
    assert b.err_list[1] < b.err_list[0]
    b.delete()
