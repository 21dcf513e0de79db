"""The bounded waits of the pipelined Born kernels (csrc/born_pipe.cu,
csrc/cols_pipe.cu) report a timeout instead of hanging, and the library
stays usable afterwards.

ODT_WAIT_LIMIT_CYCLES=0 at odt_create gives the kernels' steady mbarrier
waits a zero-cycle budget, so a wait whose bulk copy has not landed on the
first poll gives up: the CTA records the timeout, drains its copies in flight
with the default (long) limit and returns.  The solve must fail with
ODT_ERR_INTERNAL and the timeout message.  A handle created afterwards with
the default limit must solve the same case correctly (against the
single-precision oracle, relative L2 1e-5).  No GPU fault or hang is
involved: every wait ends and every copy lands before its CTA exits.

Grid: 64^3 RI with the default boundary -> 88^3 padded (pipelined plans for
88 on every axis), 2 illuminations.
"""
import os

import numpy as np
import pytest

import cases
from oracle import cbs

pytestmark = pytest.mark.gpu


def _case():
    p = cases.params([64, 64, 64], [6, 6, 6], return_3D=True)
    RI = cases.sphere_phantom([64, 64, 64], [0.1] * 3, cases.NM, seed=11, n_spheres=3, radius_um=(0.5, 1.2))
    return p, RI, cases.circle_fields(p, 2)


def test_zero_wait_limit_reports_timeout_then_fresh_handle_solves(monkeypatch):
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN
    from inverse_solver_b200._lib import OdtError

    p, RI, fields = _case()
    monkeypatch.setenv("ODT_WAIT_LIMIT_CYCLES", "0")
    monkeypatch.setenv("ODT_GRAPHS", "0")
    s = FORWARD_SOLVER_CONVERGENT_BORN(p)
    try:
        assert s.sim_size == [88, 88, 88]
        s.set_RI(RI)
        with pytest.raises(OdtError) as ei:
            s.solve(fields)
        assert ei.value.status == 8, ei.value.args     # ODT_ERR_INTERNAL
        assert "timed out" in str(ei.value)
    finally:
        s.delete()

    monkeypatch.delenv("ODT_WAIT_LIMIT_CYCLES")
    s = FORWARD_SOLVER_CONVERGENT_BORN(p)
    try:
        s.set_RI(RI)
        t, _, f3 = s.solve(fields)
    finally:
        s.delete()
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    ot, _, of3 = o.solve(fields)
    for k in range(2):
        assert cbs.rel_l2(f3[..., k], of3[..., k]) < 1e-5
        assert cbs.rel_l2(t[..., k], ot[..., k]) < 1e-5


def test_wait_limit_must_be_a_non_negative_integer(monkeypatch):
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN
    from inverse_solver_b200._lib import OdtError

    p = cases.small_params()
    monkeypatch.setenv("ODT_WAIT_LIMIT_CYCLES", "-5")
    with pytest.raises(OdtError) as ei:
        FORWARD_SOLVER_CONVERGENT_BORN(p)
    assert ei.value.status == 1 and "ODT_WAIT_LIMIT_CYCLES" in str(ei.value)
