"""Parity on the configurations that are measured, at their full sizes.

* Benchmark workload (bench.py; config 2's forward solve): 128^3 seeded
  multi-sphere phantom (seed 0) -> 152^3 padded grid, Bornmax 40, 49 ring
  illuminations solved in one batch as the benchmark solves them.  Four of
  them -- normal incidence and one plane wave on each of the NA 0.3 / 0.6 /
  0.9 rings -- against the single-precision oracle (transmitted and 3D
  fields, relative L2 <= 1e-5 each; reflected <= 3e-5) and against the FP64
  oracle's transmitted and reflected fields (tests/golden/bench_fp64.npz,
  made by tests/golden/make_bench_golden.py): the single-precision reference
  itself is 2e-5 .. 1.1e-4 from FP64 there (its Green's function setup in
  single precision), so the GPU must be within 2e-4 (transmitted) and 3e-4
  (reflected) of FP64.
* Config 3's gradient (BACKWARD_SOLVER_MULTI.get_gradiant_static,
  BACKWARD_SOLVER_MULTI.m:30-54) at its full grid, 192 x 192 x 129 RI ->
  216 x 216 x 153 padded, on two illuminations (normal and NA 0.6) of the
  ring set, measured fields from a forward solve of the seeded phantom,
  evaluated at a half-contrast estimate: gradient and misfit against the
  single-precision oracle, relative 1e-5.
* Config 2's reconstruction chain at its full size: the 49 transmitted
  fields of the benchmark solve -> wrapped phase -> Goldstein unwrapping
  (odt_unwrap_goldstein; residues, step maps, residue table, nearest lists
  and branches array_equal to the oracle, unwrapped phase bit-equal) ->
  Rytov reconstruction with Ewald scatter (odt_rytov; Count array_equal,
  RI relative L2 <= 1e-5 measured as RI - RI_bg, ORytov <= 1e-5)."""
import os

import numpy as np
import pytest

import cases
from oracle import cbs

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SEL = [0, 5, 13, 37]


@pytest.fixture(scope="module")
def bench_solve():
    """The benchmark's batch-49 solve (transmitted fields) and a batch of the
    four selected illuminations with reflected and 3D fields."""
    import bench
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN

    p = bench.workload_params()
    RI, fields = bench.workload_inputs(p)
    s = FORWARD_SOLVER_CONVERGENT_BORN(p)
    s.set_RI(RI)
    t49, _, _ = s.solve(fields)
    info = dict(sim_size=list(s.sim_size), bornmax=s.Bornmax, batch=s.batch())
    s.delete()
    p3 = dict(p, return_reflection=True, return_3D=True)
    s = FORWARD_SOLVER_CONVERGENT_BORN(p3)
    s.set_RI(RI)
    t4, r4, f4 = s.solve(np.ascontiguousarray(fields[:, :, :, SEL]))
    s.delete()
    return dict(p=p, p3=p3, RI=RI, fields=fields, t49=t49, t4=t4, r4=r4, f4=f4, info=info)


def test_bench_workload_matches_oracle(bench_solve):
    d = bench_solve
    assert d["info"]["sim_size"] == [152, 152, 152] and d["info"]["bornmax"] == 40
    assert d["info"]["batch"] == 49
    o = cbs.ForwardSolverCBS(d["p3"], single=True)
    o.set_RI(d["RI"])
    ot, orr, of = o.solve(np.ascontiguousarray(d["fields"][:, :, :, SEL]))
    for k, ill in enumerate(SEL):
        assert cbs.rel_l2(d["t49"][..., ill], d["t4"][..., k]) < 1e-6, ill     # batch 49 = batch 4
        assert cbs.rel_l2(d["t4"][..., k], ot[..., k]) < 1e-5, ill
        assert cbs.rel_l2(d["f4"][..., k], of[..., k]) < 1e-5, ill
        assert cbs.rel_l2(d["r4"][..., k], orr[..., k]) < 3e-5, ill
    g = np.load(os.path.join(ROOT, "tests", "golden", "bench_fp64.npz"))
    assert list(g["sel"]) == SEL and int(g["bornmax"]) == 40
    errs = []
    for k, ill in enumerate(SEL):
        et = cbs.rel_l2(d["t4"][..., k], g["trans64"][..., k])
        er = cbs.rel_l2(d["r4"][..., k], g["ref64"][..., k])
        errs.append((ill, et, er))
        assert et < 2e-4 and er < 3e-4, (ill, et, er)
    print("bench workload vs FP64 oracle (illumination, trans, ref):", errs)


def test_config2_chain_matches_oracle(bench_solve):
    from inverse_solver_b200.rytov import BACKWARD_SOLVER_RYTOV
    from inverse_solver_b200.unwrap import unwrap_goldstein
    from oracle import goldstein, rytov

    d = bench_solve
    fin, fout = d["fields"], d["t49"]
    wrapped = np.angle(fout[:, :, 0, :].astype(np.complex64) / fin[:, :, 0, :].astype(np.complex64)).astype(np.float32)
    assert wrapped.shape == (128, 128, 49)
    un, it = unwrap_goldstein(wrapped, intermediates=True)
    oun, oit = goldstein.unwrapp2(wrapped, return_intermediates=True)
    assert np.count_nonzero(oit["residue"]) > 0
    for k in ("residue", "step1", "step2"):
        assert np.array_equal(it[k], oit[k]), k
    assert np.array_equal(it["table"], oit["table"])
    assert np.array_equal(it["nearest"], oit["shortest"])
    assert np.array_equal(it["branches"], oit["branches"])
    assert np.array_equal(un, oun)

    rp = BACKWARD_SOLVER_RYTOV.get_default_parameters(dict(
        size=[128, 128, 128], wavelength=0.532, NA=1.2, RI_bg=1.3355, resolution=[0.1] * 3,
        vector_simulation=False))
    s = BACKWARD_SOLVER_RYTOV(rp)
    got = s.solve(fin, fout)                        # unwraps on the GPU itself
    got2 = s.solve(fin, fout, unwrapped_phase=un)
    assert np.array_equal(got, got2)
    ref, O, C = rytov.rytov_solve(rp, fin, fout, oun)
    assert C.max() >= 2 and np.array_equal(s.count, C)
    assert cbs.rel_l2(s.ORytov, O) < 1e-5
    assert cbs.rel_l2(got - 1.3355, ref - 1.3355) < 1e-5


def test_config3_gradient_matches_oracle():
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN
    from inverse_solver_b200.forward import CBSHostSetup
    from inverse_solver_b200.inputs import ring_illumination, sphere_phantom
    from oracle import multi

    size = [192, 192, 129]
    p = CBSHostSetup.get_default_parameters(dict(
        size=size, wavelength=0.532, NA=1.2, RI_bg=1.3355, resolution=[0.1] * 3,
        vector_simulation=False, return_transmission=True, return_reflection=True, return_3D=True))
    RI = sphere_phantom(size, [0.1] * 3, 1.3355, seed=1)
    fin = np.ascontiguousarray(ring_illumination(p)[:, :, :, [0, 13]])
    s = FORWARD_SOLVER_CONVERGENT_BORN(p)
    try:
        assert s.sim_size == [216, 216, 153]
        s.set_RI(RI)
        meas, _, _ = s.solve(fin)
        est = (1.3355 + 0.5 * (RI - 1.3355)).astype(RI.dtype)
        s.set_RI(est)
        s.set_RI_adjoint(est)
        grad, err = s.gradient(fin, meas)
    finally:
        s.delete()
    o = cbs.ForwardSolverCBS(p, single=True)
    ograd, oerr = multi.get_gradient_static(est, fin, meas, o)
    assert np.linalg.norm(ograd) > 0
    assert cbs.rel_l2(grad, ograd) < 1e-5
    assert abs(err - oerr) <= 1e-5 * abs(oerr)
