"""Plan autotuning (odt_autotune) and the uneven batch of config 4 through
the request loop.

  * odt_autotune times the plans that apply (fused xy-pass, separate
    pipelined passes, generic tile kernels) on an (88, 88, 88) grid, keeps
    the fastest, and a second handle of the same shape takes the choice from
    the cache; a solve with the tuned plan matches the single-precision
    oracle (relative L2 1e-5 per illumination);
  * a seeded uneven batch in the shapes of config 4 (64^3, 96x96x64, 128^3,
    192x192x96 RI grids; 1-5 illuminations each) submitted at once to the
    request loop, whose resident solvers are autotuned, gives every request
    its solo result (a fresh solver with the default plan) within 1e-5: the
    plans differ only in the order of the FFT arithmetic."""
import time

import numpy as np
import pytest

import cases
from oracle import cbs

pytestmark = pytest.mark.gpu


def test_autotune_picks_and_caches_a_plan():
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN

    size = [64, 64, 64]
    p = cases.params(size, [6, 6, 6], return_3D=True)
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=21, n_spheres=3, radius_um=(0.4, 1.0))
    fields = cases.circle_fields(p, 3)
    s = FORWARD_SOLVER_CONVERGENT_BORN(p)
    s2 = None
    try:
        s.set_RI(RI)
        r = s.autotune(3)
        assert r["batch"] == 3 and not r["cached"]
        assert set(r["ms"]) == {"fused_xy", "separate_pipelined", "generic"}
        assert r["plan"] == min(r["ms"], key=r["ms"].get)
        t, _, f = s.solve(fields)
        s2 = FORWARD_SOLVER_CONVERGENT_BORN(p)
        s2.set_RI(RI)
        r2 = s2.autotune(3)
        assert r2["cached"] and r2["plan"] == r["plan"]
    finally:
        s.delete()
        if s2 is not None:
            s2.delete()
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    ot, _, of = o.solve(fields)
    for k in range(3):
        assert cbs.rel_l2(f[..., k], of[..., k]) < 1e-5 and cbs.rel_l2(t[..., k], ot[..., k]) < 1e-5


def test_uneven_batch_equals_solo_results():
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN
    from inverse_solver_b200.serving import CONFIG4_SIZES, SolveServer, make_mix, set_ri_on_device

    reqs = make_mix(10, 7, sizes=CONFIG4_SIZES, max_ill=5, recon_every=0)
    assert len({tuple(r.params["size"]) for r in reqs}) >= 3
    solo = []
    for r in reqs:
        s = FORWARD_SOLVER_CONVERGENT_BORN(dict(r.params, max_batch=64))
        set_ri_on_device(s, r.RI)
        solo.append(s.solve(r.fields))
        s.delete()
    srv = SolveServer(slots=4, max_batch=64)
    futs = []
    for r in reqs:
        r.arrival = time.perf_counter()
        futs.append(srv.submit(r))
    got = [f.result(timeout=600) for f in futs]
    st = srv.stats()
    plans = dict(srv.plans)
    srv.close()
    assert st["requests"] == len(reqs) and plans
    for g, a in zip(got, solo):
        t, t0 = g[0], a[0]
        for k in range(t.shape[3]):
            assert cbs.rel_l2(t[..., k], t0[..., k]) < 1e-5
