"""The request loop on the GPU: a seeded mix of forward requests of four
grid sizes -- up to config 5's largest, 256 x 256 x 192 (280 x 280 x 216
padded) -- and a reconstruction, submitted while earlier ones run, gives
for every request exactly the result of solving it alone with a fresh
solver through the same path (potential built on the device; bit for bit:
the solver state is per request and the kernels are deterministic); several
requests were in flight at once."""
import time

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


def test_mixed_requests_equal_alone_results():
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN
    from inverse_solver_b200.backward import BACKWARD_SOLVER_MULTI
    from inverse_solver_b200.serving import ForwardRequest, ReconRequest, SolveServer, set_ri_on_device

    reqs = []
    for i, size in enumerate([[24, 24, 21], [30, 26, 21], [32, 32, 24], [24, 24, 21], [30, 26, 21]]):
        p = cases.params(size, [2, 2, 1.5], return_3D=True)
        RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=10 + i, n_spheres=2, radius_um=(0.3, 0.8))
        reqs.append(ForwardRequest(p, RI, cases.circle_fields(p, 1 + i % 3)))
    big = [256, 256, 192]   # config 5's largest grid, default boundary -> 280 x 280 x 216
    pb = cases.params(big, [6, 6, 6])
    RIb = cases.sphere_phantom(big, [0.1] * 3, cases.NM, seed=40, n_spheres=4, radius_um=(0.5, 2.0))
    reqs.insert(1, ForwardRequest(pb, RIb, cases.circle_fields(pb, 2)))
    # one reconstruction (2 FISTA iterations) on the small odd-z grid
    fp = cases.params([24, 24, 21], [2, 2, 1.5], return_reflection=True, return_3D=True)
    RIt = cases.sphere_phantom([24, 24, 21], [0.1] * 3, cases.NM, seed=30, n_spheres=2, radius_um=(0.3, 0.8))
    fin = cases.circle_fields(fp, 2)
    s = FORWARD_SOLVER_CONVERGENT_BORN(fp)
    s.set_RI(RIt)
    meas, _, _ = s.solve(fin)
    s.delete()
    bp = BACKWARD_SOLVER_MULTI.get_default_parameters(dict(
        forward_solver=FORWARD_SOLVER_CONVERGENT_BORN, forward_solver_parameters=fp, itter_max=2,
        inner_itt=10, tv_param=7.5e-3))
    RI0 = ((RIt + cases.NM) / 2).astype(np.float32)   # a uniform start has no potential (eps = 0)
    reqs.insert(2, ReconRequest(bp, RI0, fin, meas))

    alone = []
    for r in reqs:
        if isinstance(r, ForwardRequest):
            s = FORWARD_SOLVER_CONVERGENT_BORN(dict(r.params, max_batch=16))
            set_ri_on_device(s, r.RI)
            alone.append(s.solve(r.fields))
            if r.params is pb:
                assert s.sim_size == [280, 280, 216]
            s.delete()
        else:
            p = dict(r.params)
            p["init_solver"] = type("Init", (), {"solve": staticmethod(lambda a, b: RI0)})
            b = BACKWARD_SOLVER_MULTI(p)
            b.forward_solver.delete()
            b.forward_solver = FORWARD_SOLVER_CONVERGENT_BORN(dict(fp, max_batch=16))
            alone.append(b.solve(r.fields_in, r.fields_out))
            b.delete()

    # the alone solves use the default plan; an autotuned server could pick
    # another (results then agree to 1e-5, tests/test_autotune_gpu.py)
    srv = SolveServer(budget_bytes=16e9, slots=3, autotune=False)
    futs = []
    for r in reqs:
        r.arrival = time.perf_counter()
        futs.append(srv.submit(r))
        time.sleep(0.01)
    got = [f.result(timeout=600) for f in futs]
    st = srv.stats()
    srv.close()
    assert st["requests"] == len(reqs) and st["peak_concurrent"] >= 2
    for g, a in zip(got, alone):
        if isinstance(a, tuple):
            for x, y in zip(g, a):
                assert (x is None and y is None) or np.array_equal(x, y)
        else:
            assert np.array_equal(g, a)
