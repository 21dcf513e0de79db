"""CUDA-graph replay of a batch's solve (csrc/odt_api.cu: run_chunk_graph):
the first call of a configuration runs eagerly, the second is captured, later
ones replay the graph.  Replays must give the eager result bit for bit, and a
new potential (set_RI) or batch size must drop the stale graphs."""
import os

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


def _solver(p, graphs):
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN

    old = os.environ.get("ODT_GRAPHS")
    os.environ["ODT_GRAPHS"] = "1" if graphs else "0"
    try:
        return FORWARD_SOLVER_CONVERGENT_BORN(p)
    finally:
        if old is None:
            os.environ.pop("ODT_GRAPHS", None)
        else:
            os.environ["ODT_GRAPHS"] = old


def test_graph_replays_equal_eager_and_follow_new_potentials():
    p = cases.small_params(return_reflection=True, return_3D=True, max_batch=2)
    RI1 = cases.small_RI(seed=3)
    RI2 = cases.small_RI(seed=4)
    fields = cases.circle_fields(p, 3)       # batches of 2 and 1
    eager = _solver(p, False)
    eager.set_RI(RI1)
    ref1 = eager.solve(fields)
    eager.set_RI(RI2)
    ref2 = eager.solve(fields)
    eager.delete()
    s = _solver(p, True)
    s.set_RI(RI1)
    for _ in range(4):                          # eager, capture, replay, replay
        out = s.solve(fields)
        for a, b in zip(out, ref1):
            assert np.array_equal(a, b)
    s.set_RI(RI2)                               # drops the graphs of RI1
    for _ in range(3):
        out = s.solve(fields)
        for a, b in zip(out, ref2):
            assert np.array_equal(a, b)
    s.delete()


def test_gradient_replays_equal_eager():
    p = cases.small_params(return_transmission=True, return_reflection=True, return_3D=True)
    RI = cases.small_RI()
    fields = cases.circle_fields(p, 2)
    RI0 = (RI * 0.8 + cases.NM * 0.2).astype(np.float32)
    res = []
    for graphs in (False, True):
        s = _solver(p, graphs)
        s.set_RI(RI)
        meas, _, _ = s.solve(fields)
        s.set_RI(RI0)
        s.set_RI_adjoint(RI0)
        outs = [s.gradient(fields, meas) for _ in range(3)]
        s.delete()
        res.append(outs)
    # the misfit is a double-precision atomic sum over blocks: its last bit
    # depends on the order the blocks finish, graph or not
    for g, e in res[1]:
        assert np.array_equal(g, res[0][0][0]) and abs(e - res[0][0][1]) <= 1e-12 * res[0][0][1]
