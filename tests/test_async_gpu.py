"""Asynchronous solves through the C ABI (odt_submit / odt_poll / odt_wait,
the FORWARD_SOLVER_CONVERGENT_BORN.submit / poll / wait mirror): results
bit-identical to synchronous solves of the same fields, collected out of
order; a failing job reports its status and message to the collecting
call; destroying a handle lets its queued jobs finish."""
import ctypes as C
import time

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


def _solver():
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN

    p = cases.small_params(return_transmission=True, return_reflection=True, return_3D=True)
    s = FORWARD_SOLVER_CONVERGENT_BORN(p)
    s.set_RI(cases.small_RI())
    return s, p


def test_async_matches_sync_out_of_order():
    s, p = _solver()
    sets = [cases.circle_fields(p, n, seed=k) for k, n in enumerate((1, 3, 2))]
    ref = [s.solve(f) for f in sets]
    tickets = [s.submit(f) for f in sets]
    got = [None] * 3
    got[2] = s.wait(tickets[2])
    t0 = time.time()
    while got[0] is None and time.time() - t0 < 60:
        got[0] = s.poll(tickets[0])
        time.sleep(0.001)
    got[1] = s.wait(tickets[1])
    for r, g in zip(ref, got):
        for a, b in zip(r, g):
            assert np.array_equal(a, b)
    held, budget = s.budget()
    assert held > 0 and budget == 0
    s.delete()


def test_failing_job_reports_status_and_message():
    from inverse_solver_b200 import _lib

    s, p = _solver()
    a = _lib.SolveArgs()          # no input fields: the solve itself rejects it
    a.n_ill = 1
    a.memory = _lib.ODT_MEM_HOST
    t = C.c_uint64(0)
    assert s.lib.odt_submit(s._handle, C.byref(a), C.byref(t)) == 0
    st = C.c_int(-1)
    assert s.lib.odt_wait(s._handle, t.value, C.byref(st)) == 0
    assert st.value == 1
    assert b"NULL" in s.lib.odt_last_error() or b"fields" in s.lib.odt_last_error()
    done = C.c_int32(0)
    assert s.lib.odt_poll(s._handle, t.value, C.byref(done), C.byref(st)) == 1   # ticket released
    s.delete()


def test_destroy_lets_queued_jobs_finish():
    s, p = _solver()
    f = cases.circle_fields(p, 2)
    ref = s.solve(f)
    t1, t2 = s.submit(f), s.submit(f)
    outs = [s._jobs[t1][2], s._jobs[t2][2]]
    s.delete()
    for o in outs:
        for a, b in zip(ref, o):
            assert np.array_equal(a, b)


def test_process_exit_without_destroy_is_clean():
    """A host that exits with a job still queued and without odt_destroy
    exits normally (the worker thread does not abort the process)."""
    import subprocess
    import sys

    code = ("import sys; sys.path.insert(0, 'tests'); import cases; "
            "from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN as F; "
            "p = cases.small_params(); s = F(p); s.set_RI(cases.small_RI()); "
            "t = s.submit(cases.circle_fields(p, 1)); s.wait(t); s.submit(cases.circle_fields(p, 1)); "
            "print('done')")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "done" in r.stdout
