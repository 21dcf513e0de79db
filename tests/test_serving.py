"""Scheduler of the request loop (inverse_solver_b200/serving.py) without a
GPU: a stand-in executor with known durations and memory needs.  Admission
keeps the running requests within the memory budget, requests overlap up to
the slot count, a request that does not fit waits only for memory (later
small ones may pass it), one that can never fit fails at once, and a failing
request does not stop the loop."""
import threading
import time

import pytest

from inverse_solver_b200.serving import SolveServer


class Req:
    def __init__(self, i, need, dur, fail=False):
        self.i, self.need, self.dur, self.fail = i, need, dur, fail
        self.arrival = time.perf_counter()


def _run(reqs, budget, slots):
    live = {"n": 0, "bytes": 0.0, "max_bytes": 0.0, "max_n": 0}
    lock = threading.Lock()
    order = []

    def execute(r):
        with lock:
            live["n"] += 1
            live["bytes"] += r.need
            live["max_bytes"] = max(live["max_bytes"], live["bytes"])
            live["max_n"] = max(live["max_n"], live["n"])
            order.append(r.i)
        time.sleep(r.dur)
        with lock:
            live["n"] -= 1
            live["bytes"] -= r.need
        if r.fail:
            raise RuntimeError("request %d failed" % r.i)
        return r.i * 10

    srv = SolveServer(budget_bytes=budget, slots=slots, execute=execute, estimate=lambda r: r.need)
    futs = [srv.submit(r) for r in reqs]
    res = []
    for f in futs:
        try:
            res.append(f.result(timeout=30))
        except Exception as e:   # noqa: BLE001
            res.append(e)
    st = srv.stats()
    srv.close()
    return res, live, order, st


def test_budget_and_slots_are_respected():
    reqs = [Req(i, need=3.0 if i % 3 == 0 else 1.0, dur=0.05) for i in range(24)]
    res, live, order, st = _run(reqs, budget=5.0, slots=4)
    assert res == [i * 10 for i in range(24)]
    assert live["max_bytes"] <= 5.0 and live["max_n"] <= 4 and live["max_n"] >= 2
    assert st["requests"] == 24 and st["peak_admitted_bytes"] <= 5.0
    assert st["p99_ms"] >= st["p50_ms"] > 0


def test_large_request_waits_for_memory_small_ones_pass():
    reqs = [Req(0, 4.0, 0.2), Req(1, 4.0, 0.05), Req(2, 1.0, 0.05), Req(3, 1.0, 0.05)]
    res, live, order, _ = _run(reqs, budget=6.0, slots=4)
    assert res == [0, 10, 20, 30]
    assert order.index(2) < order.index(1)   # the small one ran while the big one waited
    assert live["max_bytes"] <= 6.0


def test_oversized_and_failing_requests():
    reqs = [Req(0, 1.0, 0.01), Req(1, 99.0, 0.01), Req(2, 1.0, 0.01, fail=True), Req(3, 1.0, 0.01)]
    res, _, _, _ = _run(reqs, budget=5.0, slots=2)
    assert res[0] == 0 and res[3] == 30
    assert isinstance(res[1], MemoryError) and isinstance(res[2], RuntimeError)


def test_device_gate_gives_autotuning_the_device_alone():
    """DeviceGate: an exclusive section (plan autotuning) starts only after
    the shared sections already running (requests) have ended, and shared
    sections arriving while it waits or runs are held back until it ends."""
    import threading
    import time as _time

    from inverse_solver_b200.serving import DeviceGate

    g = DeviceGate()
    log = []
    lock = threading.Lock()

    def note(x):
        with lock:
            log.append(x)

    def shared(name, hold):
        with g.shared():
            note(name + "+")
            _time.sleep(hold)
            note(name + "-")

    def exclusive():
        with g.exclusive():
            note("X+")
            _time.sleep(0.05)
            note("X-")

    a = threading.Thread(target=shared, args=("a", 0.2))
    a.start()
    _time.sleep(0.05)                      # a is running
    x = threading.Thread(target=exclusive)
    x.start()
    _time.sleep(0.05)                      # x waits for a
    b = threading.Thread(target=shared, args=("b", 0.0))
    b.start()                              # b arrives after x: waits for x
    for t in (a, x, b):
        t.join(5)
    assert log == ["a+", "a-", "X+", "X-", "b+", "b-"], log
