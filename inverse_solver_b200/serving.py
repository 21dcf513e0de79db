"""Request loop for forward and reconstruction solves of mixed sizes.

Requests arrive at any time and are admitted while their estimated device
memory fits the budget (HBM-budget admission).  The admitted requests run
concurrently: each runs on a device-resident solver (Green's kernels,
potential and batch buffers stay on the GPU between requests of the same
geometry), every solver has its own CUDA stream, and the library's calls
release the GIL, so the work of different requests overlaps on the device.
A request that arrives while others are running starts as soon as a slot
and its memory are free (continuous batching); its result does not depend
on what else runs, because the solver state is per request and the kernels
are deterministic.  Latency = completion - arrival on the host clock.

    srv = SolveServer(budget_bytes=40e9, slots=4)
    fut = srv.submit(ForwardRequest(params, RI, fields))
    trans, ref, field3d = fut.result()
    srv.stats()   # {"p50_ms", "p99_ms", "throughput_per_s", ...}
"""
from __future__ import annotations

import contextlib
import copy
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np


@dataclass
class ForwardRequest:
    params: dict          # FORWARD_SOLVER_CONVERGENT_BORN parameters
    RI: np.ndarray
    fields: np.ndarray    # [F_x, F_y, npol, n_ill]
    arrival: float = field(default_factory=time.perf_counter)


@dataclass
class ReconRequest:
    params: dict          # BACKWARD_SOLVER_MULTI parameters (forward_solver_parameters inside)
    RI0: np.ndarray       # starting RI of the FISTA iterations
    fields_in: np.ndarray
    fields_out: np.ndarray
    arrival: float = field(default_factory=time.perf_counter)


def geometry_key(p):
    """Solvers are reused between requests with the same geometry."""
    keys = ("size", "resolution", "wavelength", "NA", "RI_bg", "boundary_thickness",
            "boundary_sharpness", "acyclic", "vector_simulation", "use_abbe_sine",
            "return_transmission", "return_reflection", "return_3D", "RI_xy_size", "RI_center",
            "iterations_number")
    return tuple((k, repr(p.get(k))) for k in keys)


def solver_bytes(p, n_ill, max_batch=16):
    """Device memory of one solver with a batch of min(n_ill, max_batch)
    illuminations, estimated from the buffer layout of libodt (complex64):
    Green's / refocusing kernels 3 x conv-plane x z, V, and per illumination
    the Born state (3 x padded grid, or the conv volume if larger), the 3D
    fields and the 2D planes."""
    size = [int(v) for v in p["size"]]
    bt = np.asarray(p["boundary_thickness"], dtype=np.float64)
    btp = np.floor((bt * p["wavelength"] / p["RI_bg"]) / (np.asarray(p["resolution"], dtype=np.float64) * 2) + 0.5)
    sim = [size[i] + 2 * int(btp[i]) for i in range(3)]
    nvox = int(np.prod(sim))
    nri = int(np.prod(size))
    nf = size[0] * size[1]
    nc2 = (2 * size[0]) * (2 * size[1])
    nc3 = nc2 * size[2]
    comp = 3 if p.get("vector_simulation", False) else 1
    nb = min(int(n_ill), int(max_batch))
    static = 8 * (3 * nc3 + nvox)
    per = 8 * comp * (max(3 * nvox, nc3) + 2 * nri + 4 * nf + 2 * nc2)
    return static + nb * per


class DeviceGate:
    """Shared for ordinary device work, exclusive for timing.  Plan
    autotuning (odt_autotune) measures kernel times, so it must have the GPU
    to itself: exclusive() waits until the work already running in shared()
    sections has finished (the solves are synchronous host calls) and holds
    new shared sections back until it is done; a waiting exclusive section
    goes before shared sections that arrive after it."""

    def __init__(self):
        self._cv = threading.Condition()
        self._shared = 0
        self._exclusive = False
        self._waiting = 0

    @contextlib.contextmanager
    def shared(self):
        with self._cv:
            while self._exclusive or self._waiting:
                self._cv.wait()
            self._shared += 1
        try:
            yield
        finally:
            with self._cv:
                self._shared -= 1
                self._cv.notify_all()

    @contextlib.contextmanager
    def exclusive(self):
        with self._cv:
            self._waiting += 1
            while self._exclusive or self._shared:
                self._cv.wait()
            self._waiting -= 1
            self._exclusive = True
        try:
            yield
        finally:
            with self._cv:
                self._exclusive = False
                self._cv.notify_all()


class SolveServer:
    """Admits requests by device-memory budget and runs up to ``slots`` of
    them at once.  ``execute(request)`` and ``estimate(request)`` (bytes)
    may be replaced (the tests drive the scheduler with stand-ins); the
    defaults run the request on libodt."""

    def __init__(self, budget_bytes=None, slots=4, execute=None, estimate=None, max_batch=16, autotune=True):
        if budget_bytes is None:
            import torch

            free, _ = torch.cuda.mem_get_info()
            budget_bytes = int(free * 0.8)
        self.budget = float(budget_bytes)
        self.slots = int(slots)
        self.max_batch = int(max_batch)
        self.autotune = bool(autotune)   # pick each new solver's execution plan by timing (odt_autotune)
        self.plans = {}                  # geometry key -> the tuned plan
        self.execute = execute or self._execute
        self.estimate = estimate or self._estimate
        self._cv = threading.Condition()
        self._queue = []          # (request, future, bytes) in arrival order
        self._in_use = 0.0
        self._running = 0
        self._stop = False
        self._lat = []
        self._done = 0
        self._t0 = None
        self._t1 = None
        self._peak_bytes = 0.0
        self._peak_running = 0
        self._pool = {}           # geometry key -> list of idle (solver, bytes)
        self._idle = []           # (key, solver, bytes) in release order, for eviction
        self._held = 0.0          # bytes of all live solvers, idle or busy
        self._pool_lock = threading.Lock()
        self._gate = DeviceGate()   # requests run shared, autotuning exclusive
        self._threads = [threading.Thread(target=self._loop, daemon=True) for _ in range(self.slots)]
        for t in self._threads:
            t.start()

    # ------------------------------------------------------------ requests
    def submit(self, req):
        fut = Future()
        need = float(self.estimate(req))
        if need > self.budget:
            fut.set_exception(MemoryError("request needs %.3g bytes, budget is %.3g" % (need, self.budget)))
            return fut
        with self._cv:
            if self._t0 is None:
                self._t0 = time.perf_counter()
            self._queue.append((req, fut, need))
            self._cv.notify_all()
        return fut

    def close(self):
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        for t in self._threads:
            t.join()
        with self._pool_lock:
            for lst in self._pool.values():
                for s, _ in lst:
                    s.delete()
            self._pool.clear()
            self._idle.clear()
            self._held = 0.0

    def reset_stats(self):
        """Start a new measurement (latencies, span, peaks) on a running server."""
        with self._cv:
            self._lat = []
            self._done = 0
            self._t0 = self._t1 = None
            self._peak_bytes = 0
            self._peak_running = 0

    def stats(self):
        with self._cv:
            lat = np.asarray(self._lat) * 1e3
            span = (self._t1 - self._t0) if (self._t0 and self._t1) else float("nan")
            return {"requests": self._done,
                    "p50_ms": float(np.percentile(lat, 50)) if lat.size else float("nan"),
                    "p99_ms": float(np.percentile(lat, 99)) if lat.size else float("nan"),
                    "mean_ms": float(lat.mean()) if lat.size else float("nan"),
                    "throughput_per_s": self._done / span if span == span and span > 0 else float("nan"),
                    "peak_admitted_bytes": self._peak_bytes, "peak_concurrent": self._peak_running,
                    "budget_bytes": self.budget}

    # ------------------------------------------------------------ scheduler
    def _take(self):
        """First queued request whose memory fits (arrival order among those
        that fit), or None."""
        for i, (req, fut, need) in enumerate(self._queue):
            if self._in_use + need <= self.budget:
                return self._queue.pop(i)
        return None

    def _loop(self):
        while True:
            with self._cv:
                item = None
                while True:
                    if self._queue:
                        item = self._take()
                        if item is not None:
                            break
                    if self._stop and not self._queue:
                        return
                    self._cv.wait(0.05)
                req, fut, need = item
                self._in_use += need
                self._running += 1
                self._peak_bytes = max(self._peak_bytes, self._in_use)
                self._peak_running = max(self._peak_running, self._running)
            try:
                res = self.execute(req)
                done = time.perf_counter()
                fut.set_result(res)
            except BaseException as e:  # the request fails, the loop goes on
                done = time.perf_counter()
                fut.set_exception(e)
            with self._cv:
                self._in_use -= need
                self._running -= 1
                self._lat.append(done - req.arrival)
                self._done += 1
                self._t1 = done
                self._cv.notify_all()

    # ------------------------------------------------------------ execution
    def _estimate(self, req):
        if isinstance(req, ForwardRequest):
            return solver_bytes(req.params, req.fields.shape[3], self.max_batch)
        fp = req.params["forward_solver_parameters"]
        return solver_bytes(fp, req.fields_in.shape[3], self.max_batch)

    def _acquire(self, p, need):
        """An idle solver of this geometry, or a new one; idle solvers of
        other geometries are freed first (oldest first) while the live ones
        would exceed the budget."""
        from .forward import FORWARD_SOLVER_CONVERGENT_BORN

        key = geometry_key(p)
        with self._pool_lock:
            lst = self._pool.get(key)
            if lst:
                s, b = lst.pop()
                self._idle = [e for e in self._idle if e[1] is not s]
                return key, s, b
            while self._held + need > self.budget and self._idle:
                k, old, b = self._idle.pop(0)
                self._pool[k] = [e for e in self._pool[k] if e[0] is not old]
                old.delete()
                self._held -= b
            self._held += need
        q = copy.deepcopy(p)
        q["max_batch"] = self.max_batch
        s = FORWARD_SOLVER_CONVERGENT_BORN(q)
        s._needs_tune = self.autotune
        return key, s, need

    def _release(self, key, s, b):
        with self._pool_lock:
            self._pool.setdefault(key, []).append((s, b))
            self._idle.append((key, s, b))

    def _execute(self, req):
        need = self._estimate(req)
        if isinstance(req, ForwardRequest):
            with self._gate.shared():
                key, s, b = self._acquire(req.params, need)
            try:
                if getattr(s, "_needs_tune", False):   # once per solver, after its first potential,
                    s._needs_tune = False               # with the GPU to itself
                    with self._gate.exclusive():
                        set_ri_on_device(s, req.RI)
                        self.plans[key] = s.autotune(min(req.fields.shape[3], self.max_batch))
                    with self._gate.shared():
                        return s.solve(req.fields)
                with self._gate.shared():
                    set_ri_on_device(s, req.RI)
                    return s.solve(req.fields)
            finally:
                self._release(key, s, b)
        from .backward import BACKWARD_SOLVER_MULTI

        fp = req.params["forward_solver_parameters"]
        with self._gate.shared():
            key, s, b = self._acquire(fp, need)
        try:
            p = dict(req.params)
            RI0 = req.RI0
            p["init_solver"] = type("Init", (), {"solve": staticmethod(lambda a, b: RI0)})
            bs = BACKWARD_SOLVER_MULTI(p, init_solver=False)
            bs.forward_solver = s
            with self._gate.shared():
                return bs.solve(req.fields_in, req.fields_out)
        finally:
            self._release(key, s, b)


def set_ri_on_device(s, RI):
    """set_RI with the potential built on the GPU (set_RI_device): the RI map
    is uploaded once and eps_imag, Bornmax and the padded potential come from
    device kernels, so a request's set-up does not run numpy sweeps under the
    GIL while the other slots' solves wait for it.  Host set_RI where the
    device path does not apply (RI tensors of the dyadic solver)."""
    import torch

    if s.vector or np.asarray(RI).ndim != 3:
        s.set_RI(RI)
        return
    a = np.asarray(RI)
    dt = np.complex64 if np.iscomplexobj(a) else np.float32
    flat = np.ascontiguousarray(a.astype(dt).ravel(order="F"))
    dev = torch.device("cuda", int(s.parameters.get("used_gpu", 0)))
    t = torch.from_numpy(flat).to(dev)
    s.set_RI_device(t)
    torch.cuda.current_stream(dev).synchronize()


def one_at_a_time(requests):
    """Reference timing: the same requests solved one after the other, each
    with a fresh solver (create, set_RI, solve, delete): total seconds."""
    from .backward import BACKWARD_SOLVER_MULTI
    from .forward import FORWARD_SOLVER_CONVERGENT_BORN

    t0 = time.perf_counter()
    for r in requests:
        if isinstance(r, ForwardRequest):
            s = FORWARD_SOLVER_CONVERGENT_BORN(r.params)
            s.set_RI(r.RI)
            s.solve(r.fields)
            s.delete()
        else:
            p = dict(r.params)
            RI0 = r.RI0
            p["init_solver"] = type("Init", (), {"solve": staticmethod(lambda a, b: RI0)})
            b = BACKWARD_SOLVER_MULTI(p)
            b.solve(r.fields_in, r.fields_out)
            b.delete()
    return time.perf_counter() - t0


# ---------------------------------------------------------------- benchmark
CONFIG5_SIZES = ((64, 64, 64), (96, 96, 64), (128, 128, 128), (192, 192, 96), (256, 256, 192))
# reconstructions need an odd z; with the default 12-voxel boundary the padded
# lengths are 88 x 88 x 85 and 152 x 152 x 153
CONFIG5_RECON_SIZES = ((64, 64, 61), (128, 128, 129))


def make_mix(n, seed, sizes=((64, 64, 64), (96, 96, 64), (128, 128, 128)), max_ill=16,
             recon_every=0, recon_iters=10, recon_sizes=((64, 64, 61),)):
    """Seeded request mix: grids drawn from ``sizes``, 1..max_ill ring /
    circle illuminations, sphere phantoms; every ``recon_every``-th request
    (0: none) is a reconstruction of ``recon_iters`` FISTA iterations on a
    grid drawn from ``recon_sizes`` (odd z, as BACKWARD_SOLVER_MULTI.m:117-119
    requires)."""
    from .backward import BACKWARD_SOLVER_MULTI
    from .forward import CBSHostSetup, FORWARD_SOLVER_CONVERGENT_BORN
    from .inputs import FIELD_GENERATOR, sphere_phantom

    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        recon = bool(recon_every) and i % recon_every == recon_every - 1
        size = (list(recon_sizes[int(rng.integers(len(recon_sizes)))]) if recon
                else list(sizes[int(rng.integers(len(sizes)))]))
        n_ill = int(rng.integers(1, max_ill + 1))
        p = CBSHostSetup.get_default_parameters(dict(
            size=size, wavelength=0.532, NA=1.2, RI_bg=1.3355, resolution=[0.1] * 3,
            vector_simulation=False, return_transmission=True))
        RI = sphere_phantom(size, [0.1] * 3, 1.3355, seed=int(rng.integers(1 << 30)))
        fg = FIELD_GENERATOR.get_default_parameters(dict(
            size=size, wavelength=0.532, NA=1.2, RI_bg=1.3355, resolution=[0.1] * 3,
            vector_simulation=False, illumination_style="circle", percentage_NA_usage=0.6,
            illumination_number=n_ill, seed=i))
        fields = FIELD_GENERATOR(fg).get_fields()
        if recon:
            fp = dict(p, return_reflection=True, return_3D=True)
            s = FORWARD_SOLVER_CONVERGENT_BORN(fp)
            s.set_RI(RI)
            meas, _, _ = s.solve(fields)
            s.delete()
            bp = BACKWARD_SOLVER_MULTI.get_default_parameters(dict(
                forward_solver=FORWARD_SOLVER_CONVERGENT_BORN, forward_solver_parameters=fp,
                itter_max=recon_iters, inner_itt=20, tv_param=7.5e-3))
            RI0 = ((RI + 1.3355) / 2).astype(np.float32)   # a uniform start has no potential
            reqs.append(ReconRequest(bp, RI0, fields, meas))
        else:
            reqs.append(ForwardRequest(p, RI, fields))
    return reqs


def run_stream(reqs, rate_per_s, seed, budget_bytes=None, slots=4, srv=None):
    """Poisson arrivals at ``rate_per_s``: submit each request at its arrival
    time, wait for all; returns (results, stats).  With ``srv`` the given
    server (and its resident solvers) is used and left open; its statistics
    cover this stream only."""
    rng = np.random.default_rng(seed)
    gaps = (np.zeros(len(reqs)) if not np.isfinite(rate_per_s)
            else rng.exponential(1.0 / rate_per_s, size=len(reqs)))
    own = srv is None
    if own:
        srv = SolveServer(budget_bytes=budget_bytes, slots=slots)
    else:
        srv.reset_stats()
    t0 = time.perf_counter()
    futs = []
    t = 0.0
    for r, g in zip(reqs, gaps):
        t += g
        delay = t0 + t - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        r.arrival = time.perf_counter()
        futs.append(srv.submit(r))
    res = [f.result() for f in futs]
    st = srv.stats()
    if own:
        srv.close()
    return res, st


CONFIG4_SIZES = ((64, 64, 64), (96, 96, 64), (128, 128, 128), (192, 192, 96))


def run_config4(a):
    """Config 4: the seeded uneven batch through the request loop (all
    requests at once, one resident solver per shape, its plan picked by
    odt_autotune, up to 64 illuminations per launch, the shapes' solves
    overlapping on the device), against the same solves one at a time with a
    fresh default solver each.  Prints one JSON line with voxel-iter/s of
    both, the plans chosen and the clocks."""
    import json

    from .clocks import ClockSampler
    from .forward import CBSHostSetup

    n = a.requests if a.requests != 24 else 256
    reqs = make_mix(n, a.seed, sizes=CONFIG4_SIZES, max_ill=64, recon_every=0)
    vox = 0
    for r in reqs:
        h = CBSHostSetup(r.params)
        h.prepare_potential(r.RI)
        vox += h.voxel_iterations(r.fields.shape[3])
    server = SolveServer(slots=a.slots, max_batch=64)
    first = {}
    for r in reqs:   # one request of each shape makes its solver resident and tunes it
        first.setdefault(geometry_key(r.params), r)
    run_stream(list(first.values()), float("inf"), a.seed, srv=server)
    clk = ClockSampler(a.device)
    clk.start()
    _, st = run_stream(reqs, float("inf"), a.seed + 1, srv=server)
    st["clocks"] = clk.stop()
    plans = {"x".join(str(v) for v in dict(k)["size"].strip("[]").split(", ")): pl
             for k, pl in server.plans.items()} if server.plans else {}
    server.close()
    serial = one_at_a_time(reqs[: max(8, n // 8)])
    serial_vox = 0
    for r in reqs[: max(8, n // 8)]:
        h = CBSHostSetup(r.params)
        h.prepare_potential(r.RI)
        serial_vox += h.voxel_iterations(r.fields.shape[3])
    span = st["requests"] / st["throughput_per_s"]
    out = {"workload": f"config 4: {n} seeded forward solves over 64^3 / 96x96x64 / 128^3 / 192x192x96, "
                       "1-64 illuminations", "requests": n, "voxel_iterations": vox, "seconds": span,
           "voxel_iter_per_s": vox / span,
           "one_at_a_time_voxel_iter_per_s": serial_vox / serial,
           "one_at_a_time_sample": f"first {max(8, n // 8)} requests, fresh default solver each",
           "speedup": (vox / span) / (serial_vox / serial), "plans": plans, "slots": a.slots,
           "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "clocks": st["clocks"]}
    print(json.dumps(out))


def main():
    import argparse
    import json

    ap = argparse.ArgumentParser(description="request-loop latency / throughput on one GPU")
    ap.add_argument("--requests", type=int, default=24)
    ap.add_argument("--rate", type=float, default=4.0, help="mean arrivals per second")
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--recon-every", type=int, default=6)
    ap.add_argument("--uneven", action="store_true",
                    help="batched uneven solves: all requests submitted at once, forward only, "
                         "grids 64^3 / 96x96x64 / 128^3 / 192x192x96, 1-64 illuminations")
    ap.add_argument("--config5", action="store_true",
                    help="config 5: grids 64^3 .. 256x256x192 with 1-49 illuminations, every "
                         "--recon-every-th request a 10-iteration reconstruction (64x64x61 or "
                         "128x128x127); arrivals at --load times the measured capacity")
    ap.add_argument("--load", type=float, default=0.7,
                    help="with --config5: arrival rate as a fraction of the measured capacity")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--config4", action="store_true",
                    help="config 4: 256 seeded forward solves over 64^3 / 96x96x64 / 128^3 / 192x192x96 "
                         "with 1-64 illuminations, submitted at once to resident, autotuned solvers "
                         "(batches of up to 64 illuminations)")
    a = ap.parse_args()
    capacity = None
    if a.config4:
        return run_config4(a)
    if a.uneven:
        reqs = make_mix(a.requests, a.seed, sizes=((64, 64, 64), (96, 96, 64), (128, 128, 128),
                                                   (192, 192, 96)), max_ill=64, recon_every=0)
        a.rate = float("inf")
    elif a.config5:
        reqs = make_mix(a.requests, a.seed, sizes=CONFIG5_SIZES, max_ill=49, recon_every=a.recon_every,
                        recon_sizes=CONFIG5_RECON_SIZES)
        # capacity: the same requests all submitted at once, on solvers made
        # resident by a first pass (as a long-running server holds them)
        server = SolveServer(slots=a.slots)
        run_stream(reqs, float("inf"), a.seed + 1, srv=server)
        _, cap = run_stream(reqs, float("inf"), a.seed + 1, srv=server)
        capacity = cap["throughput_per_s"]
        a.rate = a.load * capacity
    else:
        reqs = make_mix(a.requests, a.seed, recon_every=a.recon_every)
    serial = one_at_a_time(reqs)
    from .clocks import ClockSampler

    clk = ClockSampler(a.device)
    clk.start()
    if capacity is not None:
        _, st = run_stream(reqs, a.rate, a.seed + 2, srv=server)
        server.close()
    else:
        _, st = run_stream(reqs, a.rate, a.seed + 1, slots=a.slots)
    st["clocks"] = clk.stop()
    if capacity is not None:
        st.update(capacity_per_s=capacity, load=a.load)
    vox = 0
    for r in reqs:
        if isinstance(r, ForwardRequest):
            from .forward import CBSHostSetup

            h = CBSHostSetup(r.params)
            h.prepare_potential(r.RI)
            vox += h.voxel_iterations(r.fields.shape[3])
    if vox:
        st["forward_voxel_iter_per_s"] = vox * st["throughput_per_s"] / len(reqs)
    st.update(one_at_a_time_s=serial, serial_throughput_per_s=len(reqs) / serial,
              rate_per_s=a.rate, slots=a.slots, seed=a.seed, n_requests=len(reqs))
    print(json.dumps(st))


if __name__ == "__main__":
    main()
