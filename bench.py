"""Benchmark: Born voxel-iterations per second of the batched CBS forward solve.

Workload (one step): the multi-illumination forward solve of a seeded
128^3 multi-sphere phantom (0.1 um voxels, RI 1.34-1.46 in 1.3355, default
6-wavelength boundary -> 152^3 padded grid), 49 plane waves (normal + 48 on
rings at NA 0.3/0.6/0.9), transmitted field returned.  Synthetic data stand in
for the reference's experimental holograms.

  value : voxel-iterations/s with inputs resident in HBM (device API), CUDA
          events on the solve stream, max over ranks
  e2e   : the same metric through the C-ABI host path (pinned host buffers,
          H2D of the input fields and D2H of the transmitted fields inside the
          timed region), wall clock around synchronous calls

usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from inverse_solver_b200.clocks import ClockSampler  # noqa: E402

METRIC = "Born voxel-iter/s"
UNIT = "voxel-iter/s"
GRID = [128, 128, 128]
N_ILL = 49
SEED = 0
# algorithmic HBM bytes per voxel and launch of each Born kernel kind
# (complex64 = 8 B): born_x reads T, Field_n, Field, V and writes T, Field_n,
# Field; born_y / born_z read and write T once.  "_pipe" = the pipelined
# (TMA-fed, persistent) variants of the same passes; "born_x_pipe_edge" = the
# pipelined x-pass of iterations 2, 3 and the final pass (56 B nominal);
# "born_xy" = the fused xy-pass (x-pass and both y-FFTs with the plane in
# shared memory: the same 56 B as the x-pass), "born_xy_edge" its launches
# for iterations 1-3 and the final pass.
ALG_BYTES_PER_VOXEL = {"born_x": 56, "born_y": 16, "born_z": 16,
                       "born_x_pipe": 56, "born_y_pipe": 16, "born_z_pipe": 16,
                       "born_x_pipe_edge": 56, "born_xy": 56, "born_xy_edge": 56}
# the same with T and Field_n in 16-bit block floating point (4 B per value
# plus one exponent byte per 8 values): xy-pass 4+4 (T) + 4+4 (Field_n) + 16
# (Field) + 8 (V) + 0.5 (exponents) = 40.5 B, z-pass 8 + 0.25 = 8.25 B; one
# iteration 48.75 B (48 B without the exponents)
ALG_BYTES_B16 = {"born_xy": 40.5, "born_xy_edge": 40.5, "born_z_pipe": 8.25}
ITER_BYTES_B16 = 48.75


def workload_params():
    from inverse_solver_b200.forward import CBSHostSetup

    return CBSHostSetup.get_default_parameters(dict(
        size=list(GRID), wavelength=0.532, NA=1.2, RI_bg=1.3355, resolution=[0.1] * 3,
        vector_simulation=False, return_transmission=True))


def workload_inputs(p, n_ill=N_ILL):
    from inverse_solver_b200.inputs import ring_illumination, sphere_phantom

    RI = sphere_phantom(GRID, [0.1] * 3, 1.3355, seed=SEED)
    fields = ring_illumination(p)
    assert fields.shape[3] == N_ILL
    return RI, np.ascontiguousarray(fields[:, :, :, :n_ill])


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_baseline(p, RI, fields, n_iter):
    """The oracle's single-precision restatement of the reference's Born loop
    (unfused sweeps + full 3D FFTs, scipy.fft with all host threads), timed on
    a bounded sample: one illumination, first n_iter Born iterations."""
    from oracle import cbs

    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    inp = o.transform_field_3D(cbs.fftc2(fields[:, :, :, :1].astype(np.complex64)))
    n_iter = min(n_iter, o.Bornmax)
    t0 = time.perf_counter()
    o.solve_raw(inp[:, :, :, 0], n_iter=n_iter)
    dt = time.perf_counter() - t0
    vox = int(np.prod(o.V.shape)) * n_iter
    return {"value": vox / dt, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": f"1 of {N_ILL} illuminations, Born iterations 1-{n_iter} of {o.Bornmax} "
                      f"on the {list(o.V.shape)} padded grid ({dt:.1f} s)"}


def plain_single_solve(p, RI, fields, n_ill=3):
    """The library's plain path on the same workload: one illumination per
    solve (batch of 1), the generic (non-pipelined) tile kernels, no graph
    replay; synchronous host calls, timed on the host clock after one warm-up
    solve.  Returns voxel-iterations/s."""
    import os as _os

    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN

    saved = {k: _os.environ.get(k) for k in ("ODT_KERNELS", "ODT_GRAPHS")}
    _os.environ["ODT_KERNELS"] = "generic"
    _os.environ["ODT_GRAPHS"] = "0"
    try:
        q = dict(p, max_batch=1)
        s = FORWARD_SOLVER_CONVERGENT_BORN(q)
    finally:
        for k, v in saved.items():
            if v is None:
                _os.environ.pop(k, None)
            else:
                _os.environ[k] = v
    s.set_RI(RI)
    one = np.ascontiguousarray(fields[:, :, :, :1])
    s.solve(one)
    t0 = time.perf_counter()
    for k in range(n_ill):
        s.solve(np.ascontiguousarray(fields[:, :, :, k:k + 1]))
    dt = time.perf_counter() - t0
    v = s.voxel_iterations(n_ill) / dt
    s.delete()
    return v


def run_reference(args, rank, world):
    if rank != 0:
        return
    p = workload_params()
    RI, fields = workload_inputs(p)
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(p, RI, fields, args.ref_iters)
        if i >= args.warmup:
            vals.append(r["value"])
    v = float(np.mean(vals))
    r["value"] = v
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
           "dtype": "fp32", "data": "synthetic",
           "config": {"workload": workload_name(), "grid": GRID, "n_ill": N_ILL},
           "cpu_baseline": r,
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "vs_baseline": None}
    print(json.dumps(out))


def workload_name():
    return ("cbs_forward: 128^3 RI grid, 0.1 um voxels, seeded multi-sphere phantom (seed 0), "
            "49 plane waves (normal + rings NA 0.3/0.6/0.9), padded 152^3, transmitted field")


def run_ours(args, rank, world, local_rank):
    import torch

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN

    p = workload_params()
    p["used_gpu"] = local_rank
    n_ill = args.n_ill
    RI, fields = workload_inputs(p, n_ill)
    s = FORWARD_SOLVER_CONVERGENT_BORN(p)
    s.set_RI(RI)
    F = s.field_size
    vox_step = s.voxel_iterations(n_ill)
    dev = torch.device("cuda", local_rank)
    fin = torch.from_numpy(np.ascontiguousarray(fields[:, :, 0, :].transpose(2, 1, 0))).to(dev)
    tout = torch.empty((n_ill, F[1], F[0]), dtype=torch.complex64, device=dev)
    stream = torch.cuda.current_stream()

    for _ in range(args.warmup):
        s.solve_device(fin, tout, stream=stream)
    torch.cuda.synchronize()
    if args.profile_run:
        s.delete()
        return

    # ---- per-kernel times and launch counts (one profiled step, not timed)
    s.set_profiling(True)
    s.solve_device(fin, tout, stream=stream)
    torch.cuda.synchronize()
    kt = s.kernel_times()
    s.set_profiling(False)
    launches_per_step = sum(n for _, n in kt.values())

    # ---- timed region (device-resident inputs); the clock sampler starts
    # first, then one untimed step brings the clocks back up after the
    # profiled step's host work before the timed steps begin
    clk = ClockSampler(local_rank)
    clk.start()
    s.solve_device(fin, tout, stream=stream)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    evs[0].record(stream)
    for i in range(args.steps):
        s.solve_device(fin, tout, stream=stream)
        evs[i + 1].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = clk.stop()
    total_ms = evs[0].elapsed_time(evs[-1])
    step_ms = [evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps)]
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = world * vox_step * args.steps / (total_ms / 1e3)

    # ---- e2e through the host C-ABI path with pinned buffers
    hin = torch.from_numpy(np.ascontiguousarray(fields[:, :, 0, :].transpose(2, 1, 0))).pin_memory()
    hout = torch.empty((n_ill, F[1], F[0]), dtype=torch.complex64).pin_memory()
    s.solve_ptrs(hin.data_ptr(), n_ill, trans=hout.data_ptr())
    if dist:
        dist.barrier()
    e2e_steps = max(1, args.steps)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        s.solve_ptrs(hin.data_ptr(), n_ill, trans=hout.data_ptr())
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_val = world * vox_step * e2e_steps / float(te.item())

    mixed = None if args.no_mixed else mixed_storage_run(args, s, fin, tout, stream, vox_step, dev, dist)
    if rank != 0:
        s.delete()
        return
    peak, peak_kind = load_peaks()
    born = {k: v for k, v in kt.items() if k in ALG_BYTES_PER_VOXEL}
    dom = max(born, key=lambda k: born[k][0])
    dom_ms, dom_n = born[dom]
    vox_launch = int(np.prod(s.sim_size)) * s.batch()
    alg_bytes = ALG_BYTES_PER_VOXEL[dom] * vox_launch
    achieved = alg_bytes / (dom_ms / dom_n / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        tj = json.load(open(tpath)).get(workload_key(), {})
        if dom in tj:
            traffic = tj[dom]
    born_ms = sum(v[0] for v in born.values())
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": {"workload": workload_name(), "grid": GRID, "padded_grid": s.sim_size,
                   "n_ill": n_ill, "bornmax": s.Bornmax, "voxel_iters_per_step": vox_step,
                   "batch": s.batch(), "l2": "inputs larger than L2 (per-step working set "
                   f"{3 * 8 * int(np.prod(s.sim_size)) * s.batch() / 1e9:.1f} GB)",
                   "parallelism": f"dp{world} (illuminations, replicas)"},
        "latency_ms": {"p50": float(np.percentile(step_ms, 50)),
                       "p99": float(np.percentile(step_ms, 99))},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic,
                     "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": dom_ms / dom_n,
                     "iteration_frac": (72.0 * vox_step / (born_ms / 1e3) / 1e9) / peak},
        "kernel_ms_per_step": {k: v[0] for k, v in kt.items()},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clocks,
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(hin.numel() * 8),
                "d2h_bytes_per_step": int(hout.numel() * 8)},
    }
    if mixed is not None:
        mk = mixed.pop("kernel_times")
        xy_ms, xy_n = mk.get("born_xy", (0.0, 0))
        mixed["roofline"] = {
            "kernel": "born_xy", "bytes_per_voxel": ALG_BYTES_B16["born_xy"], "peak": peak,
            "achieved": (ALG_BYTES_B16["born_xy"] * vox_launch / (xy_ms / xy_n / 1e3) / 1e9) if xy_n else None,
            "iteration_frac": (ITER_BYTES_B16 * vox_step / (sum(v[0] for k, v in mk.items()
                                                                if k in ALG_BYTES_B16) / 1e3) / 1e9) / peak,
            "iteration_bytes_per_voxel": ITER_BYTES_B16}
        if mixed["roofline"]["achieved"]:
            mixed["roofline"]["frac"] = mixed["roofline"]["achieved"] / peak
        mixed["speedup_vs_fp32_batched"] = mixed["value"] / value
        out["mixed_b16"] = mixed
    if world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(p, RI, fields, args.ref_iters)
    if world == 1 and not args.no_plain:
        pv = plain_single_solve(p, RI, fields)
        if mixed is not None:
            mixed["speedup_vs_plain_single_solve"] = mixed["value"] / pv
        out["plain_single_solve"] = {
            "value": pv, "unit": UNIT, "speedup_of_value": value / pv,
            "what": "same workload, one illumination per solve, generic tile kernels, no graph "
                    "replay, host calls (3 illuminations timed)"}
    s.delete()
    print(json.dumps(out))


def mixed_storage_run(args, s, fin, tout, stream, vox_step, dev, dist):
    """The same batched solve with T and Field_n in 16-bit block floating
    point (field_storage "b16"): voxel-iter/s (CUDA events, max over ranks),
    its per-kernel times, and the relative L2 distance of its transmitted
    fields from the FP32 run's (the FP64 comparison is
    tests/test_b16_storage_gpu.py)."""
    import torch

    s.set_field_storage("b16")
    t16 = torch.empty_like(tout)
    for _ in range(max(3, args.warmup)):
        s.solve_device(fin, t16, stream=stream)
    torch.cuda.synchronize()
    s.set_profiling(True)
    s.solve_device(fin, t16, stream=stream)
    torch.cuda.synchronize()
    kt = s.kernel_times()
    s.set_profiling(False)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        s.solve_device(fin, t16, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    world = dist.get_world_size() if dist else 1
    rel = float(torch.linalg.vector_norm(t16 - tout) / torch.linalg.vector_norm(tout))
    s.set_field_storage("complex64")
    return {"value": world * vox_step * args.steps / (ms / 1e3), "unit": UNIT,
            "ms_per_step": ms / args.steps, "storage": "T and Field_n: 16-bit block floating point "
            "(8 values per exponent, 15-bit mantissas); Field, V, inputs and outputs complex64; FP32 "
            "arithmetic", "trans_rel_l2_vs_fp32": rel, "kernel_times": kt,
            "kernel_ms_per_step": {k: v[0] for k, v in kt.items() if v[1]}}


def run_fista(args):
    """Inverse-solver workload (BACKWARD_SOLVER_MULTI, config-3 shape): time
    per FISTA outer iteration (forward + adjoint CBS solves of every
    illumination, TV prox with 100 inner iterations, momentum update) with
    the device-resident loop and with the host-array loop.  RI 192x192x129
    (odd z, as the reference requires), seeded multi-sphere phantom, 49
    ring illuminations, measured fields from a forward solve of the phantom,
    start from the phantom pulled halfway to the background."""
    import time

    import torch

    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN
    from inverse_solver_b200.backward import BACKWARD_SOLVER_MULTI
    from inverse_solver_b200.inputs import ring_illumination, sphere_phantom

    grid = [192, 192, 129]
    nm = 1.3355
    fp = FORWARD_SOLVER_CONVERGENT_BORN.get_default_parameters(dict(
        size=grid, wavelength=0.532, NA=1.2, RI_bg=nm, resolution=[0.1] * 3, vector_simulation=False,
        return_transmission=True, return_reflection=True, return_3D=True))
    RI = sphere_phantom(grid, [0.1] * 3, nm, seed=SEED)
    fields = np.ascontiguousarray(ring_illumination(fp)[:, :, :, :args.n_ill])
    fw = FORWARD_SOLVER_CONVERGENT_BORN(fp)
    fw.set_RI(RI)
    meas, _, _ = fw.solve(fields)
    fw.delete()
    start = (RI * 0.5 + nm * 0.5).astype(np.float32)

    class Start:
        def solve(self, input_field, output_field):
            return start

    out = {"metric": "FISTA outer iteration time", "unit": "s", "higher_is_better": False,
           "config": {"workload": "BACKWARD_SOLVER_MULTI: 192x192x129 RI grid, 0.1 um voxels, seeded "
                                  "multi-sphere phantom, %d ring illuminations, inner_itt 100, "
                                  "tv_param 7.5e-3" % fields.shape[3], "grid": grid,
                      "n_ill": int(fields.shape[3])}}
    clk = ClockSampler(0)
    clk.start()
    for device_loop in (True, False):
        bp = BACKWARD_SOLVER_MULTI.get_default_parameters(dict(
            RI_bg=nm, wavelength=0.532, NA=1.2, resolution=[0.1] * 3, size=grid,
            forward_solver=FORWARD_SOLVER_CONVERGENT_BORN, forward_solver_parameters=fp,
            init_solver=Start(), step=0.01, tv_param=7.5e-3, inner_itt=100, use_non_negativity=True,
            nmin=nm, nmax=1.5, device_loop=device_loop))
        times = []
        for iters in (1, 1 + args.steps):
            bp["itter_max"] = iters
            b = BACKWARD_SOLVER_MULTI(bp)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            b.solve(fields, meas)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
            b.delete()
        out["device_loop" if device_loop else "host_loop"] = (times[1] - times[0]) / args.steps
    out["clocks"] = clk.stop()
    out["value"] = out["device_loop"]
    out["steps"] = args.steps
    print(json.dumps(out), flush=True)


def run_bpm(args):
    """Beam-propagation workload (FORWARD_SOLVER_BPM): voxel-steps/s (field
    plane x slices x illuminations per second) of whole solves through the
    host API (inputs and outputs in host memory), RI 128^3 at 0.1 um
    (seeded multi-sphere phantom), 49 ring illuminations, cosine correction
    on, transmitted field only; beside it the single-precision oracle on
    the host cores for 2 illuminations."""
    from inverse_solver_b200 import FORWARD_SOLVER_BPM
    from inverse_solver_b200.inputs import ring_illumination, sphere_phantom
    from oracle import bpm as obpm

    nm = 1.3355
    p = FORWARD_SOLVER_BPM.get_default_parameters(dict(size=list(GRID), wavelength=0.532, NA=1.2, RI_bg=nm,
                                                       resolution=[0.1] * 3, vector_simulation=False))
    RI = sphere_phantom(GRID, [0.1] * 3, nm, seed=SEED)
    fields = np.ascontiguousarray(ring_illumination(p)[:, :, :, :args.n_ill])
    s = FORWARD_SOLVER_BPM(p)
    s.set_RI(RI)
    for _ in range(args.warmup):
        s.solve(fields)
    clk = ClockSampler(0)
    clk.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s.solve(fields)
    dt = (time.perf_counter() - t0) / args.steps
    units = int(np.prod(GRID)) * fields.shape[3]
    # device-resident solves (solve_device), timed with CUDA events
    import torch

    dev = torch.device("cuda", 0)
    fin = torch.from_numpy(np.ascontiguousarray(fields[:, :, 0, :].transpose(2, 1, 0))).to(dev)
    tout = torch.empty_like(fin)
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        s.solve_device(fin, tout, stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        s.solve_device(fin, tout, stream)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    dev_ms = e0.elapsed_time(e1) / args.steps
    o = obpm.ForwardSolverBPM(p, single=True)
    o.set_RI(RI)
    t0 = time.perf_counter()
    o.solve(fields[:, :, :, :2])
    dtc = time.perf_counter() - t0
    print(json.dumps({
        "metric": "BPM voxel-steps/s", "value": units / dt, "unit": "voxel-steps/s", "higher_is_better": True,
        "ms_per_solve": dt * 1e3, "steps": args.steps, "warmup": args.warmup, "clocks": clocks,
        "device_resident": {"value": units / (dev_ms / 1e3), "unit": "voxel-steps/s", "ms_per_solve": dev_ms},
        "config": {"workload": "FORWARD_SOLVER_BPM: 128^3 RI grid, 0.1 um voxels, seeded multi-sphere "
                               "phantom, %d ring illuminations, cos_correction, host API" % fields.shape[3]},
        "cpu_baseline": {"value": int(np.prod(GRID)) * 2 / dtc, "unit": "voxel-steps/s",
                         "cores": os.cpu_count(), "kind": "port", "sample": "2 illuminations"}}), flush=True)


GRID_LENGTH_CASES = (
    (72, "96^3 padded: fused xy-pass (12-point butterflies) + pipelined z-pass"),
    (103, "127^3 padded: 127 is prime, Bluestein transforms on every axis, unfused Born loop"),
    (104, "128^3 padded: fused xy-pass + pipelined z-pass (16-point butterflies)"),
    (112, "136^3 padded: fused xy-pass + pipelined z-pass (17-point butterflies)"),
    (128, "152^3 padded: fused xy-pass + pipelined z-pass"),
    (136, "160^3 padded: fused xy-pass + pipelined z-pass (20-point butterflies)"),
)


def run_grid_lengths(args):
    """Born-loop speed against the padded grid's lengths: scalar CBS solves
    of 16 ring illuminations (NA 1.2, 0.1 um voxels, seeded multi-sphere
    phantom, default boundary) on RI grids of 72^3, 103^3, 104^3, 112^3,
    128^3 and 136^3, which the default boundary pads to 96^3, 127^3 (prime:
    Bluestein transforms), 128^3, 136^3, 152^3 and 160^3 (fused passes on all
    but 127^3).  Device-resident solve_device calls
    timed with CUDA events;
    each solve moves more than the L2 (16 fields of >= 127^3 complex64).
    "kinds_one_solve" is one further solve with events around each kind of
    launch; on the 127^3 grid the unfused loop books born_point under
    born_x, each 3D FFT (three axis transforms) under born_y and born_green
    under born_z."""
    import torch

    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN
    from inverse_solver_b200.forward import CBSHostSetup
    from inverse_solver_b200.inputs import ring_illumination, sphere_phantom

    known = [n for n, _ in GRID_LENGTH_CASES]
    if any(n not in known for n in args.grid_lengths):
        raise SystemExit("--grid-lengths takes RI sizes from %s" % known)
    n_ill = 16
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    cases = []
    clk = ClockSampler(0)
    clk.start()
    for n, what in GRID_LENGTH_CASES:
        if args.grid_lengths and n not in args.grid_lengths:
            continue
        size = [n, n, n]
        p = CBSHostSetup.get_default_parameters(dict(size=size, wavelength=0.532, NA=1.2, RI_bg=1.3355,
                                                     resolution=[0.1] * 3, vector_simulation=False,
                                                     return_transmission=True))
        RI = sphere_phantom(size, [0.1] * 3, 1.3355, seed=SEED)
        fields = np.ascontiguousarray(ring_illumination(p)[:, :, :, :n_ill])
        s = FORWARD_SOLVER_CONVERGENT_BORN(dict(p, max_batch=n_ill))
        try:
            s.set_RI(RI)
            F = s.field_size
            fin = torch.from_numpy(np.ascontiguousarray(fields[:, :, 0, :].transpose(2, 1, 0))).to(dev)
            tout = torch.empty((n_ill, F[1], F[0]), dtype=torch.complex64, device=dev)
            for _ in range(args.warmup):
                s.solve_device(fin, tout, stream=stream)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                s.solve_device(fin, tout, stream=stream)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / args.steps
            vox = int(np.prod(s.sim_size)) * n_ill * s.Bornmax
            # one more solve with per-kind event timing (not in the timed region)
            s.set_profiling(True)
            s.solve_device(fin, tout, stream=stream)
            torch.cuda.synchronize()
            kt = {k: {"ms": round(v[0], 3), "launches": v[1]} for k, v in s.kernel_times().items() if v[1]}
            s.set_profiling(False)
            cases.append({"ri": size, "padded": list(s.sim_size), "path": what, "bornmax": s.Bornmax,
                          "ms_per_solve": ms, "voxel_iter_per_s": vox / (ms / 1e3), "kinds_one_solve": kt})
        finally:
            s.delete()
    clocks = clk.stop()
    print(json.dumps({
        "metric": "CBS Born iterations by padded-grid length", "unit": "voxel-iter/s", "higher_is_better": True,
        "steps": args.steps, "warmup": args.warmup, "clocks": clocks, "cases": cases,
        "config": {"workload": "scalar CBS, %d ring illuminations (NA 1.2), 0.1 um voxels, seeded multi-sphere "
                               "phantom, default boundary, solve_device (device-resident)" % n_ill}}), flush=True)


def run_setup(args):
    """Solver construction time (Green's / refocusing kernels, pupils, device
    plans) for the benchmark geometry (128^3 RI grid, 256^2 conv plane), with
    the plane part of truncated_green_plus on the GPU and on the host; the
    second construction of each is timed (the Hankel matrices of the radial
    part are cached per geometry within a process)."""
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN

    p = workload_params()
    out = {"metric": "solver construction time", "unit": "s", "higher_is_better": False,
           "config": {"workload": "FORWARD_SOLVER_CONVERGENT_BORN constructor, 128^3 RI grid, 0.1 um voxels"}}
    for key, dev, gemm in (("green_on_device", True, None), ("green_on_device_simt_gemm", True, "simt"),
                           ("green_on_host", False, None)):
        q = dict(p, green_on_device=dev)
        if gemm:
            os.environ["ODT_GREEN_GEMM"] = gemm
        else:
            os.environ.pop("ODT_GREEN_GEMM", None)
        FORWARD_SOLVER_CONVERGENT_BORN(q).delete()
        t0 = time.perf_counter()
        FORWARD_SOLVER_CONVERGENT_BORN(q).delete()
        out[key] = time.perf_counter() - t0
    os.environ.pop("ODT_GREEN_GEMM", None)
    out["value"] = out["green_on_device"]
    out["note"] = ("green_on_device: plane GEMMs on the tensor cores (tcgen05, TF32 parts); "
                   "green_on_device_simt_gemm: the same on the FP32 SIMT kernel")
    print(json.dumps(out), flush=True)


def run_retrieval(args):
    """Field retrieval workload (FIELD_EXPERIMENTAL_RETRIEVAL.get_fields):
    holograms per second for background / sample stacks of 49 synthetic
    off-axis holograms of 1024 x 1024 pixels (camera pixel 0.0625 um, output
    pixel 0.1 um: 640 x 640 spectra, 636 x 636 fields), the whole call
    through the host API (hologram upload, GPU transforms and unwrapping,
    host per-image steps, field download); beside it the oracle with its
    Goldstein restatement on the host for 2 holograms."""
    import sys as _sys

    _sys.path.insert(0, os.path.join(ROOT, "tests"))
    import cases

    from inverse_solver_b200.retrieval import FIELD_EXPERIMENTAL_RETRIEVAL
    from oracle import cbs, goldstein, retrieval

    N, n = 1024, args.n_ill
    bg, sp, _ = cases.off_axis_holograms(N, n, seed=SEED)
    p = FIELD_EXPERIMENTAL_RETRIEVAL.get_default_parameters(dict(
        size=[N, N, 64], resolution=[0.1, 0.1, 0.1], resolution_image=[0.0625, 0.0625], NA=1.2,
        wavelength=0.532, RI_bg=1.3355))
    r = FIELD_EXPERIMENTAL_RETRIEVAL(p)
    for _ in range(args.warmup):
        r.get_fields(bg, sp)
    clk = ClockSampler(0)
    clk.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r.get_fields(bg, sp)
    dt = (time.perf_counter() - t0) / args.steps
    clocks = clk.stop()

    def unwrap(ph):
        out = goldstein.unwrapp2(ph)
        return np.asarray(out[0] if isinstance(out, tuple) else out, dtype=np.float32)

    t0 = time.perf_counter()
    retrieval.get_fields(p, bg[:, :, :2], sp[:, :, :2], unwrap=unwrap)
    dtc = time.perf_counter() - t0
    del bg, sp
    # aberration correction and dirty-field rejection on fields of the size
    # get_fields returns here (636 x 636 = 4 * 3 * 53: Bluestein transforms)
    L = 636
    fin, fout, k0s, fp = cases.aberrated_fields(L, n, seed=SEED)
    ra = FIELD_EXPERIMENTAL_RETRIEVAL(FIELD_EXPERIMENTAL_RETRIEVAL.get_default_parameters(fp))
    cp = dict(overlap_factor=0.25, distList=[-2.0, -1.0, 0.0, 1.0, 2.0], k0s=k0s)
    side = {}
    for name, fn in (("get_aberration_pattern", lambda: ra.get_aberration_pattern(fin, fout, cp)),
                     ("correct_aberration", lambda: ra.correct_aberration(fin, fout, ab)),
                     ("remove_dirty_fields", lambda: ra.remove_dirty_fields(fin, fout))):
        for _ in range(max(1, args.warmup)):
            res = fn()
        if name == "get_aberration_pattern":
            ab = res[2]
        t0 = time.perf_counter()
        for _ in range(args.steps):
            fn()
        side[name] = {"fields_per_s": n * args.steps / (time.perf_counter() - t0)}
    t0 = time.perf_counter()
    retrieval.get_aberration_pattern(cbs.derive_optical_tool(fp, cbs.Prec(True)), fin[..., :7], fout[..., :7],
                                     dict(cp, k0s=k0s[:, :7]))
    side["get_aberration_pattern"]["cpu_port_fields_per_s"] = 7 / (time.perf_counter() - t0)
    print(json.dumps({
        "metric": "holograms/s", "value": n / dt, "unit": "holograms/s", "higher_is_better": True,
        "ms_per_stack": dt * 1e3, "steps": args.steps, "warmup": args.warmup, "clocks": clocks,
        "config": {"workload": "FIELD_EXPERIMENTAL_RETRIEVAL.get_fields: %d background / sample off-axis "
                               "holograms of %d x %d, 0.0625 um camera pixel, 0.1 um output" % (n, N, N)},
        "cpu_baseline": {"value": 2 / dtc, "unit": "holograms/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": "2 holograms"},
        "field_steps": {"config": "%d synthetic aberrated field pairs of %d x %d through the host API "
                                  "(host arrays in and out); CPU port on 7 pairs" % (n, L, L), **side}}), flush=True)


def workload_key():
    return "cbs_forward_128cube_49ill"


def free_port():
    import socket

    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def rank_launch_cmd(n, argv, port):
    """torchrun command that starts n ranks of this script on one node, each
    with its own RANK / LOCAL_RANK / WORLD_SIZE (rendezvous on 127.0.0.1)."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
            "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + list(argv)


def launch_ranks(n, argv):
    """`bench.py --gpus N` started without a launcher: start N ranks (one
    process per GPU) and return their exit status."""
    env = dict(os.environ)
    env.setdefault("NCCL_NVLS_ENABLE", "0")
    return subprocess.run(["timeout", "-k", "60", "3000"] + rank_launch_cmd(n, argv, free_port()),
                          env=env).returncode


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-iters", type=int, default=16,
                    help="Born iterations in the bounded CPU sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip the plain single-solve comparison")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the 16-bit storage (b16) measurement")
    ap.add_argument("--n-ill", type=int, default=N_ILL,
                    help="illuminations per step (profiling runs use fewer)")
    ap.add_argument("--profile-run", action="store_true",
                    help="only run --warmup solves (for ncu captures) and exit")
    ap.add_argument("--retrieval", action="store_true",
                    help="time the field retrieval from off-axis holograms")
    ap.add_argument("--setup", action="store_true",
                    help="time the solver constructor (Green's kernels on the GPU vs the host)")
    ap.add_argument("--bpm", action="store_true",
                    help="time the beam-propagation forward solver")
    ap.add_argument("--fista", action="store_true",
                    help="time FISTA outer iterations of the inverse solver (device vs host loop)")
    ap.add_argument("--grid-lengths", nargs="*", type=int, default=None, metavar="RI_SIZE",
                    help="time the Born loop on padded grids of 96^3, 127^3 (Bluestein), 128^3, 136^3, 152^3 "
                         "and 160^3 (RI sizes 72, 103, 104, 112, 128, 136; give some of them to time only those)")
    ap.add_argument("--print-rank-env", action="store_true",
                    help="print each rank's RANK / LOCAL_RANK / WORLD_SIZE and exit (launcher check)")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(launch_ranks(args.gpus, sys.argv[1:]))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.print_rank_env:
        print(json.dumps({"rank": rank, "local_rank": local_rank, "world": world, "gpus": args.gpus}),
              flush=True)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.fista:
        run_fista(args)
        return
    if args.bpm:
        run_bpm(args)
        return
    if args.setup:
        run_setup(args)
        return
    if args.retrieval:
        run_retrieval(args)
        return
    if args.grid_lengths is not None:
        run_grid_lengths(args)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
