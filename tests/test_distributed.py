"""Data-parallel gradient of BACKWARD_SOLVER_MULTI_MULTI_GPU without a GPU:
the reference's split of the scan list into per-worker shares
(BACKWARD_SOLVER_MULTI_MULTI_GPU.m:76-83) and the count-weighted all-reduce
(:92-115), run as 2 and 3 gloo ranks on CPU (127.0.0.1).  Each rank computes
its share's gradient with the oracle's get_gradiant_static
(BACKWARD_SOLVER_MULTI.m:30-54, forward + adjoint CBS solves on a tiny grid,
single precision) where the GPU ranks call odt_gradient; the all-reduced
gradient must equal the single-process gradient over all selected
illuminations.  Also: `bench.py --gpus N` started without a launcher starts
N ranks, each with its own RANK / LOCAL_RANK / WORLD_SIZE."""
import json
import os
import socket
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from inverse_solver_b200.distributed import shard_ranges


def test_shards_follow_reference_rounding():
    # nd = round(ii * 49 / 8): 6, 12, 18, 25 (24.5 rounds away), 31, 37, 43, 49
    assert [b - a for a, b in shard_ranges(49, 8)] == [6, 6, 6, 7, 6, 6, 6, 6]
    assert shard_ranges(3, 4) == [(0, 1), (1, 2), (2, 2), (2, 3)]
    for n, w in [(1, 1), (5, 2), (49, 3), (98, 8), (7, 7), (2, 5)]:
        sh = shard_ranges(n, w)
        covered = [i for a, b in sh for i in range(a, b)]
        assert covered == list(range(n))


TINY = [10, 10, 5]     # RI grid of the gradient case (padded 14 x 14 x 9)


def _tiny_params(npol):
    import cases

    p = cases.params(TINY, [1, 1, 1], return_transmission=True, return_reflection=True, return_3D=True)
    p["vector_simulation"] = npol == 2
    return p


def _oracle_gradient(fields_in, fields_out, npol):
    """One share's gradient and summed misfit: the oracle's
    get_gradiant_static (single precision), the computation odt_gradient
    fuses on the GPU."""
    from oracle import cbs, multi

    fwd = cbs.ForwardSolverCBS(_tiny_params(npol), single=True)
    g, e = multi.get_gradient_static(_tiny_RI(), fields_in, fields_out, fwd)
    return np.asarray(g, np.complex64), float(e)


def _tiny_RI():
    import cases

    return cases.sphere_phantom(TINY, [0.1] * 3, cases.NM, seed=4, n_spheres=1, radius_um=(0.2, 0.3))


def _params(n_scan):
    from inverse_solver_b200.backward import BACKWARD_SOLVER_MULTI

    p = BACKWARD_SOLVER_MULTI.get_default_parameters(dict(num_scan_per_iteration=n_scan, seed=3))
    p["forward_solver_parameters"] = dict(return_transmission=True, return_reflection=True,
                                          return_3D=True)
    return p


def _inputs(npol=1):
    """Fields [F_x, F_y, npol, 5] on the tiny grid: plane waves on a circle
    (npol = 2 for dyadic solvers, whose shares split along the illumination
    axis the same way) and "measured" fields that differ from the model's."""
    import cases

    f = cases.circle_fields(cases.params(TINY, [1, 1, 1]), 5)
    a = np.zeros((TINY[0], TINY[1], npol, 5), np.complex64)
    a[:, :, 0, :] = f[:, :, 0, :]
    if npol == 2:
        a[:, :, 1, 1::2] = f[:, :, 0, 1::2] * np.float32(0.5)
    rng = np.random.default_rng(1)
    b = (a * np.float32(0.9) + np.float32(0.05) * (rng.standard_normal(a.shape)
                                                    + 1j * rng.standard_normal(a.shape))).astype(np.complex64)
    return a, b


def _worker(rank, world, port, outdir, n_scan, npol):
    import torch.distributed as dist
    from datetime import timedelta

    from inverse_solver_b200.distributed import BACKWARD_SOLVER_MULTI_MULTI_GPU

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=timedelta(seconds=60))
    try:
        class Stub(BACKWARD_SOLVER_MULTI_MULTI_GPU):
            def local_gradient(self, RI, fi, fo):
                return (None, 0.0) if fi.shape[3] == 0 else _oracle_gradient(fi, fo, npol)

        s = Stub(_params(n_scan), init_solver=False)
        a, b = _inputs(npol)
        RI = _tiny_RI()
        g, e = s.get_gradiant(RI, a, b)
        g2, e2 = s.get_gradiant(RI, a, b)   # second draw of the scan list
        np.savez(os.path.join(outdir, f"r{rank}.npz"), g=g, e=e, g2=g2, e2=e2)
    finally:
        dist.destroy_process_group()


def _expected(world, n_scan, npol):
    """One process: the gradient over all selected illuminations at once
    (the mean in get_gradiant_static), and the reference's count-weighted
    error of the shares (:100-115)."""
    from inverse_solver_b200.backward import BACKWARD_SOLVER_MULTI

    s = BACKWARD_SOLVER_MULTI(_params(n_scan), init_solver=False)
    a, b = _inputs(npol)
    res = []
    for _ in range(2):
        sl = s.scan_list(a.shape[3])
        n = len(sl)
        g, _ = _oracle_gradient(a[:, :, :, sl], b[:, :, :, sl], npol)
        e = 0.0
        for lo, hi in shard_ranges(n, world):
            if hi > lo:
                e += _oracle_gradient(a[:, :, :, sl[lo:hi]], b[:, :, :, sl[lo:hi]], npol)[1] * (hi - lo)
        res.append((g, e / n))
    return res


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


@pytest.mark.parametrize("world,n_scan,npol", [(2, 0, 1), (3, 0, 1), (2, 4, 1), (2, 0, 2)])
def test_gloo_ranks_match_single_process(world, n_scan, npol):
    import torch.multiprocessing as mp

    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(world, _free_port(), d, n_scan, npol), nprocs=world, join=True,
                           start_method="spawn")
        outs = [np.load(os.path.join(d, f"r{r}.npz")) for r in range(world)]
    (g, e), (g2, e2) = _expected(world, n_scan, npol)
    from oracle.cbs import rel_l2

    for o in outs:   # every rank holds the single-process gradient (float32 sums in another order)
        assert rel_l2(o["g"], g) < 1e-5 and rel_l2(o["g2"], g2) < 1e-5
        assert abs(float(o["e"]) - e) <= 1e-9 * abs(e) and abs(float(o["e2"]) - e2) <= 1e-9 * abs(e2)
    assert np.linalg.norm(g) > 0
    assert np.array_equal(outs[0]["g"], outs[-1]["g"])


def test_bench_gpus_n_starts_n_ranks():
    """`python bench.py --gpus 2` without torchrun: two child processes,
    ranks 0 and 1 of a world of 2 (checked before any GPU work)."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--gpus", "2", "--print-rank-env"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert sorted((d["rank"], d["local_rank"], d["world"]) for d in lines) == [(0, 0, 2), (1, 1, 2)]


def test_bench_grid_lengths_rejects_unknown_size():
    """`python bench.py --grid-lengths 100`: the RI size is not one of the
    timed cases, so the run stops with a message naming them, before any GPU
    work."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--grid-lengths", "100"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode != 0
    assert "--grid-lengths takes RI sizes from [72, 103, 104, 112, 128, 136]" in r.stderr
