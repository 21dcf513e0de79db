"""Data-parallel gradient of BACKWARD_SOLVER_MULTI_MULTI_GPU without a GPU:
the reference's split of the scan list into per-worker shares
(BACKWARD_SOLVER_MULTI_MULTI_GPU.m:76-83) and the count-weighted all-reduce
(:92-115), run as 2 and 3 gloo ranks on CPU (127.0.0.1) with a stand-in for
the per-share GPU gradient, against the same computation in one process."""
import os
import socket
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


def _fake_gradient(fields_in, fields_out):
    """Stand-in for one share's odt_gradient: mean over the share of a
    per-field array, and the summed misfit."""
    g = np.mean(fields_in[:, :, 0, :, None] * np.conj(fields_out[:, :, 0, :, None]), axis=2)
    g = np.repeat(g, 3, axis=2).astype(np.complex64)
    err = float(np.sum(np.abs(fields_in - fields_out) ** 2))
    return g, err


def _params(n_scan):
    from inverse_solver_b200.backward import BACKWARD_SOLVER_MULTI

    p = BACKWARD_SOLVER_MULTI.get_default_parameters(dict(num_scan_per_iteration=n_scan, seed=3))
    p["forward_solver_parameters"] = dict(return_transmission=True, return_reflection=True,
                                          return_3D=True)
    return p


def _inputs(npol=1):
    """Fields [F_x, F_y, npol, n]: npol = 2 for dyadic (vector) solvers, whose
    shares split along the illumination axis the same way."""
    rng = np.random.default_rng(1)
    shp = (6, 5, npol, 7)
    a = (rng.standard_normal(shp) + 1j * rng.standard_normal(shp)).astype(np.complex64)
    b = (rng.standard_normal(shp) + 1j * rng.standard_normal(shp)).astype(np.complex64)
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
                return (None, 0.0) if fi.shape[3] == 0 else _fake_gradient(fi, fo)

        s = Stub(_params(n_scan), init_solver=False)
        a, b = _inputs(npol)
        g, e = s.get_gradiant(np.ones((6, 5, 3), np.complex64), a, b)
        g2, e2 = s.get_gradiant(np.ones((6, 5, 3), np.complex64), a, b)   # second draw of the scan list
        np.savez(os.path.join(outdir, f"r{rank}.npz"), g=g, e=e, g2=g2, e2=e2)
    finally:
        dist.destroy_process_group()


def _expected(world, n_scan, npol):
    """The reference's computation in one process."""
    from inverse_solver_b200.backward import BACKWARD_SOLVER_MULTI

    s = BACKWARD_SOLVER_MULTI(_params(n_scan), init_solver=False)
    a, b = _inputs(npol)
    res = []
    for _ in range(2):
        sl = s.scan_list(a.shape[3])
        n = len(sl)
        g = 0
        e = 0.0
        for lo, hi in shard_ranges(n, world):
            if hi > lo:
                gi, ei = _fake_gradient(a[:, :, :, sl[lo:hi]], b[:, :, :, sl[lo:hi]])
                g = g + gi * np.float32(hi - lo)
                e += ei * (hi - lo)
        res.append(((g / np.float32(n)).astype(np.complex64), e / n))
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
    for o in outs:   # every rank holds the same reduced gradient
        np.testing.assert_allclose(o["g"], g, rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(o["g2"], g2, rtol=1e-6, atol=1e-6)
        assert abs(float(o["e"]) - e) <= 1e-9 * abs(e) and abs(float(o["e2"]) - e2) <= 1e-9 * abs(e2)
    assert np.array_equal(outs[0]["g"], outs[-1]["g"])
