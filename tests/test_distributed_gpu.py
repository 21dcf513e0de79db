"""BACKWARD_SOLVER_MULTI_MULTI_GPU on the GPU: one rank with an NCCL process
group (127.0.0.1) -- the all-reduce runs on a CUDA buffer -- gives the same
gradient as BACKWARD_SOLVER_MULTI.get_gradiant; with two illumination shares
emulated in one process (each share's fused gradient weighted by its size)
the combination equals the one-share gradient to single precision; the
device-resident outer loop (gradient all-reduced in device memory) gives the
single-process device loop's reconstruction."""
import socket
from datetime import timedelta

import numpy as np
import pytest

import cases
from oracle import cbs

pytestmark = pytest.mark.gpu


def _port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def test_single_rank_nccl_gradient_matches_plain_solver():
    import torch
    import torch.distributed as dist

    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN
    from inverse_solver_b200.backward import BACKWARD_SOLVER_MULTI
    from inverse_solver_b200.distributed import BACKWARD_SOLVER_MULTI_MULTI_GPU, shard_ranges

    p = cases.small_params(return_transmission=True, return_reflection=True, return_3D=True)
    RI = cases.small_RI()
    fields = cases.circle_fields(p, 4)
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    meas, _, _ = o.solve(fields)
    RI0 = (RI * 0.7 + cases.NM * 0.3).astype(np.float32)
    bp = BACKWARD_SOLVER_MULTI.get_default_parameters(dict(forward_solver=FORWARD_SOLVER_CONVERGENT_BORN,
                                                           forward_solver_parameters=p))
    plain = BACKWARD_SOLVER_MULTI(bp)
    g_ref, e_ref = plain.get_gradiant(RI0, fields, meas)

    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_port()}", rank=0, world_size=1,
                            timeout=timedelta(seconds=60))
    try:
        dp = BACKWARD_SOLVER_MULTI_MULTI_GPU(bp)
        g, e = dp.get_gradiant(RI0, fields, meas)
        dp.delete()
    finally:
        dist.destroy_process_group()
    assert cbs.rel_l2(g, g_ref) < 1e-6 and abs(e - e_ref) <= 1e-6 * e_ref

    # two shares as two ranks would compute them
    acc, err = 0, 0.0
    for lo, hi in shard_ranges(4, 2):
        gs, es = plain.get_gradiant_static(RI0, fields[..., lo:hi], meas[..., lo:hi], plain.forward_solver)
        acc = acc + gs * np.float32(hi - lo)
        err += es * (hi - lo)
    plain.delete()
    assert cbs.rel_l2(acc / np.float32(4), g_ref) < 1e-5


def test_single_rank_nccl_device_loop_matches_single_process():
    import torch
    import torch.distributed as dist

    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN
    from inverse_solver_b200.backward import BACKWARD_SOLVER_MULTI
    from inverse_solver_b200.distributed import BACKWARD_SOLVER_MULTI_MULTI_GPU

    p = cases.small_params(return_transmission=True, return_reflection=True, return_3D=True)
    RI = cases.small_RI()
    fields = cases.circle_fields(p, 4)
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    meas, _, _ = o.solve(fields)

    class Blurred:
        def solve(self, input_field, output_field):
            return (RI * 0.5 + cases.NM * 0.5).astype(np.float32)

    bp = BACKWARD_SOLVER_MULTI.get_default_parameters(dict(
        RI_bg=cases.NM, wavelength=cases.LAM, NA=p["NA"], resolution=p["resolution"], size=p["size"],
        forward_solver=FORWARD_SOLVER_CONVERGENT_BORN, forward_solver_parameters=p, init_solver=Blurred(),
        step=0.01, tv_param=0.001, inner_itt=20, itter_max=2, use_non_negativity=True, nmin=cases.NM, nmax=1.5))
    b = BACKWARD_SOLVER_MULTI(bp)
    ref = b.solve(fields, meas)
    eref = list(b.err_list)
    b.delete()
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_port()}", rank=0, world_size=1,
                            timeout=timedelta(seconds=60))
    try:
        dp = BACKWARD_SOLVER_MULTI_MULTI_GPU(bp)
        assert dp._use_device_loop()
        got = dp.solve(fields, meas)
        egot = list(dp.err_list)
        dp.delete()
    finally:
        dist.destroy_process_group()
    assert cbs.rel_l2(got - cases.NM, ref - cases.NM) < 1e-6
    assert np.allclose(egot, eref, rtol=1e-6)
