"""Data-parallel BACKWARD_SOLVER_MULTI over several GPUs.

Mirrors Codes/BACKWARD_SOLVER_MULTI_MULTI_GPU.m: the illuminations of an
outer iteration are split into contiguous shares, one per GPU (:70-84); each
GPU computes the gradient of its share (forward + adjoint CBS solves, fused
in odt_gradient); the shares are combined as the count-weighted mean of the
gradients and of the errors (:92-115).

The reference runs one MATLAB worker per GPU and moves the gradients through
host queues.  Here every GPU has its own process (torch.distributed; NCCL
between GPUs, gloo on CPU), every rank runs the same FISTA outer loop, and
the one exchange per outer iteration is a sum all-reduce of
count * gradient (the RI-sized complex array) and count * err.  All ranks
therefore hold the same reconstruction after every iteration.
"""
from __future__ import annotations

import math

import numpy as np

from .backward import BACKWARD_SOLVER_MULTI
from .optics import C64


def mround(x):
    """MATLAB round (half away from zero) of a non-negative value."""
    return int(math.floor(x + 0.5))


def shard_ranges(num_fields, num_worker):
    """Contiguous shares of the scan list per worker, 0-based half-open
    (start, stop), as BACKWARD_SOLVER_MULTI_MULTI_GPU.m:76-83 forms them
    (nd = round(ii * num_fields / num_worker)); workers whose share is empty
    get (s, s)."""
    out = []
    st = 1
    for ii in range(1, num_worker + 1):
        nd = mround(ii * num_fields / num_worker)
        if nd >= st and st <= num_fields:
            out.append((st - 1, nd))
            st = nd + 1
        else:
            out.append((st - 1, st - 1))
    return out


def allreduce_sum(arrays, group=None):
    """Sum numpy arrays over the ranks of the process group in one collective
    per precision: complex64 / float32 arrays travel together as float32
    (complex as (re, im) pairs), float64 arrays together as float64.  With the
    NCCL backend the buffers are CUDA tensors on the rank's current device."""
    import torch
    import torch.distributed as dist

    nccl = dist.get_backend(group) == "nccl"
    out = [None] * len(arrays)
    for wide in (False, True):
        idx = [i for i, a in enumerate(arrays) if (np.asarray(a).dtype == np.float64) == wide]
        if not idx:
            continue
        dt = np.float64 if wide else np.float32
        flat = []
        for i in idx:
            a = np.ascontiguousarray(arrays[i])
            flat.append(a.view(np.float32).ravel() if np.iscomplexobj(a) else a.astype(dt).ravel())
        buf = torch.from_numpy(np.concatenate(flat))
        if nccl:
            buf = buf.cuda()
        dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
        buf = buf.cpu().numpy()
        o = 0
        for i, f in zip(idx, flat):
            part = buf[o:o + f.size]
            o += f.size
            shape = np.shape(arrays[i])
            out[i] = part.view(np.complex64).reshape(shape) if np.iscomplexobj(arrays[i]) else part.reshape(shape)
    return out


class BACKWARD_SOLVER_MULTI_MULTI_GPU(BACKWARD_SOLVER_MULTI):
    """BACKWARD_SOLVER_MULTI with the gradient of each outer iteration
    computed data-parallel across the ranks of torch.distributed's default
    process group (one process per GPU; the forward solver of each rank runs
    on its own device, ``forward_solver_parameters['used_gpu']``).  The scan
    list is drawn identically on every rank (seeded)."""

    def __init__(self, params, init_solver=True, group=None):
        import torch.distributed as dist

        super().__init__(params, init_solver=init_solver)
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def _use_device_loop(self):
        """Device-resident outer loop with the NCCL backend (the gradient is
        all-reduced in device memory); the host-array loop with gloo."""
        import torch.distributed as dist

        return super()._use_device_loop() and dist.get_backend(self.group) == "nccl"

    def _device_gradient(self, fs, fields_in, fields_meas, grad, n_sel):
        """:66-116 on device arrays: this rank's share of the selected
        illuminations, its gradient weighted by the share size, one sum
        all-reduce of the gradient and one of the weighted error."""
        import torch
        import torch.distributed as dist

        nF = fields_in.numel() // n_sel
        a, b = shard_ranges(n_sel, self.world)[self.rank]
        cnt = b - a
        e = 0.0
        if cnt > 0:
            e = fs.gradient_device(fields_in[a * nF:b * nF], fields_meas[a * nF:b * nF], grad)
            grad.mul_(float(cnt))
        else:
            grad.zero_()
        dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=self.group)
        grad.div_(float(n_sel))
        et = torch.tensor([e * cnt], dtype=torch.float64, device=grad.device)
        dist.all_reduce(et, op=dist.ReduceOp.SUM, group=self.group)
        return float(et.item()) / n_sel

    def local_gradient(self, RI, input_field, output_field):
        """Gradient and error of one share (get_gradiant_static); None for an
        empty share."""
        if input_field.shape[3] == 0:
            return None, 0.0
        return self.get_gradiant_static(RI, input_field, output_field, self.forward_solver)

    def get_gradiant(self, RI, input_field, output_field):
        """:66-116: split, compute the local share, weighted all-reduce."""
        sl = self.scan_list(input_field.shape[3])
        n = len(sl)
        a, b = shard_ranges(n, self.world)[self.rank]
        mine = sl[a:b]
        g, e = self.local_gradient(RI, input_field[:, :, :, mine], output_field[:, :, :, mine])
        cnt = b - a
        if g is None:
            g = np.zeros(np.asarray(RI).shape[:3], dtype=C64)
        # the reference weights each share's mean gradient and summed error by
        # the share's size and divides by the number of fields (:100-115)
        gsum, esum = allreduce_sum([np.asarray(g, dtype=C64) * np.float32(cnt),
                                    np.array([e * cnt], dtype=np.float64)], self.group)
        return (gsum / np.float32(n)).astype(C64), float(esum[0]) / n
