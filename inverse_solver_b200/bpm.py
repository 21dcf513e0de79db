"""Beam-propagation forward solver (Codes/FORWARD_SOLVER_BPM.m) on the B200
library: the host computes set_RI's tables in MATLAB single semantics
(:23-44) and the refocusing phases of solve (:93-95, :110-114); the slice
loop, the 2D FFTs, the cosine correction (:58-63) and the optional 3D field
run on the GPU (odt_bpm_solve).  The tables are uploaded once per set_RI and
each solve moves only its fields."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from .optics import C64, F32, OpticalTool, basic_optical_parameter, update_struct


class FORWARD_SOLVER_BPM:
    """Codes/FORWARD_SOLVER_BPM.m: scalar beam propagation, one slice per z
    of the RI grid (whose xy size is the field size)."""

    @staticmethod
    def get_default_parameters(init_params=None):
        """FORWARD_SOLVER.m:9-20 + FORWARD_SOLVER_BPM.m:9-19."""
        p = basic_optical_parameter()
        p.update(return_transmission=True, return_reflection=False, return_3D=False, use_GPU=True)
        p.update(iterations_number=-1, use_GPU=True, cos_correction=True)
        return update_struct(p, init_params) if init_params else p

    def __init__(self, params):
        """FORWARD_SOLVER_BPM.m:21-23 (DERIVE_OPTICAL_TOOL of the parameters)."""
        self.parameters = dict(params)
        self.utility = OpticalTool(self.parameters)
        self.lib = _lib.load()
        self.RI = None

    def set_RI(self, RI):
        """:23-44 in single precision."""
        p, u = self.parameters, self.utility
        RI = np.asarray(RI)
        RI = RI.astype(C64 if np.iscomplexobj(RI) else F32)
        if RI.ndim != 3 or list(RI.shape[:2]) != [int(p["size"][0]), int(p["size"][1])]:
            raise ValueError("the RI must be [size(1), size(2), Nz]")
        self.RI = RI
        c = 1j * 2 * math.pi * u.k0
        self.field_multiplier = ((c * (RI - p["RI_bg"])).astype(C64) * p["resolution"][2]).astype(C64)
        self.filter_out = np.fft.ifftshift(u.NA_circle).astype(F32)
        rk = np.asarray(u.refocusing_kernel, dtype=C64)
        self.refocus_kernel = np.fft.ifftshift((np.exp((rk * p["resolution"][2]).astype(C64)) * u.NA_circle)
                                               .astype(C64))
        self._dev = None   # device copies of the tables, made by the first solve

    def _device_tables(self):
        """The RI-dependent tables and the slice-independent phases in device
        memory (column-major), uploaded once per set_RI."""
        import torch

        if self._dev is None:
            dev = torch.device("cuda", int(self.parameters.get("used_gpu", 0)))

            def up(a, dt):
                return torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=dt).ravel(order="F"))).to(dev)

            pre, post = self._phases()
            self._dev = dict(fm=up(self.field_multiplier, C64), rk=up(self.refocus_kernel, C64),
                             fo=up(self.filter_out, F32), pre=up(pre, C64), post=up(post, C64),
                             ct=up(self.utility.cos_theta, F32), device=dev)
        return self._dev

    def _phases(self):
        p, u = self.parameters, self.utility
        nz = self.field_multiplier.shape[2]
        rk = (np.asarray(u.refocusing_kernel, dtype=C64) * p["resolution"][2]).astype(C64)
        pre = np.exp((rk * (-math.floor(nz / 2) - 1)).astype(C64)).astype(C64)
        post = np.exp((rk * (-(nz - math.floor(nz / 2) - 1))).astype(C64)).astype(C64)
        return pre, post

    def solve_device(self, fields_in, trans, stream=None):
        """Device-resident solve: fields_in / trans contiguous complex64 CUDA
        tensors of F_x*F_y*n_ill elements (column-major [F_x, F_y, n_ill]);
        transmitted field only.  Work is queued on ``stream`` (default: the
        current torch stream) and the call returns without synchronising."""
        import torch

        n1, n2, nz = self.field_multiplier.shape
        plane = n1 * n2
        for t in (fields_in, trans):
            if not t.is_cuda or not t.is_contiguous() or t.dtype != torch.complex64:
                raise ValueError("solve_device expects contiguous complex64 CUDA tensors")
        nill = fields_in.numel() // plane
        if nill < 1 or fields_in.numel() != nill * plane or trans.numel() != fields_in.numel():
            raise ValueError("fields must be [F_x, F_y, n] alike")
        d = self._device_tables()
        a = _lib.BPMArgs()
        a.size[:] = [n1, n2, nz]
        a.field_multiplier, a.refocus_kernel = d["fm"].data_ptr(), d["rk"].data_ptr()
        a.filter_out = d["fo"].data_ptr()
        a.pre, a.post = d["pre"].data_ptr(), d["post"].data_ptr()
        a.cos_theta = d["ct"].data_ptr() if self.parameters["cos_correction"] else None
        a.fields_in = fields_in.data_ptr()
        a.n_ill = nill
        a.trans = trans.data_ptr()
        a.field3d = None
        a.memory = _lib.ODT_MEM_DEVICE
        if stream is None:
            stream = torch.cuda.current_stream(fields_in.device)
        a.stream = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        _lib.check(self.lib.odt_bpm_solve(C.byref(a)))

    def solve(self, input_field):
        """:45-117 -> (fields_trans, fields_ref, fields_3D); fields_ref is
        the reference's untouched ones(...) array when return_reflection."""
        if self.RI is None:
            raise RuntimeError("call set_RI first")
        p = self.parameters
        f = np.asarray(input_field)
        if f.ndim == 3:
            f = f[:, :, :, None]
        if f.shape[2] > 1:
            if f.shape[2] != 2:
                raise ValueError("must give far field polarisation with 2 pols only")
            raise ValueError("Look at the old version for polarised version but it is useless")
        n1, n2, nz = self.field_multiplier.shape
        if list(f.shape[:2]) != [n1, n2]:
            raise ValueError("input fields must be [size(1), size(2), 1, n]")
        import torch

        nill = f.shape[3]
        d = self._device_tables()
        dev = d["device"]
        fin = torch.from_numpy(np.ascontiguousarray(np.asarray(f[:, :, 0, :], dtype=C64).transpose(2, 1, 0))).to(dev)
        trans_d = torch.empty_like(fin)
        f3_d = torch.empty((nill, nz, n2, n1), dtype=torch.complex64, device=dev) if p["return_3D"] else None
        a = _lib.BPMArgs()
        a.size[:] = [n1, n2, nz]
        a.field_multiplier, a.refocus_kernel = d["fm"].data_ptr(), d["rk"].data_ptr()
        a.filter_out = d["fo"].data_ptr()
        a.pre, a.post = d["pre"].data_ptr(), d["post"].data_ptr()
        a.cos_theta = d["ct"].data_ptr() if p["cos_correction"] else None
        a.fields_in = fin.data_ptr()
        a.n_ill = nill
        a.trans = trans_d.data_ptr()
        a.field3d = f3_d.data_ptr() if f3_d is not None else None
        a.memory = _lib.ODT_MEM_DEVICE
        s = torch.cuda.current_stream(dev)
        a.stream = s.cuda_stream
        _lib.check(self.lib.odt_bpm_solve(C.byref(a)))
        trans = trans_d.cpu().numpy().transpose(2, 1, 0)
        f3 = f3_d.cpu().numpy().transpose(3, 2, 1, 0) if f3_d is not None else None
        fields_trans = trans[:, :, None, :]
        fields_ref = np.ones(fields_trans.shape, dtype=C64) if p["return_reflection"] else None
        fields_3D = f3[:, :, :, None, :] if f3 is not None else None
        return fields_trans, fields_ref, fields_3D
