"""BACKWARD_SOLVER_RYTOV and OVERLAP_COUNTER on the B200 library.

Mirrors Codes/BACKWARD_SOLVER_RYTOV.m (Rytov field -> Ewald-sphere scatter ->
normalise -> ifftn -> RI), the overlap counting of
Codes/BACKWARD_SOLVER_RYTOV_precompute.m:87-137 and Codes/OVERLAP_COUNTER.m
(whose get_overlap calls a solve that has no overlap_3D in the reference; the
counting it intends is the _precompute one, done here).  All per-pixel work
runs in odt_rytov on the GPU; the host computes DERIVE_OPTICAL_TOOL's grids.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from .optics import C64, F32, OpticalTool, basic_optical_parameter, update_struct


def _f(x, dt):
    return np.asfortranarray(np.asarray(x, dtype=dt))


def vector2scalarfield(input_field, output_field):
    """sub_code/vector2scalarfield.m for one polarisation (pass-through)."""
    if input_field.shape[2] != 1:
        raise NotImplementedError("two-polarisation fields are not supported")
    return input_field[:, :, 0, :], output_field[:, :, 0, :]


class BACKWARD_SOLVER_RYTOV:
    @staticmethod
    def get_default_parameters(init_params=None):
        """BACKWARD_SOLVER_RYTOV.m:6-16 (+ ``unwrap``: the phase unwrapper,
        default the GPU Goldstein unwrapper of unwrapp2_gpu.m)."""
        p = basic_optical_parameter()
        p.update(use_non_negativity=False, non_negativity_iteration=100)
        return update_struct(p, init_params) if init_params else p

    def __init__(self, params):
        self.parameters = params
        self.ORytov = None
        self.count = None

    def _check(self, input_field, output_field):
        p = self.parameters
        if input_field.ndim != 4:
            raise ValueError("You need to provide the field with 4 dimenssion")
        if input_field.shape[0] != input_field.shape[1]:
            raise ValueError("Please input a square field")
        if input_field.shape != output_field.shape:
            raise ValueError("Please input field and bg of same size")
        if p["resolution"][0] != p["resolution"][1]:
            raise ValueError("x/y input resolution must be isotropic")
        if p["size"][0] != p["size"][1]:
            raise ValueError("x/y output size must be isotropic")
        if p["size"][0] != input_field.shape[0] or p["size"][1] != input_field.shape[1]:
            raise ValueError("declare size in the parameter must be the same as the field size")

    def _run(self, bg, sp, phase, count_one, nn_iter, want_ri=True, want_overlap=False):
        p = self.parameters
        u = OpticalTool(p)
        N = [int(v) for v in p["size"]]
        n = bg.shape[2]
        a = _lib.RytovArgs()
        a.size[:] = N
        a.resolution[:] = [float(r) for r in p["resolution"]]
        a.fourier_res[:] = u.fourier_res
        a.k0_nm, a.ri_bg, a.wavelength = u.k0_nm, float(p["RI_bg"]), float(p["wavelength"])
        keep = [_f(u.fourier_coor[0], F32), _f(u.fourier_coor[1], F32), _f(u.k3, F32),
                _f(u.NA_circle, np.uint8), _f(u.coorxy < (2 * p["NA"] / p["wavelength"]), np.uint8),
                _f(bg, C64), _f(sp, C64) if sp is not None else None,
                _f(phase, F32) if phase is not None else None]
        a.coor1, a.coor2, a.k3, a.na_circle, a.emask, a.bg, a.sp, a.phase = [_lib.ptr(k) for k in keep]
        a.n_ill = n
        a.count_one = 1 if count_one else 0
        a.non_negativity_iteration = int(nn_iter)
        RI = np.empty(N, dtype=C64, order="F") if want_ri else None
        O = np.empty(N, dtype=C64, order="F")
        cnt = np.empty(N, dtype=F32, order="F")
        ov = np.empty((N[0], N[1], n), dtype=F32, order="F") if want_overlap else None
        sh = np.zeros(2 * n, dtype=np.int32)
        a.RI, a.ORytov, a.count, a.overlap_field = (_lib.ptr(RI), _lib.ptr(O), _lib.ptr(cnt),
                                                    _lib.ptr(ov))
        a.shifts = sh.ctypes.data
        a.memory = _lib.ODT_MEM_HOST
        a.stream = None
        _lib.check(_lib.load().odt_rytov(C.byref(a)))
        return RI, O, cnt, ov, sh.reshape(n, 2)

    def solve(self, input_field, output_field, unwrapped_phase=None):
        """:22-127; ``unwrapped_phase`` overrides the unwrapping of
        angle(sp./bg) (the reference unwraps with unwrapp2_gpu, :49)."""
        input_field = np.asarray(input_field)
        output_field = np.asarray(output_field)
        self._check(input_field, output_field)
        bg, sp = vector2scalarfield(input_field, output_field)
        if unwrapped_phase is None:
            from .unwrap import unwrapp2_gpu
            wrapped = np.angle((sp.astype(C64) / bg.astype(C64))).astype(F32)
            unwrapped_phase = unwrapp2_gpu(wrapped)
        p = self.parameters
        nn = p["non_negativity_iteration"] if p["use_non_negativity"] else 0
        RI, O, cnt, _, _ = self._run(bg, sp, unwrapped_phase, False, nn)
        self.ORytov, self.count = O, cnt
        return RI


class OVERLAP_COUNTER(BACKWARD_SOLVER_RYTOV):
    """OVERLAP_COUNTER.m:1-25 with the counting of
    BACKWARD_SOLVER_RYTOV_precompute.m:87-137."""

    def get_overlap(self, input_field):
        input_field = np.asarray(input_field)
        self._check(input_field, input_field)
        bg, _ = vector2scalarfield(input_field, input_field)
        _, _, cnt, ov, _ = self._run(bg, None, None, True, 0, want_ri=False, want_overlap=True)
        return cnt, ov
