"""CPU restatement of the beam-propagation forward solver
(Codes/FORWARD_SOLVER_BPM.m) -- test infrastructure (the oracle): only the
tests, the smoke check and the benchmark's CPU baseline import it.

Follows FORWARD_SOLVER_BPM.m line by line in MATLAB single precision (or
double with ``single=False``): set_RI :23-44 (field multiplier, output
filter, ifftshifted refocus kernel), solve :45-117 (cosine correction from
the peak of each illumination's centred spectrum, refocus to the first slice,
the slice loop of :97-109, refocus back to the focal plane).  Parity is
unpinned: the reference ships no outputs for this path.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.fft as sfft

from .cbs import Prec, basic_optical_parameter, derive_optical_tool, fftc2, update_struct


def bpm_default_parameters(init=None):
    """FORWARD_SOLVER.m:9-20 + FORWARD_SOLVER_BPM.m:9-19."""
    p = basic_optical_parameter()
    p.update(return_transmission=True, return_reflection=False, return_3D=False, use_GPU=True)
    p.update(iterations_number=-1, use_GPU=True, cos_correction=True)
    if init is not None:
        p = update_struct(p, init)
    return p


def _fft2(x, inverse=False):
    return (sfft.ifft2 if inverse else sfft.fft2)(x, axes=(0, 1))


class ForwardSolverBPM:
    def __init__(self, params, single=True):
        self.parameters = dict(params)
        self.P = Prec(single)
        self.u = derive_optical_tool(self.parameters, self.P)

    def set_RI(self, RI):
        """:23-44."""
        P, u, p = self.P, self.u, self.parameters
        RI = P.S(np.asarray(RI)) if self.P.single else np.asarray(RI, dtype=np.complex128)
        self.RI = RI
        c = 1j * 2 * math.pi * u["k0"]
        self.field_multiplier = P.C(P.S(P.S(c * (RI - p["RI_bg"])) * p["resolution"][2]))
        self.filter_out = np.fft.ifftshift(u["NA_circle"])
        rk = P.C(u["refocusing_kernel"])
        self.refocus_kernel = np.fft.ifftshift(P.C(np.exp(P.C(rk * p["resolution"][2])) * u["NA_circle"]))

    def cos_coeffs(self, input_field):
        """:58-63: cos_theta at the first maximum (column-major) of |centred spectrum| per illumination."""
        spec = np.abs(fftc2(input_field))
        n = spec.shape[3]
        out = np.empty(n, dtype=self.P.r)
        ct = np.asarray(self.u["cos_theta"]).ravel(order="F")
        for k in range(n):
            out[k] = ct[int(np.argmax(spec[:, :, :, k].ravel(order="F"))) % ct.size]
        return out

    def solve(self, input_field):
        """:45-117 -> (fields_trans, fields_ref, fields_3D)."""
        P, u, p = self.P, self.u, self.parameters
        f = P.C(np.asarray(input_field))
        if f.ndim == 3:
            f = f[:, :, :, None]
        if f.shape[2] > 1:
            raise ValueError("must give far field polarisation with 2 pols only")
        fm = self.field_multiplier
        nz = fm.shape[2]
        cos = self.cos_coeffs(f) if p["cos_correction"] else None
        ref = np.ones(f.shape, dtype=P.c) if p["return_reflection"] else None
        f3 = np.ones((f.shape[0], f.shape[1], nz, 1, f.shape[3]), dtype=P.c) if p["return_3D"] else None
        rk = P.C(u["refocusing_kernel"])
        dz = p["resolution"][2]
        f = P.C(fftc2(f))
        f = P.C(f * P.C(np.exp(P.C(P.C(rk * dz) * (-math.floor(nz / 2) - 1))))[:, :, None, None])
        f = P.C(fftc2(f, inverse=True))
        f = P.C(_fft2(f))
        for step in range(nz):
            f = P.C(f * self.refocus_kernel[:, :, None, None])
            f = P.C(_fft2(f, inverse=True))
            if cos is not None:
                e = P.C((P.R(1) / cos)[None, None, None, :] * fm[:, :, step][:, :, None, None])
            else:
                e = fm[:, :, step][:, :, None, None]
            f = P.C(f * P.C(np.exp(e)))
            f = P.C(_fft2(f))
            if f3 is not None:
                f3[:, :, step, :, :] = P.C(_fft2(f * self.filter_out[:, :, None, None], inverse=True))
        f = P.C(_fft2(f, inverse=True))
        f = P.C(fftc2(f))
        f = P.C(f * P.C(np.exp(P.C(P.C(rk * dz) * (-(nz - math.floor(nz / 2) - 1)))))[:, :, None, None])
        f = P.C(fftc2(f, inverse=True))
        return f, ref, f3
