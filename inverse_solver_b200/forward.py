"""FORWARD_SOLVER_CONVERGENT_BORN on the B200 library.

Same constructor / ``set_RI`` / ``solve`` surface and parameter struct as
Codes/FORWARD_SOLVER_CONVERGENT_BORN.m; the geometry-dependent setup is done
on the host in MATLAB single semantics (as the reference's CUDA variant does,
FORWARD_SOLVER_CONVERGENT_BORN_CUDA.m:18-63) and every illumination is solved
by libodt (include/odt.h) on the GPU.  There is no CPU path for the solve: if
the library is missing the constructor raises.

Arrays are numpy arrays indexed like MATLAB, ``a[x, y, z, pol, ill]``.
"""
from __future__ import annotations

import copy
import ctypes as C
import math

import numpy as np

from . import _lib
from .optics import (C64, F32, OpticalTool, basic_optical_parameter, centered_fft2,
                     centered_fftn, mround, polarisation_basis, potential2ri, ri2potential,
                     green_plane_maps, truncated_green_plus, truncated_green_radial, update_struct)


def _f32(x):
    return np.asfortranarray(np.asarray(x, dtype=F32))


def _c64(x):
    return np.asfortranarray(np.asarray(x, dtype=C64))


class CBSHostSetup:
    """Host-side part of FORWARD_SOLVER_CONVERGENT_BORN: everything the MATLAB
    class computes before the GPU takes over (Green's kernels, pupils, the
    padded potential and its separable tables).  Needs no GPU."""

    @staticmethod
    def get_default_parameters(init_params=None):
        """FORWARD_SOLVER.m:9-20 + FORWARD_SOLVER_CONVERGENT_BORN.m:32-45, plus
        the CUDA class's ``used_gpu`` (device ordinal) and this library's
        ``max_batch`` (illuminations resident per launch, 0 = automatic),
        ``mem_budget`` (bytes, 0 = half of free HBM) and ``field_storage``
        ("complex64", the reference's precision, or "b16": the Born loop's
        spectral array and Field_n in 16-bit block floating point, see
        odt_set_field_storage)."""
        p = basic_optical_parameter()
        p.update(return_transmission=True, return_reflection=False, return_3D=False,
                 use_GPU=True)
        p.update(iterations_number=-1, boundary_thickness=[6, 6, 6], boundary_sharpness=1,
                 verbose=False, acyclic=True, RI_xy_size=[0, 0], RI_center=[0, 0])
        p.update(used_gpu=0, max_batch=0, mem_budget=0, field_storage="complex64")
        return update_struct(p, init_params) if init_params else p

    # ------------------------------------------------------------ ctor
    def __init__(self, params):
        """Constructor (FORWARD_SOLVER_CONVERGENT_BORN.m:48-133)."""
        p = self.parameters = copy.deepcopy(params)
        # pole_num (:293-296): 3 field components with the dyadic Green's function
        self.vector = bool(p.get("vector_simulation", True))
        self.pole_num = 3 if self.vector else 1
        for key, val in (("used_gpu", 0), ("max_batch", 0), ("mem_budget", 0)):
            p.setdefault(key, val)
        self.utility = u = OpticalTool(p)
        p["RI_xy_size"] = list(p["RI_xy_size"])
        for i in range(2):
            if p["RI_xy_size"][i] == 0:
                p["RI_xy_size"][i] = p["size"][i]
        self.expected_RI_size = [int(p["RI_xy_size"][0]), int(p["RI_xy_size"][1]), int(p["size"][2])]
        bt = [float(b) for b in p["boundary_thickness"]]
        if len(bt) != 3:
            raise ValueError('Boundary in only one direction is not precise; enter '
                             '"boundary_thickness" as an array of size 3')
        self.cyclic_boundary_xy = (bt[0] == 0 and bt[1] == 0
                                   and self.expected_RI_size[0] == p["size"][0]
                                   and self.expected_RI_size[1] == p["size"][1])
        rc = [int(c) for c in p["RI_center"]]
        if self.cyclic_boundary_xy:                                   # :65-72
            ru = np.exp(u.refocusing_kernel[:, :, None] * u.image_coor[2][None, None, :])
            ru = ru * u.NA_circle[:, :, None]
            fsg = ru / (1j * 4 * math.pi)
            fsg = fsg * (u.NA_circle / (u.k3 + (~u.NA_circle)))[:, :, None]
            fsg = fsg / (u.image_res[0] * u.image_res[1])
            fsg = centered_fft2(fsg, inverse=True)
        else:                                                         # :74-108
            ptg = copy.deepcopy(p)
            ptg["size"] = [p["size"][0] + self.expected_RI_size[0] + rc[0],
                           p["size"][1] + self.expected_RI_size[1] + rc[1], p["size"][2]]
            ru = self._crop_shift(self._truncated_green(ptg, True), rc)
            ru = centered_fft2(centered_fftn(ru, inverse=True))
            ru = ru * (u.image_res[0] * u.image_res[1])
            fsg = self._crop_shift(self._truncated_green(ptg, False), rc)
            fsg = centered_fftn(fsg, inverse=True)
        self.refocusing_util = ru.astype(C64)
        self.kernel_trans = centered_fft2(np.conj(fsg)).astype(C64)   # :114
        self.kernel_ref = centered_fft2(fsg).astype(C64)              # :115
        self.boundary_thickness_pixel = mround(
            (np.asarray(bt) * p["wavelength"] / p["RI_bg"]) / (np.asarray(p["resolution"], dtype=np.float64) * 2)
        ).astype(int)                                                 # :129
        ri = self.expected_RI_size
        self.sim_size = [ri[i] + 2 * int(self.boundary_thickness_pixel[i]) for i in range(3)]
        self.field_size = [int(p["size"][0]), int(p["size"][1])]
        self.conv_size = (list(self.field_size) if self.cyclic_boundary_xy
                          else [self.field_size[0] + ri[0], self.field_size[1] + ri[1]])
        self.pupil_in, self.pupil_out = self._pupils()
        if self.vector:
            self.polarisation = polarisation_basis(self.field_size, p)

    def _truncated_green(self, params, refocus_version):
        """truncated_green_plus on the host (MATLAB single semantics)."""
        return truncated_green_plus(params, refocus_version)

    @staticmethod
    def _crop_shift(a, rc):
        a = a[-min(0, rc[0]):a.shape[0] - max(0, rc[0]), -min(0, rc[1]):a.shape[1] - max(0, rc[1]), :]
        return np.roll(a, (-rc[0], -rc[1]), axis=(0, 1))

    def _pupils(self):
        """transform_field_3D / transform_field_2D filters (FORWARD_SOLVER.m:38-97),
        scalar case, as one real factor each."""
        u = self.utility
        NA = u.NA_circle
        pin = NA.astype(F32)
        pout = NA.astype(F32)
        if self.parameters["use_abbe_sine"]:
            pin[NA] = pin[NA] / np.sqrt(u.cos_theta[NA])
            pout = (pout * np.sqrt(u.cos_theta)) * NA
        return pin, pout

    # ------------------------------------------------------------ set_RI
    def prepare_potential(self, RI):
        """condition_RI -> create_boundary_RI -> init
        (FORWARD_SOLVER_CONVERGENT_BORN.m:180-396): fills V, the separable
        tables and the scalars, and returns the PotentialParams struct plus
        the arrays it points into (keep them alive until the call returns)."""
        RI = np.asarray(RI)
        if list(RI.shape[:3]) != list(self.expected_RI_size) or (RI.ndim > 3 and RI.shape[3] > 1):
            raise ValueError("The refractive index does not have the expected size : %d %d %d"
                             % tuple(self.expected_RI_size))
        RI = RI.reshape(RI.shape[:3]).astype(C64 if np.iscomplexobj(RI) else F32)
        p = self.parameters
        lam, nm = p["wavelength"], p["RI_bg"]
        # condition_RI :199-222
        self.eps_imag = F32(np.abs(ri2potential(RI.ravel(), lam, nm)).max() * 1.01)
        btp = [int(b) for b in self.boundary_thickness_pixel]
        old = RI.shape
        # create_boundary_RI :223-279
        RIp = np.pad(ri2potential(RI, lam, nm), [(btp[0], btp[0]), (btp[1], btp[1]), (btp[2], btp[2])])
        RIp = potential2ri(RIp, lam, nm)
        self.ROI = [btp[0] + 1, btp[0] + old[0], btp[1] + 1, btp[1] + old[1], btp[2] + 1, btp[2] + old[2]]
        V_temp = ri2potential(RIp, lam, nm)
        self.RI = potential2ri(V_temp, lam, nm)
        V = (ri2potential(self.RI, lam, nm) - 1j * self.eps_imag).astype(C64)
        pp, keep = self.potential_params(self.eps_imag)
        self.V = V
        self.tensor = False
        return pp, keep + [_c64(V)]

    def prepare_tensor_potential(self, RI):
        """prepare_potential for an RI tensor [x, y, z, 3, 3]
        (FORWARD_SOLVER_CONVERGENT_BORN.m:199-279 with size(RI,4) > 1):
        eps_imag = 1.01 max |potential| over all nine components (the
        reference's pagesvd runs on the 1 x 1 pages of pott(:)), every
        component padded with zero potential and passed through the
        RI2potential / potential2RI round trips, V(:,:,:,j,j) -= 1i eps_imag.
        Returns the PotentialParams and the arrays it points into, V
        ([sim, 3, 3], column-major) last."""
        if not self.vector:
            raise ValueError("a tensor RI needs vector_simulation (the dyadic Green's function)")
        RI = np.asarray(RI)
        if list(RI.shape[:3]) != list(self.expected_RI_size) or RI.shape[3:] != (3, 3):
            raise ValueError("The refractive index tensor must be [%d %d %d 3 3]" % tuple(self.expected_RI_size))
        RI = RI.astype(C64 if np.iscomplexobj(RI) else F32)
        p = self.parameters
        lam, nm = p["wavelength"], p["RI_bg"]
        self.eps_imag = F32(np.abs(ri2potential(RI.ravel(), lam, nm)).max() * 1.01)
        btp = [int(b) for b in self.boundary_thickness_pixel]
        RIp = np.pad(ri2potential(RI, lam, nm), [(btp[0], btp[0]), (btp[1], btp[1]), (btp[2], btp[2]), (0, 0), (0, 0)])
        V_temp = ri2potential(potential2ri(RIp, lam, nm), lam, nm)
        self.RI = potential2ri(V_temp, lam, nm)
        V = ri2potential(self.RI, lam, nm).astype(C64)
        for j in range(3):
            V[:, :, :, j, j] = V[:, :, :, j, j] - 1j * self.eps_imag
        pp, keep = self.potential_params(self.eps_imag)
        self.V = V
        self.tensor = True
        return pp, keep + [_c64(V)]

    def potential_params(self, eps_imag):
        """The RI-independent part of create_boundary_RI and init
        (FORWARD_SOLVER_CONVERGENT_BORN.m:251-396) for a given eps_imag:
        attenuation masks, ramps, Green's coordinates, Bornmax and the
        scalars, as the PotentialParams struct plus the arrays it points
        into (keep them alive until the call returns)."""
        p = self.parameters
        self.eps_imag = F32(eps_imag)
        btp = [int(b) for b in self.boundary_thickness_pixel]
        old = list(self.expected_RI_size)
        self.ROI = [btp[0] + 1, btp[0] + old[0], btp[1] + 1, btp[1] + old[1], btp[2] + 1, btp[2] + old[2]]
        shape = tuple(old[j] + 2 * btp[j] for j in range(3))
        masks = []
        for j in range(3):
            n = shape[j]
            x = (np.abs(np.arange(1, n + 1) - math.floor(n / 2 + 1) + 0.5) - 0.5).astype(F32)
            x = np.roll(x, -(n // 2)) / (btp[j] - 0.5)
            v0 = x.copy()
            v0[np.abs(x) >= 1] = 1
            v0 = 1 - np.abs(v0)
            sh = p["boundary_sharpness"]
            v0[v0 > sh] = sh
            v0 = v0 / sh
            if btp[j] == 0:
                v0[:] = 0
            masks.append((1 - v0 * 1).astype(F32))
        # init :280-396
        pb = copy.deepcopy(p)
        pb["size"] = list(shape)
        ub = self.utility_border = OpticalTool(pb)
        if p["acyclic"] and self.cyclic_boundary_xy:
            sc = [ub.fourier_coor[0], ub.fourier_coor[1], ub.fourier_coor[2] + ub.fourier_res[2] / 4]
        elif p["acyclic"]:
            sc = [ub.fourier_coor[i] + ub.fourier_res[i] / 4 for i in range(3)]
        else:
            sc = list(ub.fourier_coor)
        kq2 = [np.fft.ifftshift(c * c).astype(F32) for c in sc]
        # dyadic Green's function: rads = shifted coordinate / k0_nm (:316-319),
        # ifftshifted (:385), and the absorptive correction (:322)
        rads = [np.fft.ifftshift((np.asarray(c, dtype=F32) / ub.k0_nm).astype(F32)) for c in sc]
        a2 = F32((2 * math.pi * ub.k0_nm) ** 2)
        absorb = C64(a2 / C64(a2 + 1j * self.eps_imag))
        step = F32(abs(2 * (2 * math.pi * ub.k0_nm) / self.eps_imag))
        nrm = float(np.linalg.norm(np.asarray(shape, dtype=np.float64) * np.asarray(p["resolution"], dtype=np.float64)))
        bopt = int(math.ceil(float(F32(F32(nrm / step) / 2 + 1)))) * 2
        it = p["iterations_number"]
        self.Bornmax = 0 if it == 0 else (bopt * abs(int(it)) if it < 0 else int(it))
        ramps = []
        if p["acyclic"]:
            for j in range(3):
                n = shape[j]
                if self.boundary_thickness_pixel[0] == 0 and self.boundary_thickness_pixel[1] == 0:
                    if j < 2:
                        ramps.append(np.ones(n, dtype=C64))
                        continue
                    x = np.exp(-1j * math.pi * (np.arange(1, n + 1) - 1) / n / 2)
                    ramps.append((x / x[n // 2]).astype(C64))
                else:
                    x = np.exp(-1j * math.pi * (np.arange(1, n + 1) - 1) / n / 2).astype(C64)
                    ramps.append(x / x[n // 2])
        else:
            ramps = [np.ones(shape[j], dtype=C64) for j in range(3)]
        pp = _lib.PotentialParams()
        pp.eps_imag = float(self.eps_imag)
        pp.green_scale = float(F32(4 * math.pi ** 2))
        pp.green_offset = float(F32((2 * math.pi * ub.k0_nm) ** 2))
        pp.dV = float(F32(ub.dV))
        pp.roi[:] = [int(r) for r in self.ROI]
        pp.bornmax = int(self.Bornmax)
        pp.acyclic = 1 if p["acyclic"] else 0
        keep = ([_f32(m) for m in masks] + [_c64(r) for r in ramps] + [_f32(k) for k in kq2]
                + [_f32(r) for r in rads])
        for j in range(3):
            pp.mask[j] = _lib.ptr(keep[j])
            pp.ramp[j] = _lib.ptr(keep[3 + j])
            pp.kq2[j] = _lib.ptr(keep[6 + j])
            pp.rad[j] = _lib.ptr(keep[9 + j])
        pp.absorb[:] = [float(absorb.real), float(absorb.imag)]
        self.rads1d = rads
        self.green_absorbtion_correction = absorb
        self.attenuation_mask1d = masks
        self.ramp1d = ramps
        self.kq2 = kq2
        return pp, keep

    def voxel_iterations(self, n_ill):
        """Born voxel-iterations of one solve of n_ill illuminations."""
        return int(np.prod(self.sim_size)) * int(self.Bornmax) * int(n_ill)


class FORWARD_SOLVER_CONVERGENT_BORN(CBSHostSetup):
    """Convergent Born series forward solver (scalar Green's function, or the
    dyadic one with vector_simulation) whose per-illumination work runs in
    libodt on the GPU."""

    def __init__(self, params):
        """Constructor + CudaBorn action 0 (FORWARD_SOLVER_CONVERGENT_BORN_CUDA.m:18-41)."""
        self._handle = 0
        self._jobs = {}
        self.lib = _lib.load()
        super().__init__(params)
        self._create_handle()

    def _truncated_green(self, params, refocus_version):
        """truncated_green_plus with its plane part (interpolation onto the
        oversized grid, the centred 2D and z FFTs and crops: most of the
        set-up time) on the GPU (odt_green_planes); the radial profile and the
        interpolation maps come from the host.  The result equals the host
        path's to single-precision rounding (the FFTs are the library's).
        Parameter ``green_on_device=False`` keeps the host path."""
        if not self.parameters.get("green_on_device", True):
            return super()._truncated_green(params, refocus_version)
        r = truncated_green_radial(params, refocus_version, hankel_filter=self._device_hankel)
        keep = [np.asfortranarray(np.asarray(r["green"], dtype=C64)),
                np.asfortranarray(np.asarray(r["near"], dtype=np.int32)),
                np.asfortranarray(np.asarray(r["near2"], dtype=np.int32)),
                np.asfortranarray(np.asarray(r["w"], dtype=F32))]
        keep += [np.asfortranarray(m) for m in green_plane_maps(r)]
        out = np.empty(r["out_px"], dtype=C64, order="F")
        a = _lib.GreenArgs()
        a.radial = _lib.ptr(keep[0])
        a.n_r = keep[0].shape[0]
        a.near1, a.near2, a.w = _lib.ptr(keep[1]), _lib.ptr(keep[2]), _lib.ptr(keep[3])
        a.creation[:] = r["creation"]
        a.out_size[:] = r["out_px"]
        a.scale = float(r["scale"])
        a.m1, a.m2, a.mz = _lib.ptr(keep[4]), _lib.ptr(keep[5]), _lib.ptr(keep[6])
        a.out = _lib.ptr(out)
        a.device = int(self.parameters.get("used_gpu", 0))
        _lib.check(self.lib.odt_green_planes(C.byref(a)))
        return out

    def _device_hankel(self, hk, green, band):
        """The cropped Hankel transform pair and band window of
        truncated_green_plus (:33-66) on the GPU (odt_hankel_filter): the
        Bessel matrix is built on the device from the zeros of J_0."""
        if hk.order != 0 or float(hk.R) != 1.0:
            raise ValueError("odt_hankel_filter covers the order-0, unit-radius transform only")
        vals = np.asfortranarray(np.asarray(green, dtype=C64))
        roots = np.ascontiguousarray(hk.roots64, dtype=np.float64)
        b = np.ascontiguousarray(band, dtype=F32)
        out = np.empty_like(vals, order="F")
        a = _lib.HankelArgs()
        a.roots, a.n, a.pos, a.nz = _lib.ptr(roots), len(hk.c), int(hk.pos), vals.shape[1]
        a.values, a.band, a.out = _lib.ptr(vals), _lib.ptr(b), _lib.ptr(out)
        a.device = int(self.parameters.get("used_gpu", 0))
        _lib.check(self.lib.odt_hankel_filter(C.byref(a)))
        return out

    def _create_handle(self):
        p = self.parameters
        ri, sim, field, conv = self.expected_RI_size, self.sim_size, self.field_size, self.conv_size
        if p["RI_center"][0] != 0 or p["RI_center"][1] != 0 or ri[0] != field[0] or ri[1] != field[1]:
            raise ValueError("RI_xy_size must equal size(1:2) and RI_center must be [0 0] "
                             "(the reference's crop_field2RI / V(ROI).*source need it)")
        g = _lib.Geometry()
        g.sim_size[:] = sim
        g.ri_size[:] = ri
        g.field_size[:] = field
        g.conv_size[:] = conv
        g.device = int(p["used_gpu"])
        g.max_batch = int(p["max_batch"])
        g.mem_budget = int(p["mem_budget"])
        g.pol = self.pole_num
        self._keep = [_c64(self.refocusing_util), _c64(self.kernel_trans), _c64(self.kernel_ref),
                      _f32(self.pupil_in), _f32(self.pupil_out)]
        h = C.c_uint32(0)
        _lib.check(self.lib.odt_create(C.byref(g), *[_lib.ptr(a) for a in self._keep], C.byref(h)))
        self._handle = h.value
        self._keep = None
        self.set_field_storage(p.get("field_storage", "complex64"))
        if self.vector:
            rad, perp, tan, km = self.polarisation
            keep = [_f32(rad), _f32(perp), _f32(tan), np.asfortranarray(km.astype(np.uint8))]
            _lib.check(self.lib.odt_set_polarisation(self._handle, *[_lib.ptr(k) for k in keep]))

    def set_RI(self, RI):
        """set_RI (FORWARD_SOLVER_CONVERGENT_BORN.m:180-198) + CudaBorn action 1
        (FORWARD_SOLVER_CONVERGENT_BORN_CUDA.m:42-63).  An RI tensor
        [x, y, z, 3, 3] (or the struct form {"scatt_pott": tensor}, :181-186)
        goes to odt_set_tensor_potential (vector_simulation only)."""
        if isinstance(RI, dict):
            RI = np.asarray(RI["scatt_pott"])
            if RI.ndim < 4 or RI.shape[3] <= 1:
                raise ValueError("Structur form only allowed for tensor RI")
        RI = np.asarray(RI)
        if RI.ndim >= 4 and RI.shape[3] > 1:
            pp, keep = self.prepare_tensor_potential(RI)
            _lib.check(self.lib.odt_set_tensor_potential(self._handle, C.byref(pp), _lib.ptr(keep[-1])))
            return
        pp, keep = self.prepare_potential(RI)
        _lib.check(self.lib.odt_set_potential(self._handle, C.byref(pp), _lib.ptr(keep[-1])))

    _STATE = ("eps_imag", "ROI", "RI", "V", "Bornmax", "utility_border", "attenuation_mask1d",
              "ramp1d", "kq2")

    def set_RI_adjoint(self, RI):
        """Potential of the adjoint solve, conj(flip(RI, 3))
        (BACKWARD_SOLVER_MULTI.m:48), uploaded to the adjoint slot; the
        forward state of this object is left unchanged."""
        saved = {k: getattr(self, k) for k in self._STATE if hasattr(self, k)}
        try:
            pp, keep = self.prepare_potential(np.conj(np.flip(np.asarray(RI), axis=2)))
            _lib.check(self.lib.odt_set_adjoint_potential(self._handle, C.byref(pp),
                                                          _lib.ptr(keep[-1])))
            self.adjoint_Bornmax = self.Bornmax
        finally:
            for k, v in saved.items():
                setattr(self, k, v)

    def _ri_device_args(self, ri, adjoint, stream):
        import torch

        n = int(np.prod(self.expected_RI_size))
        if not (isinstance(ri, torch.Tensor) and ri.is_cuda and ri.is_contiguous() and ri.numel() == n):
            raise ValueError("set_RI_device: RI must be a contiguous CUDA tensor of %d elements "
                             "(the column-major [RI_x, RI_y, RI_z] grid)" % n)
        if ri.dtype not in (torch.complex64, torch.float32):
            raise ValueError("set_RI_device: RI must be complex64 or float32")
        a = _lib.RIDeviceArgs()
        a.ri = ri.data_ptr()
        a.is_complex = 1 if ri.dtype == torch.complex64 else 0
        a.adjoint = 1 if adjoint else 0
        a.wavelength = float(self.parameters["wavelength"])
        a.ri_bg = float(self.parameters["RI_bg"])
        a.stream = torch.cuda.current_stream(ri.device).cuda_stream if stream is None else stream
        return a

    def set_RI_device(self, ri, adjoint=False, stream=None):
        """set_RI (or, with adjoint=True, set_RI_adjoint) for an RI array that
        is already in device memory: a contiguous CUDA tensor holding the
        column-major [RI_x, RI_y, RI_z] grid (complex64 or float32).  eps_imag
        and the padded potential are computed on the GPU
        (odt_potential_eps_device, odt_set_potential_device); only the
        RI-independent tables come from the host.  Used by the device-resident
        outer loop of BACKWARD_SOLVER_MULTI."""
        a = self._ri_device_args(ri, adjoint, stream)
        eps = C.c_float(0)
        _lib.check(self.lib.odt_potential_eps_device(self._handle, C.byref(a), C.byref(eps)))
        saved = {k: getattr(self, k) for k in self._STATE if hasattr(self, k)} if adjoint else {}
        try:
            pp, keep = self.potential_params(eps.value)
            _lib.check(self.lib.odt_set_potential_device(self._handle, C.byref(pp), C.byref(a)))
            if adjoint:
                self.adjoint_Bornmax = self.Bornmax
        finally:
            for k, v in saved.items():
                setattr(self, k, v)

    def gradient_device(self, fields_in, fields_meas, grad, stream=None):
        """gradient() on device arrays: fields_in / fields_meas contiguous CUDA
        complex64 tensors of F_x*F_y*npol*n_ill elements (column-major
        [F_x, F_y, npol, n_ill]; npol = 2 with vector_simulation, else 1),
        grad a CUDA complex64 tensor of the RI grid's size; returns err."""
        import torch

        nF = int(self.field_size[0] * self.field_size[1]) * (2 if self.vector else 1)
        n_ill = fields_in.numel() // nF
        if fields_in.numel() != nF * n_ill or fields_meas.numel() != fields_in.numel() or n_ill < 1:
            raise ValueError("input and output fields must be [F_x, F_y, npol, n] alike")
        err = C.c_double(0)
        a = _lib.GradientArgs()
        a.fields_in, a.fields_meas = fields_in.data_ptr(), fields_meas.data_ptr()
        a.n_ill = n_ill
        a.grad = grad.data_ptr()
        a.err = C.addressof(err)
        a.memory = _lib.ODT_MEM_DEVICE
        s = torch.cuda.current_stream(grad.device) if stream is None else stream
        a.stream = s.cuda_stream
        _lib.check(self.lib.odt_gradient(self._handle, C.byref(a)))
        s.synchronize()
        return err.value

    def gradient(self, input_field, output_field):
        """Fused forward + adjoint gradient of get_gradiant_static
        (BACKWARD_SOLVER_MULTI.m:30-54) after set_RI(RI) and
        set_RI_adjoint(RI): returns (gradient [RI size] complex64, err).  With
        vector_simulation the fields are [F_x, F_y, 2, n] and the gradient is
        the mean over the three field components and the illuminations."""
        x = np.asarray(input_field)
        y = np.asarray(output_field)
        if x.ndim == 3:
            x = x[:, :, :, None]
        if y.ndim == 3:
            y = y[:, :, :, None]
        npol = 2 if self.vector else 1
        if x.shape != y.shape or x.shape[2] != npol:
            raise ValueError("input and output fields must be [F_x, F_y, %d, n] alike" % npol)
        xin, yin = _c64(x), _c64(y)
        g = np.empty(self.expected_RI_size, dtype=C64, order="F")
        err = C.c_double(0)
        a = _lib.GradientArgs()
        a.fields_in, a.fields_meas = _lib.ptr(xin), _lib.ptr(yin)
        a.n_ill = x.shape[3]
        a.grad = _lib.ptr(g)
        a.err = C.addressof(err)
        a.memory = _lib.ODT_MEM_HOST
        a.stream = None
        _lib.check(self.lib.odt_gradient(self._handle, C.byref(a)))
        return g, err.value

    # ------------------------------------------------------------ solve
    def _outputs(self, n_ill, on_device=False):
        p = self.parameters
        F = self.field_size
        R = self.expected_RI_size
        shp_t = (F[0], F[1], 2 if self.vector else 1, n_ill)
        shp_3 = (R[0], R[1], R[2], self.pole_num, n_ill)
        mk = (lambda s: np.empty(s, dtype=C64, order="F"))
        return (mk(shp_t) if p["return_transmission"] else None,
                mk(shp_t) if p["return_reflection"] else None,
                mk(shp_3) if p["return_3D"] else None)

    def solve(self, input_field):
        """solve (FORWARD_SOLVER_CONVERGENT_BORN.m:397-520): input_field is the
        spatial field [F_x, F_y, npol, n_ill] (npol = 1, or 2 with
        vector_simulation); returns (fields_trans, fields_ref, fields_3D),
        each None when its return_* flag is false ([F_x, F_y, npol, n_ill],
        and [x, y, z, pole_num, n_ill] for the 3D field)."""
        x = np.asarray(input_field)
        if x.ndim == 2:
            x = x[:, :, None, None]
        elif x.ndim == 3:
            x = x[:, :, :, None]
        if x.shape[2] > 1 and not self.vector:                         # :404-414
            raise ValueError("the source is 2D but parameter indicate a vectorial simulation")
        if x.shape[2] == 1 and self.vector:
            raise ValueError("the source is 3D but parameter indicate a non-vectorial simulation")
        if x.shape[2] > 2:
            raise ValueError("Input field must be either a scalar or a 2D vector")
        if list(x.shape[:2]) != list(self.field_size):
            raise ValueError("input field must be %d x %d" % tuple(self.field_size))
        a, keep, out = self._host_args(x)
        _lib.check(self.lib.odt_solve(self._handle, C.byref(a)))
        return out

    def _host_args(self, x):
        n_ill = x.shape[3]
        xin = _c64(x)
        ft, fr, f3 = self._outputs(n_ill)
        a = _lib.SolveArgs()
        a.fields_in = _lib.ptr(xin)
        a.n_ill = n_ill
        a.trans = _lib.ptr(ft)
        a.ref = _lib.ptr(fr)
        a.field3d = _lib.ptr(f3)
        a.memory = _lib.ODT_MEM_HOST
        a.stream = None
        return a, xin, (ft, fr, f3)

    # ------------------------------------------------- asynchronous solves
    def submit(self, input_field):
        """odt_submit: queue the solve of input_field (as for solve) on the
        handle's worker thread and return a ticket for poll / wait; the
        buffers are held until the ticket is collected."""
        x = np.asarray(input_field)
        if x.ndim == 3:
            x = x[:, :, :, None]
        if x.ndim != 4 or list(x.shape[:2]) != list(self.field_size):
            raise ValueError("input field must be [F_x, F_y, npol, n_ill]")
        a, keep, out = self._host_args(x)
        t = C.c_uint64(0)
        _lib.check(self.lib.odt_submit(self._handle, C.byref(a), C.byref(t)))
        self._jobs[t.value] = (a, keep, out)
        return t.value

    def poll(self, ticket):
        """odt_poll: None while the solve runs, then its outputs (raises
        OdtError if it failed)."""
        done, st = C.c_int32(0), C.c_int(0)
        _lib.check(self.lib.odt_poll(self._handle, C.c_uint64(ticket), C.byref(done), C.byref(st)))
        if not done.value:
            return None
        _, _, out = self._jobs.pop(ticket)
        _lib.check(st.value)
        return out

    def wait(self, ticket):
        """odt_wait: block until the ticket's solve finishes; its outputs."""
        st = C.c_int(0)
        _lib.check(self.lib.odt_wait(self._handle, C.c_uint64(ticket), C.byref(st)))
        _, _, out = self._jobs.pop(ticket)
        _lib.check(st.value)
        return out

    def budget(self):
        """odt_budget: (bytes held on the device, budget in bytes or 0)."""
        held, bud = C.c_int64(0), C.c_int64(0)
        _lib.check(self.lib.odt_budget(self._handle, C.byref(held), C.byref(bud)))
        return held.value, bud.value

    def solve_device(self, fields_in, trans=None, ref=None, field3d=None, stream=None):
        """Device-resident solve: arguments are CUDA tensors (torch) whose memory
        is the column-major MATLAB layout, e.g. a contiguous complex64 tensor of
        shape (n_ill, F_y, F_x) for [F_x, F_y, n_ill].  Work is queued on
        ``stream`` (a torch.cuda.Stream or raw handle; default: the current
        torch stream) and the call returns without synchronising."""
        import torch

        if stream is None:
            stream = torch.cuda.current_stream()
        sh = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        nF = self.field_size[0] * self.field_size[1] * (2 if self.vector else 1)
        n_ill = fields_in.numel() // nF
        for t in (fields_in, trans, ref, field3d):
            if t is not None and (not t.is_cuda or not t.is_contiguous() or t.dtype != torch.complex64):
                raise ValueError("solve_device expects contiguous complex64 CUDA tensors")
        a = _lib.SolveArgs()
        a.fields_in = fields_in.data_ptr()
        a.n_ill = n_ill
        a.trans = trans.data_ptr() if trans is not None else None
        a.ref = ref.data_ptr() if ref is not None else None
        a.field3d = field3d.data_ptr() if field3d is not None else None
        a.memory = _lib.ODT_MEM_DEVICE
        a.stream = sh
        _lib.check(self.lib.odt_solve(self._handle, C.byref(a)))

    def solve_ptrs(self, fields_in, n_ill, trans=None, ref=None, field3d=None, device=False,
                   stream=None):
        """odt_solve on raw addresses (e.g. pinned host tensors); column-major
        [F_x, F_y, n_ill] / [ri, n_ill] complex64 buffers."""
        a = _lib.SolveArgs()
        a.fields_in = fields_in
        a.n_ill = int(n_ill)
        a.trans, a.ref, a.field3d = trans, ref, field3d
        a.memory = _lib.ODT_MEM_DEVICE if device else _lib.ODT_MEM_HOST
        a.stream = stream
        _lib.check(self.lib.odt_solve(self._handle, C.byref(a)))

    # ------------------------------------------------------------ misc
    def batch(self):
        b = C.c_int32(0)
        _lib.check(self.lib.odt_get_batch(self._handle, C.byref(b)))
        return b.value

    def set_field_storage(self, storage):
        """Storage of the Born loop's spectral array and Field_n: "complex64"
        (default) or "b16" (16-bit block floating point, odt_set_field_storage;
        square x-y grids of 88, 120 or 152 with a scalar potential)."""
        modes = {"complex64": _lib.ODT_STORAGE_COMPLEX64, "b16": _lib.ODT_STORAGE_B16}
        if storage not in modes:
            raise ValueError('field_storage must be "complex64" or "b16", got %r' % (storage,))
        _lib.check(self.lib.odt_set_field_storage(self._handle, modes[storage]))
        self.parameters["field_storage"] = storage

    def solve_source(self, source):
        """CudaBorn's action 2 (CUDA_CODE/main.cpp:139-163): the Born series
        driven by 3D incident fields over the RI grid, source [RI_x, RI_y,
        RI_z, n] (or [RI_x, RI_y, RI_z, 3, n] with vector_simulation; one field
        may omit the last axis); returns Field(ROI) + source in the same
        layout (odt_solve_source)."""
        x = np.asarray(source)
        ri = list(self.expected_RI_size)
        comp = (3,) if self.vector else ()
        single = x.ndim == 3 + len(comp)
        if single:
            x = x[..., None]
        if list(x.shape[:3]) != ri or tuple(x.shape[3:-1]) != comp:
            raise ValueError("source must be [%d, %d, %d%s, n]" % (ri[0], ri[1], ri[2], ", 3" if comp else ""))
        xin = _c64(x)
        out = np.empty(x.shape, dtype=C64, order="F")
        a = _lib.SourceArgs()
        a.source, a.n, a.field3d = _lib.ptr(xin), x.shape[-1], _lib.ptr(out)
        a.memory = _lib.ODT_MEM_HOST
        a.stream = None
        _lib.check(self.lib.odt_solve_source(self._handle, C.byref(a)))
        return out[..., 0] if single else out

    def autotune(self, n_ill=None):
        """Time the execution plans that apply to this geometry (fused xy-pass,
        separate pipelined passes, generic tile kernels) on one solve of
        n_ill plane waves (default: the batch) with the current potential,
        keep the fastest (odt_autotune; cached process-wide per shape) and
        return {"plan", "batch", "cached", "ms": {plan: ms per solve}}."""
        r = _lib.TuneResult()
        n = int(n_ill) if n_ill else max(1, int(self.batch()) or int(self.parameters.get("max_batch") or 16))
        _lib.check(self.lib.odt_autotune(self._handle, n, C.byref(r)))
        names = ("fused_xy", "separate_pipelined", "generic")
        plan = "fused_xy" if r.fused_xy else ("separate_pipelined" if r.pipelined else "generic")
        return {"plan": plan, "batch": r.batch, "cached": bool(r.cached),
                "ms": {nm: r.ms[i] for i, nm in enumerate(names) if r.ms[i] >= 0}}

    def set_profiling(self, on: bool):
        _lib.check(self.lib.odt_set_profiling(self._handle, 1 if on else 0))

    def kernel_times(self):
        """{kind: (total ms, launches)} accumulated while profiling was on."""
        cap = 16
        names = (C.c_char_p * cap)()
        ms = (C.c_double * cap)()
        nl = (C.c_int64 * cap)()
        n = C.c_int32(0)
        _lib.check(self.lib.odt_get_kernel_times(self._handle, names, ms, nl, cap, C.byref(n)))
        return {names[i].decode(): (ms[i], nl[i]) for i in range(min(n.value, cap))}

    def delete(self):
        """CudaBorn action 3 (FORWARD_SOLVER_CONVERGENT_BORN_CUDA.m:64-68)."""
        if getattr(self, "_handle", 0):
            h, self._handle = self._handle, 0
            _lib.check(self.lib.odt_destroy(h))

    def __del__(self):
        try:
            self.delete()
        except Exception:
            pass
