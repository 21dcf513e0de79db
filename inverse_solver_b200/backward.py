"""BACKWARD_SOLVER_MULTI and TV_FISTA_inner_v2 on the B200 library.

Mirrors Codes/BACKWARD_SOLVER_MULTI.m (FISTA on u = RI^2/RI_bg^2 - 1 with a
TV proximal step) and Codes/sub_code/TV_FISTA_inner_v2.m.  The gradient
(forward + adjoint CBS solves and the reduction) runs fused on the GPU
(odt_gradient); the TV prox runs on the GPU (odt_tv_prox) with the FISTA
scalars in double on the host; the outer-loop momentum is a few elementwise
array updates in single precision, as the reference does them.

With ``device_loop`` (the default when the forward solver is the scalar GPU
solver) the whole outer loop stays in device memory: the potentials are built
on the GPU from the device RI (set_RI_device), the gradient, prox input, TV
prox and momentum update work on device arrays, and the host only handles the
FISTA scalars and the RI-independent potential tables.  ``device_loop=False``
keeps the host-array loop (numpy between the GPU calls).
"""
from __future__ import annotations

import copy
import ctypes as C
import math

import numpy as np

from . import _lib
from .optics import C64, F32, basic_optical_parameter, update_struct


def TV_FISTA_inner_v2(in_mat, lam, Vmin, Vmax, Vimag_max, non_neg, dirichlet_boundary, inner_itt,
                      use_gpu=True):
    """Isotropic-TV prox (sub_code/TV_FISTA_inner_v2.m:1-53) on the GPU.
    Real result when Vimag_max == 0 (the reference keeps the real part)."""
    x = np.asarray(in_mat)
    cplx = Vimag_max > 0
    x = np.asfortranarray(x.astype(C64) if cplx else np.real(x).astype(F32))
    if x.ndim == 2:
        x = x[:, :, None]
    out = np.empty_like(x, order="F")
    a = _lib.TVArgs()
    a.size[:] = list(x.shape[:3])
    a.inp, a.out = _lib.ptr(x), _lib.ptr(out)
    a.is_complex = 1 if cplx else 0
    a.lam = float(lam)
    a.vmin, a.vmax, a.vimag_max = float(Vmin), float(Vmax), float(Vimag_max)
    a.non_neg = 1 if non_neg else 0
    a.dirichlet = 1 if dirichlet_boundary else 0
    a.inner_itt = int(inner_itt)
    a.memory = _lib.ODT_MEM_HOST
    a.stream = None
    _lib.check(_lib.load().odt_tv_prox(C.byref(a)))
    return out.reshape(np.asarray(in_mat).shape) if np.asarray(in_mat).ndim == 2 else out


def _tv_prox_device(inp, out, shape, cplx, lam, Vmin, Vmax, Vimag_max, non_neg, dirichlet_boundary, inner_itt,
                    stream):
    """TV_FISTA_inner_v2 on device arrays (column-major [shape], float32 or
    complex64 CUDA tensors), ordered on `stream`."""
    a = _lib.TVArgs()
    a.size[:] = list(shape)
    a.inp, a.out = inp.data_ptr(), out.data_ptr()
    a.is_complex = 1 if cplx else 0
    a.lam = float(lam)
    a.vmin, a.vmax, a.vimag_max = float(Vmin), float(Vmax), float(Vimag_max)
    a.non_neg = 1 if non_neg else 0
    a.dirichlet = 1 if dirichlet_boundary else 0
    a.inner_itt = int(inner_itt)
    a.memory = _lib.ODT_MEM_DEVICE
    a.stream = stream.cuda_stream
    _lib.check(_lib.load().odt_tv_prox(C.byref(a)))


class BACKWARD_SOLVER_MULTI:
    """Multiple-scattering inverse solver (Codes/BACKWARD_SOLVER_MULTI.m)."""

    @staticmethod
    def get_default_parameters(init_params=None):
        """BACKWARD_SOLVER_MULTI.m:9-29 (+ ``seed`` for the random scan subsets,
        which the reference draws with an unseeded randperm)."""
        p = basic_optical_parameter()
        p.update(forward_solver=None, forward_solver_parameters=None, init_solver=None,
                 step=0.01, tv_param=0.001, use_non_negativity=False, nmin=-math.inf,
                 nmax=math.inf, kappamax=0, inner_itt=100, itter_max=100,
                 num_scan_per_iteration=0, verbose=False, seed=0, device_loop=True)
        return update_struct(p, init_params) if init_params else p

    def __init__(self, params, init_solver=True):
        """Constructor (:58-79): the forward solver must return transmission,
        reflection and the 3D field."""
        self.parameters = params
        fp = params["forward_solver_parameters"]
        if not (fp["return_transmission"] and fp["return_reflection"] and fp["return_3D"]):
            raise ValueError("need to set all return parameter to true in the forward solver")
        self.forward_solver = None
        if init_solver:
            self.forward_solver = params["forward_solver"](fp)
        self.RI_inter = None
        self.err_list = []
        self._rng = np.random.default_rng(params.get("seed", 0))

    @staticmethod
    def get_gradiant_static(RI, input_field, output_field, forward_solver):
        """:30-54 -- fused on the GPU by odt_gradient."""
        forward_solver.set_RI(RI)
        forward_solver.set_RI_adjoint(RI)
        return forward_solver.gradient(input_field, output_field)

    def scan_list(self, n):
        """:82-88 (seeded instead of randperm's global stream)."""
        k = self.parameters["num_scan_per_iteration"]
        if k == 0:
            return np.arange(n)
        sl = np.unique(np.concatenate([[0], self._rng.permutation(n)[:k]]))
        return sl[:k]

    def get_gradiant(self, RI, input_field, output_field):
        """:80-91."""
        sl = self.scan_list(input_field.shape[3])
        return self.get_gradiant_static(RI, input_field[:, :, :, sl], output_field[:, :, :, sl],
                                        self.forward_solver)

    def _use_device_loop(self):
        fs = self.forward_solver
        return self.parameters.get("device_loop", True) and fs is not None and hasattr(fs, "set_RI_device")

    def solve(self, input_field, output_field):
        """:92-196: FISTA outer loop."""
        if self._use_device_loop():
            return self._solve_device(input_field, output_field)
        p = self.parameters
        RI = p["init_solver"].solve(input_field, output_field)
        RI = np.asarray(RI).astype(C64)
        alpha = 1 / p["step"]
        t_np = 1.0
        nb2 = p["RI_bg"] ** 2
        u_n = RI ** 2 / nb2 - 1
        x_n = RI ** 2 / nb2 - 1
        if RI.shape[2] % 2 == 0:
            raise ValueError("need to be odd size")
        Vmin = (p["nmin"] ** 2 - p["kappamax"] ** 2) / nb2 - 1
        Vmax = p["nmax"] ** 2 / nb2 - 1
        Vimag_max = 2 * p["kappamax"] * p["nmax"] / nb2
        self.err_list = []
        for _ in range(p["itter_max"]):
            grad, err = self.get_gradiant(RI, input_field, output_field)
            self.err_list.append(err)
            t_n = t_np
            s_n = TV_FISTA_inner_v2(u_n - (1 / alpha) * grad, p["tv_param"] / alpha, Vmin, Vmax,
                                    Vimag_max, p["use_non_negativity"], False, p["inner_itt"])
            t_np = (1 + math.sqrt(1 + 4 * t_n ** 2)) / 2
            u_n = s_n + (t_n - 1) / t_np * (s_n - x_n)
            x_n = s_n
            RI = p["RI_bg"] * np.sqrt(np.asarray(u_n).astype(C64) + 1)
            self.RI_inter = RI
        return RI

    def _device_gradient(self, fs, fields_in, fields_meas, grad, n_sel):
        """Gradient of the selected illuminations into `grad` (device), err."""
        return fs.gradient_device(fields_in, fields_meas, grad)

    def _solve_device(self, input_field, output_field):
        """:92-196 with the iterates in device memory (see the module docstring)."""
        import torch

        p = self.parameters
        fs = self.forward_solver
        dev = torch.device("cuda", int(fs.parameters["used_gpu"]))
        RI = np.asarray(p["init_solver"].solve(input_field, output_field)).astype(C64)
        if RI.shape[2] % 2 == 0:
            raise ValueError("need to be odd size")
        alpha = 1 / p["step"]
        t_np = 1.0
        nb2 = p["RI_bg"] ** 2
        Vmin = (p["nmin"] ** 2 - p["kappamax"] ** 2) / nb2 - 1
        Vmax = p["nmax"] ** 2 / nb2 - 1
        Vimag_max = 2 * p["kappamax"] * p["nmax"] / nb2
        cplx = Vimag_max > 0
        shape = RI.shape[:3]
        n = int(np.prod(shape))

        def up(a):
            return torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=C64).ravel(order="F"))).to(dev)

        u = up(RI ** 2 / nb2 - 1)
        x = u.clone()
        ri = up(RI)
        grad = torch.empty(n, dtype=torch.complex64, device=dev)
        pdt = torch.complex64 if cplx else torch.float32
        prox_in = torch.empty(n, dtype=pdt, device=dev)
        prox_out = torch.empty(n, dtype=pdt, device=dev)
        xin = np.asarray(input_field)
        yin = np.asarray(output_field)
        if xin.ndim == 3:
            xin, yin = xin[:, :, :, None], yin[:, :, :, None]
        npol = 2 if getattr(fs, "vector", False) else 1
        if xin.shape != yin.shape or xin.shape[2] != npol:
            raise ValueError("input and output fields must be [F_x, F_y, %d, n] alike" % npol)
        nill = xin.shape[3]
        fin = up(xin)
        fmeas = up(yin)
        nF = xin.shape[0] * xin.shape[1] * npol
        s = torch.cuda.current_stream(dev)
        fa = _lib.FistaArgs()
        fa.n = n
        fa.grad, fa.u, fa.x, fa.ri = grad.data_ptr(), u.data_ptr(), x.data_ptr(), ri.data_ptr()
        fa.prox_in, fa.prox_out = prox_in.data_ptr(), prox_out.data_ptr()
        fa.prox_complex = 1 if cplx else 0
        fa.step = 1 / alpha
        fa.ri_bg = float(p["RI_bg"])
        fa.stream = s.cuda_stream
        lib = _lib.load()
        self.err_list = []
        for _ in range(p["itter_max"]):
            sl = self.scan_list(nill)
            if len(sl) == nill:
                f1, f2 = fin, fmeas
            else:
                idx = torch.as_tensor(np.asarray(sl), device=dev)
                f1 = fin.view(nill, nF).index_select(0, idx).reshape(-1)
                f2 = fmeas.view(nill, nF).index_select(0, idx).reshape(-1)
            fs.set_RI_device(ri)
            fs.set_RI_device(ri, adjoint=True)
            err = self._device_gradient(fs, f1, f2, grad, len(sl))
            self.err_list.append(err)
            t_n = t_np
            _lib.check(lib.odt_fista_prox_input(C.byref(fa)))
            _tv_prox_device(prox_in, prox_out, shape, cplx, p["tv_param"] / alpha, Vmin, Vmax, Vimag_max,
                            p["use_non_negativity"], False, p["inner_itt"], s)
            t_np = (1 + math.sqrt(1 + 4 * t_n ** 2)) / 2
            fa.coef = (t_n - 1) / t_np
            _lib.check(lib.odt_fista_update(C.byref(fa)))
        s.synchronize()
        out = ri.cpu().numpy().reshape(shape, order="F")
        self.RI_inter = out
        return out

    def delete(self):
        if self.forward_solver is not None:
            self.forward_solver.delete()
