"""Oracle: CPU restatement of the convergent-Born-series (CBS) forward solver.

TEST INFRASTRUCTURE ONLY -- imported by tests/, __graft_entry__.smoke() and
bench.py's CPU baseline legs; never by the product package.

Parity unpinned: the reference is MATLAB R2021a (no MATLAB/Octave here, no
stored outputs in the reference), so this module restates it line by line and
is pinned by known-answer properties only (see ``oracle/__init__.py``).

Two precisions:

* ``single=True``  -- MATLAB ``single`` semantics: every array op runs in
  float32 / complex64 and a double scalar meeting a single array is first
  converted to single (numpy's NEP-50 weak-scalar rule does exactly this for
  Python floats).  This is "the reference in single precision".
* ``single=False`` -- the same code in float64 / complex128: the FP64 oracle.

Array convention: numpy arrays indexed ``a[x, y, z, ...]`` where axis 0 is
MATLAB's first (fastest) dimension.  Column-major memory is only a concern
at the C-ABI boundary, not here.

The Born loop (``solve_raw``) is restated literally -- separate elementwise
sweeps, ``fft_flip`` of the Green's function and conjugation of the phase
ramp on every iteration, full 3D FFTs -- because that unfused form is also
what the CPU baseline times.
"""
from __future__ import annotations

import copy
import math
import os

import numpy as np
import scipy.fft as sfft
import scipy.special as ssp

_WORKERS = os.cpu_count() or 1


# ---------------------------------------------------------------- precision
class Prec:
    """float32 (MATLAB single) or float64 working precision."""

    def __init__(self, single: bool):
        self.single = bool(single)
        self.r = np.float32 if single else np.float64
        self.c = np.complex64 if single else np.complex128

    def R(self, x):
        return np.asarray(x, dtype=self.r)

    def C(self, x):
        return np.asarray(x, dtype=self.c)

    def S(self, x):
        """MATLAB ``single(x)`` in single mode, identity cast otherwise."""
        x = np.asarray(x)
        if np.iscomplexobj(x):
            return x.astype(self.c)
        return x.astype(self.r)


def mround(x):
    """MATLAB ``round``: half away from zero."""
    x = np.asarray(x, dtype=np.float64)
    return np.sign(x) * np.floor(np.abs(x) + 0.5)


# ------------------------------------------------------------- FFT helpers
def fftc2(x, inverse=False):
    """``fftshift(fft2(ifftshift(x)))`` on the first two axes (MATLAB's
    shifts over the remaining axes cancel because fft2 does not touch them)."""
    ax = (0, 1)
    y = np.fft.ifftshift(x, axes=ax)
    y = (sfft.ifft2 if inverse else sfft.fft2)(y, axes=ax, workers=_WORKERS)
    return np.fft.fftshift(y, axes=ax)


def fftc_axis(x, axis, inverse=False):
    y = np.fft.ifftshift(x, axes=(axis,))
    y = (sfft.ifft if inverse else sfft.fft)(y, axis=axis, workers=_WORKERS)
    return np.fft.fftshift(y, axes=(axis,))


def fftcn(x, inverse=False):
    y = np.fft.ifftshift(x)
    y = (sfft.ifftn if inverse else sfft.fftn)(y, workers=_WORKERS)
    return np.fft.fftshift(y)


# ------------------------------------------------------------ parameters
def basic_optical_parameter(init=None):
    """``sub_code/BASIC_OPTICAL_PARAMETER.m:1-15``."""
    p = dict(size=[100, 100, 100], wavelength=0.532, NA=1.2, RI_bg=1.336,
             resolution=[0.1, 0.1, 0.1], vector_simulation=True,
             use_abbe_sine=True)
    if init is not None:
        p = update_struct(p, init)
    return p


def update_struct(base, update):
    """``sub_code/update_struct.m:1-16`` (unknown fields are copied too)."""
    out = copy.deepcopy(base)
    for k, v in update.items():
        out[k] = copy.deepcopy(v)
    return out


def cbs_default_parameters(init=None):
    """``FORWARD_SOLVER.m:9-20`` + ``FORWARD_SOLVER_CONVERGENT_BORN.m:32-45``."""
    p = basic_optical_parameter()
    p.update(return_transmission=True, return_reflection=False,
             return_3D=False, use_GPU=True)
    p.update(iterations_number=-1, boundary_thickness=[6, 6, 6],
             boundary_sharpness=1, verbose=False, acyclic=True,
             RI_xy_size=[0, 0], RI_center=[0, 0])
    if init is not None:
        p = update_struct(p, init)
    return p


# ------------------------------------------------------ optical utilities
def derive_optical_tool(params, P: Prec):
    """``sub_code/DERIVE_OPTICAL_TOOL.m:1-81``."""
    res = [float(r) for r in params["resolution"]]
    size = [int(s) for s in params["size"]]
    u = {}
    ci, cf, fres = [], [], []
    for i in range(3):
        n = size[i]
        idx = P.R(np.arange(1, n + 1) - (n // 2 + 1))
        ci.append(idx * res[i])                       # :22-27
        fres.append(1.0 / (res[i] * n))               # :34-36
        cf.append(idx * fres[i])                      # :42-47
    u["image_coor"] = ci
    u["fourier_coor"] = cf
    u["fourier_res"] = fres
    u["image_res"] = res
    u["size"] = size
    coorxy = np.sqrt(cf[0][:, None] ** 2 + cf[1][None, :] ** 2)  # :51-53
    u["coorxy"] = coorxy
    lam = float(params["wavelength"])
    u["k0"] = 1.0 / lam
    u["k0_nm"] = u["k0"] * float(params["RI_bg"])
    u["nm"] = float(params["RI_bg"])
    u["kmax"] = float(params["NA"]) / lam
    u["NA_circle"] = coorxy < u["kmax"]                           # :60
    k3 = u["k0_nm"] ** 2 - coorxy ** 2                            # :61
    k3[k3 < 0] = 0
    k3 = np.sqrt(k3)
    u["k3"] = k3
    u["dV"] = res[0] * res[1] * res[2]                            # :62
    u["refocusing_kernel"] = (1j * 2 * math.pi) * k3              # :64
    u["cos_theta"] = k3 / u["k0_nm"]                              # :65
    return u


def ri2potential(RI, wavelength, base_RI, P: Prec):
    """``sub_code/RI2potential.m:1-5``."""
    k0 = 1.0 / wavelength
    k = 2 * math.pi * base_RI * k0
    return P.S(k ** 2 * (RI ** 2 / base_RI ** 2 - 1))


def potential2ri(pot, wavelength, base_RI, P: Prec):
    """``sub_code/potential2RI.m:1-5`` (MATLAB sqrt of a negative real is
    complex; the real-valued path is the one the configs use)."""
    k0 = 1.0 / wavelength
    k = 2 * math.pi * base_RI * k0
    arg = 1 + pot / k ** 2
    if not np.iscomplexobj(arg) and np.any(arg < 0):
        arg = arg.astype(P.c)
    return P.S(base_RI * np.sqrt(arg))


def fft_flip(a, flip_bool, use_shift):
    """``sub_code/fft_flip.m:1-11``."""
    for ii, fb in enumerate(flip_bool):
        if fb:
            a = np.flip(a, axis=ii)
            if a.shape[ii] % 2 == 0 or not use_shift:
                a = np.roll(a, 1, axis=ii)
    return a


# ------------------------------------------------ truncated Green function
def jn_roots(n, N):
    """Roots of J_n: ``hankel_transform/JnRoots.m:10-36`` (Gauss-Newton
    with a finite-difference slope, 100 rounds at most)."""
    eps = np.finfo(np.float64).eps

    def jv(order, x):
        return ssp.j0(x) if order == 0 else (ssp.j1(x) if order == 1 else ssp.jv(order, x))

    def step(r):
        b = (1 - eps / 2) * r
        f = (1 + eps) * r
        with np.errstate(invalid="ignore", divide="ignore"):
            f = np.real(jv(n, r)) * (f - b) / np.real(jv(n, f) - jv(n, b))
        f[np.abs(f) > 0.05] = 0.05
        f[np.isnan(f)] = 0
        return r - f

    r = n * math.pi / 2 - math.pi / 4 + math.pi * np.arange(1, N + 1, dtype=np.float64)
    r = step(r)
    m = np.ones(N, dtype=bool)
    K = 100
    while m.any() and K:
        R = step(r[m])
        k = r[m] != R
        r[m] = R
        m[m] = k
        K -= 1
    if n:
        r = np.concatenate([[0.0], r[r > 0]])[:N]
    return r


def _besselj(order, x):
    if order == 0:
        return ssp.j0(x)
    if order == 1:
        return ssp.j1(x)
    return ssp.jv(order, x)


class DiscreteHankelCroppedFourier:
    """``hankel_transform/discrete_hankel_croped_fourier.m:19-65``."""

    def __init__(self, max_r, samples, order, cropping, P: Prec):
        self.P = P
        n = order
        R = P.R(max_r)
        roots = P.S(jn_roots(n, samples + 1))
        C = roots[-1]
        c = roots[:-1]
        self.r = R / C * c                                        # :31
        k = c / R                                                 # :32
        self.pos = int(np.argmin(np.abs(k - k.max() * cropping))) + 1   # :34
        pos = self.pos
        I = np.abs(P.S(_besselj(1 + n, c.astype(np.float64))))   # :37
        self.K = 2 * math.pi * R / C * I                          # :38
        self.Rv = I / R                                           # :39
        I = np.sqrt(P.R(2) / C) / I                               # :40
        bess = P.S(_besselj(n, (c[:pos, None] / C * c[None, :]).astype(np.float64)))   # :41
        bess2 = P.S(_besselj(n, (c[:, None] / C * c[None, :pos]).astype(np.float64)))  # :42
        self.I2 = I[:, None] * I[None, :pos] * bess2              # :43
        self.I = I[:pos, None] * I[None, :] * bess                # :44
        self.k = k[:pos]                                          # :46

    def forward(self, vals):                                      # :54-59
        return (self.I @ (vals / self.Rv[:, None])) * self.K[:self.pos, None]

    def backward(self, vals):                                     # :60-65
        return (self.I2 @ (vals / self.K[:self.pos, None])) * self.Rv[:, None]


def _bin_search_nearest(value, searched_pos):
    """``truncated_green_plus.m:111-129`` (1-based indices returned)."""
    sp = searched_pos.ravel()
    nearest = np.ones(value.shape, dtype=np.int64)
    dist = sp.size
    step_up = dist
    while step_up > 1:
        step_up = int(math.ceil(step_up / 2))
        upper = nearest + step_up
        upper[upper > dist] = dist
        flag = sp[upper - 1] < value
        nearest = np.where(flag, upper, nearest)
    nearest2 = nearest.copy()
    sel = sp[nearest - 1] < value
    nearest2[sel] += 1
    nearest2[nearest2 > dist] = dist
    with np.errstate(invalid="ignore", divide="ignore"):
        blend = (value - sp[nearest - 1]) / (sp[nearest2 - 1] - sp[nearest - 1])
    blend[nearest2 == nearest] = 1
    return nearest, nearest2, blend


def truncated_green_plus(params, refocus_version, P: Prec):
    """``sub_code/truncated_green_plus.m:1-110`` (Vico-Greengard style
    xy-truncated Green's function through a cropped discrete Hankel
    transform)."""
    req = basic_optical_parameter()
    req.update(use_GPU=True, oversize_z=10, oversample_xy=20000,
               oversample_xy_fourier=2, simultanous_process=30)
    params = update_struct(req, params)
    res = np.asarray(params["resolution"], dtype=np.float64)
    out_px = np.asarray(params["size"], dtype=np.float64)
    crea_px = out_px * np.array([math.sqrt(2) * 1.1, math.sqrt(2) * 1.1, 1.0]) + params["oversize_z"]
    crea = crea_px * res
    max_size = crea[:2].max()
    crea_px[:2] = np.ceil(max_size / res[:2])
    params["size"] = [int(round(v)) for v in crea_px]
    out_px = [int(v) for v in out_px]
    u = derive_optical_tool(params, P)
    samples = params["oversample_xy"] * params["oversample_xy_fourier"]
    S1, S2, Nz = params["size"]
    if samples < math.sqrt(S1 ** 2 + S2 ** 2) * 5:
        raise ValueError("the code might not be valid for such big array")
    hk = DiscreteHankelCroppedFourier(
        1, samples, 0,
        (math.sqrt(S1 ** 2 + S2 ** 2) * params["oversample_xy_fourier"]) / (2 * samples), P)
    H = hk.r
    H = H / H.max()
    H = H * (u["coorxy"].max() * params["oversample_xy_fourier"])   # :43
    Hk3 = u["k0_nm"] ** 2 - H ** 2
    Hk3[Hk3 < 0] = 0
    Hk3 = np.sqrt(Hk3)
    Hcirc = H < u["kmax"]
    fz = u["fourier_coor"][2]
    fres3 = u["fourier_res"][2]
    ratio = (Nz - params["oversize_z"] / 2) / Nz
    arg = (Hk3[:, None] - fz[None, :]) / fres3 * ratio
    green = np.sinc(arg) * ratio                                  # :47-49
    green = P.S(green)
    if not refocus_version:
        green = green * Hcirc[:, None] / (Hk3 + (~Hcirc))[:, None]
        green = green / (1j * 4 * math.pi)
    else:
        green = green * Hcirc[:, None]
    img = hk.forward(green)
    nk = hk.k / hk.k.max()
    mask = (nk < 0.9) + (nk < 1) * (nk > 0.9) * (1 - nk) * 10     # :62
    img = img * P.S(mask)[:, None]
    green = hk.backward(img)
    near, near2, blend = _bin_search_nearest(u["coorxy"], H)
    green_out = np.zeros((out_px[0], out_px[1], Nz), dtype=P.c)
    slices = list(range(1, Nz + 1, params["simultanous_process"]))
    if len(slices) == 1 or slices[-1] != Nz:
        slices.append(Nz)
    scale = Nz / (u["image_res"][0] * u["image_res"][1])
    for ii in range(len(slices) - 1):
        zi = np.arange(slices[ii], slices[ii + 1] + 1)
        g = green[:, zi - 1]
        gs = g[near - 1, :] * blend[:, :, None] + g[near2 - 1, :] * (1 - blend)[:, :, None]
        gs = gs * scale
        gs = fftc2(gs, inverse=True)
        rs = [S1 // 2 + 1 - out_px[0] // 2, S2 // 2 + 1 - out_px[1] // 2]
        gs = gs[rs[0] - 1:rs[0] - 1 + out_px[0], rs[1] - 1:rs[1] - 1 + out_px[1], :]
        gs = fftc2(gs)
        green_out[:, :, zi - 1] = gs
    green_out = fftc_axis(green_out, 2, inverse=True)
    zs = Nz // 2 + 1 - out_px[2] // 2
    green_out = green_out[:, :, zs - 1:zs - 1 + out_px[2]]
    green_out = fftc_axis(green_out, 2)
    return green_out


def polarisation_utility(ZP, params, P: Prec):
    """``FORWARD_SOLVER.m:131-180``: per k-pixel radial / perpendicular unit
    vectors of the pupil plane, the unit tangent of the Ewald sphere and the
    propagating-wave mask.  Returns (Radial_2D [N1,N2,2], Perp_2D [N1,N2,2],
    ewald_TanVec [N1,N2,3], K_mask [N1,N2]).  The reference builds K_2 with
    ZP(1) as the end of its range (:139), so the field must be square."""
    N1, N2 = int(ZP[0]), int(ZP[1])
    if N1 != N2:
        raise ValueError("the polarisation basis needs a square field")
    lam = float(params["wavelength"])
    dx = [float(v) for v in params["resolution"]]
    k0 = 1.0 / lam
    k = 2 * math.pi * float(params["RI_bg"]) * k0
    kres = [1.0 / dx[0] / N1, 1.0 / dx[1] / N2]
    K1 = P.R(2 * math.pi * kres[0] / k * np.arange(-(N1 // 2), N1 - N1 // 2, dtype=np.float64))[:, None]
    K2 = P.R(2 * math.pi * kres[1] / k * np.arange(-(N2 // 2), N1 - N2 // 2, dtype=np.float64))[None, :]
    s3 = P.R(1) - (K1 ** 2 + K2 ** 2)
    K3 = np.sqrt(np.maximum(s3, 0)).astype(P.r)        # real(sqrt(.)) of a negative is 0
    K_mask = ~(K3 == 0)
    nr = np.sqrt(K1 ** 2 + K2 ** 2)
    with np.errstate(invalid="ignore", divide="ignore"):
        t1 = K1 / nr
        t2 = K2 / nr
    t1 = np.where(nr == 0, P.R(1), t1)
    t2 = np.where(nr == 0, P.R(0), t2)
    R2 = np.stack([t1, t2], axis=2).astype(P.r)
    P2 = np.stack([t2, -t1], axis=2).astype(P.r)
    ns = np.sqrt((K1 ** 2 + K2 ** 2) + K3 ** 2)
    R3 = np.stack([np.broadcast_to(K1 / ns, ns.shape), np.broadcast_to(K2 / ns, ns.shape), K3 / ns], axis=2).astype(P.r)
    proj = R3[:, :, 0] * R2[:, :, 0] + R3[:, :, 1] * R2[:, :, 1]
    E = np.zeros((N1, N1, 3), dtype=P.r)
    E[:, :, 0:2] = R2
    E = (E - proj[:, :, None] * R3).astype(P.r)
    en = np.sqrt((E[:, :, 0] ** 2 + E[:, :, 1] ** 2) + E[:, :, 2] ** 2)
    en[~K_mask] = 1
    E = (E / en[:, :, None]).astype(P.r)
    return R2, P2, E, K_mask


# ---------------------------------------------------------- the solver
class ForwardSolverCBS:
    """Restatement of ``Codes/FORWARD_SOLVER_CONVERGENT_BORN.m``: the scalar
    Green's function, and with ``vector_simulation`` the dyadic one
    (``pole_num = 3``), for an isotropic RI ``[x, y, z]`` or, with the dyadic
    Green's function, an RI tensor ``[x, y, z, 3, 3]`` (``size(RI,4) > 1``)."""

    def __init__(self, params, single=True):
        """Constructor ``:48-133``."""
        self.P = P = Prec(single)
        self.parameters = p = copy.deepcopy(params)
        self.vector = bool(p.get("vector_simulation", False))
        self.utility = derive_optical_tool(p, P)
        p["RI_xy_size"] = list(p["RI_xy_size"])
        if p["RI_xy_size"][0] == 0:
            p["RI_xy_size"][0] = p["size"][0]
        if p["RI_xy_size"][1] == 0:
            p["RI_xy_size"][1] = p["size"][1]
        self.expected_RI_size = [p["RI_xy_size"][0], p["RI_xy_size"][1], p["size"][2]]
        bt = p["boundary_thickness"]
        self.cyclic_boundary_xy = (bt[0] == 0 and bt[1] == 0
                                   and self.expected_RI_size[0] == p["size"][0]
                                   and self.expected_RI_size[1] == p["size"][1])
        u = self.utility
        rc = p["RI_center"]
        if self.cyclic_boundary_xy:                                   # :65-72
            ru = np.exp(u["refocusing_kernel"][:, :, None] * u["image_coor"][2][None, None, :])
            ru = ru * u["NA_circle"][:, :, None]
            fsg = ru / (1j * 4 * math.pi)
            fsg = fsg * (u["NA_circle"] / (u["k3"] + (~u["NA_circle"])))[:, :, None]
            fsg = fsg / (u["image_res"][0] * u["image_res"][1])
            fsg = fftc2(fsg, inverse=True)
            self.refocusing_util = ru
        else:                                                         # :74-108
            ptg = copy.deepcopy(p)
            ptg["size"] = [p["size"][0] + self.expected_RI_size[0] + rc[0],
                           p["size"][1] + self.expected_RI_size[1] + rc[1],
                           p["size"][2]]
            ru = truncated_green_plus(ptg, True, P)
            ru = self._crop_center_shift(ru, rc)
            ru = fftcn(ru, inverse=True)
            ru = fftc2(ru)
            ru = ru * (u["image_res"][0] * u["image_res"][1])
            self.refocusing_util = ru
            fsg = truncated_green_plus(ptg, False, P)
            fsg = self._crop_center_shift(fsg, rc)
            fsg = fftcn(fsg, inverse=True)
        self.kernel_trans = fftc2(np.conj(fsg))                       # :114
        self.kernel_ref = fftc2(fsg)                                  # :115
        bt = np.asarray(bt, dtype=np.float64)
        if bt.size != 3:
            raise ValueError("boundary_thickness must have 3 entries")
        self.boundary_thickness_pixel = mround(
            (bt * p["wavelength"] / p["RI_bg"]) / (np.asarray(p["resolution"], dtype=np.float64) * 2)
        ).astype(int)                                                 # :129

    @staticmethod
    def _crop_center_shift(a, rc):
        a = a[-min(0, rc[0]):a.shape[0] - max(0, rc[0]), -min(0, rc[1]):a.shape[1] - max(0, rc[1]), :]
        return np.roll(a, (-rc[0], -rc[1]), axis=(0, 1))

    # --- padding / cropping helpers :134-179
    def _conv_size(self):
        p = self.parameters
        return [p["size"][0] + self.expected_RI_size[0], p["size"][1] + self.expected_RI_size[1]]

    def padd_RI2conv(self, m):
        if self.cyclic_boundary_xy:
            return m
        C = self._conv_size()
        rc = self.parameters["RI_center"]
        add_start = [-(m.shape[i] // 2 - C[i] // 2) + rc[i] for i in range(2)]
        add_end = [C[i] - m.shape[i] - add_start[i] for i in range(2)]
        pad = [(add_start[0], add_end[0]), (add_start[1], add_end[1])] + [(0, 0)] * (m.ndim - 2)
        return np.pad(m, pad)

    def padd_field2conv(self, m):
        if self.cyclic_boundary_xy:
            return m
        C = self._conv_size()
        add_start = [-(m.shape[i] // 2 - C[i] // 2) for i in range(2)]
        add_end = [C[i] - m.shape[i] - add_start[i] for i in range(2)]
        pad = [(add_start[0], add_end[0]), (add_start[1], add_end[1])] + [(0, 0)] * (m.ndim - 2)
        return np.pad(m, pad)

    def crop_conv2field(self, m):
        if self.cyclic_boundary_xy:
            return m
        sz = self.parameters["size"]
        s = [m.shape[i] // 2 + 1 - sz[i] // 2 for i in range(2)]
        return m[s[0] - 1:s[0] - 1 + sz[0], s[1] - 1:s[1] - 1 + sz[1], ...]

    def crop_field2RI(self, m):
        sz = self.parameters["size"]
        rc = self.parameters["RI_center"]
        s = [m.shape[i] // 2 + 1 - sz[i] // 2 + rc[i] for i in range(2)]
        return m[s[0] - 1:s[0] - 1 + sz[0], s[1] - 1:s[1] - 1 + sz[1], ...]

    def crop_conv2RI(self, m):
        return self.crop_field2RI(self.crop_conv2field(m))

    # --- set_RI :180-198
    def set_RI(self, RI):
        """``:180-198``; the struct form ``{"scatt_pott": RI}`` is accepted for
        a tensor RI only (``:181-186``)."""
        if isinstance(RI, dict):
            RI = np.asarray(RI["scatt_pott"])
            if RI.ndim < 4 or RI.shape[3] <= 1:
                raise ValueError("Structur form only allowed for tensor RI")
        RI = np.asarray(RI)
        if list(RI.shape[:3]) != list(self.expected_RI_size):
            raise ValueError("The refractive index does not have the expected size")
        self.tensor = RI.ndim >= 4 and RI.shape[3] > 1
        if self.tensor and (RI.shape[3:] != (3, 3) or not self.vector):
            raise ValueError("a tensor RI is [x, y, z, 3, 3] and needs vector_simulation")
        if not self.tensor:
            RI = RI.reshape(RI.shape[:3])
        self.RI = self.P.S(RI)
        self.condition_RI()
        self.init()

    def condition_RI(self):
        """``:199-222``.  For a tensor RI the reference takes the largest
        singular value of ``pagesvd(permute(pott(:), [4 5 1 2 3]))``: the pages
        of the flattened column are 1 x 1, so that is max |potential| over all
        nine components, as for the scalar case."""
        P, p = self.P, self.parameters
        pot = ri2potential(self.RI.ravel(), p["wavelength"], p["RI_bg"], P)
        self.eps_imag = P.S(np.abs(pot).max() * 1.01)                 # :201-205
        self.ROI = self.create_boundary_RI()
        V = ri2potential(self.RI, p["wavelength"], p["RI_bg"], P)
        if self.tensor:                                               # :216-219
            V = P.S(V).astype(P.c)
            for j1 in range(3):
                V[:, :, :, j1, j1] = V[:, :, :, j1, j1] - 1j * self.eps_imag
            self.V = V
        else:
            self.V = V - 1j * self.eps_imag                           # :215
            self.V = P.S(self.V)

    def create_boundary_RI(self):
        """``:223-279``: zero-potential padding, ROI, attenuation mask."""
        P, p = self.P, self.parameters
        btp = [int(b) for b in self.boundary_thickness_pixel]  # Python ints keep single ops single
        old = self.RI.shape
        RIp = ri2potential(self.RI, p["wavelength"], p["RI_bg"], P)
        RIp = np.pad(RIp, [(btp[0], btp[0]), (btp[1], btp[1]), (btp[2], btp[2])]
                     + [(0, 0)] * (RIp.ndim - 3))
        RIp = potential2ri(RIp, p["wavelength"], p["RI_bg"], P)
        ROI = [btp[0] + 1, btp[0] + old[0], btp[1] + 1, btp[1] + old[1], btp[2] + 1, btp[2] + old[2]]
        V_temp = ri2potential(RIp, p["wavelength"], p["RI_bg"], P)
        mask = None
        self.mask1d = []
        for j1 in range(3):
            n = V_temp.shape[j1]
            x = P.R(np.abs(np.arange(1, n + 1) - math.floor(n / 2 + 1) + 0.5) - 0.5)
            x = np.roll(x, -(n // 2))
            x = x / (btp[j1] - 0.5)
            val0 = x.copy()
            val0[np.abs(x) >= 1] = 1
            val0 = np.abs(val0)
            val0 = 1 - val0
            sh = p["boundary_sharpness"]
            val0[val0 > sh] = sh
            val0 = val0 / sh
            if btp[j1] == 0:
                val0[:] = 0
            fac = 1 - val0 * 1
            self.mask1d.append(fac)
            shp = [1, 1, 1]
            shp[j1] = n
            mask = fac.reshape(shp) if mask is None else mask * fac.reshape(shp)
        self.attenuation_mask = mask
        self.RI = potential2ri(V_temp, p["wavelength"], p["RI_bg"], P)
        return ROI

    def init(self):
        """``:280-396``: Green's function, phase ramp, iteration count."""
        P, p = self.P, self.parameters
        pb = copy.deepcopy(p)
        pb["size"] = list(self.RI.shape[:3])
        ub = self.utility_border = derive_optical_tool(pb, P)
        self.pole_num = 3 if self.vector else 1                      # :293-296
        fc, fr = ub["fourier_coor"], ub["fourier_res"]
        if p["acyclic"] and self.cyclic_boundary_xy:
            sc = [fc[0], fc[1], fc[2] + fr[2] / 4]
        elif p["acyclic"]:
            sc = [fc[0] + fr[0] / 4, fc[1] + fr[1] / 4, fc[2] + fr[2] / 4]
        else:
            sc = list(fc)
        self.shifted_coordinate = sc
        k0nm = ub["k0_nm"]
        # rads(:,:,:,i) = shifted_coordinate{i} / k0_nm (:316-319); the
        # absorptive correction of the dyadic Green's function (:322)
        self.rads1d = [P.S(P.S(sc[i]) / k0nm) for i in range(3)]
        a2 = P.S((2 * math.pi * k0nm) ** 2)
        self.green_absorbtion_correction = P.S(a2 / P.S(a2 + 1j * self.eps_imag))
        step = P.S(abs(2 * (2 * math.pi * k0nm) / self.eps_imag))     # :326
        nrm = float(np.linalg.norm(np.asarray(self.RI.shape[:3], dtype=np.float64) * np.asarray(p["resolution"], dtype=np.float64)))
        Bopt = math.ceil(float(P.S(P.S(nrm / step) / 2 + 1))) * 2      # :327
        it = p["iterations_number"]
        if it == 0:
            self.Bornmax = 0
        elif it < 0:
            self.Bornmax = Bopt * abs(it)
        else:
            self.Bornmax = int(it)
        A = (sc[0] ** 2)[:, None, None] + (sc[1] ** 2)[None, :, None] + (sc[2] ** 2)[None, None, :]
        G = 4 * math.pi ** 2 * np.abs(A) - (2 * math.pi * k0nm) ** 2 - 1j * self.eps_imag
        self.Greenp = P.S(1 / P.S(G))                                # :347-351
        if p["acyclic"]:
            if self.boundary_thickness_pixel[0] == 0 and self.boundary_thickness_pixel[1] == 0:
                n = self.V.shape[2]
                x = np.exp(-1j * math.pi * (np.arange(1, n + 1) - 1) / n / 2)
                x = x / x[n // 2]
                ramp = x.reshape(1, 1, n)
                self.ramp1d = [np.ones(self.V.shape[0]), np.ones(self.V.shape[1]), x]
            else:
                ramp = None
                self.ramp1d = []
                for j1 in range(3):
                    n = self.V.shape[j1]
                    x = P.S(np.exp(-1j * math.pi * (np.arange(1, n + 1) - 1) / n / 2))
                    x = x / x[n // 2]
                    self.ramp1d.append(x)
                    shp = [1, 1, 1]
                    shp[j1] = n
                    ramp = x.reshape(shp) if ramp is None else ramp * x.reshape(shp)
            self.phase_ramp = P.S(ramp)
            self.ramp1d = [P.S(r) for r in self.ramp1d]
        else:
            self.phase_ramp = np.ones((1, 1, 1), dtype=P.c)
            self.ramp1d = None
        self.Greenp = np.fft.ifftshift(self.Greenp)                  # :384
        if self.pole_num == 3:                                        # :385
            n = self.V.shape[:3]
            r = np.zeros(tuple(n) + (3,), dtype=P.r)
            r[..., 0] = self.rads1d[0][:, None, None]
            r[..., 1] = self.rads1d[1][None, :, None]
            r[..., 2] = self.rads1d[2][None, None, :]
            self.rads = np.fft.ifftshift(r, axes=(0, 1, 2))

    # --- solve :397-520
    def transform_field_3D(self, f):
        """``FORWARD_SOLVER.m:38-68``: pupil (NA, Abbe sine) and, for two
        polarisations, the 2 -> 3 component change of basis."""
        u = self.utility
        NA = u["NA_circle"]
        f = f * NA.reshape(NA.shape + (1,) * (f.ndim - 2))
        if self.parameters["use_abbe_sine"]:
            filt = self.P.R(NA)
            filt[NA] = filt[NA] / np.sqrt(u["cos_theta"][NA])
            f = f * filt.reshape(filt.shape + (1,) * (f.ndim - 2))
        if f.ndim < 3 or f.shape[2] == 1:
            return f
        if f.shape[2] != 2:
            raise ValueError("Far field has two polarisation")
        R2, P2, E, K = polarisation_utility(f.shape[:2], self.parameters, self.P)
        f = f * K[:, :, None, None]
        b1 = f[:, :, 0] * R2[:, :, 0, None] + f[:, :, 1] * R2[:, :, 1, None]
        b2 = f[:, :, 0] * P2[:, :, 0, None] + f[:, :, 1] * P2[:, :, 1, None]
        out = np.zeros((f.shape[0], f.shape[1], 3, f.shape[3]), dtype=self.P.c)
        out = out + b1[:, :, None, :] * E[:, :, :, None]
        out[:, :, 0:2] = out[:, :, 0:2] + b2[:, :, None, :] * P2[:, :, :, None]
        return out

    def transform_field_2D(self, f, reflection=False):
        """``FORWARD_SOLVER.m:69-128``: pupil (NA, Abbe sine) and, for three
        components, the 3 -> 2 polarisation change of basis (the reflection
        variant flips the axial component of the tangent vector, :113)."""
        u = self.utility
        NA = u["NA_circle"]
        sh = NA.shape + (1,) * (f.ndim - 2)
        f = f * NA.reshape(sh)
        if self.parameters["use_abbe_sine"]:
            f = f * np.sqrt(u["cos_theta"]).reshape(sh) * NA.reshape(sh)
        if f.ndim < 3 or f.shape[2] == 1:
            return f
        if f.shape[2] != 3:
            raise ValueError("Near field has three polarisation")
        R2, P2, E, K = polarisation_utility(f.shape[:2], self.parameters, self.P)
        if reflection:
            E = E.copy()
            E[:, :, 2] = -E[:, :, 2]
        f = f * K.reshape(K.shape + (1,) * (f.ndim - 2))
        x = f if f.ndim == 4 else f[..., None]
        b1 = (x[:, :, 0] * E[:, :, 0, None] + x[:, :, 1] * E[:, :, 1, None]) + x[:, :, 2] * E[:, :, 2, None]
        b2 = x[:, :, 0] * P2[:, :, 0, None] + x[:, :, 1] * P2[:, :, 1, None]
        out = np.zeros((x.shape[0], x.shape[1], 2, x.shape[3]), dtype=self.P.c)
        out = out + b1[:, :, None, :] * R2[:, :, :, None]
        out = out + b2[:, :, None, :] * P2[:, :, :, None]
        return out if f.ndim == 4 else out[..., 0]

    def solve(self, input_field):
        P, p = self.P, self.parameters
        inp = P.S(np.asarray(input_field))
        if inp.ndim == 2:
            inp = inp[:, :, None, None]
        elif inp.ndim == 3:
            inp = inp[:, :, :, None]
        if inp.shape[2] > 1 and not self.vector:                      # :404-414
            raise ValueError("the source is 2D but parameter indicate a vectorial simulation")
        if inp.shape[2] == 1 and self.vector:
            raise ValueError("the source is 3D but parameter indicate a non-vectorial simulation")
        if inp.shape[2] > 2:
            raise ValueError("Input field must be either a scalar or a 2D vector")
        inp = fftc2(inp)
        inp = self.transform_field_3D(inp)
        R = self.ROI
        nx, ny, nz = R[1] - R[0] + 1, R[3] - R[2] + 1, R[5] - R[4] + 1
        nill = inp.shape[3]
        npol = inp.shape[2]
        out_pol = 2 if self.pole_num == 3 else 1
        ft = np.ones((nx, ny, out_pol, nill), dtype=P.c) if p["return_transmission"] else None
        fr = np.ones((nx, ny, out_pol, nill), dtype=P.c) if p["return_reflection"] else None
        f3 = np.ones((nx, ny, nz, npol, nill), dtype=P.c) if p["return_3D"] else None
        for k in range(nill):
            src = inp[:, :, :, k] if self.vector else inp[:, :, 0, k]
            Field = self.solve_raw(src)
            F4 = Field if self.vector else Field[..., None]
            if p["return_3D"]:
                f3[:, :, :, :, k] = F4
            if p["return_transmission"] or p["return_reflection"]:
                pot = ri2potential(self.RI[R[0] - 1:R[1], R[2] - 1:R[3], R[4] - 1:R[5]], p["wavelength"], p["RI_bg"], P)
                if self.tensor:                                       # :451-455
                    em = 0
                    for j1 in range(3):
                        em = em + F4[..., j1:j1 + 1] * pot[:, :, :, :, j1] * self.utility_border["dV"]
                else:
                    em = F4 * pot[..., None] * self.utility_border["dV"]
                em = self.padd_RI2conv(em)
                em = fftc2(em)
            if p["return_transmission"]:
                t = self.crop_conv2field(fftc2(np.sum(em * self.kernel_trans[..., None], axis=2), inverse=True))
                t = fftc2(t) + inp[:, :, :, k]
                t = self.transform_field_2D(t)
                ft[:, :, :, k] = fftc2(t, inverse=True)
            if p["return_reflection"]:
                r = self.crop_conv2field(fftc2(np.sum(em * self.kernel_ref[..., None], axis=2), inverse=True))
                r = fftc2(r)
                r = self.transform_field_2D(r, reflection=True)
                fr[:, :, :, k] = fftc2(r, inverse=True)
        return ft, fr, f3

    def refocus_source(self, source):
        """``solve_raw :543-554``: 2D input spectrum -> 3D incident field."""
        s = fftc2(source, inverse=True)
        s = self.padd_field2conv(s)
        s = fftc2(s)
        if s.ndim == 3:   # components: [C, C, 1, 3] .* refocusing_util
            s = s[:, :, None, :] * self.refocusing_util[:, :, :, None]
        else:
            s = s[:, :, None] * self.refocusing_util
        s = fftc2(s, inverse=True)
        return self.crop_conv2RI(s)

    def solve_raw(self, source, n_iter=None):
        """``:521-654``: the Born loop, restated literally.  ``n_iter``
        truncates the loop (used only to time a bounded CPU sample)."""
        P = self.P
        vec = self.pole_num == 3
        if source.ndim == 3 and not vec:
            source = source[:, :, 0]
        V = self.V
        ten = getattr(self, "tensor", False)
        shp = V.shape[:3] + ((3,) if vec else ())
        psi = np.zeros(shp, dtype=P.c)
        Field = np.zeros(shp, dtype=P.c)
        Field_n = np.zeros(shp, dtype=P.c)
        source = self.refocus_source(source)
        incident = source
        R = self.ROI
        roi = (slice(R[0] - 1, R[1]), slice(R[2] - 1, R[3]), slice(R[4] - 1, R[5]))
        Vx = V[..., None] if vec else V
        if ten:                                                       # :567-574
            src0 = source
            source = np.zeros_like(src0)
            for j1 in range(3):
                source = source + V[roi][:, :, :, :, j1] * src0[..., j1:j1 + 1]
            source = source + 1j * self.eps_imag * src0
        else:
            source = ((V[roi] + 1j * self.eps_imag)[..., None] if vec else (V[roi] + 1j * self.eps_imag)) * source  # :566
        Greenp = self.Greenp
        ramp = self.phase_ramp
        rads = self.rads if vec else None
        corr = self.green_absorbtion_correction
        acyc = self.parameters["acyclic"]
        c = 1j / self.eps_imag
        nB = self.Bornmax if n_iter is None else min(n_iter, self.Bornmax)
        temp = None
        for jj in range(1, nB + 1):
            if acyc:
                Greenp = fft_flip(Greenp, [1, 1, 1], False)
                if vec:
                    rads = fft_flip(rads, [1, 1, 1], False)
                ramp = np.conj(ramp)
            psi[...] = 0
            if jj in (1, 2):
                Field_n[...] = 0
                psi[roi] = c * source / 2
            elif ten:                                                 # :592-594
                for j1 in range(3):
                    psi = psi + c * Field_n[..., j1:j1 + 1] * V[:, :, :, :, j1]
            else:
                psi = c * Field_n * Vx
            if vec:   # dyadic absorptive Green's function (:597-601)
                PSI = np.zeros(shp, dtype=P.c)
                for j2 in range(3):
                    coeff = sfft.fftn(psi[..., j2] * ramp, workers=_WORKERS)
                    eye = np.zeros(3, dtype=P.r)
                    eye[j2] = 1
                    d = eye - (corr * rads) * rads[..., j2:j2 + 1]
                    PSI = PSI + (Greenp[..., None] * d) * coeff[..., None]
                for j1 in range(3):
                    PSI[..., j1] = sfft.ifftn(PSI[..., j1], workers=_WORKERS) * np.conj(ramp)
            else:
                PSI = Greenp * sfft.fftn(psi * ramp, workers=_WORKERS)
                PSI = sfft.ifftn(PSI, workers=_WORKERS) * np.conj(ramp)
            if jj not in (1, 2):
                Field_n = Field_n - psi
            if ten:                                                   # :624-627
                for j1 in range(3):
                    Field_n = Field_n + V[:, :, :, :, j1] * PSI[..., j1:j1 + 1]
            else:
                Field_n = Field_n + Vx * PSI
            Field_n = Field_n * (self.attenuation_mask[..., None] if vec else self.attenuation_mask)
            if jj == 2:
                temp = Field
            Field = Field + Field_n
            if jj == 3:
                Field_n = Field_n + temp
                temp = None
        return Field[roi] + incident


# ---------------------------------------------------------- convenience
def rel_l2(a, b):
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return float(d / n) if n > 0 else float(d)
