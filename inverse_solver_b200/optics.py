"""Host-side optical setup in MATLAB ``single`` semantics.

These are the geometry-dependent quantities the MATLAB classes compute before
handing work to the GPU (in the reference's CUDA variant they are computed on
the host as well: FORWARD_SOLVER_CONVERGENT_BORN_CUDA.m:20 sets use_GPU=false
for the setup).  Everything runs in float32 / complex64 with double scalars
converted to single before each operation, which is what MATLAB does for
single arrays (numpy's weak Python-scalar rule gives the same behaviour).

Arrays are indexed ``a[x, y, z]`` (axis 0 = MATLAB's first dimension).
"""
from __future__ import annotations

import copy
import math
import os

import numpy as np
import scipy.fft as sfft
import scipy.special as ssp

F32 = np.float32
C64 = np.complex64
_WORKERS = os.cpu_count() or 1


def basic_optical_parameter(init=None):
    """BASIC_OPTICAL_PARAMETER (sub_code/BASIC_OPTICAL_PARAMETER.m:1-15)."""
    p = {"size": [100, 100, 100], "wavelength": 0.532, "NA": 1.2, "RI_bg": 1.336,
         "resolution": [0.1, 0.1, 0.1], "vector_simulation": True, "use_abbe_sine": True}
    return update_struct(p, init) if init else p


def update_struct(base, update):
    """update_struct (sub_code/update_struct.m:1-16): unknown fields are kept."""
    out = copy.deepcopy(base)
    if update:
        for k, v in update.items():
            out[k] = copy.deepcopy(v)
    return out


def mround(x):
    """MATLAB round (half away from zero)."""
    x = np.asarray(x, dtype=np.float64)
    return np.sign(x) * np.floor(np.abs(x) + 0.5)


def centered_fft2(x, inverse=False):
    """fftshift(fft2(ifftshift(x))) over the first two axes, single precision."""
    y = np.fft.ifftshift(x, axes=(0, 1))
    y = (sfft.ifft2 if inverse else sfft.fft2)(y, axes=(0, 1), workers=_WORKERS)
    return np.fft.fftshift(y, axes=(0, 1))


def centered_fft_axis(x, axis, inverse=False):
    y = np.fft.ifftshift(x, axes=(axis,))
    y = (sfft.ifft if inverse else sfft.fft)(y, axis=axis, workers=_WORKERS)
    return np.fft.fftshift(y, axes=(axis,))


def centered_fftn(x, inverse=False):
    y = np.fft.ifftshift(x)
    y = (sfft.ifftn if inverse else sfft.fftn)(y, workers=_WORKERS)
    return np.fft.fftshift(y)


class OpticalTool:
    """DERIVE_OPTICAL_TOOL (sub_code/DERIVE_OPTICAL_TOOL.m:1-81)."""

    def __init__(self, params):
        self.image_res = [float(r) for r in params["resolution"]]
        self.size = [int(s) for s in params["size"]]
        self.image_coor, self.fourier_coor, self.fourier_res = [], [], []
        for i in range(3):
            n = self.size[i]
            idx = np.arange(1, n + 1, dtype=F32) - F32(n // 2 + 1)
            self.image_coor.append(idx * self.image_res[i])
            fr = 1.0 / (self.image_res[i] * n)
            self.fourier_res.append(fr)
            self.fourier_coor.append(idx * fr)
        c0, c1 = self.fourier_coor[0], self.fourier_coor[1]
        self.coorxy = np.sqrt(c0[:, None] ** 2 + c1[None, :] ** 2)
        lam = float(params["wavelength"])
        self.k0 = 1.0 / lam
        self.k0_nm = self.k0 * float(params["RI_bg"])
        self.kmax = float(params["NA"]) / lam
        self.NA_circle = self.coorxy < self.kmax
        k3 = self.k0_nm ** 2 - self.coorxy ** 2
        k3[k3 < 0] = 0
        self.k3 = np.sqrt(k3)
        self.dV = self.image_res[0] * self.image_res[1] * self.image_res[2]
        self.refocusing_kernel = (1j * 2 * math.pi) * self.k3
        self.cos_theta = self.k3 / self.k0_nm


def polarisation_basis(field_size, params):
    """polarisation_utility (FORWARD_SOLVER.m:131-180) in single precision:
    per pixel of the centred [N, N] field spectrum the pupil-plane radial and
    perpendicular unit vectors, the unit tangent of the Ewald sphere and the
    mask of propagating waves.  Returns (radial [N,N,2], perp [N,N,2],
    tangent [N,N,3], kmask [N,N] bool).  Square fields only: the reference
    builds its second coordinate with the first size as the range end."""
    n1, n2 = int(field_size[0]), int(field_size[1])
    if n1 != n2:
        raise ValueError("the dyadic solver needs a square field (polarisation_utility)")
    k = 2 * math.pi * float(params["RI_bg"]) / float(params["wavelength"])
    res = [float(r) for r in params["resolution"]]
    kx = (2 * math.pi * (1.0 / res[0] / n1) / k
          * np.arange(-(n1 // 2), n1 - n1 // 2, dtype=np.float64)).astype(F32)[:, None]
    ky = (2 * math.pi * (1.0 / res[1] / n2) / k
          * np.arange(-(n2 // 2), n1 - n2 // 2, dtype=np.float64)).astype(F32)[None, :]
    kxy2 = kx * kx + ky * ky
    kz = np.sqrt(np.maximum(F32(1) - kxy2, F32(0)))
    kmask = kz != 0
    rho = np.sqrt(kxy2)
    with np.errstate(invalid="ignore", divide="ignore"):
        ux, uy = kx / rho, ky / rho
    ux = np.where(rho == 0, F32(1), ux).astype(F32)
    uy = np.where(rho == 0, F32(0), uy).astype(F32)
    radial = np.stack([ux, uy], axis=2)
    perp = np.stack([uy, -ux], axis=2)
    rn = np.sqrt(kxy2 + kz * kz)
    s3 = [np.broadcast_to(kx / rn, rn.shape), np.broadcast_to(ky / rn, rn.shape), kz / rn]
    proj = s3[0] * ux + s3[1] * uy
    t = [(ux - proj * s3[0]).astype(F32), (uy - proj * s3[1]).astype(F32), (F32(0) - proj * s3[2]).astype(F32)]
    tn = np.sqrt((t[0] * t[0] + t[1] * t[1]) + t[2] * t[2])
    tn[~kmask] = 1
    tangent = np.stack([c / tn for c in t], axis=2).astype(F32)
    return radial.astype(F32), perp.astype(F32), tangent, kmask


def ri2potential(RI, wavelength, base_RI):
    """RI2potential (sub_code/RI2potential.m:1-5)."""
    k = 2 * math.pi * base_RI * (1.0 / wavelength)
    RI = np.asarray(RI)
    if RI.dtype not in (np.float32, np.complex64):
        RI = RI.astype(C64 if np.iscomplexobj(RI) else F32)
    return k ** 2 * (RI ** 2 / base_RI ** 2 - 1)


def potential2ri(pot, wavelength, base_RI):
    """potential2RI (sub_code/potential2RI.m:1-5); sqrt of a negative real
    argument is complex as in MATLAB."""
    k = 2 * math.pi * base_RI * (1.0 / wavelength)
    arg = 1 + pot / k ** 2
    if not np.iscomplexobj(arg) and np.any(arg < 0):
        arg = arg.astype(C64)
    return base_RI * np.sqrt(arg)


# ------------------------------------------------ truncated Green's function
def bessel_j(order, x):
    if order == 0:
        return ssp.j0(x)
    if order == 1:
        return ssp.j1(x)
    return ssp.jv(order, x)


def bessel_zeros(n, N):
    """First N positive zeros of J_n by the Gauss-Newton iteration with a
    finite-difference slope of hankel_transform/JnRoots.m:10-36."""
    eps = np.finfo(np.float64).eps

    def step(r):
        lo = (1 - eps / 2) * r
        hi = (1 + eps) * r
        with np.errstate(invalid="ignore", divide="ignore"):
            d = np.real(bessel_j(n, r)) * (hi - lo) / np.real(bessel_j(n, hi) - bessel_j(n, lo))
        d[np.abs(d) > 0.05] = 0.05
        d[np.isnan(d)] = 0
        return r - d

    r = n * math.pi / 2 - math.pi / 4 + math.pi * np.arange(1, N + 1, dtype=np.float64)
    r = step(r)
    active = np.ones(N, dtype=bool)
    for _ in range(100):
        if not active.any():
            break
        nr = step(r[active])
        changed = r[active] != nr
        r[active] = nr
        active[active] = changed
    if n:
        r = np.concatenate([[0.0], r[r > 0]])[:N]
    return r


class CroppedHankel:
    """Discrete Hankel transform restricted to the low-k band
    (hankel_transform/discrete_hankel_croped_fourier.m:19-65)."""

    def __init__(self, max_r, samples, order, cropping):
        R = F32(max_r)
        self.roots64 = bessel_zeros(order, samples + 1)
        roots = self.roots64.astype(F32)
        C = roots[-1]
        c = roots[:-1]
        self.r = R / C * c
        k = c / R
        self.pos = int(np.argmin(np.abs(k - k.max() * cropping))) + 1
        self.order, self.R, self.C, self.c = order, R, C, c
        I = np.abs(bessel_j(1 + order, c.astype(np.float64)).astype(F32))
        self.K = 2 * math.pi * R / C * I
        self.Rv = I / R
        self.scale = np.sqrt(F32(2) / C) / I
        self.k = k[:self.pos]
        self._fwd = self._bwd = None

    def _matrices(self):
        """The Bessel matrices (:41-42), built on first use (most of the
        set-up time on the host; the GPU path builds them on the device)."""
        if self._fwd is None:
            p, c, C, s = self.pos, self.c, self.C, self.scale
            b1 = bessel_j(self.order, (c[:p, None] / C * c[None, :]).astype(np.float64)).astype(F32)
            b2 = bessel_j(self.order, (c[:, None] / C * c[None, :p]).astype(np.float64)).astype(F32)
            self._fwd = s[:p, None] * s[None, :] * b1
            self._bwd = s[:, None] * s[None, :p] * b2
        return self._fwd, self._bwd

    def forward(self, vals):
        fwd, _ = self._matrices()
        return (fwd @ (vals / self.Rv[:, None])) * self.K[:self.pos, None]

    def backward(self, vals):
        _, bwd = self._matrices()
        return (bwd @ (vals / self.K[:self.pos, None])) * self.Rv[:, None]


_HANKEL_CACHE = {}


def _cropped_hankel(samples, cropping):
    """The order-0 unit-radius transform of truncated_green_plus; the
    refocusing kernel and the Green's function of one geometry use the same
    one, so it is built once (its Bessel matrices are most of the set-up
    time).  Keeps the last few."""
    key = (int(samples), float(cropping))
    hk = _HANKEL_CACHE.get(key)
    if hk is None:
        if len(_HANKEL_CACHE) >= 4:
            _HANKEL_CACHE.pop(next(iter(_HANKEL_CACHE)))
        hk = _HANKEL_CACHE[key] = CroppedHankel(1, samples, 0, cropping)
    return hk


def _nearest_bins(value, grid):
    """Bracketing sample indices and linear weight of `value` in the sorted
    `grid` (truncated_green_plus.m:111-129), 1-based like the reference."""
    g = grid.ravel()
    n = g.size
    near = np.ones(value.shape, dtype=np.int64)
    step = n
    while step > 1:
        step = int(math.ceil(step / 2))
        up = np.minimum(near + step, n)
        near = np.where(g[up - 1] < value, up, near)
    near2 = near.copy()
    near2[g[near - 1] < value] += 1
    near2[near2 > n] = n
    with np.errstate(invalid="ignore", divide="ignore"):
        w = (value - g[near - 1]) / (g[near2 - 1] - g[near - 1])
    w[near2 == near] = 1
    return near, near2, w


def truncated_green_radial(params, refocus_version=False, hankel_filter=None):
    """The radial part of truncated_green_plus (sub_code/truncated_green_plus.m
    :1-66 and bin_search_nearest :111-129): the band-limited radial profile
    [samples, Nz] and the interpolation maps of the oversized xy grid.
    Returns a dict (green, near, near2, w, creation [S1, S2, Nz], out_px,
    scale).  ``hankel_filter(hk, green, band)``, if given, replaces the host
    forward transform / band window / backward transform (:45-53)."""
    req = basic_optical_parameter()
    req.update(use_GPU=True, oversize_z=10, oversample_xy=20000, oversample_xy_fourier=2,
               simultanous_process=30)
    params = update_struct(req, params)
    res = np.asarray(params["resolution"], dtype=np.float64)
    out_px = [int(v) for v in params["size"]]
    crea = np.asarray(out_px, dtype=np.float64) * np.array([math.sqrt(2) * 1.1, math.sqrt(2) * 1.1, 1.0])
    crea = crea + params["oversize_z"]
    size_um = crea * res
    crea[:2] = np.ceil(size_um[:2].max() / res[:2])
    params["size"] = [int(round(v)) for v in crea]
    S1, S2, Nz = params["size"]
    u = OpticalTool(params)
    ovf = params["oversample_xy_fourier"]
    samples = params["oversample_xy"] * ovf
    if samples < math.sqrt(S1 ** 2 + S2 ** 2) * 5:
        raise ValueError("truncated_green_plus: grid too large for the Hankel sampling")
    hk = _cropped_hankel(samples, (math.sqrt(S1 ** 2 + S2 ** 2) * ovf) / (2 * samples))
    H = hk.r / hk.r.max()
    H = H * (u.coorxy.max() * ovf)
    Hk3 = u.k0_nm ** 2 - H ** 2
    Hk3[Hk3 < 0] = 0
    Hk3 = np.sqrt(Hk3)
    Hin = H < u.kmax
    ratio = (Nz - params["oversize_z"] / 2) / Nz
    green = np.sinc((Hk3[:, None] - u.fourier_coor[2][None, :]) / u.fourier_res[2] * ratio) * ratio
    green = green.astype(F32)
    if refocus_version:
        green = green * Hin[:, None]
    else:
        green = green * Hin[:, None] / (Hk3 + (~Hin))[:, None]
        green = green / (1j * 4 * math.pi)
    nk = hk.k / hk.k.max()
    band = ((nk < 0.9) + (nk < 1) * (nk > 0.9) * (1 - nk) * 10).astype(F32)
    if hankel_filter is not None:
        green = hankel_filter(hk, green, band)
    else:
        img = hk.forward(green)
        green = hk.backward(img * band[:, None])
    near, near2, w = _nearest_bins(u.coorxy, H)
    return dict(green=green, near=near, near2=near2, w=w, creation=[S1, S2, Nz], out_px=out_px,
                scale=Nz / (u.image_res[0] * u.image_res[1]), simultanous_process=params["simultanous_process"])


def centred_dft_matrix(n, inverse=False):
    """C[k, j] with C @ x = fftshift(fft(ifftshift(x))) (ifft with 1/n for
    inverse), in double."""
    c = n // 2
    k = np.arange(n) - c
    e = np.exp((2j if inverse else -2j) * math.pi * np.outer(k, k) / n)
    return e / n if inverse else e


def green_plane_maps(r):
    """The linear maps of truncated_green_plus's plane part (:67-110) for the
    GPU path: centred inverse DFT of the oversized length, crop to the output
    length, centred forward DFT, per axis, as [out, S] complex64 matrices."""
    S1, S2, Nz = r["creation"]
    o = r["out_px"]
    offs = [S1 // 2 - o[0] // 2, S2 // 2 - o[1] // 2, Nz // 2 - o[2] // 2]
    maps = []
    for n, m, r0 in zip((S1, S2, Nz), o, offs):
        maps.append((centred_dft_matrix(m) @ centred_dft_matrix(n, inverse=True)[r0:r0 + m, :]).astype(C64))
    return maps


def truncated_green_planes(r):
    """The plane part of truncated_green_plus (:67-110) on the host: the
    radial profile interpolated onto the oversized xy grid per z, centred
    inverse 2D FFT, crop to the output xy size, centred forward 2D FFT, then
    the centred inverse z-FFT, crop to the output z size and forward z-FFT."""
    green, near, near2, w = r["green"], r["near"], r["near2"], r["w"]
    S1, S2, Nz = r["creation"]
    out_px = r["out_px"]
    out = np.zeros((out_px[0], out_px[1], Nz), dtype=C64)
    slices = list(range(1, Nz + 1, r["simultanous_process"]))
    if len(slices) == 1 or slices[-1] != Nz:
        slices.append(Nz)
    r0 = S1 // 2 - out_px[0] // 2
    r1 = S2 // 2 - out_px[1] // 2
    for a, b in zip(slices[:-1], slices[1:]):
        zi = np.arange(a - 1, b)
        g = green[:, zi]
        gs = g[near - 1, :] * w[:, :, None] + g[near2 - 1, :] * (1 - w)[:, :, None]
        gs = centered_fft2(gs * r["scale"], inverse=True)
        gs = centered_fft2(gs[r0:r0 + out_px[0], r1:r1 + out_px[1], :])
        out[:, :, zi] = gs
    out = centered_fft_axis(out, 2, inverse=True)
    z0 = Nz // 2 - out_px[2] // 2
    out = out[:, :, z0:z0 + out_px[2]]
    return centered_fft_axis(out, 2)


def truncated_green_plus(params, refocus_version=False):
    """xy-truncated free-space Green's function (or refocusing kernel) on the
    [size(1), size(2), size(3)] grid, Fourier in xy and z
    (sub_code/truncated_green_plus.m:1-110)."""
    return truncated_green_planes(truncated_green_radial(params, refocus_version))
