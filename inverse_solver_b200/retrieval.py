"""Field retrieval from off-axis holograms (Codes/FIELD_EXPERIMENTAL_RETRIEVAL.m)
on the B200 library.  get_fields keeps the hologram stacks on the GPU from
upload to result: the transforms (centred FFTs of the background and sample
holograms, the sideband search and re-centring, the resolution crop / pad,
the NA circle, the inverse transforms: odt_hologram_fields), the
normalisation and the phase / amplitude of sp ./ bg (odt_hologram_phase),
Goldstein unwrapping (unwrap_goldstein_device) and the recombination with
the ramp-free phase (odt_hologram_combine).  Only the per-image scalar steps
run on the host, in MATLAB single semantics: the sub-pixel peak positions
and the border plane fit of PhiShiftMS, for which the unwrapped phase on the
border band (a few percent of the pixels) comes back from the device.  The
interactive branches of the reference (the "rectangle" ROI picker,
PhiShiftMS's hand-drawn masks) are not mirrored: ROI is numeric or absent.
"""
from __future__ import annotations

import copy
import ctypes as C
import math

import numpy as np

from . import _lib
from .optics import C64, F32, OpticalTool, basic_optical_parameter, mround, update_struct


def load_tiff(fname, num_images=None):
    """loadTIFF (FIELD_EXPERIMENTAL_RETRIEVAL.m:451-466): the pages of a TIFF
    file as a single-precision stack [rows, cols, pages] (squeezed to 2D for
    one page)."""
    from PIL import Image

    img = Image.open(fname)
    n = getattr(img, "n_frames", 1) if num_images is None else int(num_images)
    pages = []
    for k in range(n):
        img.seek(k)
        pages.append(np.asarray(img, dtype=F32))
    out = np.stack(pages, axis=2)
    return out[:, :, 0] if n == 1 else out


def _subpixel(pk, M):
    """peak_subpixel_positioner.m:1-67 on the peak data of one image (i1, i2
    1-based, |F| at the peak and at its neighbours along each axis): the
    position relative to the centre floor(M/2)+1 plus the neighbour-ratio
    refinement, in single precision."""
    i1, i2, v0, a1, b1, a2, b2 = (F32(x) for x in pk)
    centre = M // 2 + 1

    def refine(lo, hi):
        nb, sgn = (lo, -1) if lo >= hi else (hi, 1)   # max([lo, hi]): the first on ties
        d = np.array([nb / (nb + v0), nb / (nb - v0)], dtype=F32)
        d[np.abs(d) > 1] = 0
        return F32(sgn * d.max())

    return F32(F32(i1 - centre) + refine(a1, b1)), F32(F32(i2 - centre) + refine(a2, b2))


def _omit_outliers(v):
    lst = v[v != 0].astype(np.float64)
    p25, p75 = np.percentile(lst, [25, 75], method="hazen")        # MATLAB prctile
    lo, hi = p25 - 1.5 * (p75 - p25), p75 + 1.5 * (p75 - p25)
    out = v.copy()
    out[(out < lo) | (out > hi)] = 0
    return out


_BORDER = {}


def _border(imY, imX, bsize):
    """Column-major indices of the border of width bsize - 1 (PhiShiftMS's
    mask) with their x / y coordinates, and the full coordinate grids, per
    image shape."""
    key = (imY, imX, bsize)
    if key not in _BORDER:
        mask = np.ones((imY, imX), bool)
        mask[bsize - 1:imY - bsize + 1, bsize - 1:imX - bsize + 1] = False
        idx = np.flatnonzero(mask.ravel(order="F"))
        XX, YY = np.meshgrid(np.arange(1, imX + 1, dtype=np.float64), np.arange(1, imY + 1, dtype=np.float64))
        _BORDER[key] = (idx, XX.ravel(order="F")[idx], YY.ravel(order="F")[idx], XX.astype(F32),
                        YY.astype(F32))
    return _BORDER[key]


def _plane_coef(vb, bx, by):
    """D2_LSAms (n = 1) on the border values vb (column-major order, with
    their x / y coordinates): outliers and exact zeros left out, A'A in
    double, A'p and the solve in single, as MATLAB evaluates them; returns
    (x slope, y slope, height) in single."""
    v = _omit_outliers(vb)
    keep = v != 0
    A = np.stack([bx[keep], by[keep], np.ones(int(keep.sum()))], axis=1)
    return np.linalg.solve((A.T @ A).astype(F32), (A.astype(F32).T @ v[keep]).astype(F32)).astype(F32)


def phi_shift_ms(p2, bsize=8):
    """PhiShiftMS(p2, 1, 1) (sub_code/PhiShiftMS.m, D2_LSAms with n = 1 and
    omit_outliers): a + b x + c y fitted by least squares to the border of
    width bsize - 1 and subtracted; only the border pixels are visited, in
    the reference's column-major order."""
    imY, imX = p2.shape
    idx, bx, by, XX, YY = _border(imY, imX, bsize)
    coef = _plane_coef(np.asarray(p2, dtype=F32).ravel(order="F")[idx], bx, by)
    g = (p2 - coef[2]).astype(F32)
    g = (g - coef[0] * XX).astype(F32)
    return (g - coef[1] * YY).astype(F32)


ISOUTLIER_SCALE = 1.4826022185056018   # -1 / (sqrt(2) erfcinv(3/2)): MAD -> standard deviation


def _isoutlier(x):
    """MATLAB isoutlier(x), default 'median' method: more than three scaled
    median absolute deviations from the median."""
    x = np.asarray(x, dtype=np.float64)
    med = np.median(x)
    mad = ISOUTLIER_SCALE * np.median(np.abs(x - med))
    return (x < med - 3 * mad) | (x > med + 3 * mad)


def _stack(field):
    """A field array [N1, N2(, 1), n] as a Fortran-ordered complex64 stack
    [N1, N2, n]."""
    f = np.asarray(field, dtype=C64)
    return np.asfortranarray(f.reshape(f.shape[0], f.shape[1], -1, order="F"))


def _rmul(x, m):
    """MATLAB's real-times-complex product: both parts scaled by m."""
    out = np.empty(x.shape, dtype=C64)
    out.real = x.real * m
    out.imag = x.imag * m
    return out


def _col_major(a, device):
    """A CUDA tensor whose storage is the column-major layout of the numpy
    array a (its shape reversed)."""
    import torch

    if a.flags.f_contiguous:
        return torch.from_numpy(a.T).to(device)
    t = torch.from_numpy(np.ascontiguousarray(a)).to(device)
    return t.permute(*reversed(range(t.dim()))).contiguous()


class FIELD_EXPERIMENTAL_RETRIEVAL:
    """Codes/FIELD_EXPERIMENTAL_RETRIEVAL.m: complex fields from off-axis
    background / sample hologram pairs."""

    @staticmethod
    def get_default_parameters(init_params=None):
        """:8-22."""
        p = basic_optical_parameter()
        p.update(resolution_image=[0.1, 0.1], use_abbe_correction=True, cutout_portion=1 / 3,
                 other_corner=False, conjugate_field=False, use_GPU=True)
        return update_struct(p, init_params) if init_params else p

    def __init__(self, params):
        self.parameters = copy.deepcopy(params)
        self.utility = None
        self.lib = _lib.load()

    def get_fields(self, bg_file, sp_file, ROI=None):
        """:27-229 (numeric ROI [r0 r1 c0 c1], 1-based inclusive, or None):
        returns (input_field, output_field, updated_optical_parameters, k0s,
        is_overexposed, ROI); the holograms are TIFF file names or arrays
        [N, N(, n)]."""
        from .unwrap import unwrapp2_gpu

        p = self.parameters
        bg = load_tiff(bg_file) if isinstance(bg_file, str) else np.asarray(bg_file, dtype=F32)
        sp = load_tiff(sp_file) if isinstance(sp_file, str) else np.asarray(sp_file, dtype=F32)
        if bg.shape != sp.shape:
            raise ValueError("Background and sample field must be of same size")
        if bg.shape[0] != bg.shape[1]:
            raise ValueError("the image must be a square")
        if p["resolution_image"][0] != p["resolution_image"][1]:
            raise ValueError("please enter an isotropic resolution for the image")
        if p["resolution"][0] != p["resolution"][1]:
            raise ValueError("please enter an isotropic resolution for the output image")
        if ROI is not None:
            if isinstance(ROI, str):
                raise ValueError("the interactive ROI picker is not available; give [r0 r1 c0 c1]")
            bg = bg[ROI[0] - 1:ROI[1], ROI[2] - 1:ROI[3]]
            sp = sp[ROI[0] - 1:ROI[1], ROI[2] - 1:ROI[3]]
        if bg.ndim == 2:
            bg, sp = bg[:, :, None], sp[:, :, None]
        if bg.shape[0] != bg.shape[1]:
            raise ValueError("the image must be a square")
        N, nimg = bg.shape[0], bg.shape[2]
        # resolution matching (:131-145)
        ratio = p["resolution"][0] / p["resolution_image"][0]
        if ratio >= 1:
            d = int(mround(0.5 * (N - N / ratio)))
            M = N - 2 * d
        else:
            pad = -int(mround(0.5 * (N - N / ratio)))
            d, M = -pad, N + 2 * pad
        p["resolution"] = list(p["resolution"])
        p["resolution"][0] = p["resolution_image"][0] * N / M
        p["resolution"][1] = p["resolution_image"][1] * N / M
        p["size"] = list(p["size"])
        p["size"][0], p["size"][1] = M, M
        import torch

        dev = torch.device("cuda", torch.cuda.current_device())
        stream = torch.cuda.current_stream(dev)
        na = np.asfortranarray(OpticalTool(p).NA_circle.astype(np.uint8))
        hb, hs = _col_major(np.asarray(bg, dtype=F32), dev), _col_major(np.asarray(sp, dtype=F32), dev)
        over = (torch.maximum(hb, hs).amax(dim=(1, 2)) > 254).cpu().numpy()
        bgf = torch.empty((nimg, M - 4, M - 4), dtype=torch.complex64, device=dev)   # column-major [M-4, M-4, n]
        spf = torch.empty_like(bgf)
        peaks = torch.empty((nimg, 7), dtype=torch.float32, device=dev)
        nat = torch.from_numpy(na.T).to(dev)
        side = np.zeros(2, dtype=np.int32)
        a = _lib.HologramArgs()
        a.size[:] = [N, N, nimg]
        a.bg, a.sp = hb.data_ptr(), hs.data_ptr()
        a.cutout_portion = float(p["cutout_portion"])
        a.other_corner = 1 if p["other_corner"] else 0
        a.out_size, a.crop = M, d
        a.na_circle = nat.data_ptr()
        a.bg_field, a.sp_field = bgf.data_ptr(), spf.data_ptr()
        a.peaks, a.sideband = peaks.data_ptr(), _lib.ptr(side)
        a.memory = _lib.ODT_MEM_DEVICE
        a.stream = stream.cuda_stream
        _lib.check(self.lib.odt_hologram_fields(C.byref(a)))
        del hb, hs
        pk = peaks.cpu().numpy().T
        k0s = np.zeros((2, nimg), dtype=F32)
        for jj in range(nimg):
            k0s[0, jj], k0s[1, jj] = _subpixel(pk[:, jj], M)
        # normalisation, phase, unwrapping, ramp removal (:179-204)
        L = M - 4
        p["size"][0], p["size"][1] = L, L
        phase = torch.empty((nimg, L, L), dtype=torch.float32, device=dev)
        amp = torch.empty_like(phase)
        g = _lib.HologramPhaseArgs()
        g.size[:] = [L, L, nimg]
        g.bg, g.sp = bgf.data_ptr(), spf.data_ptr()
        g.conjugate = 1 if p["conjugate_field"] else 0
        g.phase, g.amp = phase.data_ptr(), amp.data_ptr()
        g.stream = stream.cuda_stream
        _lib.check(self.lib.odt_hologram_phase(C.byref(g)))
        phase = unwrapp2_gpu(phase.permute(2, 1, 0)).permute(2, 1, 0)   # column-major again, no copy
        idx, bx, by, _, _ = _border(L, L, 8)
        vb = phase.reshape(nimg, L * L)[:, torch.from_numpy(idx).to(dev)].cpu().numpy()
        coef = np.empty((nimg, 3), dtype=F32)
        for jj in range(nimg):
            cx, cy, c0 = _plane_coef(vb[jj], bx, by)
            coef[jj] = (c0, cx, cy)
        coef_d = torch.from_numpy(coef).to(dev)
        c = _lib.HologramCombineArgs()
        c.size[:] = [L, L, nimg]
        c.bg, c.amp, c.phase, c.coef = bgf.data_ptr(), amp.data_ptr(), phase.data_ptr(), coef_d.data_ptr()
        c.sp = spf.data_ptr()
        c.stream = stream.cuda_stream
        _lib.check(self.lib.odt_hologram_combine(C.byref(c)))
        bgh, sph = bgf.cpu().numpy().T, spf.cpu().numpy().T      # Fortran-ordered [L, L, n] views
        self.utility = OpticalTool(p)
        base = basic_optical_parameter()
        updated = {k: copy.deepcopy(p[k]) for k in base}
        return bgh[:, :, None, :], sph[:, :, None, :], updated, k0s, over, ROI

    def _utility(self):
        return self.utility if self.utility is not None else OpticalTool(self.parameters)

    def _fft2c(self, x, inverse=False):
        f = np.asfortranarray(np.asarray(x, dtype=C64)).copy(order="F")
        a = _lib.Fft2cArgs()
        a.size[:] = [f.shape[0], f.shape[1], 1 if f.ndim == 2 else f.shape[2]]
        a.data = _lib.ptr(f)
        a.inverse = 1 if inverse else 0
        a.memory = _lib.ODT_MEM_HOST
        a.stream = None
        _lib.check(self.lib.odt_fft2c(C.byref(a)))
        return f

    def get_aberration_pattern(self, input_field, output_field, correct_params):
        """:216-352 on the GPU (odt_aberration_pattern) with the optical tool
        of the last get_fields (or of the parameters).  correct_params holds
        overlap_factor, k0s [2, n] (get_fields' sub-pixel positions) and
        distList.  Returns (input_field_f, output_field_f, aberration_params
        = {pattern, distance, utility})."""
        u = self._utility()
        fin, fout = _stack(input_field), _stack(output_field)
        N1, N2, n = fin.shape
        if fout.shape != fin.shape:
            raise ValueError("input and output fields differ in size")
        if (N1, N2) != tuple(u.NA_circle.shape):
            raise ValueError("field and optical grid sizes differ")
        coorxy = np.asarray(u.coorxy, dtype=F32)
        fmask = np.asfortranarray(coorxy < coorxy.max() * F32(correct_params["overlap_factor"])).astype(np.uint8)
        na = np.asfortranarray(u.NA_circle.astype(np.uint8))
        rk = np.asfortranarray(np.asarray(u.refocusing_kernel, dtype=C64))
        k0s = np.asfortranarray(np.asarray(correct_params["k0s"], dtype=F32).reshape(2, -1))
        if k0s.shape[1] != n:
            raise ValueError("k0s must hold one position per field")
        dl = np.ascontiguousarray(np.atleast_1d(np.asarray(correct_params["distList"], dtype=np.float64)))
        pattern = np.empty((N1, N2), dtype=C64, order="F")
        oi, oo = np.empty_like(fin, order="F"), np.empty_like(fin, order="F")
        chosen = C.c_int32(0)
        a = _lib.AberrationArgs()
        a.size[:] = [N1, N2, n]
        a.input_field, a.output_field = _lib.ptr(fin), _lib.ptr(fout)
        a.k0s, a.pupil_mask, a.na_circle = _lib.ptr(k0s), _lib.ptr(fmask), _lib.ptr(na)
        a.refocusing_kernel = _lib.ptr(rk)
        a.dist_list, a.n_dist = _lib.ptr(dl), len(dl)
        a.pattern, a.input_out, a.output_out = _lib.ptr(pattern), _lib.ptr(oi), _lib.ptr(oo)
        a.chosen = C.cast(C.byref(chosen), C.c_void_p)
        a.memory = _lib.ODT_MEM_HOST
        a.stream = None
        _lib.check(self.lib.odt_aberration_pattern(C.byref(a)))
        shape = np.shape(input_field)
        return (oi.reshape(shape, order="F"), oo.reshape(shape, order="F"),
                {"pattern": pattern, "distance": float(dl[chosen.value]), "utility": u})

    def correct_aberration(self, input_field, field_trans, aberration_params):
        """:354-390: the pattern of get_aberration_pattern brought to these
        fields' Fourier resolution and field of view (the reference's steps,
        transforms on the GPU), masked by the NA circle of the pattern's
        coordinates, then both stacks filtered by exp(-1i angle(pattern)) on
        the GPU (odt_refocus_2d)."""
        u = self._utility()
        pattern = np.asarray(aberration_params["pattern"], dtype=C64)
        ua = aberration_params["utility"]
        N = np.shape(input_field)[0]
        target = int(mround(N * ua.fourier_res[0] / u.fourier_res[0] / 2) * 2)

        def half(a, b):
            d = float(np.floor(a - b)) / 2
            if d != int(d):
                raise ValueError("odd size difference in correct_aberration")
            return int(d)

        if target > N:
            p = self._fft2c(pattern)
            c = half(target, p.shape[0])
            p0 = np.zeros((target, target), dtype=C64)
            p0[c:target - c, c:target - c] = p
            pattern = self._fft2c(p0, inverse=True)
        elif target < N:
            p = self._fft2c(pattern)
            c = half(p.shape[0], target)
            pattern = self._fft2c(p[c:p.shape[0] - c, c:p.shape[1] - c], inverse=True)
        if pattern.shape[0] > N:
            c = half(pattern.shape[0], N)
            pattern = self._fft2c(pattern[c:pattern.shape[0] - c, c:pattern.shape[1] - c], inverse=True)
        elif pattern.shape[0] < N:
            c = half(target, pattern.shape[0])
            p0 = np.zeros((target, target), dtype=C64)
            p0[c:target - c, c:target - c] = pattern
            pattern = p0
        f1 = (np.asarray(ua.fourier_coor[0], dtype=F32) * F32(pattern.shape[0])) / F32(target)
        f2 = (np.asarray(ua.fourier_coor[1], dtype=F32) * F32(pattern.shape[1])) / F32(target)
        na = np.sqrt(f1[:, None] ** 2 + f2[None, :] ** 2) < u.kmax
        if na.shape != pattern.shape:
            raise ValueError("aberration pattern and optical grid sizes differ")
        filt = np.asfortranarray(np.exp(-1j * np.angle(_rmul(pattern, na.astype(F32))).astype(F32)).astype(C64))
        return self._filter(input_field, filt), self._filter(field_trans, filt)

    def _filter(self, field, kernel):
        f = _stack(field)
        if f.shape[:2] != kernel.shape:
            raise ValueError("field and pattern sizes differ")
        out = np.empty_like(f, order="F")
        a = _lib.RefocusArgs()
        a.size[:] = list(f.shape)
        a.field, a.kernel, a.out = _lib.ptr(f), _lib.ptr(kernel), _lib.ptr(out)
        _lib.check(self.lib.odt_refocus_2d(C.byref(a)))
        return out.reshape(np.shape(field), order="F")

    def remove_dirty_fields(self, input_field, output_field, prctile=95, manual_on=False):
        """:399-452 for scalar fields: per image the standard deviation of the
        gradient energy of |sp/bg|_k - |sp/bg|_1 and the fraction of the
        (GPU-unwrapped) phase outside 1.5 x [min, max] of the first image's
        (odt_field_quality); keeps the first field and those that are neither
        isoutlier nor above the fraction prctile / 100.  The manual review
        (manual_on) is interactive and not available."""
        if manual_on:
            raise ValueError("the manual review of remove_dirty_fields is interactive and not available")
        if np.ndim(input_field) == 4 and np.shape(input_field)[2] != 1:
            raise ValueError("remove_dirty_fields takes scalar fields (one polarisation)")
        bg, sp = _stack(input_field), _stack(output_field)
        if bg.shape != sp.shape:
            raise ValueError("input and output fields differ in size")
        N1, N2, n = bg.shape
        sd = np.empty(n, dtype=F32)
        cnt = np.empty(n, dtype=np.int64)
        a = _lib.FieldQualityArgs()
        a.size[:] = [N1, N2, n]
        a.bg, a.sp = _lib.ptr(bg), _lib.ptr(sp)
        a.gradient_std, a.outside_count = _lib.ptr(sd), _lib.ptr(cnt)
        a.memory = _lib.ODT_MEM_HOST
        a.stream = None
        _lib.check(self.lib.odt_field_quality(C.byref(a)))
        bad = cnt / float(N1 * N2) > prctile / 100
        keep = np.flatnonzero(~_isoutlier(sd) & ~bad)
        F = np.unique(np.concatenate([[0], keep])).astype(int)
        return bg[:, :, F].reshape(N1, N2, 1, len(F), order="F"), sp[:, :, F].reshape(N1, N2, 1, len(F), order="F")

    def refocus(self, field_trans, z):
        """:392-394 on the GPU (odt_refocus_2d), with the utility of the last
        get_fields (or of the parameters)."""
        u = self.utility if self.utility is not None else OpticalTool(self.parameters)
        f = np.asarray(field_trans, dtype=C64)
        shape = f.shape
        f = np.asfortranarray(f.reshape(shape[0], shape[1], -1, order="F"))
        k = np.asfortranarray(np.exp(z * np.asarray(u.refocusing_kernel)).astype(C64))
        if k.shape != shape[:2]:
            raise ValueError("field and optical grid sizes differ")
        out = np.empty_like(f, order="F")
        a = _lib.RefocusArgs()
        a.size[:] = [shape[0], shape[1], f.shape[2]]
        a.field, a.kernel, a.out = _lib.ptr(f), _lib.ptr(k), _lib.ptr(out)
        _lib.check(self.lib.odt_refocus_2d(C.byref(a)))
        return out.reshape(shape, order="F")
