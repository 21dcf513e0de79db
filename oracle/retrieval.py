"""CPU restatement of the field retrieval front-end
(Codes/FIELD_EXPERIMENTAL_RETRIEVAL.m) -- test infrastructure (the oracle):
only the tests and the benchmark's CPU baseline import it.

Covers the non-interactive path of get_fields (:27-229; the "rectangle" ROI
picker and the GUI branches of PhiShiftMS are interactive and out of scope)
with its helpers sub_code/CPU_placement_finder_prepare.m:1-19,
sub_code/peak_subpixel_positioner.m:1-67 and sub_code/PhiShiftMS.m (mask
style 1, D2_LSAms with n = 1, omit_outliers: :1-44, :103-166), and refocus
(:392-394), get_aberration_pattern (:216-352), correct_aberration
(:354-390) and remove_dirty_fields (:399-452; without the manual review).
MATLAB single semantics: single(x) * double(y) is single,
prctile is numpy's "hazen" percentile, find / max return the first hit in
column-major order.  Parity is unpinned: the reference ships no holograms.
"""
from __future__ import annotations

import copy
import math

import numpy as np

from .cbs import basic_optical_parameter, derive_optical_tool, fftc2, mround, update_struct, Prec

F32 = np.float32
C64 = np.complex64


def retrieval_default_parameters(init=None):
    """FIELD_EXPERIMENTAL_RETRIEVAL.m:8-22."""
    p = basic_optical_parameter()
    p.update(resolution_image=[0.1, 0.1], use_abbe_correction=True, cutout_portion=1 / 3,
             other_corner=False, conjugate_field=False, use_GPU=True)
    if init is not None:
        p = update_struct(p, init)
    return p


def placement_finder_prepare(size1, size2, size3, limit):
    """CPU_placement_finder_prepare.m:1-19 (grids of positions relative to
    the centre floor(n/2)+1, 1-based)."""
    g1 = (np.arange(1, size1 + 1, dtype=F32) - (size1 // 2 + 1))[:, None, None] * np.ones((1, size2, size3), F32)
    g2 = (np.arange(1, size2 + 1, dtype=F32) - (size2 // 2 + 1))[None, :, None] * np.ones((size1, 1, size3), F32)
    g3 = (np.arange(1, size3 + 1, dtype=F32) - (size3 // 2 + 1))[None, None, :] * np.ones((size1, size2, 1), F32)
    g4 = (np.abs(g1) <= limit) * (np.abs(g2) <= limit) * (np.abs(g3) <= limit)
    return g1, g2, g3, g4


def peak_subpixel_positioner(peak_img, p1, p2):
    """peak_subpixel_positioner.m:1-67 for a 2D image: position of the
    maximum (first in column-major order) relative to the centre, refined
    by the ratio of the larger neighbour along each axis."""
    img = np.asarray(peak_img)
    flat = img.ravel(order="F")
    m = int(np.argmax(flat))
    pos1 = float(p1.ravel(order="F")[m])
    pos2 = float(p2.ravel(order="F")[m])
    i1, i2 = m % img.shape[0], m // img.shape[0]
    c = [i1 - 1, i1 + 1]
    i1b = c[int(np.argmax([img[i1 - 1, i2], img[i1 + 1, i2]]))]
    c = [i2 - 1, i2 + 1]
    i2b = c[int(np.argmax([img[i1, i2 - 1], img[i1, i2 + 1]]))]

    def frac(nb):
        v0 = img[i1, i2]
        d = np.array([nb / (nb + v0), nb / (nb - v0)], dtype=img.dtype)
        d = np.real(d)
        d[np.abs(d) > 1] = 0
        return d

    d1 = np.sign(i1b - i1) * frac(img[i1b, i2]).max()
    d2 = np.sign(i2b - i2) * frac(img[i1, i2b]).max()
    return F32(pos1 + d1), F32(pos2 + d2)


def omit_outliers(p2mask):
    """PhiShiftMS.m omit_outliers: zero the values outside
    [p25 - 1.5 IQR, p75 + 1.5 IQR] of the non-zero entries."""
    lst = p2mask.ravel(order="F")
    lst = lst[lst != 0].astype(np.float64)
    p25, p75 = np.percentile(lst, [25, 75], method="hazen")
    cmin = p25 - 1.5 * (p75 - p25)
    cmax = p75 + 1.5 * (p75 - p25)
    out = p2mask.copy()
    out[out < cmin] = 0
    out[out > cmax] = 0
    return out


def d2_lsams(p2, n, mask):
    """PhiShiftMS.m D2_LSAms with a mask: least-squares fit of
    a0 + sum_i (c_i x^i + d_i y^i) to the masked, outlier-free non-zero
    pixels (A'A in double; A'p and the solve in single, as MATLAB evaluates a
    double matrix against single data), subtracted from p2."""
    imY, imX = p2.shape
    XX, YY = np.meshgrid(np.arange(1, imX + 1, dtype=np.float64), np.arange(1, imY + 1, dtype=np.float64))
    p2mask = omit_outliers((p2 * mask).astype(F32))
    v = p2mask.ravel(order="F")
    keep = v != 0
    cols = [(XX ** i).ravel(order="F")[keep] for i in range(1, n + 1)]
    cols += [(YY ** i).ravel(order="F")[keep] for i in range(1, n + 1)]
    cols.append(np.ones(int(keep.sum())))
    AA = np.stack(cols, axis=1)                 # double, as MATLAB builds it
    rhs = v[keep].astype(F32)
    AtA = (AA.T @ AA).astype(F32)               # double product, then single for the mixed solve
    Atp = (AA.astype(F32).T @ rhs).astype(F32)  # double * single -> single
    coef = np.linalg.solve(AtA, Atp).astype(F32)
    good = (p2 - coef[-1]).astype(F32)
    for i in range(1, n + 1):
        good = (good - coef[i - 1] * (XX ** i).astype(F32)).astype(F32)
        good = (good - coef[n + i - 1] * (YY ** i).astype(F32)).astype(F32)
    return good, coef


def phi_shift_ms(p2):
    """PhiShiftMS(p2, 1, 1): first-order ramp fitted on the border (bsize 8)."""
    imY, imX = p2.shape
    bsize = 8
    mask = np.ones((imY, imX), F32)
    mask[bsize - 1:imY - bsize + 1, bsize - 1:imX - bsize + 1] = 0
    good, _ = d2_lsams(p2, 1, mask)
    return good


def _delete_bands(n1, n2, cutout, other_corner):
    b1 = np.arange(int(mround(n1 * cutout)), n1 + 1) - 1
    if other_corner:
        b2 = np.arange(1, int(mround(n2 * (1 - cutout))) + 1) - 1
    else:
        b2 = np.arange(int(mround(n2 * cutout)), n2 + 1) - 1
    return b1, b2


def get_fields(params, bg, sp, roi=None, unwrap=None):
    """:27-229 without the interactive ROI: returns (input_field,
    output_field, updated_optical_parameters, k0s, is_overexposed).  `unwrap`
    is the phase unwrapper (unwrapp2_gpu); the oracle passes its own
    Goldstein restatement."""
    p = copy.deepcopy(params)
    P = Prec(True)
    bg = np.asarray(bg, dtype=F32)
    sp = np.asarray(sp, dtype=F32)
    if bg.ndim == 2:
        bg, sp = bg[:, :, None], sp[:, :, None]
    if bg.shape != sp.shape:
        raise ValueError("Background and sample field must be of same size")
    if bg.shape[0] != bg.shape[1]:
        raise ValueError("the image must be a square")
    if roi is not None:
        bg = bg[roi[0] - 1:roi[1], roi[2] - 1:roi[3]]
        sp = sp[roi[0] - 1:roi[1], roi[2] - 1:roi[3]]
    over = np.maximum(bg, sp).max(axis=(0, 1)) > 254
    fb = fftc2(bg.astype(C64)).astype(C64)
    fs = fftc2(sp.astype(C64)).astype(C64)
    n1, n2 = fb.shape[:2]
    b1, b2 = _delete_bands(n1, n2, p["cutout_portion"], p["other_corner"])
    nb = fb[:, :, 0].copy()
    nb[b1, :] = 0
    nb[:, b2] = 0
    a = np.abs(nb)
    m = int(np.argmax(a.ravel(order="F")))
    c1, c2 = m % n1 + 1, m // n1 + 1
    def centre(f):
        f = np.roll(f, (1 - c1, 1 - c2), axis=(0, 1))
        return np.fft.fftshift(np.fft.fftshift(f, axes=0), axes=1)
    fb, fs = centre(fb), centre(fs)
    old = fb.shape[0]
    ratio = p["resolution"][0] / p["resolution_image"][0]
    if ratio >= 1:
        c = int(mround(0.5 * (fb.shape[0] - fb.shape[0] / ratio)))
        fb = fb[c:fb.shape[0] - c, c:fb.shape[1] - c]
        fs = fs[c:fs.shape[0] - c, c:fs.shape[1] - c]
    else:
        pd = -int(mround(0.5 * (fb.shape[0] - fb.shape[0] / ratio)))
        fb = np.pad(fb, ((pd, pd), (pd, pd), (0, 0)))
        fs = np.pad(fs, ((pd, pd), (pd, pd), (0, 0)))
    p["resolution"] = list(p["resolution"])
    p["resolution"][0] = p["resolution_image"][0] * old / fb.shape[0]
    p["resolution"][1] = p["resolution_image"][1] * old / fb.shape[1]
    p["size"] = list(p["size"])
    p["size"][0], p["size"][1] = fb.shape[0], fb.shape[1]
    u = derive_optical_tool(p, P)
    na = np.asarray(u["NA_circle"])[:, :, None]
    fb = (fb * na).astype(C64)
    fs = (fs * na).astype(C64)
    p1, p2, _, _ = placement_finder_prepare(fb.shape[0], fb.shape[1], 1, 1)
    k0s = np.zeros((2, fb.shape[2]), F32)
    for jj in range(fb.shape[2]):
        k0s[0, jj], k0s[1, jj] = peak_subpixel_positioner(np.abs(fb[:, :, jj]), p1[:, :, 0], p2[:, :, 0])
    bgf = fftc2(fb, inverse=True).astype(C64)
    spf = fftc2(fs, inverse=True).astype(C64)
    bgf = bgf[2:-2, 2:-2]
    spf = spf[2:-2, 2:-2]
    p["size"][0], p["size"][1] = bgf.shape[0], bgf.shape[1]
    amean = (np.abs(bgf).sum(axis=(0, 1)) / (bgf.shape[0] * bgf.shape[1])).astype(F32)
    bgf = (bgf / amean).astype(C64)
    spf = (spf / amean).astype(C64)
    if p["conjugate_field"]:
        bgf, spf = np.conj(bgf), np.conj(spf)
    ratio_f = (spf / bgf).astype(C64)
    phase = np.angle(ratio_f).astype(F32)
    phase = unwrap(phase) if unwrap is not None else phase
    amp = np.abs(ratio_f).astype(F32)
    for jj in range(phase.shape[2]):
        phase[:, :, jj] = phi_shift_ms(phase[:, :, jj])
    spf = (amp * bgf * np.exp(1j * phase).astype(C64)).astype(C64)
    bgf = bgf[:, :, None, :]
    spf = spf[:, :, None, :]
    base = basic_optical_parameter()
    upd = {k: p[k] for k in base}
    return bgf, spf, upd, k0s, over


def refocus(params, field, z):
    """:392-394: fftshift(ifft2(ifftshift(fftshift(fft2(ifftshift(f))) .*
    exp(z .* refocusing_kernel))))."""
    u = derive_optical_tool(params, Prec(True))
    k = np.exp(z * np.asarray(u["refocusing_kernel"])).astype(C64)
    f = fftc2(np.asarray(field, dtype=C64)).astype(C64)
    sh = (slice(None), slice(None)) + (None,) * (f.ndim - 2)
    return fftc2((f * k[sh]).astype(C64), inverse=True).astype(C64)


# ------------------------------------------------ aberration and dirty fields
def _rmul(x, m):
    """MATLAB's real-times-complex product: both parts scaled by the real m
    (which fixes the signed zeros that angle() sees where m is 0)."""
    x = np.asarray(x, dtype=C64)
    out = np.empty(np.broadcast_shapes(x.shape, np.shape(m)), dtype=C64)
    out.real = x.real * m
    out.imag = x.imag * m
    return out


def _stack(field):
    f = np.asarray(field, dtype=C64)
    return f.reshape(f.shape[0], f.shape[1], -1, order="F")


def _phasor(z):
    return np.exp(1j * np.angle(z).astype(F32)).astype(C64)


def get_aberration_pattern(u, input_field, output_field, correct_params):
    """FIELD_EXPERIMENTAL_RETRIEVAL.m:216-352 (get_aberration_pattern) with
    the optical tool u of the fields (derive_optical_tool) and correct_params
    {overlap_factor, k0s [2, n], distList}; returns (input_field_f,
    output_field_f, aberration_params = {pattern, distance, utility}).  The
    pixel sums are taken in double (the reference sums in single; the order
    of a single-precision sum is not defined there)."""
    fin, fout = _stack(input_field), _stack(output_field)
    N1, N2, n = fin.shape
    NA = np.asarray(u["NA_circle"]).astype(F32)
    coorxy = np.asarray(u["coorxy"], dtype=F32)
    rk = np.asarray(u["refocusing_kernel"], dtype=C64)
    # stitch pupil (:217-227)
    fE = fftc2((fout / fin).astype(C64)).astype(C64)
    fmask = (coorxy < coorxy.max() * F32(correct_params["overlap_factor"])).astype(F32)
    fdp = _rmul(_phasor((fE * np.conj(fE[:, :, :1])).astype(C64)), fmask[:, :, None])
    k0s = np.asarray(correct_params["k0s"], dtype=F32).reshape(2, -1)
    sh = mround(k0s).astype(int)
    P = np.empty_like(fdp)
    for k in range(n):
        P[:, :, k] = np.roll(fdp[:, :, k], (sh[0, k], sh[1, k]), axis=(0, 1))
    P = _rmul(P, NA[:, :, None])
    # relative phase (:235-276), images in the order of |k0s| (stable sort)
    seq = np.argsort(np.sqrt(k0s[0] * k0s[0] + k0s[1] * k0s[1]), kind="stable")
    S = np.zeros((N1, N2), dtype=C64)
    for ii in range(1, n):
        S = (S + P[:, :, seq[ii - 1]]).astype(C64)
        cur = P[:, :, seq[ii]]
        keep = (np.abs(S) > 0) & (np.abs(cur) > 0)
        t = (S * np.conj(cur)).astype(C64)[keep]
        b = np.angle(np.complex64(t.astype(np.complex128).sum())).astype(F32)
        P[:, :, seq[ii]] = (cur * np.exp(1j * b).astype(C64)).astype(C64)
    P2 = P[:, :, 0].copy()
    for k in range(1, n):
        P2 = (P2 + P[:, :, k]).astype(C64)
    # defocus search (:284-296)
    dl = np.atleast_1d(np.asarray(correct_params["distList"], dtype=np.float64))
    cc = np.zeros(len(dl), dtype=F32)
    ph2 = np.exp(-1j * np.angle(P2).astype(F32)).astype(C64)
    for i, d in enumerate(dl):
        t = _rmul((np.exp((rk * F32(d)).astype(C64)) * ph2).astype(C64), NA)
        cc[i] = np.abs(np.complex64(t.astype(np.complex128).sum()))
    cmax = int(np.argmax(cc))
    approx = (rk * F32(dl[cmax])).astype(C64)
    approx = (approx - approx[N1 // 2, N2 // 2]).astype(C64)
    ea = np.exp(1j * approx).astype(C64)
    # low-pass box from the most frequent sideband step (:307-326)
    k2 = mround(k0s[1]).astype(F32)
    vals, counts = np.unique(np.diff(k2), return_counts=True)
    if len(vals) == 0:
        raise ValueError("get_aberration_pattern needs at least two fields")
    dist = F32(abs(vals[int(np.argmax(counts))]) * F32(2))
    if not dist > 0:
        raise ValueError("the most frequent step of round(k0s(2,:)) is 0 (no low-pass box)")
    c1, c2 = N1 // 2, N2 // 2
    r0, r1 = c1 - int(np.floor(F32(N1) / dist)), c1 + int(np.ceil(F32(N1) / dist))
    q0, q1 = c2 - int(np.floor(F32(N2) / dist)), c2 + int(np.ceil(F32(N2) / dist))
    if r0 < 0 or q0 < 0 or r1 > N1 - 1 or q1 > N2 - 1:
        raise ValueError("the low-pass box leaves the image")
    lpf = np.zeros((N1, N2), dtype=F32)
    lpf[r0:r1 + 1, q0:q1 + 1] = 1
    psf = fftc2((P2 * ea).astype(C64), inverse=True).astype(C64)
    psf = _rmul(psf, lpf)
    P3 = (fftc2(psf).astype(C64) * ea).astype(C64)
    # pattern and corrected fields (:343-351)
    pattern = _rmul((P3 * np.exp(-1j * np.angle(P3[c1, c2]).astype(F32))).astype(C64), NA)
    filt = np.exp(-1j * np.angle(pattern).astype(F32)).astype(C64)

    def apply(f):
        g = fftc2((fftc2(f).astype(C64) * filt[:, :, None]).astype(C64), inverse=True).astype(C64)
        return g.reshape(np.shape(input_field), order="F")

    return apply(fin), apply(fout), {"pattern": pattern, "distance": float(dl[cmax]), "utility": u}


def correct_aberration(u, input_field, field_trans, aberration_params):
    """:354-390 (correct_aberration): the pattern brought to the fields'
    Fourier resolution and field of view (the reference's steps, including
    the inverse transform after the field-of-view crop), masked by the NA
    circle of the pattern's coordinates, then
    ifft2c(fft2c(field) .* exp(-1i angle(pattern))) for both stacks."""
    pattern = np.asarray(aberration_params["pattern"], dtype=C64)
    ua = aberration_params["utility"]
    N = np.shape(input_field)[0]
    target = int(mround(N * ua["fourier_res"][0] / u["fourier_res"][0] / 2) * 2)

    def half(a, b):
        d = float(np.floor(a - b)) / 2
        if d != int(d):
            raise ValueError("odd size difference in correct_aberration")
        return int(d)

    if target > N:
        p = fftc2(pattern).astype(C64)
        c = half(target, p.shape[0])
        p0 = np.zeros((target, target), dtype=C64)
        p0[c:target - c, c:target - c] = p
        pattern = fftc2(p0, inverse=True).astype(C64)
    elif target < N:
        p = fftc2(pattern).astype(C64)
        c = half(p.shape[0], target)
        pattern = fftc2(p[c:p.shape[0] - c, c:p.shape[1] - c], inverse=True).astype(C64)
    if pattern.shape[0] > N:
        c = half(pattern.shape[0], N)
        pattern = fftc2(pattern[c:pattern.shape[0] - c, c:pattern.shape[1] - c], inverse=True).astype(C64)
    elif pattern.shape[0] < N:
        c = half(target, pattern.shape[0])
        p0 = np.zeros((target, target), dtype=C64)
        p0[c:target - c, c:target - c] = pattern
        pattern = p0
    f1 = (np.asarray(ua["fourier_coor"][0], dtype=F32) * F32(pattern.shape[0])) / F32(target)
    f2 = (np.asarray(ua["fourier_coor"][1], dtype=F32) * F32(pattern.shape[1])) / F32(target)
    na = np.sqrt(f1[:, None] ** 2 + f2[None, :] ** 2) < u["kmax"]
    if na.shape != pattern.shape:
        raise ValueError("aberration pattern and optical grid sizes differ")
    pattern = _rmul(pattern, na.astype(F32))
    filt = np.exp(-1j * np.angle(pattern).astype(F32)).astype(C64)

    def apply(f):
        s = _stack(f)
        g = fftc2((fftc2(s).astype(C64) * filt[:, :, None]).astype(C64), inverse=True).astype(C64)
        return g.reshape(np.shape(f), order="F")

    return apply(input_field), apply(field_trans)


ISOUTLIER_SCALE = 1.4826022185056018   # -1 / (sqrt(2) erfcinv(3/2)): MAD -> standard deviation


def isoutlier(x):
    """MATLAB isoutlier(x) (default 'median' method): more than three scaled
    median absolute deviations from the median."""
    x = np.asarray(x, dtype=np.float64)
    med = np.median(x)
    mad = ISOUTLIER_SCALE * np.median(np.abs(x - med))
    return (x < med - 3 * mad) | (x > med + 3 * mad)


def remove_dirty_fields(input_field, output_field, prctile=95, unwrap=None):
    """:399-452 (remove_dirty_fields) for scalar fields without the manual
    review: per image the standard deviation of the gradient energy of
    |sp/bg|_k - |sp/bg|_1 and the fraction of unwrapped phase outside
    1.5 x [min, max] of the first image's; keeps the first field and those
    that are neither isoutlier nor above the fraction prctile / 100.
    Returns (input_field_f, output_field_f, gradient_std, outside_count)."""
    bg, sp = _stack(input_field), _stack(output_field)
    q = (sp / bg).astype(C64)
    amp = np.abs(q).astype(F32)
    ph = np.angle(q).astype(F32)
    ph = np.asarray(unwrap(ph) if unwrap is not None else ph, dtype=F32).reshape(amp.shape, order="F")
    p0 = ph[:, :, 0]
    hi, lo = F32(p0.max() * F32(1.5)), F32(p0.min() * F32(1.5))
    n = amp.shape[2]
    sd = np.zeros(n, dtype=F32)
    cnt = np.zeros(n, dtype=np.int64)
    for k in range(n):
        f1 = (amp[:, :, k] - amp[:, :, 0]).astype(F32)
        gy, gx = np.gradient(f1)
        g = (gx * gx + gy * gy).astype(F32)
        sd[k] = F32(np.std(g.astype(np.float64), ddof=1))
        cnt[k] = np.count_nonzero(ph[:, :, k] > hi) + np.count_nonzero(ph[:, :, k] < lo)
    bad2 = cnt / float(p0.size) > prctile / 100
    keep = np.flatnonzero(~isoutlier(sd.astype(np.float64)) & ~bad2)
    F = np.unique(np.concatenate([[0], keep])).astype(int)
    N1, N2 = bg.shape[:2]
    return (bg[:, :, F].reshape(N1, N2, 1, len(F), order="F"), sp[:, :, F].reshape(N1, N2, 1, len(F), order="F"),
            sd, cnt)
