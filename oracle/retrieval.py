"""CPU restatement of the field retrieval front-end
(Codes/FIELD_EXPERIMENTAL_RETRIEVAL.m) -- test infrastructure (the oracle):
only the tests and the benchmark's CPU baseline import it.

Covers the non-interactive path of get_fields (:27-229; the "rectangle" ROI
picker and the GUI branches of PhiShiftMS are interactive and out of scope)
with its helpers sub_code/CPU_placement_finder_prepare.m:1-19,
sub_code/peak_subpixel_positioner.m:1-67 and sub_code/PhiShiftMS.m (mask
style 1, D2_LSAms with n = 1, omit_outliers: :1-44, :103-166), and refocus
(:392-394).  MATLAB single semantics: single(x) * double(y) is single,
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
