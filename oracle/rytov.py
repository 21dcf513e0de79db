"""Oracle: CPU restatement of BACKWARD_SOLVER_RYTOV and the overlap counting
of BACKWARD_SOLVER_RYTOV_precompute / OVERLAP_COUNTER.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py); parity unpinned.

Index arithmetic follows MATLAB single semantics exactly (it decides the
integer Ewald-sphere voxel of every pixel, so the counts are bit-exact
targets): a double scalar meeting a single array is rounded to single and
the operation is done in single; comparisons between single arrays and
double scalars are exact (done in double).  ``x`` is MATLAB's dimension 2
and ``y`` dimension 1 in this code, as in the reference.
"""
from __future__ import annotations

import math

import numpy as np

from . import cbs

F32 = np.float32


def mround32(x):
    """MATLAB round on a single array (half away from zero)."""
    return (np.sign(x) * np.floor(np.abs(x) + F32(0.5))).astype(F32)


def vector2scalarfield(input_field, output_field):
    """sub_code/vector2scalarfield.m:1-13 for one polarisation (pass-through)."""
    if input_field.shape[2] != 1:
        raise NotImplementedError("two-polarisation fields are not restated")
    return input_field[:, :, 0, :], output_field[:, :, 0, :]


def find_peak(F):
    """[mj, mi] = find(F == max(F(:))) (BACKWARD_SOLVER_RYTOV.m:63): MATLAB's
    max of a complex array compares abs, then angle; the first match in
    column-major order is returned (0-based row, col)."""
    a = np.abs(F.astype(np.complex64)).astype(F32)
    m = a.max()
    cand = np.argwhere(a.T == m)  # column-major order: iterate columns first
    cand = [(int(c[1]), int(c[0])) for c in cand]  # (row, col)
    if len(cand) > 1:
        ang = [np.angle(F[r, c]) for r, c in cand]
        best = max(ang)
        cand = [rc for rc, g in zip(cand, ang) if g == best]
    return cand[0]


def _geometry(params):
    u = cbs.derive_optical_tool(params, cbs.Prec(True))
    return u


def illumination_shifts(params, bg):
    """f_dx, f_dy, k0_x, k0_y, k0_z (BACKWARD_SOLVER_RYTOV.m:55-74), double."""
    u = _geometry(params)
    n = bg.shape[2]
    f_dx = np.zeros(n)
    f_dy = np.zeros(n)
    mj0 = mi0 = 0
    for ii in range(n):
        Fbg = cbs.fftc2(bg[:, :, ii].astype(np.complex64))
        mj, mi = find_peak(Fbg)
        if ii == 0:
            mj0, mi0 = mj, mi
        f_dy[ii] = mj - mj0
        f_dx[ii] = mi - mi0
    k0_x = u["fourier_res"][1] * f_dx
    k0_y = u["fourier_res"][0] * f_dy
    k0_z = np.real(np.sqrt((u["k0_nm"] ** 2 - k0_x ** 2 - k0_y ** 2).astype(np.complex128)))
    return f_dx, f_dy, k0_x, k0_y, k0_z


def ewald_indices(params, u, k0x, k0y, k0z):
    """Per-pixel Ewald-sphere voxel of one illumination
    (BACKWARD_SOLVER_RYTOV.m:84-101): (mask, Ky, Kx, Kz) with 1-based
    integer-valued single indices; rows = dim 1 (y), columns = dim 2 (x)."""
    N = params["size"]
    res = u["fourier_res"]
    kz = u["k3"]                                       # single [N1, N2]
    kx = u["fourier_coor"][1][None, :] + np.zeros((N[0], N[1]), F32)
    ky = u["fourier_coor"][0][:, None] + np.zeros((N[0], N[1]), F32)
    Kx = kx - F32(k0x)
    Ky = ky - F32(k0y)
    Kz = kz - F32(k0z)
    d = np.float64
    mask = ((kz > 0) & u["NA_circle"]
            & (Kx.astype(d) > res[1] * (-math.floor(N[1] / 2)))
            & (Ky.astype(d) > res[0] * (-math.floor(N[0] / 2)))
            & (Kz.astype(d) > res[2] * (-math.floor(N[2] / 2)))
            & (Kx.astype(d) < res[1] * (math.floor(N[1] / 2) - 1))
            & (Ky.astype(d) < res[0] * (math.floor(N[0] / 2) - 1))
            & (Kz.astype(d) < res[2] * (math.floor(N[2] / 2) - 1)))
    iKx = mround32((Kx / F32(res[1]) + F32(math.floor(N[1] / 2))) + F32(1))
    iKy = mround32((Ky / F32(res[0]) + F32(math.floor(N[0] / 2))) + F32(1))
    iKz = mround32((Kz / F32(res[2]) + F32(math.floor(N[2] / 2))) + F32(1))
    return mask, iKy, iKx, iKz


def rytov_scatter(params, bg, sp, ret_phase, count_one=False):
    """The Ewald scatter loop and normalisation of BACKWARD_SOLVER_RYTOV.solve
    (:55-107); ``count_one`` selects the _precompute counting (Count += 1,
    BACKWARD_SOLVER_RYTOV_precompute.m:126) instead of Count += (Uprime ~= 0).
    Returns ORytov (normalised), Count, overlap_field, shifts."""
    u = _geometry(params)
    N = params["size"]
    res = params["resolution"]
    f_dx, f_dy, k0_x, k0_y, k0_z = illumination_shifts(params, bg)
    amp = np.abs((sp / bg).astype(np.complex64)).astype(F32)
    O = np.zeros(N, dtype=np.complex64)
    C = np.zeros(N, dtype=F32)
    kz_map = []
    for kk in range(bg.shape[2]):
        FR = (np.log(amp[:, :, kk]) + 1j * ret_phase[:, :, kk]).astype(np.complex64)
        Us = cbs.fftc2(FR) * (res[0] * res[1])
        Us = np.roll(Us, (int(round(k0_y[kk] / u["fourier_res"][0])), int(round(k0_x[kk] / u["fourier_res"][1]))), axis=(0, 1))
        Us = Us * u["NA_circle"]
        kz = u["k3"]
        Up = (kz / 1j) * Us
        mask, iKy, iKx, iKz = ewald_indices(params, u, k0_x[kk], k0_y[kk], k0_z[kk])
        sel = np.nonzero(mask.T.ravel())[0]          # find(): column-major order
        rows, cols = sel % N[0], sel // N[0]
        ky, kx, kzz = (iKy[rows, cols].astype(np.int64) - 1, iKx[rows, cols].astype(np.int64) - 1,
                       iKz[rows, cols].astype(np.int64) - 1)
        up = Up[rows, cols].astype(np.complex64)
        O[ky, kx, kzz] = O[ky, kx, kzz] + up
        C[ky, kx, kzz] = C[ky, kx, kzz] + (F32(1) if count_one else (up != 0).astype(F32))
        m = np.full((N[0], N[1]), -1, dtype=np.int64)
        m[ky, kx] = kzz * N[0] * N[1] + kx * N[0] + ky
        kz_map.append(m)
    pos = C > 0
    O[pos] = (O[pos] / C[pos]) / F32(np.prod(np.asarray(res, dtype=np.float64)))
    ov = np.zeros((N[0], N[1], bg.shape[2]), dtype=F32)
    Cf = C.ravel(order="F")
    for kk, m in enumerate(kz_map):
        sl = np.zeros((N[0], N[1]), dtype=F32)
        hit = m >= 0
        sl[hit] = Cf[m[hit]]
        ov[:, :, kk] = np.roll(sl, (int(round(k0_y[kk] / u["fourier_res"][0])), int(round(k0_x[kk] / u["fourier_res"][1]))), axis=(0, 1))
    return O, C, ov, (f_dx, f_dy)


def rytov_solve(params, input_field, output_field, ret_phase, non_negativity_iteration=0):
    """BACKWARD_SOLVER_RYTOV.solve (:22-127) with the unwrapped phase given
    (the reference unwraps angle(sp./bg) with unwrapp2_gpu at :49).  Returns
    RI (complex single), ORytov, Count."""
    bg, sp = vector2scalarfield(input_field, output_field)
    bg = bg.astype(np.complex64)
    sp = sp.astype(np.complex64)
    O, C, _, _ = rytov_scatter(params, bg, sp, ret_phase)
    P = cbs.Prec(True)
    rec = cbs.fftcn(O, inverse=True).astype(np.complex64)
    RI = cbs.potential2ri(rec * F32(4 * math.pi), params["wavelength"], params["RI_bg"], P)
    if non_negativity_iteration:
        u = _geometry(params)
        Emask = u["coorxy"] < (2 * params["NA"] / params["wavelength"])
        rec = cbs.fftcn(O, inverse=True).astype(np.complex64)
        zero_O = np.abs(O) == 0
        for _ in range(non_negativity_iteration):
            neg = rec.real < 0
            rec[neg] = 0 + 1j * rec.imag[neg]
            On = cbs.fftcn(rec).astype(np.complex64)
            On = (Emask[:, :, None] * On * zero_O + O).astype(np.complex64)
            rec = cbs.fftcn(On, inverse=True).astype(np.complex64)
        neg = rec.real < 0
        rec[neg] = 0 + 1j * rec.imag[neg]
        RI = cbs.potential2ri(rec * F32(4 * math.pi), params["wavelength"], params["RI_bg"], P)
    return RI.astype(np.complex64), O, C


def overlap_counts(params, input_field):
    """OVERLAP_COUNTER.get_overlap (OVERLAP_COUNTER.m:19-23) with the working
    count logic of BACKWARD_SOLVER_RYTOV_precompute.m:87-137: Count += 1 per
    illumination whose Ewald cap hits a voxel; overlap_field(:,:,kk) is that
    count read back at each pixel of illumination kk and shifted back."""
    bg, _ = vector2scalarfield(input_field, input_field)
    bg = bg.astype(np.complex64)
    phase = np.zeros(bg.shape, dtype=F32)
    _, C, ov, _ = rytov_scatter(params, bg, bg, phase, count_one=True)
    return C, ov
