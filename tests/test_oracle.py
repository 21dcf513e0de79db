"""CPU checks of the oracle: known-answer pins and regression fixtures."""
import math

import numpy as np
import scipy.special as ssp

import cases
from oracle import cbs


def test_hankel_disk_known_answer():
    """hankel_transform/test_hankel.m: the transform of the disk r<1 is
    2*pi*J1(k)/k.  The cropped discrete transform must reproduce it on the
    retained band (Gibbs ripple of the discontinuous disk bounds the error)."""
    P = cbs.Prec(False)
    hk = cbs.DiscreteHankelCroppedFourier(10, 4000, 0, 0.2, P)
    f = (hk.r < 1).astype(np.float64)
    H = hk.forward(f[:, None])[:, 0]
    ref = 2 * math.pi * ssp.j1(hk.k) / hk.k
    err = np.abs(H - ref).max() / (2 * math.pi * 0.5)
    assert err < 0.02, err
    # round trip forward -> backward on a smooth band-limited profile
    g = np.exp(-hk.r ** 2)
    back = hk.backward(hk.forward(g[:, None]))[:, 0]
    assert np.abs(back - g).max() < 1e-3


def test_bessel_roots():
    r = cbs.jn_roots(0, 200)
    assert np.abs(ssp.j0(r)).max() < 1e-12
    assert np.all(np.diff(r) > 3.0)


def test_cfg1_scalars():
    """The survey's computed table: cfg1 -> bt_px 16, padded 96^3, eps 49.32, 28 iterations."""
    s = cbs.ForwardSolverCBS.__new__(cbs.ForwardSolverCBS)
    p = cases.cfg1_params()
    btp = cbs.mround((np.asarray(p["boundary_thickness"]) * p["wavelength"] / p["RI_bg"]) /
                     (np.asarray(p["resolution"]) * 2))
    assert list(btp) == [16, 16, 16]
    RI = cases.cfg1_RI()
    pot = cbs.ri2potential(RI.ravel(), p["wavelength"], p["RI_bg"], cbs.Prec(True))
    eps = np.float32(np.abs(pot).max() * 1.01)
    assert abs(float(eps) - 49.32) < 0.01
    step = np.float32(abs(2 * (2 * math.pi * p["RI_bg"] / p["wavelength"]) / eps))
    nrm = float(np.linalg.norm(np.array([96.0] * 3) * 0.1))
    assert math.ceil(float(np.float32(np.float32(nrm / step) / 2 + 1))) * 2 == 28
    del s


def test_fft_flip_negates_frequency():
    a = np.arange(7 * 6).reshape(7, 6).astype(float)
    f = cbs.fft_flip(a, [1, 1], False)
    for i in range(7):
        for j in range(6):
            assert f[i, j] == a[(-i) % 7, (-j) % 6]


def test_golden_regression():
    g = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "cbs_small.npz"))
    p = cases.small_params(return_reflection=True, return_3D=True)
    s = cbs.ForwardSolverCBS(p, single=True)
    s.set_RI(g["RI"])
    assert s.Bornmax == int(g["bornmax"])
    t, r, f = s.solve(g["fields"])
    assert cbs.rel_l2(t, g["trans32"]) < 1e-6
    assert cbs.rel_l2(r, g["ref32"]) < 1e-6
    assert cbs.rel_l2(f, g["field3d32"]) < 1e-6
    # single vs double restatement: the reference's own single-precision error
    assert cbs.rel_l2(g["trans32"], g["trans64"]) < 2e-4
    assert cbs.rel_l2(g["ref32"], g["ref64"]) < 2e-4


def test_zero_potential_gives_incident_field():
    """RI == single(RI_bg) everywhere: the potential is only the rounding
    residue of single(RI_bg)^2/RI_bg^2 - 1 (exactly 0 would make eps_imag 0,
    which the reference divides by), so the 3D field is the refocused incident
    field and the transmitted field the pupil-filtered input to ~1e-6."""
    p = cases.small_params(return_reflection=True, return_3D=True)
    s = cbs.ForwardSolverCBS(p, single=False)
    s.set_RI(np.full(cases.SMALL_SIZE, cases.NM, dtype=np.float32))
    fields = cases.circle_fields(p, 2)
    t, r, f = s.solve(fields)
    for k in range(2):
        inc = s.refocus_source(s.transform_field_3D(cbs.fftc2(fields[:, :, :, k].astype(np.complex128)))[:, :, 0])
        assert cbs.rel_l2(f[:, :, :, 0, k], inc) < 1e-5
        filt = s.transform_field_2D(s.transform_field_3D(cbs.fftc2(fields[:, :, 0, k].astype(np.complex128))))
        assert cbs.rel_l2(t[:, :, 0, k], cbs.fftc2(filt, inverse=True)) < 1e-5
    assert np.abs(r).max() < 1e-5 * np.abs(t).max()
