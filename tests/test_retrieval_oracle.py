"""The field-retrieval oracle (oracle/retrieval.py,
FIELD_EXPERIMENTAL_RETRIEVAL.m) and the library's host helpers on CPU:
  * PhiShiftMS removes a pure first-order ramp (known answer) and the
    library's phi_shift_ms equals the oracle's;
  * the sub-pixel peak refinement of the library (from the peak data the GPU
    returns) equals peak_subpixel_positioner on the same image;
  * get_fields on synthetic off-axis holograms recovers the sample's phase
    bump (up to the sign convention of the sideband) and a flat border."""
import numpy as np

import cases
from oracle import goldstein, retrieval


def _unwrap(ph):
    out = goldstein.unwrapp2(ph)
    return np.asarray(out[0] if isinstance(out, tuple) else out, dtype=np.float32)


def test_ramp_is_removed_and_library_helper_matches():
    from inverse_solver_b200.retrieval import phi_shift_ms

    y, x = np.meshgrid(np.arange(1, 65, dtype=np.float64), np.arange(1, 61, dtype=np.float64), indexing="ij")
    ramp = (0.3 + 0.02 * x - 0.015 * y).astype(np.float32)
    assert np.abs(retrieval.phi_shift_ms(ramp)).max() < 1e-4
    rng = np.random.default_rng(1)
    p = (ramp + 0.1 * rng.standard_normal(ramp.shape)).astype(np.float32)
    assert np.array_equal(phi_shift_ms(p), retrieval.phi_shift_ms(p))


def test_subpixel_from_peak_data_matches_positioner():
    from inverse_solver_b200.retrieval import _subpixel

    rng = np.random.default_rng(2)
    for M in (40, 41):
        img = rng.random((M, M)).astype(np.float32)
        i1, i2 = 11, 27
        img[i1, i2] = 5.0
        img[i1 + 1, i2] = 3.0
        img[i1, i2 - 1] = 2.5
        p1, p2, _, _ = retrieval.placement_finder_prepare(M, M, 1, 1)
        ref = retrieval.peak_subpixel_positioner(img, p1[:, :, 0], p2[:, :, 0])
        pk = [i1 + 1, i2 + 1, img[i1, i2], img[i1 - 1, i2], img[i1 + 1, i2], img[i1, i2 - 1], img[i1, i2 + 1]]
        assert _subpixel(np.asarray(pk, np.float32), M) == ref


def test_get_fields_recovers_the_phase_object():
    bg, sp, phi = cases.off_axis_holograms(128, 3)
    p = retrieval.retrieval_default_parameters(dict(size=[128, 128, 64], resolution=[0.1, 0.1, 0.1],
                                                    resolution_image=[0.08, 0.08], NA=1.2, wavelength=0.532,
                                                    RI_bg=1.3355))
    bgf, spf, upd, k0s, over = retrieval.get_fields(p, bg, sp, unwrap=_unwrap)
    assert bgf.shape == (98, 98, 1, 3) and upd["size"][:2] == [98, 98]
    assert not over.any() and np.isfinite(k0s).all()
    ph = np.angle(spf[:, :, 0, :] / bgf[:, :, 0, :])
    assert np.abs(ph[:8]).max() < 0.1                 # flat border after the ramp fit
    assert 2.0 < np.abs(ph).max() < 3.0              # the 2.5 rad bump
