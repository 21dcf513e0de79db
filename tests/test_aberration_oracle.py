"""The oracle's aberration correction and dirty-field rejection
(FIELD_EXPERIMENTAL_RETRIEVAL.m:216-452) on synthetic aberrated fields:
self-consistency (get_aberration_pattern's corrected fields are
correct_aberration's with the same pattern), the reference's error cases,
MATLAB isoutlier on small known cases, and dirty-field rejection of planted
bad fields."""
import numpy as np
import pytest

import cases
from oracle import cbs, goldstein, retrieval


def _unwrap(ph):
    out = goldstein.unwrapp2(ph)
    return np.asarray(out[0] if isinstance(out, tuple) else out, dtype=np.float32)


def _tool(params):
    return cbs.derive_optical_tool(params, cbs.Prec(True))


CP = dict(overlap_factor=0.25, distList=[-2.0, -1.0, 0.0, 1.0, 2.0])


def test_pattern_then_correct_is_consistent():
    inp, out, k0s, params = cases.aberrated_fields(64, 5, seed=1)
    u = _tool(params)
    fi, fo, ab = retrieval.get_aberration_pattern(u, inp, out, dict(CP, k0s=k0s))
    assert fi.shape == inp.shape and ab["pattern"].shape == (64, 64)
    assert ab["distance"] in CP["distList"]
    ci, co = retrieval.correct_aberration(u, inp, out, ab)
    assert cbs.rel_l2(ci, fi) < 1e-6 and cbs.rel_l2(co, fo) < 1e-6
    # the pattern is unit-phased at the centre and zero outside the NA circle
    p = ab["pattern"]
    assert abs(np.angle(p[32, 32])) < 1e-5
    assert np.all(p[~np.asarray(u["NA_circle"])] == 0)


def test_reference_error_cases():
    inp, out, k0s, params = cases.aberrated_fields(64, 5, seed=1)
    u = _tool(params)
    flat = k0s.copy()
    flat[1] = 0.2        # every step of round(k0s(2,:)) is 0: no low-pass box
    with pytest.raises(ValueError):
        retrieval.get_aberration_pattern(u, inp, out, dict(CP, k0s=flat))
    with pytest.raises(ValueError):
        retrieval.get_aberration_pattern(u, inp[..., :1], out[..., :1], dict(CP, k0s=k0s[:, :1]))


def test_isoutlier_known_cases():
    assert retrieval.isoutlier([1, 2, 3, 4, 100]).tolist() == [False, False, False, False, True]
    # median 3, MAD 1 -> bounds 3 -/+ 4.4478
    x = np.array([3.0, 2.0, 4.0, 3.0 + 4.44, 3.0 - 4.46])
    assert retrieval.isoutlier(x).tolist() == [False, False, False, False, True]
    assert not retrieval.isoutlier(np.full(6, 2.5)).any()


def test_remove_dirty_fields_rejects_planted_fields():
    inp, out, k0s, params = cases.aberrated_fields(64, 7, seed=2)
    out = out.copy()
    rng = np.random.default_rng(0)
    out[:, :, 0, 3] *= (1 + 0.5 * rng.standard_normal((64, 64))).astype(np.float32)   # amplitude noise
    x = np.arange(64)[None, :]
    out[:, :, 0, 5] *= np.exp(2j * np.pi * 8 * x / 64).astype(np.complex64)          # phase ramp (8 cycles)
    fi, fo, sd, cnt = retrieval.remove_dirty_fields(inp, out, 80, unwrap=_unwrap)
    kept = [k for k in range(7) if any(np.array_equal(fi[:, :, 0, j], inp[:, :, 0, k]) for j in range(fi.shape[3]))]
    assert 3 not in kept and 5 not in kept and 0 in kept
    assert fi.shape == (64, 64, 1, len(kept)) and fo.shape == fi.shape
