"""GPU field retrieval (odt_hologram_fields + the host mirror of
FIELD_EXPERIMENTAL_RETRIEVAL.get_fields, GPU phase unwrapping) against the
oracle on synthetic off-axis holograms: background and sample fields within
rel-L2 1e-5, sub-pixel peak positions within 1e-3 pixel, the same updated
parameters and exposure flags; resolution matching by cropping and by
padding, a numeric ROI, the other-corner sideband; refocus within 1e-5."""
import numpy as np
import pytest

import cases
from oracle import cbs, goldstein, retrieval

pytestmark = pytest.mark.gpu


def _unwrap(ph):
    out = goldstein.unwrapp2(ph)
    return np.asarray(out[0] if isinstance(out, tuple) else out, dtype=np.float32)


def _params(**kw):
    base = dict(size=[128, 128, 64], resolution=[0.1, 0.1, 0.1], resolution_image=[0.08, 0.08], NA=1.2,
                wavelength=0.532, RI_bg=1.3355)
    base.update(kw)
    return retrieval.retrieval_default_parameters(base)


@pytest.mark.parametrize("case", ["crop", "pad", "roi", "other_corner"])
def test_get_fields_matches_oracle(case):
    from inverse_solver_b200.retrieval import FIELD_EXPERIMENTAL_RETRIEVAL

    kw, roi, carrier = {}, None, (-0.23, -0.27)
    if case == "pad":
        kw = dict(resolution=[0.06, 0.06, 0.1])
    elif case == "roi":
        roi = [5, 124, 5, 124]
    elif case == "other_corner":
        kw = dict(other_corner=True)
        carrier = (-0.23, 0.27)
    bg, sp, _ = cases.off_axis_holograms(128, 3, seed=4, carrier=carrier)
    p = _params(**kw)
    ob, os_, oupd, ok0, oover = retrieval.get_fields(p, bg, sp, roi=roi, unwrap=_unwrap)
    r = FIELD_EXPERIMENTAL_RETRIEVAL(p)
    gb, gs, gupd, gk0, gover, _ = r.get_fields(bg, sp, roi)
    assert gb.shape == ob.shape and gs.shape == os_.shape
    assert cbs.rel_l2(gb, ob) < 1e-5 and cbs.rel_l2(gs, os_) < 1e-5
    assert np.abs(gk0 - ok0).max() < 1e-3
    assert np.array_equal(gover, oover)
    assert gupd["size"] == oupd["size"] and np.allclose(gupd["resolution"], oupd["resolution"])
    if case == "crop":
        rp = dict(p, size=list(gupd["size"]), resolution=list(gupd["resolution"]))
        assert cbs.rel_l2(r.refocus(gs, 0.7), retrieval.refocus(rp, os_, 0.7)) < 1e-5
