"""GPU parity of the beam-propagation solver (odt_bpm_solve through
FORWARD_SOLVER_BPM) against the single-precision oracle (oracle/bpm.py):
transmitted and 3D fields within rel-L2 1e-5 per illumination, with and
without the cosine correction; the homogeneous-medium known answer."""
import numpy as np
import pytest

import cases
from oracle import bpm, cbs

pytestmark = pytest.mark.gpu


def _params(size, **kw):
    return bpm.bpm_default_parameters(dict(size=list(size), wavelength=cases.LAM, NA=1.2, RI_bg=cases.NM,
                                           resolution=[0.1] * 3, vector_simulation=False, **kw))


def worst(a, b):
    return max(cbs.rel_l2(a[..., k], b[..., k]) for k in range(a.shape[-1]))


@pytest.mark.parametrize("cos_correction", [True, False])
@pytest.mark.parametrize("size", [[32, 28, 20], [48, 48, 33]])
def test_bpm_matches_oracle(size, cos_correction):
    from inverse_solver_b200 import FORWARD_SOLVER_BPM

    p = _params(size, return_3D=True, return_reflection=True, cos_correction=cos_correction)
    RI = cases.sphere_phantom(size, [0.1] * 3, cases.NM, seed=sum(size), n_spheres=3, radius_um=(0.3, 0.7))
    fields = cases.circle_fields(p, 4)
    s = FORWARD_SOLVER_BPM(p)
    s.set_RI(RI)
    t, r, f3 = s.solve(fields)
    o = bpm.ForwardSolverBPM(p, single=True)
    o.set_RI(RI)
    ot, orr, of3 = o.solve(fields)
    assert t.shape == ot.shape and f3.shape == of3.shape
    assert worst(t, ot) < 1e-5
    assert worst(f3, of3) < 1e-5
    assert np.array_equal(r, orr)


def test_bpm_homogeneous_known_answer():
    from inverse_solver_b200 import FORWARD_SOLVER_BPM

    p = _params([40, 36, 25])
    fields = cases.circle_fields(p, 3)
    s = FORWARD_SOLVER_BPM(p)
    s.set_RI(np.full(p["size"], cases.NM, dtype=np.float32))
    t, _, _ = s.solve(fields)
    assert cbs.rel_l2(t, fields) < 1e-5
