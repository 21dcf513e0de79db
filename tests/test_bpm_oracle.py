"""The BPM oracle (oracle/bpm.py, FORWARD_SOLVER_BPM.m) on CPU:
  * known answer: in a homogeneous medium (RI = RI_bg) the refocusing phases
    before and after the slice loop undo the Nz free-space steps, so the
    transmitted field is the input restricted to the NA circle (a plane wave
    inside the NA comes back unchanged);
  * single against double precision on a phantom: rel-L2 <= 1e-5;
  * the library's host tables (FORWARD_SOLVER_BPM.set_RI) equal the
    oracle's single-precision ones."""
import numpy as np

import cases
from oracle import bpm, cbs


def _params(size=(32, 28, 20), **kw):
    return bpm.bpm_default_parameters(dict(size=list(size), wavelength=cases.LAM, NA=1.2, RI_bg=cases.NM,
                                           resolution=[0.1] * 3, vector_simulation=False, **kw))


def test_homogeneous_medium_returns_the_band_limited_input():
    p = _params(return_3D=True)
    fields = cases.circle_fields(p, 3)
    o = bpm.ForwardSolverBPM(p, single=False)
    o.set_RI(np.full(p["size"], cases.NM))
    t, _, f3 = o.solve(fields)
    na = np.asarray(o.u["NA_circle"])
    want = cbs.fftc2(cbs.fftc2(fields.astype(np.complex128)) * na[:, :, None, None], inverse=True)
    assert cbs.rel_l2(t, want) < 1e-12
    assert cbs.rel_l2(t, fields) < 1e-6      # plane waves inside the NA (single-precision inputs)
    assert f3.shape == (32, 28, 20, 1, 3)


def test_single_matches_double_on_a_phantom():
    p = _params(return_3D=True)
    RI = cases.sphere_phantom(p["size"], [0.1] * 3, cases.NM, seed=5, n_spheres=3, radius_um=(0.3, 0.7))
    fields = cases.circle_fields(p, 3)
    out = []
    for single in (True, False):
        o = bpm.ForwardSolverBPM(p, single=single)
        o.set_RI(RI)
        out.append(o.solve(fields))
    assert cbs.rel_l2(out[0][0], out[1][0]) < 1e-5
    assert cbs.rel_l2(out[0][2], out[1][2]) < 1e-5


def test_host_tables_equal_the_oracle():
    from inverse_solver_b200.bpm import FORWARD_SOLVER_BPM

    p = _params()
    RI = cases.sphere_phantom(p["size"], [0.1] * 3, cases.NM, seed=6, n_spheres=2, radius_um=(0.3, 0.7))
    o = bpm.ForwardSolverBPM(p, single=True)
    o.set_RI(RI)
    s = FORWARD_SOLVER_BPM.__new__(FORWARD_SOLVER_BPM)   # tables only: no library call
    from inverse_solver_b200.optics import OpticalTool
    s.parameters, s.utility = dict(p), OpticalTool(p)
    s.set_RI(RI)
    assert np.array_equal(s.field_multiplier, o.field_multiplier)
    assert np.array_equal(s.refocus_kernel, o.refocus_kernel)
    assert np.array_equal(s.filter_out.astype(bool), o.filter_out)
