"""GPU parity of the Rytov reconstruction (BACKWARD_SOLVER_RYTOV.m) and of the
overlap counts (BACKWARD_SOLVER_RYTOV_precompute.m / OVERLAP_COUNTER.m)
against the oracle.  Count and overlap_field are integers computed with the
reference's single-precision index arithmetic: bit-exact.  ORytov and the RI
map: relative L2 <= 1e-5 (RI measured as RI - RI_bg)."""
import numpy as np
import pytest

import cases
from oracle import cbs, rytov

pytestmark = pytest.mark.gpu

SIZE = [32, 32, 21]


def _params():
    from inverse_solver_b200.rytov import BACKWARD_SOLVER_RYTOV

    return BACKWARD_SOLVER_RYTOV.get_default_parameters(dict(
        size=SIZE, wavelength=cases.LAM, NA=1.2, RI_bg=cases.NM, resolution=[0.1] * 3,
        vector_simulation=False))


def _fields(p):
    from inverse_solver_b200.inputs import ring_illumination

    return ring_illumination(p, rings=((0.3, 8), (0.6, 8), (0.9, 12)))


def test_overlap_counts_bit_exact():
    from inverse_solver_b200.rytov import OVERLAP_COUNTER

    p = _params()
    f = _fields(p)
    cnt, ov = OVERLAP_COUNTER(p).get_overlap(f)
    ocnt, oov = rytov.overlap_counts(p, f)
    assert cnt.max() >= 3
    assert np.array_equal(cnt, ocnt)
    assert np.array_equal(ov, oov)


@pytest.mark.parametrize("nn", [0, 5])
def test_rytov_matches_oracle(nn):
    from inverse_solver_b200.rytov import BACKWARD_SOLVER_RYTOV

    p = _params()
    p["use_non_negativity"] = nn > 0
    p["non_negativity_iteration"] = nn
    fin = _fields(p)
    fp = cases.params(SIZE, [2, 2, 2], NA=1.2)
    RI = cases.sphere_phantom(SIZE, [0.1] * 3, cases.NM, seed=11, n_spheres=2, radius_um=(0.4, 0.8))
    o = cbs.ForwardSolverCBS(fp, single=True)
    o.set_RI(RI)
    fout, _, _ = o.solve(fin)
    phase = np.angle(fout[:, :, 0, :] / fin[:, :, 0, :]).astype(np.float32)
    s = BACKWARD_SOLVER_RYTOV(p)
    got = s.solve(fin, fout, unwrapped_phase=phase)
    ref, O, C = rytov.rytov_solve(p, fin, fout, phase, non_negativity_iteration=nn)
    assert np.array_equal(s.count, C)
    assert cbs.rel_l2(s.ORytov, O) < 1e-5
    assert cbs.rel_l2(got - cases.NM, ref - cases.NM) < 1e-5
