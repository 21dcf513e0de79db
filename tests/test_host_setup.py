"""The package's host-side setup must equal the oracle's single-precision
setup bit for bit (same operations in the same order)."""
import numpy as np

import cases
from inverse_solver_b200.forward import CBSHostSetup
from oracle import cbs


def _compare(p, RI):
    h = CBSHostSetup(p)
    o = cbs.ForwardSolverCBS(p, single=True)
    h.prepare_potential(RI)
    o.set_RI(RI)
    for name in ("refocusing_util", "kernel_trans", "kernel_ref"):
        assert np.array_equal(getattr(h, name), getattr(o, name)), name
    assert np.array_equal(h.V, o.V)
    assert float(h.eps_imag) == float(o.eps_imag)
    assert h.Bornmax == o.Bornmax
    assert [int(v) for v in h.ROI] == [int(v) for v in o.ROI]
    m3 = (h.attenuation_mask1d[0][:, None, None] * h.attenuation_mask1d[1][None, :, None]) * \
        h.attenuation_mask1d[2][None, None, :]
    assert np.array_equal(m3, o.attenuation_mask)
    r3 = (h.ramp1d[0][:, None, None] * h.ramp1d[1][None, :, None]) * h.ramp1d[2][None, None, :]
    assert np.array_equal(r3, np.broadcast_to(o.phase_ramp, r3.shape))
    k0nm = h.utility_border.k0_nm
    A = (h.kq2[0][:, None, None] + h.kq2[1][None, :, None]) + h.kq2[2][None, None, :]
    G = 1 / (4 * np.pi ** 2 * np.abs(A) - (2 * np.pi * k0nm) ** 2 - 1j * h.eps_imag)
    assert np.array_equal(G.astype(np.complex64), o.Greenp)
    return h


def test_small_case_setup_matches_oracle():
    _compare(cases.small_params(), cases.small_RI())


def test_cyclic_xy_setup_matches_oracle():
    p = cases.params([24, 20, 18], [0, 0, 2])
    h = _compare(p, cases.small_RI()[:24, :20, :18])
    assert h.cyclic_boundary_xy and h.conv_size == h.field_size
