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


def test_tensor_potential_matches_oracle():
    """prepare_tensor_potential (set_RI with an RI tensor [x, y, z, 3, 3])
    equals the oracle's tensor condition_RI / create_boundary_RI bit for bit:
    V with -1i eps_imag on the diagonal, eps_imag over all nine components."""
    p = cases.params([24, 24, 18], [1.5, 1.5, 1.5])
    p["vector_simulation"] = True
    RI = cases.small_RI()[:24, :24, :18]
    T = np.empty(RI.shape + (3, 3), np.float32)
    T[...] = np.float32(cases.NM)
    for i in range(3):
        T[:, :, :, i, i] = cases.NM + (RI - cases.NM) * (1 - 0.2 * i)
    T[:, :, :, 0, 1] = T[:, :, :, 1, 0] = cases.NM + (RI - cases.NM) * 0.1
    h = CBSHostSetup(p)
    o = cbs.ForwardSolverCBS(p, single=True)
    pp, keep = h.prepare_tensor_potential(T)
    o.set_RI(T)
    assert h.tensor and o.tensor
    assert h.V.shape == o.V.shape == tuple(h.sim_size) + (3, 3)
    assert np.array_equal(h.V, o.V)
    assert np.array_equal(keep[-1], o.V) and keep[-1].flags.f_contiguous
    assert float(h.eps_imag) == float(o.eps_imag) and h.Bornmax == o.Bornmax


def test_tensor_potential_argument_checks():
    """A tensor RI needs the dyadic Green's function and the [x, y, z, 3, 3]
    shape; the struct form needs a tensor (FORWARD_SOLVER_CONVERGENT_BORN.m
    :181-186)."""
    import pytest

    RI = cases.small_RI()[:24, :24, :18]
    T = np.full(RI.shape + (3, 3), cases.NM, np.float32)
    for i in range(3):
        T[:, :, :, i, i] = RI
    scalar = CBSHostSetup(cases.params([24, 24, 18], [1.5, 1.5, 1.5]))
    with pytest.raises(ValueError):
        scalar.prepare_tensor_potential(T)
    p = cases.params([24, 24, 18], [1.5, 1.5, 1.5])
    p["vector_simulation"] = True
    vec = CBSHostSetup(p)
    with pytest.raises(ValueError):
        vec.prepare_tensor_potential(T[..., :2])
    with pytest.raises(ValueError):
        vec.prepare_tensor_potential(T[:20])
    vec.prepare_tensor_potential(T)
    assert vec.tensor and np.all(vec.V[:, :, :, 0, 1] == 0)
    assert vec.eps_imag > 0 and np.all(vec.V[:, :, :, 0, 0].imag == -vec.eps_imag)
