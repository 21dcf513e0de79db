"""GPU parity of the Goldstein unwrapper (odt_unwrap_goldstein through the
C ABI) against the oracle and the reference's own linker results
(tests/golden/goldstein_small.npz).  Residues, step maps, residue table,
nearest lists and branches are integers: bit-exact.  The unwrapped phase is
the same sequence of single-precision operations as the oracle: bit-exact."""
import numpy as np
import pytest

import cases
from oracle import goldstein as g

pytestmark = pytest.mark.gpu

GOLD = "tests/golden/goldstein_small.npz"


@pytest.fixture(scope="module")
def gold():
    import os

    return np.load(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), GOLD))


def test_chain_matches_reference_golden(gold):
    from inverse_solver_b200.unwrap import unwrap_goldstein

    for k in range(int(gold["n_cases"])):
        ph = gold[f"c{k}_phase"]
        out, it = unwrap_goldstein(ph, intermediates=True)
        assert np.array_equal(it["residue"], gold[f"c{k}_residue"]), k
        assert np.array_equal(it["table"], gold[f"c{k}_table"]), k
        assert np.array_equal(it["nearest"], gold[f"c{k}_ref_nearest"]), k
        assert np.array_equal(it["branches"], gold[f"c{k}_ref_branches"]), k
        assert np.array_equal(it["step1"], gold[f"c{k}_step1"]), k
        assert np.array_equal(it["step2"], np.asarray(_oracle_step2(ph))), k
        assert np.array_equal(out, gold[f"c{k}_unwrapped"]), k


def _oracle_step2(ph):
    _, it = g.unwrapp2(ph, return_intermediates=True)
    return it["step2"]


@pytest.mark.parametrize("shape,seed,noise", [((128, 128, 4), 31, 1.0), ((96, 72, 3), 32, 2.5),
                                              ((64, 64, 1), 33, 0.3)])
def test_larger_stacks_match_oracle(shape, seed, noise):
    from inverse_solver_b200.unwrap import unwrap_goldstein

    ph = cases.wrapped_phase(shape, seed, noise)
    ref, oit = g.unwrapp2(ph, return_intermediates=True)
    out, it = unwrap_goldstein(ph, intermediates=True)
    assert np.array_equal(it["residue"], oit["residue"])
    assert np.array_equal(it["step1"], oit["step1"])
    assert np.array_equal(it["step2"], oit["step2"])
    if "table" in oit:
        assert np.array_equal(it["nearest"], oit["shortest"])
        assert np.array_equal(it["branches"], oit["branches"])
    assert np.array_equal(out, ref)


def test_two_dimensional_input_and_thread_counts():
    from inverse_solver_b200.unwrap import unwrap_goldstein, unwrapp2_gpu

    ph = cases.wrapped_phase((50, 44, 1), 40, 1.5)
    ref = g.unwrapp2(ph)
    a = unwrapp2_gpu(ph[:, :, 0])
    assert a.shape == (50, 44)
    assert np.array_equal(a, ref[:, :, 0])
    for t in (1, 2, 7):
        assert np.array_equal(unwrap_goldstein(ph, link_threads=t), ref)


def test_device_memory_path_matches_host():
    import torch

    from inverse_solver_b200.unwrap import unwrapp2_gpu

    ph = cases.wrapped_phase((64, 48, 5), 41, 1.2)
    host = unwrapp2_gpu(ph)
    dev = unwrapp2_gpu(torch.from_numpy(ph).cuda())
    torch.cuda.synchronize()
    assert np.array_equal(dev.cpu().numpy(), host)


def test_residue_free_and_tiny_maps():
    from inverse_solver_b200.unwrap import unwrap_goldstein

    y, x = np.meshgrid(np.linspace(-1, 1, 40), np.linspace(-1, 1, 36), indexing="ij")
    true = (14.0 * np.exp(-(x ** 2 + y ** 2) / 0.3)).astype(np.float32)
    w = np.angle(np.exp(1j * true.astype(np.float64))).astype(np.float32)[:, :, None]
    out, it = unwrap_goldstein(w, intermediates=True)
    assert it["branches"].shape[1] == 0 and not np.any(it["step1"])
    assert np.array_equal(out, g.unwrapp2(w))
    tiny = cases.wrapped_phase((2, 2, 3), 42, 3.0)
    assert np.array_equal(unwrap_goldstein(tiny), g.unwrapp2(tiny))


def test_bad_sizes_rejected():
    from inverse_solver_b200 import _lib
    from inverse_solver_b200.unwrap import unwrap_goldstein

    with pytest.raises(_lib.OdtError) as e:
        unwrap_goldstein(np.zeros((1, 5, 2), np.float32))
    assert e.value.status == 1


def test_rytov_default_unwrap_matches_oracle():
    """BACKWARD_SOLVER_RYTOV.solve with its default unwrapping (unwrapp2_gpu
    of angle(sp./bg), BACKWARD_SOLVER_RYTOV.m:49) against the oracle fed with
    the oracle's unwrapped phase."""
    from inverse_solver_b200.inputs import ring_illumination
    from inverse_solver_b200.rytov import BACKWARD_SOLVER_RYTOV
    from oracle import rytov

    p = BACKWARD_SOLVER_RYTOV.get_default_parameters(dict(
        size=[32, 32, 21], wavelength=cases.LAM, NA=1.2, RI_bg=cases.NM, resolution=[0.1] * 3,
        vector_simulation=False))
    bg = ring_illumination(p, rings=((0.3, 4), (0.6, 6)))
    rng = np.random.default_rng(7)
    ph = cases.wrapped_phase((32, 32, bg.shape[3]), 43, 0.8, amp=6.0)
    amp = (1 + 0.05 * rng.standard_normal(ph.shape)).astype(np.float32)
    sp = (bg[:, :, 0, :] * amp * np.exp(1j * ph)).astype(np.complex64)[:, :, None, :]
    RI = BACKWARD_SOLVER_RYTOV(p).solve(bg, sp)
    wrapped = np.angle(sp[:, :, 0, :] / bg[:, :, 0, :]).astype(np.float32)
    uw = g.unwrapp2(wrapped)
    oRI, _, _ = rytov.rytov_solve(p, bg, sp, uw)
    num = np.linalg.norm((RI - oRI).ravel())
    den = np.linalg.norm((oRI - cases.NM).ravel())
    assert num / den < 1e-5
