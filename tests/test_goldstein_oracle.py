"""Goldstein branch-cut unwrapping without a GPU:
  * known answers of the oracle's residue and dipole stages (a single
    vortex, a vortex/antivortex pair, a residue-free ramp);
  * the oracle's nearest-residue lists and branch list equal the reference's
    own code (compiled from its sources: tests/golden/goldstein_small.npz,
    and fresh seeds when oracle/_ref is built);
  * the library's host stages (residue table, nearest search, threaded
    linker from inverse_solver_b200/csrc, compiled as plain C++) equal the
    oracle / reference bit for bit;
  * properties of the unwrapped phase (multiples of 2*pi from the input,
    exact recovery of a residue-free phase)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import cases
from oracle import goldstein as g

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "inverse_solver_b200", "csrc")
GOLD = os.path.join(ROOT, "tests", "golden", "goldstein_small.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def _cases(gold):
    return range(int(gold["n_cases"]))


def vortex(N1, N2, c1, c2, sign=1):
    y, x = np.meshgrid(np.arange(N1, dtype=np.float64), np.arange(N2, dtype=np.float64), indexing="ij")
    return np.angle((y - c1) + 1j * sign * (x - c2)).astype(np.float32)


# ---------------------------------------------------------------- known answers
def test_residue_free_ramp():
    y, x = np.meshgrid(np.arange(20.0), np.arange(24.0), indexing="ij")
    true = (0.9 * x + 0.4 * y).astype(np.float32)
    w = np.angle(np.exp(1j * true)).astype(np.float32)[:, :, None]
    assert not np.any(g.get_residue(w))
    out, it = g.unwrapp2(w, return_intermediates=True)
    assert it["branches"].shape[1] == 0
    np.testing.assert_allclose(out[:, :, 0] - out[0, 0, 0], true - true[0, 0], atol=2e-5)


@pytest.mark.parametrize("sign", [1, -1])
def test_single_vortex_residue(sign):
    w = vortex(16, 18, 7.5, 9.5, sign)[:, :, None]
    r = g.get_residue(w)
    nz = np.argwhere(r != 0)
    assert nz.tolist() == [[7, 9, 0]]
    v = r[7, 9, 0]
    assert abs(v) == 1
    # opposite vortex sense flips the charge
    r2 = g.get_residue(vortex(16, 18, 7.5, 9.5, -sign)[:, :, None])
    assert r2[7, 9, 0] == -v


@pytest.mark.parametrize("pos_d2,neg_d2,step", [(8, 9, -1), (9, 8, 1)])
def test_dipole_pair_along_dim2(pos_d2, neg_d2, step):
    """A +1/-1 pair side by side along dimension 2 cancels; the step goes to
    (d1 + 1, min(d2) + 1): +charge when the partner is at d2 - 1 (direction
    1), -charge when it is at d2 + 1 (direction 3)."""
    r = np.zeros((15, 19, 1), np.float32)
    r[7, pos_d2, 0] = 2
    r[7, neg_d2, 0] = -1
    r2, s1, s2 = g.remove_dipoles(r)
    assert r2[7, pos_d2, 0] == 1 and r2[7, neg_d2, 0] == 0 and np.count_nonzero(r2) == 1
    exp = np.zeros_like(s1)
    exp[8, 9, 0] = step
    assert np.array_equal(s1, exp) and not np.any(s2)


def test_dipole_pair_along_dim1_leaves_no_step():
    r = np.zeros((15, 19, 2), np.float32)
    r[6, 9, 1] = 1
    r[7, 9, 1] = -1
    r2, s1, _ = g.remove_dipoles(r)
    assert not np.any(r2) and not np.any(s1)


def test_dipole_direction_order():
    """Directions run d1-1, d2-1, d1+1, d2+1: a +1 with partners on two sides
    pairs with the first one only."""
    r = np.zeros((10, 10, 1), np.float32)
    r[5, 5, 0] = 1
    r[5, 6, 0] = -1       # direction 3
    r[4, 5, 0] = -1       # direction 0, taken first
    r2, s1, _ = g.remove_dipoles(r)
    assert r2[4, 5, 0] == 0 and r2[5, 6, 0] == -1 and r2[5, 5, 0] == 0
    assert not np.any(s1)


# ---------------------------------------------------------------- pinned on the reference
def test_oracle_matches_reference_golden(gold):
    for k in _cases(gold):
        ph = gold[f"c{k}_phase"]
        uw, it = g.unwrapp2(ph, return_intermediates=True)
        assert np.array_equal(it["residue"], gold[f"c{k}_residue"])
        assert np.array_equal(it["table"], gold[f"c{k}_table"])
        assert np.array_equal(it["shortest"], gold[f"c{k}_ref_nearest"]), k
        assert np.array_equal(it["branches"], gold[f"c{k}_ref_branches"]), k
        assert np.array_equal(it["step1"], gold[f"c{k}_step1"])
        assert np.array_equal(uw, gold[f"c{k}_unwrapped"])


@pytest.mark.skipif(g.ref_lib() is None, reason="oracle/_ref not built (needs the reference sources)")
@pytest.mark.parametrize("seed", [11, 12, 13])
def test_oracle_matches_reference_fresh(seed):
    lib = g.ref_lib()
    rng = np.random.default_rng(seed)
    shape = (int(rng.integers(12, 56)), int(rng.integers(12, 56)), int(rng.integers(1, 4)))
    ph = cases.wrapped_phase(shape, seed, noise=float(rng.uniform(0.5, 2.5)))
    _, it = g.unwrapp2(ph, return_intermediates=True)
    if "table" not in it:
        pytest.skip("no residues")
    M = it["residue"].shape
    near = g.ref_nearest(lib, it["table"], it["lookup"], it["lookup_z_start"], it["square_size"], 8, M)
    assert np.array_equal(near, it["shortest"])
    br = g.ref_branches(lib, it["table"], near, it["square_size"], it["lookup"], it["lookup_z_start"], M)
    assert np.array_equal(br, it["branches"])


# ---------------------------------------------------------------- library host stages
@pytest.fixture(scope="module")
def host(tmp_path_factory):
    so = str(tmp_path_factory.mktemp("gs") / "gs_host.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", "-I" + CSRC,
                    os.path.join(ROOT, "tests", "native", "goldstein_host_check.cpp"),
                    os.path.join(CSRC, "goldstein_link.cpp"), "-o", so], check=True)
    lib = C.CDLL(so)
    P = C.POINTER(C.c_int32)
    lib.gs_table.argtypes = [P, P, C.c_longlong, C.c_int, C.c_int, C.c_int, P, P, P]
    lib.gs_table.restype = C.c_int
    lib.gs_lookup.argtypes = [P]
    lib.gs_nearest.argtypes = [P]
    lib.gs_link.argtypes = [P, C.c_int, P, C.c_longlong]
    lib.gs_link.restype = C.c_longlong
    return lib


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def host_chain(lib, residue, threads):
    M1, M2, nz = residue.shape
    flat = residue.reshape(-1, order="F")
    idx = np.nonzero(flat)[0].astype(np.int32)
    val = flat[idx].astype(np.int32)
    R = idx.size
    rows = np.zeros((R, 6), np.int32)
    sq = np.zeros(nz, np.int32)
    zs = np.zeros(nz, np.int32)
    n_look = lib.gs_table(_p(idx), _p(val), R, M1, M2, nz, _p(rows), _p(sq), _p(zs))
    look = np.zeros(n_look, np.int32)
    lib.gs_lookup(_p(look))
    near = np.zeros((R, 8, 2), np.int32)
    lib.gs_nearest(_p(near))
    cap = 4 * R + 16
    br = np.zeros((cap, 6), np.int32)
    nb = lib.gs_link(_p(near), threads, _p(br), cap)
    return (rows.T, sq, zs, look, np.ascontiguousarray(near.transpose(2, 1, 0)), br[:nb].T)


@pytest.mark.parametrize("threads", [1, 3])
def test_host_stages_match_reference(gold, host, threads):
    for k in _cases(gold):
        res = gold[f"c{k}_residue"]
        rows, sq, zs, look, near, br = host_chain(host, res, threads)
        tab, osq, olook, ozs = g.residue_table(res)
        assert np.array_equal(rows, gold[f"c{k}_table"])
        assert np.array_equal(sq, osq) and np.array_equal(zs, ozs) and np.array_equal(look, olook)
        assert np.array_equal(near, gold[f"c{k}_ref_nearest"]), k
        assert np.array_equal(br, gold[f"c{k}_ref_branches"]), k


def test_host_linker_dense_residues(host):
    """Near-random phase: dense residues, many overflow searches beyond the
    8 precomputed neighbours."""
    ph = cases.wrapped_phase((48, 48, 3), 21, noise=3.0)
    _, it = g.unwrapp2(ph, return_intermediates=True)
    rows, _, _, _, near, br = host_chain(host, it["residue"], 4)
    assert np.array_equal(rows, it["table"])
    assert np.array_equal(near, it["shortest"])
    assert np.array_equal(br, it["branches"])


# ---------------------------------------------------------------- properties
def test_unwrapped_differs_by_multiples_of_2pi(gold):
    for k in _cases(gold):
        ph = gold[f"c{k}_phase"]
        uw = gold[f"c{k}_unwrapped"]
        q = (uw.astype(np.float64) - ph) / (2 * np.pi)
        assert np.max(np.abs(q - np.round(q))) < 1e-3


def test_smooth_phase_recovered_exactly():
    y, x = np.meshgrid(np.linspace(-1, 1, 40), np.linspace(-1, 1, 36), indexing="ij")
    true = (14.0 * np.exp(-(x ** 2 + y ** 2) / 0.3)).astype(np.float32)
    w = np.angle(np.exp(1j * true.astype(np.float64))).astype(np.float32)[:, :, None]
    assert not np.any(g.get_residue(w))
    out = g.unwrapp2(w)[:, :, 0]
    np.testing.assert_allclose(out - out[0, 0], true - true[0, 0], atol=5e-5)


def _wrapping(u):
    """The wrap count of show_unwrapping_performance.m:10-17: pixels whose
    differences exceed pi along both axes."""
    dx = u[:-1, 1:] - u[1:, 1:]
    dy = u[1:, :-1] - u[1:, 1:]
    f = 0.9999
    return int((((np.abs(dx) >= f * np.pi).astype(int) + (np.abs(dy) >= f * np.pi)) > 1).sum())


def test_unwrapping_removes_most_wraps(gold):
    for k in _cases(gold):
        ph, uw = gold[f"c{k}_phase"], gold[f"c{k}_unwrapped"]
        for z in range(ph.shape[2]):
            assert _wrapping(uw[:, :, z]) <= _wrapping(ph[:, :, z]) // 2
