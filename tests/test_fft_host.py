"""CPU check of the Stockham pass logic in fft_core.cuh: the device functions
compile as plain C++ and run pass by pass with one thread (exact, since each
pass is a pure src -> dst map); results are compared with numpy."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "inverse_solver_b200", "csrc")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("fft") / "fft_host_check")
    cuda_inc = os.environ.get("CUDA_HOME", "/usr/local/cuda") + "/include"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + cuda_inc, "-I" + CSRC,
                    os.path.join(ROOT, "tests", "native", "fft_host_check.cpp"),
                    os.path.join(CSRC, "fft_plan.cpp"), "-o", exe], check=True)
    return exe


def _run(exe, n, W, inv, x, order=0):
    inp = "\n".join(f"{v.real:.9g} {v.imag:.9g}" for v in x.ravel())
    r = subprocess.run([exe, str(n), str(W), str(int(inv)), str(order)], input=inp,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return np.array([complex(*map(float, l.split())) for l in r.stdout.split("\n") if l]).reshape(W, n)


SIZES = [1, 2, 3, 5, 8, 9, 12, 16, 19, 24, 27, 29, 31, 64, 88, 96, 120, 128, 144, 152, 200,
         216, 256, 280, 3 * 17, 5 * 23, 625, 1000]


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("inv", [False, True])
@pytest.mark.parametrize("order", [0, 1])
def test_stockham_matches_numpy(checker, n, inv, order):
    rng = np.random.default_rng(n)
    W = 4
    x = (rng.standard_normal((W, n)) + 1j * rng.standard_normal((W, n))).astype(np.complex64)
    y = _run(checker, n, W, inv, x, order)
    xd = x.astype(np.complex128)
    ref = np.fft.ifft(xd, axis=1) * n if inv else np.fft.fft(xd, axis=1)
    err = np.linalg.norm(y - ref) / np.linalg.norm(ref)
    assert err < 3e-7, err


def test_unsupported_prime_is_rejected(checker):
    r = subprocess.run([checker, "37", "4", "0"], input="", capture_output=True, text=True)
    assert r.returncode == 4 and "prime factor 37" in r.stderr


TILE_SIZES = [3, 7, 9, 15, 16, 19, 21, 24, 26, 27, 35, 38, 52, 56, 88, 96]


@pytest.fixture(scope="module")
def tile_checker(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("tfft") / "fft_tile_host_check")
    cuda_inc = os.environ.get("CUDA_HOME", "/usr/local/cuda") + "/include"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + cuda_inc, "-I" + CSRC,
                    os.path.join(ROOT, "tests", "native", "fft_tile_host_check.cpp"),
                    os.path.join(CSRC, "fft_plan.cpp"), "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("n", TILE_SIZES)
@pytest.mark.parametrize("kind", [0, 1])
def test_tile_fft_bodies_with_centring_shifts(tile_checker, n, kind):
    """The line / column FFT kernel bodies (dispatched on the plan's radix
    class, as on the GPU) against numpy's centred FFT, both directions."""
    rng = np.random.default_rng(n + 100 * kind)
    n0, n2 = 20, 3
    if kind == 0:
        x = (rng.standard_normal((n, n0 * n2)) + 1j * rng.standard_normal((n, n0 * n2))).astype(np.complex64)
        ax = 0
    else:
        x = (rng.standard_normal((n0, n, n2)) + 1j * rng.standard_normal((n0, n, n2))).astype(np.complex64)
        ax = 1
    inp = "\n".join(f"{v.real:.9g} {v.imag:.9g}" for v in x.ravel(order="F"))
    for inv in (False, True):
        r = subprocess.run([tile_checker, str(kind), str(n0), str(n), str(n2), str(int(inv)),
                            str(n // 2), "0"], input=inp, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        y = np.array([complex(*map(float, l.split())) for l in r.stdout.split("\n") if l])
        y = y.reshape(x.shape, order="F")
        xd = np.fft.ifftshift(x.astype(np.complex128), axes=ax)
        ref = np.fft.fftshift((np.fft.ifft if inv else np.fft.fft)(xd, axis=ax), axes=ax)
        assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 3e-7
