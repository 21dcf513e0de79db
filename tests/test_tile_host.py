"""The GPU tile-kernel bodies (inverse_solver_b200/csrc/tile_bodies.cuh),
compiled as plain C++ and run CTA by CTA on the CPU in the launch order of
the library, reproduce the oracle's Born series (field inside the ROI) to
single-precision accuracy.  Covers 1-, 2- and 3-pass FFT plans and the short
half-series cases (Bornmax 1, 2, 3)."""
import os
import subprocess

import numpy as np
import pytest

import cases
from inverse_solver_b200.forward import CBSHostSetup
from oracle import cbs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "inverse_solver_b200", "csrc")


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("tile") / "tile_host_check")
    inc = os.environ.get("CUDA_HOME", "/usr/local/cuda") + "/include"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + inc, "-I" + CSRC,
                    os.path.join(ROOT, "tests", "native", "tile_host_check.cpp"),
                    os.path.join(CSRC, "fft_plan.cpp"), "-o", exe], check=True)
    return exe


def run_case(exe, tmp, p, RI, fields):
    h = CBSHostSetup(p)
    h.prepare_potential(RI)
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    inp = o.transform_field_3D(cbs.fftc2(fields.astype(np.complex64)))
    nb = fields.shape[3]
    einc = np.stack([o.refocus_source(inp[:, :, 0, k]) for k in range(nb)], axis=3)
    ref = np.stack([o.solve_raw(inp[:, :, :, k]) for k in range(nb)], axis=3)
    P = h.sim_size
    R = h.ROI
    hdr = np.array(P + [R[0] - 1, R[2] - 1, R[4] - 1] + list(h.expected_RI_size) +
                   [nb, h.Bornmax, 1 if p["acyclic"] else 0, 16, 4, 4, 0], dtype=np.int32)
    eps = np.float32(h.eps_imag)
    sc = np.array([eps, np.float32(1) / eps, np.float32(4 * np.pi ** 2),
                   np.float32((2 * np.pi * h.utility_border.k0_nm) ** 2),
                   1.0 / (P[0] * P[1] * P[2])], dtype=np.float32)
    fin = os.path.join(tmp, "in.bin")
    fout = os.path.join(tmp, "out.bin")
    with open(fin, "wb") as f:
        f.write(hdr.tobytes())
        f.write(sc.tobytes())
        for m in h.attenuation_mask1d:
            f.write(np.asarray(m, np.float32).tobytes())
        for r in h.ramp1d:
            f.write(np.asarray(r, np.complex64).tobytes())
        for k in h.kq2:
            f.write(np.asarray(k, np.float32).tobytes())
        f.write(np.asfortranarray(h.V.astype(np.complex64)).tobytes(order="F"))
        f.write(np.asfortranarray(einc.astype(np.complex64)).tobytes(order="F"))
    subprocess.run([exe, fin, fout], check=True)
    got = np.fromfile(fout, dtype=np.complex64).reshape(einc.shape, order="F")
    return got, ref


@pytest.mark.parametrize("iters", [-1, 1, 2, 3])
def test_small_case(harness, tmp_path, iters):
    p = cases.small_params(iterations_number=iters)
    got, ref = run_case(harness, str(tmp_path), p, cases.small_RI(), cases.circle_fields(p, 2))
    assert cbs.rel_l2(got, ref) < 1e-5


def test_radix7_plan(harness, tmp_path):
    # padded [56, 38, 24]: plans [7,8], [19,2], [8,3]
    p = cases.params([48, 30, 20], [2, 2, 1])
    RI = cases.sphere_phantom([48, 30, 20], [0.1] * 3, cases.NM, seed=7, n_spheres=2,
                              radius_um=(0.3, 0.8))
    got, ref = run_case(harness, str(tmp_path), p, RI, cases.circle_fields(p, 1))
    assert cbs.rel_l2(got, ref) < 1e-5


def test_one_and_three_pass_plans(harness, tmp_path):
    # padded [48, 38, 19]: plans [3,8,2], [19,2], [19]
    p = cases.params([40, 26, 11], [2, 3, 2])
    RI = cases.sphere_phantom([40, 26, 11], [0.1] * 3, cases.NM, seed=5, n_spheres=2,
                              radius_um=(0.3, 0.6))
    got, ref = run_case(harness, str(tmp_path), p, RI, cases.circle_fields(p, 1))
    assert cbs.rel_l2(got, ref) < 1e-5
