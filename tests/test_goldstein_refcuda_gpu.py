"""The library's Goldstein GPU stages against the reference's own CUDA
kernels, built from the reference sources into oracle/_ref/
libref_goldstein_cuda.so (oracle/ref_goldstein/Makefile; skipped when that
library was not built):

  residues  get_residue_cuda.cu:34-66            -> with the dipole pass,
  dipoles   remove_dipoles_cuda.cu:52-146           residue_out: array_equal
  raster    raster_branches_cuda.cu:68-161       -> step1_out / step2_out:
                                                    array_equal
  integrate unwrapp_phase_goldstein_cuda.cu:63-157 -> phase_out: within 8
                                                    units in the last place
                                                    of the slice's largest
                                                    magnitude

The reference chain is driven as unwrapp2_gpu.m / goldstein_branch_cut.m
drive it: find(residue > 0) as 1-based int32 positives for the dipole pass,
step 1 from the dipole pass converted to int32, step 2 [N1, n] zeros (the
dipole gateway returns its zero-filled second output), then the raster of
the branch list and the integration.  The branch list fed to the
reference's raster is the library's, which equals the reference's own
linker output (tests/test_goldstein_gpu.py).  Maps are square because the
reference's step 2 is [N1, n] while its raster and integration index it
with stride N2.  The integration may differ in the last places where a step
is non-zero: the reference's kernels are built with nvcc's defaults, which
may contract `last + d - step*2*pi` into one multiply-add, and the library
rounds the product and the sum separately, as the oracle does; each pixel's
wrapped difference is taken against the previous unwrapped value, so such
a difference stays at the rounding level of the running (unwrapped) value
instead of growing along the path."""

import ctypes as C
import os

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                   "libref_goldstein_cuda.so")


def _assert_ulps(a, b, n=8):
    """Equal within n units in the last place of each slice's largest
    unwrapped magnitude (the integration carries the running value, so a
    rounding difference is an absolute one at that magnitude)."""
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32).reshape(a.shape, order="F")
    a3 = a.reshape(a.shape[0], a.shape[1], -1)
    b3 = b.reshape(a3.shape)
    big = np.maximum(np.abs(a3), np.abs(b3)).max(axis=(0, 1))
    ulp = np.spacing(big.astype(np.float32))[None, None, :]
    d = np.abs(a3.astype(np.float64) - b3)
    assert np.all(d <= n * ulp), float(np.max(d / ulp))


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(LIB):
        pytest.skip("reference CUDA kernels not built (oracle/ref_goldstein/Makefile)")
    lib = C.CDLL(LIB)
    for f in ("ref_cuda_residue", "ref_cuda_dipoles", "ref_cuda_raster", "ref_cuda_unwrap"):
        getattr(lib, f).restype = C.c_int
    return lib


def _reference_chain(lib, phase, branches):
    import torch

    dev = torch.device("cuda", 0)
    n1, n2, n3 = phase.shape
    ph = torch.from_numpy(np.ascontiguousarray(phase.ravel(order="F"))).to(dev)
    res = torch.zeros((n1 - 1) * (n2 - 1) * n3, dtype=torch.float32, device=dev)
    assert lib.ref_cuda_residue(C.c_void_p(ph.data_ptr()), C.c_void_p(res.data_ptr()), n1, n2, n3) == 0
    pos = np.flatnonzero(res.cpu().numpy() > 0).astype(np.int32) + 1    # find(residue_map(:) > 0)
    pos_d = torch.from_numpy(pos).to(dev) if pos.size else torch.zeros(1, dtype=torch.int32, device=dev)
    step1f = torch.zeros(n1 * n2 * n3, dtype=torch.float32, device=dev)
    assert lib.ref_cuda_dipoles(C.c_void_p(res.data_ptr()), C.c_void_p(pos_d.data_ptr()), int(pos.size),
                                C.c_void_p(step1f.data_ptr()), n1, n2, n3) == 0
    step1 = step1f.to(torch.int32)
    step2 = torch.zeros(n1 * n3, dtype=torch.int32, device=dev)
    br = np.ascontiguousarray(np.asarray(branches, np.int32).T)          # [6, B] column-major
    br_d = torch.from_numpy(br.ravel()).to(dev) if br.size else torch.zeros(6, dtype=torch.int32, device=dev)
    assert lib.ref_cuda_raster(C.c_void_p(br_d.data_ptr()), int(br.shape[0]), C.c_void_p(step1.data_ptr()),
                               C.c_void_p(step2.data_ptr()), n1, n2, n3) == 0
    out = ph.clone()
    assert lib.ref_cuda_unwrap(C.c_void_p(out.data_ptr()), C.c_void_p(step1.data_ptr()),
                               C.c_void_p(step2.data_ptr()), n1, n2, n3) == 0
    f = lambda t, shp: t.cpu().numpy().reshape(shp, order="F")  # noqa: E731
    return (f(res, (n1 - 1, n2 - 1, n3)), f(step1, (n1, n2, n3)), f(step2, (n1, n3)), f(out, (n1, n2, n3)))


def _golden_phases():
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "goldstein_small.npz"))
    out = []
    for k in range(int(g["n_cases"])):
        ph = g[f"c{k}_phase"]
        ph = ph if ph.ndim == 3 else ph[:, :, None]
        if ph.shape[0] == ph.shape[1]:
            out.append(ph)
    return out


CASES = [((128, 128, 4), 41, 1.0), ((96, 96, 3), 42, 2.5), ((64, 64, 2), 43, 0.9), ((128, 128, 49), 44, 0.8)]


@pytest.mark.parametrize("shape,seed,noise", CASES)
def test_library_stages_equal_reference_cuda_kernels(ref, shape, seed, noise):
    from inverse_solver_b200.unwrap import unwrap_goldstein

    ph = cases.wrapped_phase(shape, seed, noise)
    out, it = unwrap_goldstein(ph, intermediates=True)
    rres, rs1, rs2, rout = _reference_chain(ref, ph, it["branches"])
    assert np.array_equal(it["residue"], rres)
    assert np.count_nonzero(rres) > 0
    assert np.array_equal(it["step1"], rs1)
    assert np.array_equal(np.asarray(it["step2"]).reshape(rs2.shape, order="F"), rs2)
    _assert_ulps(out, rout)


def test_golden_cases_equal_reference_cuda_kernels(ref):
    from inverse_solver_b200.unwrap import unwrap_goldstein

    phases = _golden_phases()
    assert phases
    for ph in phases:
        out, it = unwrap_goldstein(ph, intermediates=True)
        rres, rs1, rs2, rout = _reference_chain(ref, ph, it["branches"])
        assert np.array_equal(np.asarray(it["residue"]).reshape(rres.shape, order="F"), rres)
        assert np.array_equal(np.asarray(it["step1"]).reshape(rs1.shape, order="F"), rs1)
        _assert_ulps(out, rout)
