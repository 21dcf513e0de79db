"""GPU aberration correction and dirty-field rejection
(odt_aberration_pattern, odt_field_quality, odt_fft2c and the host mirror
of FIELD_EXPERIMENTAL_RETRIEVAL.get_aberration_pattern / correct_aberration
/ remove_dirty_fields) against the oracle on synthetic aberrated fields.
Bounds: pattern and corrected fields rel-L2 <= 1e-4 (the pattern enters
through angle(), which amplifies the ulp-level differences of the device
FFTs at its smallest values, and the phase-matching sums run in a
different order); the same defocus distance; gradient statistics within
1e-4 relative, the same outside counts and the same kept fields; the
centred FFT within 1e-5 for any length (radix tiles, or Bluestein's
algorithm for lengths with a prime factor above 31)."""
import ctypes as C

import numpy as np
import pytest

import cases
from oracle import cbs, goldstein, retrieval

pytestmark = pytest.mark.gpu

CP = dict(overlap_factor=0.25, distList=[-2.0, -1.0, 0.0, 1.0, 2.0])


def _unwrap(ph):
    out = goldstein.unwrapp2(ph)
    return np.asarray(out[0] if isinstance(out, tuple) else out, dtype=np.float32)


def _solver(params):
    from inverse_solver_b200.retrieval import FIELD_EXPERIMENTAL_RETRIEVAL

    return FIELD_EXPERIMENTAL_RETRIEVAL(FIELD_EXPERIMENTAL_RETRIEVAL.get_default_parameters(params))


def _tool(params):
    return cbs.derive_optical_tool(params, cbs.Prec(True))


@pytest.mark.parametrize("N,n,seed", [(96, 7, 0), (120, 9, 3), (106, 7, 11)])
def test_aberration_pattern_matches_oracle(N, n, seed):
    inp, out, k0s, params = cases.aberrated_fields(N, n, seed=seed)
    ofi, ofo, oab = retrieval.get_aberration_pattern(_tool(params), inp, out, dict(CP, k0s=k0s))
    gfi, gfo, gab = _solver(params).get_aberration_pattern(inp, out, dict(CP, k0s=k0s))
    assert gab["distance"] == oab["distance"]
    assert gfi.shape == ofi.shape and gfo.shape == ofo.shape
    assert cbs.rel_l2(gab["pattern"], oab["pattern"]) < 1e-4
    assert cbs.rel_l2(gfi, ofi) < 1e-4 and cbs.rel_l2(gfo, ofo) < 1e-4


def test_correct_aberration_matches_oracle():
    inp, out, k0s, params = cases.aberrated_fields(96, 7, seed=5)
    r = _solver(params)
    _, _, gab = r.get_aberration_pattern(inp, out, dict(CP, k0s=k0s))
    oab = dict(gab, utility=_tool(params))
    # same optical grid: the pattern is used as it is
    gi, go = r.correct_aberration(inp, out, gab)
    oi, oo = retrieval.correct_aberration(_tool(params), inp, out, oab)
    assert cbs.rel_l2(gi, oi) < 1e-5 and cbs.rel_l2(go, oo) < 1e-5
    # pattern measured on a finer Fourier grid: transform, pad, crop, inverse
    pa = dict(params, resolution=[0.096, 0.096, 0.1])
    ra = _solver(pa)
    _, _, gab_a = ra.get_aberration_pattern(inp, out, dict(CP, k0s=k0s))
    gi, go = r.correct_aberration(inp, out, gab_a)
    oi, oo = retrieval.correct_aberration(_tool(params), inp, out, dict(gab_a, utility=_tool(pa)))
    assert cbs.rel_l2(gi, oi) < 1e-4 and cbs.rel_l2(go, oo) < 1e-4
    # coarser grid: the reference's steps leave mismatched sizes (an error in both)
    pb = dict(params, resolution=[0.104, 0.104, 0.1])
    _, _, gab_b = _solver(pb).get_aberration_pattern(inp, out, dict(CP, k0s=k0s))
    with pytest.raises(ValueError):
        r.correct_aberration(inp, out, gab_b)
    with pytest.raises(ValueError):
        retrieval.correct_aberration(_tool(params), inp, out, dict(gab_b, utility=_tool(pb)))


def test_remove_dirty_fields_matches_oracle():
    inp, out, k0s, params = cases.aberrated_fields(96, 9, seed=7)
    out = out.copy()
    rng = np.random.default_rng(1)
    out[:, :, 0, 2] *= (1 + 0.5 * rng.standard_normal((96, 96))).astype(np.float32)
    out[:, :, 0, 6] *= np.exp(2j * np.pi * 12 * np.arange(96)[None, :] / 96).astype(np.complex64)
    ofi, ofo, osd, ocnt = retrieval.remove_dirty_fields(inp, out, 80, unwrap=_unwrap)
    r = _solver(params)
    gfi, gfo = r.remove_dirty_fields(inp, out, 80)
    assert np.array_equal(gfi, ofi) and np.array_equal(gfo, ofo)
    kept = [k for k in range(9) if any(np.array_equal(gfi[:, :, 0, j], inp[:, :, 0, k]) for j in range(gfi.shape[3]))]
    assert 0 in kept and 2 not in kept and 6 not in kept
    from inverse_solver_b200 import _lib
    sd = np.empty(9, np.float32)
    cnt = np.empty(9, np.int64)
    a = _lib.FieldQualityArgs()
    a.size[:] = [96, 96, 9]
    bg = np.asfortranarray(inp.reshape(96, 96, 9, order="F"))
    sp = np.asfortranarray(out.reshape(96, 96, 9, order="F"))
    a.bg, a.sp, a.gradient_std, a.outside_count = _lib.ptr(bg), _lib.ptr(sp), _lib.ptr(sd), _lib.ptr(cnt)
    a.memory = _lib.ODT_MEM_HOST
    _lib.check(_lib.load().odt_field_quality(C.byref(a)))
    assert np.allclose(sd, osd, rtol=1e-4, atol=1e-12)
    assert np.array_equal(cnt, ocnt)


def test_device_memory_matches_host():
    import torch

    from inverse_solver_b200 import _lib

    inp, out, k0s, params = cases.aberrated_fields(96, 5, seed=4)
    r = _solver(params)
    hi, ho, hab = r.get_aberration_pattern(inp, out, dict(CP, k0s=k0s))
    u = r._utility()
    fin = torch.from_numpy(np.ascontiguousarray(inp.reshape(96, 96, 5, order="F").T)).cuda()
    fout = torch.from_numpy(np.ascontiguousarray(out.reshape(96, 96, 5, order="F").T)).cuda()
    pat = torch.empty((96, 96), dtype=torch.complex64, device="cuda")
    di, do = torch.empty_like(fin), torch.empty_like(fout)
    coorxy = np.asarray(u.coorxy, dtype=np.float32)
    fmask = np.asfortranarray(coorxy < coorxy.max() * np.float32(0.25)).astype(np.uint8)
    na = np.asfortranarray(u.NA_circle.astype(np.uint8))
    rk = np.asfortranarray(np.asarray(u.refocusing_kernel, dtype=np.complex64))
    k0 = np.asfortranarray(k0s)
    dl = np.asarray(CP["distList"], dtype=np.float64)
    a = _lib.AberrationArgs()
    a.size[:] = [96, 96, 5]
    a.input_field, a.output_field = fin.data_ptr(), fout.data_ptr()
    a.k0s, a.pupil_mask, a.na_circle, a.refocusing_kernel = _lib.ptr(k0), _lib.ptr(fmask), _lib.ptr(na), _lib.ptr(rk)
    a.dist_list, a.n_dist = _lib.ptr(dl), len(dl)
    a.pattern, a.input_out, a.output_out = pat.data_ptr(), di.data_ptr(), do.data_ptr()
    a.memory = _lib.ODT_MEM_DEVICE
    a.stream = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.load().odt_aberration_pattern(C.byref(a)))
    torch.cuda.synchronize()
    assert np.array_equal(pat.cpu().numpy().T, hab["pattern"])
    assert np.array_equal(di.cpu().numpy().T, hi.reshape(96, 96, 5, order="F"))
    assert np.array_equal(do.cpu().numpy().T, ho.reshape(96, 96, 5, order="F"))


# sizes: radix tiles on both axes; Bluestein on both (2 * 37, 2 * 53); a
# Bluestein line axis and a Bluestein column axis of padded length 1280 (8
# pencils per tile: the largest tiles of the Bluestein kernels); a Bluestein
# column axis of padded length 2048 and direct lengths of 1536 (4 pencils)
FFT_SIZES = [(60, 84, 3), (74, 106, 2), (37, 53, 1), (636, 96, 1), (96, 636, 1), (64, 1016, 1), (1536, 8, 1),
             (8, 1536, 1)]


@pytest.mark.parametrize("inverse", [False, True])
@pytest.mark.parametrize("shape", FFT_SIZES)
def test_fft2c_matches_numpy(inverse, shape):
    import torch

    from inverse_solver_b200 import _lib

    rng = np.random.default_rng(2)
    x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    ref = cbs.fftc2(x.astype(np.complex128), inverse=inverse)
    h = np.asfortranarray(x.copy())
    a = _lib.Fft2cArgs()
    a.size[:] = list(shape)
    a.data, a.inverse, a.memory = _lib.ptr(h), int(inverse), _lib.ODT_MEM_HOST
    _lib.check(_lib.load().odt_fft2c(C.byref(a)))
    assert cbs.rel_l2(h, ref) < 1e-5
    d = torch.from_numpy(np.ascontiguousarray(x.transpose(2, 1, 0))).cuda()
    a.data, a.memory, a.stream = d.data_ptr(), _lib.ODT_MEM_DEVICE, torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.load().odt_fft2c(C.byref(a)))
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy().transpose(2, 1, 0), h)


def test_refocus_any_length_matches_oracle():
    from inverse_solver_b200.retrieval import FIELD_EXPERIMENTAL_RETRIEVAL

    inp, out, k0s, params = cases.aberrated_fields(106, 3, seed=12)     # 106 = 2 * 53: Bluestein axes
    p = FIELD_EXPERIMENTAL_RETRIEVAL.get_default_parameters(params)
    got = FIELD_EXPERIMENTAL_RETRIEVAL(p).refocus(out, 0.7)
    ref = retrieval.refocus(params, out, 0.7)
    assert cbs.rel_l2(got, ref) < 1e-5
