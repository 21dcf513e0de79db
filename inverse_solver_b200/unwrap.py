"""Goldstein branch-cut phase unwrapping on the B200 library.

Mirrors Codes/sub_code/goldstein_GPU/unwrapp2_gpu.m: residues, dipole
removal, branch cuts (goldstein_branch_cut.m) and integration, all in one
call of odt_unwrap_goldstein (GPU kernels plus the host branch linker).
Arrays are indexed as in MATLAB (a[d1, d2, slice]); a 2D map is one slice.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

F32 = np.float32
NEAREST = 8   # precomputed_shortest_number of goldstein_branch_cut.m:24


def _size(shape):
    if len(shape) not in (2, 3):
        raise ValueError("wrapped phase must be 2D or 3D")
    n = shape[2] if len(shape) == 3 else 1
    return [int(shape[0]), int(shape[1]), int(n)]


def _run(args):
    _lib.check(_lib.load().odt_unwrap_goldstein(C.byref(args)))


def unwrap_goldstein(wrapped_phase, intermediates=False, link_threads=0):
    """Unwrap a 2D or 3D single-precision phase (numpy).  With
    ``intermediates`` also return a dict of the chain's products: residue
    (after dipole removal), step1, step2, table [6, R], nearest [2, 8, R] and
    branches [6, B] in the reference's layouts."""
    w = np.asfortranarray(np.asarray(wrapped_phase, dtype=F32))
    size = _size(w.shape)
    out = np.empty(w.shape, dtype=F32, order="F")
    a = _lib.UnwrapArgs()
    a.size[:] = size
    a.phase_in, a.phase_out = _lib.ptr(w), _lib.ptr(out)
    a.link_threads = int(link_threads)
    a.memory = _lib.ODT_MEM_HOST
    a.stream = None
    nres, nbr = C.c_int64(0), C.c_int64(0)
    a.n_residues = C.cast(C.byref(nres), C.c_void_p)
    a.n_branches = C.cast(C.byref(nbr), C.c_void_p)
    if not intermediates:
        _run(a)
        return out
    N1, N2, n = size
    res = np.empty((N1 - 1, N2 - 1, n), dtype=F32, order="F")
    s1 = np.empty((N1, N2, n), dtype=np.int32, order="F")
    s2 = np.empty((N2, n), dtype=np.int32, order="F")
    a.residue_out, a.step1_out, a.step2_out = _lib.ptr(res), _lib.ptr(s1), _lib.ptr(s2)
    _run(a)
    # second pass with tables sized from the counts of the first
    R, B = int(nres.value), int(nbr.value)
    tab = np.zeros((6, max(R, 1)), dtype=np.int32, order="F")
    near = np.zeros((2, NEAREST, max(R, 1)), dtype=np.int32, order="F")
    br = np.zeros((6, max(B, 1)), dtype=np.int32, order="F")
    out2 = np.empty(w.shape, dtype=F32, order="F")
    a.phase_out = _lib.ptr(out2)
    a.residue_out = a.step1_out = a.step2_out = None
    a.table_out, a.nearest_out, a.residue_cap = _lib.ptr(tab), _lib.ptr(near), R
    a.branches_out, a.branch_cap = _lib.ptr(br), B
    _run(a)
    shp = w.shape
    inter = {"residue": res.reshape(res.shape[:2] + ((n,) if len(shp) == 3 else ())),
             "step1": s1.reshape(s1.shape[:2] + ((n,) if len(shp) == 3 else ())),
             "step2": s2, "table": tab[:, :R], "nearest": near[:, :, :R], "branches": br[:, :B]}
    return out, inter


def unwrap_goldstein_device(wrapped, out=None, link_threads=0):
    """Unwrap a CUDA torch tensor indexed [d1, d2(, slice)] (MATLAB order;
    the tensor's memory is converted to column-major for the library) on the
    current stream; returns a tensor of the same shape."""
    import torch

    if wrapped.dtype != torch.float32 or not wrapped.is_cuda:
        raise TypeError("expected a float32 CUDA tensor")
    size = _size(tuple(wrapped.shape))
    col = wrapped.permute(*reversed(range(wrapped.dim()))).contiguous()   # column-major storage
    res = torch.empty_like(col)
    a = _lib.UnwrapArgs()
    a.size[:] = size
    a.phase_in, a.phase_out = col.data_ptr(), res.data_ptr()
    a.link_threads = int(link_threads)
    a.memory = _lib.ODT_MEM_DEVICE
    a.stream = torch.cuda.current_stream(wrapped.device).cuda_stream
    with torch.cuda.device(wrapped.device):
        _run(a)
    r = res.permute(*reversed(range(res.dim())))
    if out is not None:
        out.copy_(r)
        return out
    return r


def unwrapp2_gpu(wrapped_phase):
    """unwrapp2_gpu.m:1-6: the unwrapped phase, same shape and type family
    as the input (numpy array or CUDA torch tensor)."""
    if type(wrapped_phase).__module__.startswith("torch"):
        return unwrap_goldstein_device(wrapped_phase)
    return unwrap_goldstein(wrapped_phase)
