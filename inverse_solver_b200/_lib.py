"""ctypes binding of libodt.so (the C ABI declared in include/odt.h).

The shared library is built in-tree (``inverse_solver_b200/libodt.so``).  If
it is missing or does not load, every entry point raises ``OdtError`` -- there
is no CPU fallback for the Born loop.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libodt.so")

ODT_MEM_HOST = 0
ODT_MEM_DEVICE = 1
ODT_STORAGE_COMPLEX64 = 0
ODT_STORAGE_B16 = 1

STATUS_NAMES = {
    0: "ODT_OK",
    1: "ODT_ERR_INVALID_ARGUMENT",
    2: "ODT_ERR_BAD_HANDLE",
    3: "ODT_ERR_CUDA",
    4: "ODT_ERR_OUT_OF_MEMORY",
    5: "ODT_ERR_NOT_READY",
    6: "ODT_ERR_UNSUPPORTED",
    7: "ODT_ERR_NUMERIC",
    8: "ODT_ERR_INTERNAL",
}


class OdtError(RuntimeError):
    """A libodt call failed; ``status`` is the odt_status code."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


class Geometry(C.Structure):
    _fields_ = [
        ("sim_size", C.c_int32 * 3),
        ("ri_size", C.c_int32 * 3),
        ("field_size", C.c_int32 * 2),
        ("conv_size", C.c_int32 * 2),
        ("device", C.c_int32),
        ("max_batch", C.c_int32),
        ("mem_budget", C.c_int64),
        ("pol", C.c_int32),
    ]


class PotentialParams(C.Structure):
    _fields_ = [
        ("eps_imag", C.c_float),
        ("green_scale", C.c_float),
        ("green_offset", C.c_float),
        ("dV", C.c_float),
        ("roi", C.c_int32 * 6),
        ("bornmax", C.c_int32),
        ("acyclic", C.c_int32),
        ("mask", C.c_void_p * 3),
        ("ramp", C.c_void_p * 3),
        ("kq2", C.c_void_p * 3),
        ("rad", C.c_void_p * 3),
        ("absorb", C.c_float * 2),
    ]


class SolveArgs(C.Structure):
    _fields_ = [
        ("fields_in", C.c_void_p),
        ("n_ill", C.c_int32),
        ("trans", C.c_void_p),
        ("ref", C.c_void_p),
        ("field3d", C.c_void_p),
        ("memory", C.c_int32),
        ("stream", C.c_void_p),
    ]


class NoallocBornArgs(C.Structure):
    _fields_ = [
        ("sim_size", C.c_int32 * 3),
        ("roi", C.c_int32 * 6),
        ("bornmax", C.c_int32),
        ("acyclic", C.c_int32),
        ("eps_imag", C.c_float),
        ("green_scale", C.c_float),
        ("green_offset", C.c_float),
        ("mask", C.c_void_p * 3),
        ("ramp", C.c_void_p * 3),
        ("kq2", C.c_void_p * 3),
        ("V", C.c_void_p),
        ("einc", C.c_void_p),
        ("fout", C.c_void_p),
        ("stream", C.c_void_p),
    ]


class GradientArgs(C.Structure):
    _fields_ = [
        ("fields_in", C.c_void_p),
        ("fields_meas", C.c_void_p),
        ("n_ill", C.c_int32),
        ("grad", C.c_void_p),
        ("err", C.c_void_p),
        ("memory", C.c_int32),
        ("stream", C.c_void_p),
    ]


class RIDeviceArgs(C.Structure):
    _fields_ = [
        ("ri", C.c_void_p),
        ("is_complex", C.c_int32),
        ("adjoint", C.c_int32),
        ("wavelength", C.c_double),
        ("ri_bg", C.c_double),
        ("stream", C.c_void_p),
    ]


class FistaArgs(C.Structure):
    _fields_ = [
        ("n", C.c_int64),
        ("grad", C.c_void_p),
        ("u", C.c_void_p),
        ("x", C.c_void_p),
        ("ri", C.c_void_p),
        ("prox_in", C.c_void_p),
        ("prox_out", C.c_void_p),
        ("prox_complex", C.c_int32),
        ("step", C.c_double),
        ("coef", C.c_double),
        ("ri_bg", C.c_double),
        ("stream", C.c_void_p),
    ]


class HologramArgs(C.Structure):
    _fields_ = [
        ("size", C.c_int32 * 3),
        ("bg", C.c_void_p),
        ("sp", C.c_void_p),
        ("cutout_portion", C.c_double),
        ("other_corner", C.c_int32),
        ("out_size", C.c_int32),
        ("crop", C.c_int32),
        ("na_circle", C.c_void_p),
        ("bg_field", C.c_void_p),
        ("sp_field", C.c_void_p),
        ("peaks", C.c_void_p),
        ("sideband", C.c_void_p),
        ("memory", C.c_int32),
        ("stream", C.c_void_p),
    ]


class HologramPhaseArgs(C.Structure):
    _fields_ = [
        ("size", C.c_int32 * 3),
        ("bg", C.c_void_p),
        ("sp", C.c_void_p),
        ("conjugate", C.c_int32),
        ("phase", C.c_void_p),
        ("amp", C.c_void_p),
        ("stream", C.c_void_p),
    ]


class HologramCombineArgs(C.Structure):
    _fields_ = [
        ("size", C.c_int32 * 3),
        ("bg", C.c_void_p),
        ("amp", C.c_void_p),
        ("phase", C.c_void_p),
        ("coef", C.c_void_p),
        ("sp", C.c_void_p),
        ("stream", C.c_void_p),
    ]


class AberrationArgs(C.Structure):
    _fields_ = [
        ("size", C.c_int32 * 3),
        ("input_field", C.c_void_p),
        ("output_field", C.c_void_p),
        ("k0s", C.c_void_p),
        ("pupil_mask", C.c_void_p),
        ("na_circle", C.c_void_p),
        ("refocusing_kernel", C.c_void_p),
        ("dist_list", C.c_void_p),
        ("n_dist", C.c_int32),
        ("pattern", C.c_void_p),
        ("input_out", C.c_void_p),
        ("output_out", C.c_void_p),
        ("chosen", C.c_void_p),
        ("memory", C.c_int32),
        ("stream", C.c_void_p),
    ]


class Fft2cArgs(C.Structure):
    _fields_ = [
        ("size", C.c_int32 * 3),
        ("data", C.c_void_p),
        ("inverse", C.c_int32),
        ("memory", C.c_int32),
        ("stream", C.c_void_p),
    ]


class FieldQualityArgs(C.Structure):
    _fields_ = [
        ("size", C.c_int32 * 3),
        ("bg", C.c_void_p),
        ("sp", C.c_void_p),
        ("gradient_std", C.c_void_p),
        ("outside_count", C.c_void_p),
        ("memory", C.c_int32),
        ("stream", C.c_void_p),
    ]


class RefocusArgs(C.Structure):
    _fields_ = [
        ("size", C.c_int32 * 3),
        ("field", C.c_void_p),
        ("kernel", C.c_void_p),
        ("out", C.c_void_p),
    ]


class GreenArgs(C.Structure):
    _fields_ = [
        ("radial", C.c_void_p),
        ("n_r", C.c_int32),
        ("near1", C.c_void_p),
        ("near2", C.c_void_p),
        ("w", C.c_void_p),
        ("creation", C.c_int32 * 3),
        ("out_size", C.c_int32 * 3),
        ("scale", C.c_float),
        ("m1", C.c_void_p),
        ("m2", C.c_void_p),
        ("mz", C.c_void_p),
        ("out", C.c_void_p),
        ("device", C.c_int32),
    ]


class HankelArgs(C.Structure):
    _fields_ = [
        ("roots", C.c_void_p),
        ("n", C.c_int32),
        ("pos", C.c_int32),
        ("nz", C.c_int32),
        ("values", C.c_void_p),
        ("band", C.c_void_p),
        ("out", C.c_void_p),
        ("device", C.c_int32),
    ]


class SourceArgs(C.Structure):
    _fields_ = [
        ("source", C.c_void_p),
        ("n", C.c_int32),
        ("field3d", C.c_void_p),
        ("memory", C.c_int32),
        ("stream", C.c_void_p),
    ]


class TuneResult(C.Structure):
    _fields_ = [
        ("fused_xy", C.c_int32),
        ("pipelined", C.c_int32),
        ("batch", C.c_int32),
        ("cached", C.c_int32),
        ("ms", C.c_double * 3),
    ]


class BPMArgs(C.Structure):
    _fields_ = [
        ("size", C.c_int32 * 3),
        ("field_multiplier", C.c_void_p),
        ("refocus_kernel", C.c_void_p),
        ("filter_out", C.c_void_p),
        ("pre", C.c_void_p),
        ("post", C.c_void_p),
        ("cos_theta", C.c_void_p),
        ("fields_in", C.c_void_p),
        ("n_ill", C.c_int32),
        ("trans", C.c_void_p),
        ("field3d", C.c_void_p),
        ("memory", C.c_int32),
        ("stream", C.c_void_p),
    ]


class TVArgs(C.Structure):
    _fields_ = [
        ("size", C.c_int32 * 3),
        ("inp", C.c_void_p),
        ("out", C.c_void_p),
        ("is_complex", C.c_int32),
        ("lam", C.c_double),
        ("vmin", C.c_double),
        ("vmax", C.c_double),
        ("vimag_max", C.c_double),
        ("non_neg", C.c_int32),
        ("dirichlet", C.c_int32),
        ("inner_itt", C.c_int32),
        ("memory", C.c_int32),
        ("stream", C.c_void_p),
    ]


class RytovArgs(C.Structure):
    _fields_ = [
        ("size", C.c_int32 * 3),
        ("resolution", C.c_double * 3),
        ("fourier_res", C.c_double * 3),
        ("k0_nm", C.c_double),
        ("ri_bg", C.c_double),
        ("wavelength", C.c_double),
        ("coor1", C.c_void_p),
        ("coor2", C.c_void_p),
        ("k3", C.c_void_p),
        ("na_circle", C.c_void_p),
        ("emask", C.c_void_p),
        ("bg", C.c_void_p),
        ("sp", C.c_void_p),
        ("phase", C.c_void_p),
        ("n_ill", C.c_int32),
        ("count_one", C.c_int32),
        ("non_negativity_iteration", C.c_int32),
        ("RI", C.c_void_p),
        ("ORytov", C.c_void_p),
        ("count", C.c_void_p),
        ("overlap_field", C.c_void_p),
        ("shifts", C.c_void_p),
        ("memory", C.c_int32),
        ("stream", C.c_void_p),
    ]


# every symbol include/odt.h declares: name -> (restype, argtypes)
class UnwrapArgs(C.Structure):
    _fields_ = [
        ("size", C.c_int32 * 3),
        ("phase_in", C.c_void_p),
        ("phase_out", C.c_void_p),
        ("residue_out", C.c_void_p),
        ("step1_out", C.c_void_p),
        ("step2_out", C.c_void_p),
        ("table_out", C.c_void_p),
        ("nearest_out", C.c_void_p),
        ("residue_cap", C.c_int64),
        ("branches_out", C.c_void_p),
        ("branch_cap", C.c_int64),
        ("n_residues", C.c_void_p),
        ("n_branches", C.c_void_p),
        ("link_threads", C.c_int32),
        ("memory", C.c_int32),
        ("stream", C.c_void_p),
    ]


SIGNATURES = {
    "odt_create": (C.c_int, [C.POINTER(Geometry), C.c_void_p, C.c_void_p, C.c_void_p,
                             C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32)]),
    "odt_set_potential": (C.c_int, [C.c_uint32, C.POINTER(PotentialParams), C.c_void_p]),
    "odt_set_polarisation": (C.c_int, [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "odt_solve": (C.c_int, [C.c_uint32, C.POINTER(SolveArgs)]),
    "odt_destroy": (C.c_int, [C.c_uint32]),
    "odt_get_batch": (C.c_int, [C.c_uint32, C.POINTER(C.c_int32)]),
    "odt_set_profiling": (C.c_int, [C.c_uint32, C.c_int32]),
    "odt_set_field_storage": (C.c_int, [C.c_uint32, C.c_int32]),
    "odt_hankel_filter": (C.c_int, [C.POINTER(HankelArgs)]),
    "odt_autotune": (C.c_int, [C.c_uint32, C.c_int32, C.POINTER(TuneResult)]),
    "odt_solve_source": (C.c_int, [C.c_uint32, C.POINTER(SourceArgs)]),
    "odt_get_kernel_times": (C.c_int, [C.c_uint32, C.POINTER(C.c_char_p),
                                       C.POINTER(C.c_double), C.POINTER(C.c_int64),
                                       C.c_int32, C.POINTER(C.c_int32)]),
    "odt_born_series_noalloc": (C.c_int, [C.POINTER(NoallocBornArgs)]),
    "odt_set_adjoint_potential": (C.c_int, [C.c_uint32, C.POINTER(PotentialParams), C.c_void_p]),
    "odt_set_tensor_potential": (C.c_int, [C.c_uint32, C.POINTER(PotentialParams), C.c_void_p]),
    "odt_gradient": (C.c_int, [C.c_uint32, C.POINTER(GradientArgs)]),
    "odt_tv_prox": (C.c_int, [C.POINTER(TVArgs)]),
    "odt_potential_eps_device": (C.c_int, [C.c_uint32, C.POINTER(RIDeviceArgs), C.POINTER(C.c_float)]),
    "odt_set_potential_device": (C.c_int, [C.c_uint32, C.POINTER(PotentialParams), C.POINTER(RIDeviceArgs)]),
    "odt_fista_prox_input": (C.c_int, [C.POINTER(FistaArgs)]),
    "odt_fista_update": (C.c_int, [C.POINTER(FistaArgs)]),
    "odt_bpm_solve": (C.c_int, [C.POINTER(BPMArgs)]),
    "odt_green_planes": (C.c_int, [C.POINTER(GreenArgs)]),
    "odt_hologram_fields": (C.c_int, [C.POINTER(HologramArgs)]),
    "odt_refocus_2d": (C.c_int, [C.POINTER(RefocusArgs)]),
    "odt_hologram_phase": (C.c_int, [C.POINTER(HologramPhaseArgs)]),
    "odt_hologram_combine": (C.c_int, [C.POINTER(HologramCombineArgs)]),
    "odt_aberration_pattern": (C.c_int, [C.POINTER(AberrationArgs)]),
    "odt_field_quality": (C.c_int, [C.POINTER(FieldQualityArgs)]),
    "odt_fft2c": (C.c_int, [C.POINTER(Fft2cArgs)]),
    "odt_submit": (C.c_int, [C.c_uint32, C.POINTER(SolveArgs), C.POINTER(C.c_uint64)]),
    "odt_poll": (C.c_int, [C.c_uint32, C.c_uint64, C.POINTER(C.c_int32), C.POINTER(C.c_int)]),
    "odt_wait": (C.c_int, [C.c_uint32, C.c_uint64, C.POINTER(C.c_int)]),
    "odt_budget": (C.c_int, [C.c_uint32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "odt_rytov": (C.c_int, [C.POINTER(RytovArgs)]),
    "odt_unwrap_goldstein": (C.c_int, [C.POINTER(UnwrapArgs)]),
    "odt_last_error": (C.c_char_p, []),
    "odt_abi_version": (C.c_int32, []),
}

_lock = threading.Lock()
_lib = None


def load():
    """Load libodt.so once and attach signatures; raises OdtError if absent."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise OdtError(8, f"{LIB_PATH} not built (run __graft_entry__.build() or make -C "
                              "inverse_solver_b200/csrc)")
        try:
            lib = C.CDLL(LIB_PATH)
        except OSError as e:
            raise OdtError(8, f"cannot load {LIB_PATH}: {e}") from e
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(status: int):
    if status != 0:
        msg = load().odt_last_error()
        raise OdtError(status, msg.decode() if msg else "")


def ptr(a) -> int:
    """Address of a numpy array or torch tensor (contiguous)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data
