"""The asynchronous entry points (odt_submit / odt_poll / odt_wait /
odt_budget) reject an unknown handle with ODT_ERR_BAD_HANDLE before touching
the GPU (CPU-only check of the argument paths)."""
import ctypes as C

from inverse_solver_b200 import _lib


def test_unknown_handle_is_rejected():
    lib = _lib.load()
    a = _lib.SolveArgs()
    t = C.c_uint64(0)
    done, st = C.c_int32(0), C.c_int(0)
    held, bud = C.c_int64(0), C.c_int64(0)
    assert lib.odt_submit(987654, C.byref(a), C.byref(t)) == 2
    assert lib.odt_poll(987654, 1, C.byref(done), C.byref(st)) == 2
    assert lib.odt_wait(987654, 1, C.byref(st)) == 2
    assert lib.odt_budget(987654, C.byref(held), C.byref(bud)) == 2
    assert b"unknown handle" in lib.odt_last_error()
