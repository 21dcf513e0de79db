"""C-ABI library checks that need no GPU: it loads, exports every symbol
include/odt.h declares, and its argument checks fail cleanly."""
import ctypes as C
import os
import re

import pytest

from inverse_solver_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "odt.h")).read()
    return sorted(set(re.findall(r"^\s*(?:odt_status|const char\*|int32_t)\s+(odt_\w+)\s*\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_symbols()
    assert "odt_create" in names and "odt_solve" in names and len(names) >= 9
    for n in names:
        assert hasattr(lib, n), n
        assert n in _lib.SIGNATURES, n
    assert lib.odt_abi_version() == 2


def test_bad_handle_and_null_arguments():
    lib = _lib.load()
    st = lib.odt_destroy(123456)
    assert st == 2
    assert b"unknown handle" in lib.odt_last_error()
    assert lib.odt_create(None, None, None, None, None, None, None) == 1
    assert b"NULL" in lib.odt_last_error()
    b = C.c_int32(0)
    assert lib.odt_get_batch(99, C.byref(b)) == 2
    with pytest.raises(_lib.OdtError) as e:
        _lib.check(lib.odt_solve(77, None))
    assert e.value.status == 2
    # RI-tensor potential: NULL V, then an unknown handle (no device call)
    pp = _lib.PotentialParams()
    assert lib.odt_set_tensor_potential(77, C.byref(pp), None) == 1
    v = (C.c_float * 18)()
    assert lib.odt_set_tensor_potential(77, C.byref(pp), C.cast(v, C.c_void_p)) == 2
    assert b"unknown handle" in lib.odt_last_error()


def test_unwrap_argument_checks():
    lib = _lib.load()
    assert lib.odt_unwrap_goldstein(None) == 1
    a = _lib.UnwrapArgs()
    a.size[:] = [1, 8, 1]
    assert lib.odt_unwrap_goldstein(C.byref(a)) == 1          # NULL phase
    import numpy as np
    buf = np.zeros(64, np.float32)
    a.phase_in = a.phase_out = buf.ctypes.data
    assert lib.odt_unwrap_goldstein(C.byref(a)) == 1          # size0 < 2
    assert b"size" in lib.odt_last_error()
    a.size[:] = [65536, 65536, 1]
    assert lib.odt_unwrap_goldstein(C.byref(a)) == 1          # 2^32 elements
    a.size[:] = [8, 8, 1]
    a.memory = 5
    assert lib.odt_unwrap_goldstein(C.byref(a)) == 1          # bad memory flag


def test_mex_gateway_compiles_against_the_header():
    """The MATLAB gateway (inverse_solver_b200/mex/odt_mex.cpp) type-checks
    against include/odt.h, with a declarations-only stand-in for MATLAB's
    mex.h (MATLAB is absent here, so it is not linked)."""
    import shutil
    import subprocess

    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([gxx, "-std=c++17", "-fsyntax-only", "-Wall", "-Werror",
                        "-I" + os.path.join(root, "tests", "native", "mex_stub"),
                        "-I" + os.path.join(root, "include"),
                        os.path.join(root, "inverse_solver_b200", "mex", "odt_mex.cpp")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
