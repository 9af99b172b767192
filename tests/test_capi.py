"""The C-ABI library builds, loads and exports every symbol that include/*.h declares.

Only argument validation is exercised here (it runs before any device call)."""
import ctypes as C
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from qgn_fortran_b200 import _lib, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "qgn_gpu.h")
HEADERS = sorted(glob.glob(os.path.join(ROOT, "include", "*.h")))


def header_symbols(paths=HEADERS):
    text = "".join(open(p).read() for p in paths)
    return sorted(set(re.findall(r"^\s*(?:int|const char\s*\*)\s+(qgn_\w+)\s*\(", text, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.load()


def test_header_declares_the_boundary():
    syms = header_symbols([HEADER])
    # test and debugging hooks live in their own header, outside the drop-in boundary
    assert not any("debug" in s for s in syms)
    for s in ("qgn_create", "qgn_step", "qgn_advance", "qgn_rhs", "qgn_set_state", "qgn_get_state",
              "qgn_diagnostics", "qgn_last_error", "qgn_destroy"):
        assert s in syms


def test_every_declared_symbol_is_exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (qgn_\w+)", out))
    for s in header_symbols():
        assert s in exported, s
        assert hasattr(lib, s)
        assert s in _lib.SIGNATURES, s


def test_argument_validation_without_device(lib):
    ctx = C.c_void_p()
    z = np.zeros(4)
    dp = z.ctypes.data_as(C.POINTER(C.c_double))
    assert lib.qgn_create(None, dp, dp, dp, dp, dp, dp, 0, 0, C.byref(ctx)) == _lib.QGN_ERR_ARG
    p = _lib.qgn_params(nx=384, ny=256, nz=2, Lx=1e6, Ly=1e6, Htot=4000.0)
    H = np.array([1000.0, 3000.0])
    M = np.eye(2)
    assert lib.qgn_create(C.byref(p), _lib.dptr(H), None, _lib.dptr(H), _lib.dptr(H), _lib.dptr(M),
                          _lib.dptr(H), 0, 0, C.byref(ctx)) == _lib.QGN_ERR_CONFIG     # nx not 2^k
    p.nx = 256
    p.nz = 1
    assert lib.qgn_create(C.byref(p), _lib.dptr(H), None, _lib.dptr(H), _lib.dptr(H), _lib.dptr(M),
                          _lib.dptr(H), 0, 0, C.byref(ctx)) == _lib.QGN_ERR_CONFIG     # nz < 2
    p.nz = 2
    Hbad = np.array([1000.0, np.nan])
    assert lib.qgn_create(C.byref(p), _lib.dptr(Hbad), None, _lib.dptr(H), _lib.dptr(H), _lib.dptr(M),
                          _lib.dptr(H), 0, 0, C.byref(ctx)) == _lib.QGN_ERR_CONFIG     # non-finite H
    assert lib.qgn_create(C.byref(p), _lib.dptr(H), None, _lib.dptr(H), _lib.dptr(H), _lib.dptr(M),
                          _lib.dptr(H), 9, 0, C.byref(ctx)) == _lib.QGN_ERR_CONFIG     # scheme
    assert lib.qgn_step(None, None, None, None) == _lib.QGN_ERR_ARG
    assert lib.qgn_destroy(None) == 0
    assert lib.qgn_probe_fp64_fma(0, None, None) == _lib.QGN_ERR_ARG
    r = C.c_int()
    assert lib.qgn_ens_fft_radix(None, 0, C.byref(r)) == _lib.QGN_ERR_ARG
    assert lib.qgn_ens_set_tiles(None, 0, 128, 16, 0) == _lib.QGN_ERR_ARG
    assert lib.qgn_last_error(None) == b"null context"
