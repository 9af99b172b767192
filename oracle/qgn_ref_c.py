"""ctypes wrapper of oracle/qgn_ref.c, the C / OpenMP FP64 restatement of QGN.

TEST INFRASTRUCTURE ONLY (large-size oracle and timed CPU baseline).  Parity unpinned, as
for oracle/qgn_oracle.py, with which tests/test_oracle_c.py cross-checks it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from .qgn_oracle import Params, QGNOracle

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "qgn_ref.c")
LIB = os.path.join(HERE, "_build", "libqgn_ref.so")
SCHEMES = {"ark43_qgleith": 0, "ark43": 1, "bsrk3": 2, "rk4": 3, "ab3": 4}


def build(force: bool = False) -> str:
    """gcc -O3 -fopenmp; x86-64-v3 so the library also runs on the GPU hosts' CPUs."""
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        cmd = ["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-std=c11", "-o", LIB, SRC, "-lm"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("gcc failed:\n" + r.stderr)
    return LIB


_lib = None


def load():
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(LIB)
        dp = C.POINTER(C.c_double)
        lib.qgn_ref_create.restype = C.c_void_p
        lib.qgn_ref_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, dp, dp, dp, dp, dp, dp]
        lib.qgn_ref_destroy.argtypes = [C.c_void_p]
        lib.qgn_ref_rhs.argtypes = [C.c_void_p, dp, dp]
        lib.qgn_ref_forward.argtypes = [C.c_void_p, dp, dp]
        lib.qgn_ref_step.restype = C.c_int
        lib.qgn_ref_step.argtypes = [C.c_void_p, dp, dp, dp, C.c_int]
        lib.qgn_ref_rejects.restype = C.c_longlong
        lib.qgn_ref_rejects.argtypes = [C.c_void_p]
        lib.qgn_ref_threads.restype = C.c_int
        _lib = lib
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class RefC:
    """The C restatement of one QGN model; host set-up (modes) shared with the numpy oracle."""

    def __init__(self, p: Params, H_raw, S, uBar, scheme="ark43_qgleith"):
        self.lib = load()
        self.m = QGNOracle(p, H_raw, S, uBar)
        self.p = p
        prm = np.array([p.Lx, p.Ly, p.Htot, p.beta, p.A2, p.A8, p.r0, p.C_d, p.TOL, p.dt_max], dtype=np.float64)
        m = self.m
        self._keep = [prm, np.ascontiguousarray(m.H), np.ascontiguousarray(m.uBar),
                      np.ascontiguousarray(m.qyBar), np.asfortranarray(m.Modes), np.ascontiguousarray(m.EVals)]
        self.h = self.lib.qgn_ref_create(p.nx, p.ny, p.nz, SCHEMES[scheme], int(bool(p.is_explicit)),
                                         *[_dp(a) for a in self._keep])

    def __del__(self):
        try:
            self.lib.qgn_ref_destroy(self.h)
        except Exception:
            pass

    def shape(self):
        return (self.p.nz, self.p.ny, self.p.nx // 2 + 1)

    def initialize_spec(self, qp):
        qp = np.ascontiguousarray(qp, dtype=np.float64)
        out = np.empty(self.shape(), dtype=np.complex128)
        self.lib.qgn_ref_forward(self.h, _dp(qp), _dp(out))
        return out

    def get_rhs(self, q):
        q = np.ascontiguousarray(q, dtype=np.complex128)
        out = np.empty_like(q)
        self.lib.qgn_ref_rhs(self.h, _dp(q), _dp(out))
        return out

    def step(self, q, t, dt, max_rejects=10_000):
        """TimeStep in place on q (complex128 C-contiguous); returns (t, dt)."""
        tt, dd = C.c_double(t), C.c_double(dt)
        rc = self.lib.qgn_ref_step(self.h, _dp(q), C.byref(tt), C.byref(dd), int(max_rejects))
        if rc != 0:
            raise RuntimeError("reject limit")
        return tt.value, dd.value

    def rejects(self):
        return self.lib.qgn_ref_rejects(self.h)

    def threads(self):
        return self.lib.qgn_ref_threads()
