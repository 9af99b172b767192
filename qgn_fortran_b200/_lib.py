"""ctypes binding of include/qgn_gpu.h (and the test hooks of include/qgn_gpu_debug.h).

This is the same binding a Python host makes through ctypes.
Loading fails loudly when the CUDA library has not been built: there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqgn_b200.so")
# the bounds-checked debug build (qgn_fortran_b200.build(check=True)), loaded only by its test
CHECK_LIB_PATH = os.path.join(HERE, "libqgn_b200_check.so")

QGN_OK = 0
QGN_ERR_CONFIG = 1
QGN_ERR_CUDA = 2
QGN_ERR_NONFINITE = 3
QGN_ERR_REJECT_LIMIT = 4
QGN_ERR_ARG = 5
QGN_ERR_NO_DEVICE = 6
QGN_ERR_TOO_LARGE = 7
QGN_STATIC_SCRATCH_BYTES = 32 * 1024 * 1024
QGN_OUTPUT_KEPT = 0
QGN_OUTPUT_FULL = 1
QGN_KERNEL_FAMILIES = 14

SCHEMES = {"ark43_qgleith": 0, "ark43": 1, "bsrk3": 2, "rk4": 3, "ab3": 4}
PRECISIONS = {"fp64": 0, "mixed": 1}

ERROR_NAMES = {
    QGN_ERR_CONFIG: "QGN_ERR_CONFIG",
    QGN_ERR_CUDA: "QGN_ERR_CUDA",
    QGN_ERR_NONFINITE: "QGN_ERR_NONFINITE",
    QGN_ERR_REJECT_LIMIT: "QGN_ERR_REJECT_LIMIT",
    QGN_ERR_ARG: "QGN_ERR_ARG",
    QGN_ERR_NO_DEVICE: "QGN_ERR_NO_DEVICE",
    QGN_ERR_TOO_LARGE: "QGN_ERR_TOO_LARGE",
}


class qgn_params(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("is_explicit", C.c_int),
        ("Lx", C.c_double), ("Ly", C.c_double), ("Htot", C.c_double),
        ("f0", C.c_double), ("beta", C.c_double),
        ("A2", C.c_double), ("A8", C.c_double), ("r0", C.c_double), ("C_d", C.c_double),
        ("TOL", C.c_double), ("dt_max", C.c_double),
        ("max_rejects", C.c_int), ("reserved", C.c_int),
    ]


# every symbol include/qgn_gpu.h declares, with its ctypes signature
_dp = C.POINTER(C.c_double)
_ctxp = C.c_void_p
SIGNATURES = {
    "qgn_create": (C.c_int, [C.POINTER(qgn_params), _dp, _dp, _dp, _dp, _dp, _dp, C.c_int, C.c_int,
                             C.POINTER(C.c_void_p)]),
    "qgn_step": (C.c_int, [_ctxp, _dp, _dp, _dp]),
    "qgn_advance": (C.c_int, [_ctxp, _dp, _dp, _dp, C.c_int]),
    "qgn_set_output": (C.c_int, [_ctxp, C.c_int]),
    "qgn_set_state": (C.c_int, [_ctxp, _dp, C.c_double, C.c_double]),
    "qgn_get_state": (C.c_int, [_ctxp, _dp, _dp, _dp]),
    "qgn_advance_resident": (C.c_int, [_ctxp, C.c_int]),
    "qgn_get_time": (C.c_int, [_ctxp, _dp, _dp]),
    "qgn_rhs": (C.c_int, [_ctxp, _dp, _dp]),
    "qgn_psi": (C.c_int, [_ctxp, _dp, _dp]),
    "qgn_leith": (C.c_int, [_ctxp, _dp]),
    "qgn_energetics": (C.c_int, [_ctxp, _dp, _dp, _dp]),
    "qgn_diagnostics": (C.c_int, [_ctxp, _dp, _dp, C.c_int]),
    "qgn_physical": (C.c_int, [_ctxp, _dp, _dp, _dp]),
    "qgn_set_state_physical": (C.c_int, [_ctxp, _dp, C.c_double, C.c_double]),
    "qgn_physical_modal": (C.c_int, [_ctxp, _dp, _dp, _dp, _dp]),
    "qgn_cnn_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_ulonglong,
                                 C.POINTER(C.c_void_p)]),
    "qgn_cnn_padded_channels": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "qgn_cnn_num_params": (C.c_longlong, [C.c_void_p]),
    "qgn_cnn_get_weights": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "qgn_cnn_set_weights": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "qgn_cnn_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "qgn_cnn_gradients": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_float),
                                    C.POINTER(C.c_double)]),
    "qgn_cnn_train_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float,
                                     C.POINTER(C.c_double)]),
    "qgn_cnn_set_engine": (C.c_int, [C.c_void_p, C.c_int]),
    "qgn_cnn_check": (C.c_int, [C.c_void_p]),
    "qgn_cnn_debug_set_counter": (C.c_int, [C.c_void_p, C.c_int, C.c_uint]),
    "qgn_cnn_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "qgn_cnn_last_error": (C.c_char_p, [C.c_void_p]),
    "qgn_cnn_destroy": (C.c_int, [C.c_void_p]),
    "qgn_coarse_grain": (C.c_int, [_ctxp, _ctxp]),
    "qgn_closure_snapshot": (C.c_int, [_ctxp, _ctxp, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_void_p,
                                       C.c_void_p, C.c_int, C.c_int]),
    "qgn_closure_attach": (C.c_int, [_ctxp, C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_double,
                                     C.c_double]),
    "qgn_closure_stats": (C.c_int, [_ctxp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), _dp]),
    "qgn_ens_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "qgn_ens_advance": (C.c_int, [C.c_void_p, C.c_int]),
    "qgn_ens_tuning": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                 C.POINTER(C.c_float)]),
    "qgn_ens_fft_radix": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    "qgn_ens_set_tiles": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]),
    "qgn_ens_profile_enable": (C.c_int, [C.c_void_p, C.c_int]),
    "qgn_ens_profile_read": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp, C.POINTER(C.c_longlong),
                                       C.POINTER(C.c_longlong)]),
    "qgn_ens_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "qgn_ens_last_error": (C.c_char_p, [C.c_void_p]),
    "qgn_ens_destroy": (C.c_int, [C.c_void_p]),
    "qgn_rejects": (C.c_int, [_ctxp, C.POINTER(C.c_longlong)]),
    "qgn_profile_enable": (C.c_int, [_ctxp, C.c_int]),
    "qgn_profile_read": (C.c_int, [_ctxp, C.c_int, _dp, _dp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "qgn_kernel_name": (C.c_char_p, [C.c_int]),
    "qgn_stream": (C.c_int, [_ctxp, C.POINTER(C.c_void_p)]),
    "qgn_debug_read": (C.c_int, [_ctxp, C.c_int, _dp, C.c_longlong]),
    "qgn_check_failures": (C.c_int, [_ctxp, C.POINTER(C.c_longlong)]),
    "qgn_probe_fp64_fma": (C.c_int, [C.c_int, _dp, _dp]),
    "qgn_rhs_static": (C.c_int, [C.POINTER(qgn_params), _dp, _dp, _dp, _dp, _dp, C.c_void_p, C.c_void_p,
                                 C.c_void_p]),
    "qgn_last_error": (C.c_char_p, [_ctxp]),
    "qgn_destroy": (C.c_int, [_ctxp]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load libqgn_b200.so; raises if it is missing (build it with qgn_fortran_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build the CUDA library first (python -m qgn_fortran_b200.build)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class QGNError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


def dptr(a):
    """double* of a contiguous numpy array (complex arrays as interleaved doubles)."""
    return a.ctypes.data_as(_dp)
