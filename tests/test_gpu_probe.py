"""FP64 FMA throughput probe (include/qgn_probe.h): the denominator of the transforms' FLOP fraction."""
import ctypes

import pytest

from qgn_fortran_b200 import _lib

pytestmark = pytest.mark.gpu


def test_fp64_fma_probe_measures_a_plausible_peak(cuda_ok):
    lib = _lib.load()
    tf, ms = ctypes.c_double(), ctypes.c_double()
    assert lib.qgn_probe_fp64_fma(3, ctypes.byref(tf), ctypes.byref(ms)) == _lib.QGN_OK
    print(f"FP64 FMA probe: {tf.value:.2f} TFLOP/s, {ms.value:.3f} ms per launch")
    # a B200 issues 64 FP64 FMAs per SM per clock: ~37 TFLOP/s at 1.965 GHz on 148 SMs; the
    # bounds only reject a probe that does not measure FMA throughput at all
    assert 10.0 < tf.value < 80.0
    assert ms.value > 0.1
