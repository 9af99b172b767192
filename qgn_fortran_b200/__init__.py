"""B200-native (sm_100a) QGN pseudo-spectral right-hand side and time steppers.

Drop-in for the TimeStep path of iangrooms/QGN_Fortran behind the C-ABI in
``include/qgn_gpu.h`` (``libqgn_b200.so``).  ``QGNModule`` mirrors the reference's
``QGN_Module`` public API from Python.
"""
from .model import QGNEnsemble, QGNModule, full_params, host_initialize  # noqa: F401
from . import inputs  # noqa: F401

__all__ = ["QGNEnsemble", "QGNModule", "full_params", "host_initialize", "inputs"]
