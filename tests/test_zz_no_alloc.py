"""qgn_rhs_static: the GetRHS entry point that allocates no device memory.

Some hosts cannot call cudaMalloc where they evaluate the model: a component inside a
larger application that owns every device array (an OpenACC or OpenMP-offload data
region, or a memory pool carved up at start-up), or a time loop that must not take
cudaMalloc's implicit synchronisation.  For them qgn_rhs_static keeps its intermediates
in a fixed device array inside the library.  This test calls it through the C-ABI with
device arrays the caller owns and checks two calls in a row against the allocating entry
point qgn_rhs, at the RHS tolerance of the parity suite (per-layer relative L2 <= 1e-12).
The file sorts last so that a run stopping at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from qgn_fortran_b200 import QGNModule, _lib
from qgn_fortran_b200.inputs import exponential_stratification, seeded_random_pv

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-12


def layer_rel(a, b):
    num = np.sqrt(np.sum(np.abs(a - b) ** 2, axis=(1, 2)))
    den = np.sqrt(np.sum(np.abs(b) ** 2, axis=(1, 2)))
    return num / np.where(den > 0, den, 1.0)


def call_static(g, q_dev, out_dev, stream):
    H = np.ascontiguousarray(g.H)
    modes = np.asfortranarray(g.Modes)
    return g.lib.qgn_rhs_static(C.byref(g._cp), _lib.dptr(H), _lib.dptr(np.ascontiguousarray(g.uBar)),
                                _lib.dptr(np.ascontiguousarray(g.qyBar)),
                                modes.ctypes.data_as(C.POINTER(C.c_double)),
                                _lib.dptr(np.ascontiguousarray(g.EVals)),
                                C.c_void_p(q_dev.data_ptr()), C.c_void_p(out_dev.data_ptr()), C.c_void_p(stream))


def test_rhs_static_matches_allocating_entry_point(cuda_ok):
    import torch

    nx, ny, nz = 128, 256, 4
    H, S, U = exponential_stratification(nz)
    params = dict(nx=nx, ny=ny, nz=nz, Lx=2.0e6, Ly=4.0e6, Htot=4000.0, beta=2.0e-11, A2=2.0, A8=1.0e20,
                  r0=1.0e-7, C_d=1.0e-5, TOL=1.0e-12, is_explicit=True)
    g = QGNModule(params, H, S, U, scheme="ark43_qgleith")
    stream = torch.cuda.current_stream().cuda_stream
    # a call on another geometry first: it leaves data at other offsets of the shared array
    # (padding columns included), which the calls below must not pick up
    H8, S8, U8 = exponential_stratification(8)
    p8 = dict(params, nx=256, ny=256, nz=8, Ly=2.0e6, C_d=0.0)
    g8 = QGNModule(p8, H8, S8, U8, scheme="ark43_qgleith")
    q8 = g8.initialize(seeded_random_pv(256, 256, 8, 8.0, 1.0e-6, seed=5))
    q8_dev = torch.from_numpy(q8).to("cuda")
    out8_dev = torch.empty_like(q8_dev)
    assert call_static(g8, q8_dev, out8_dev, stream) == _lib.QGN_OK
    torch.cuda.synchronize()
    assert np.all(layer_rel(out8_dev.cpu().numpy(), g8.get_rhs(q8)) <= RHS_TOL)
    for seed in (11, 12):     # two calls in a row: the second must not see the first's scratch
        q = g.initialize(seeded_random_pv(nx, ny, nz, 8.0, 1.0e-6, seed=seed))
        ref = g.get_rhs(q)
        q_dev = torch.from_numpy(q).to("cuda")
        out_dev = torch.full_like(q_dev, complex(np.nan, np.nan))
        rc = call_static(g, q_dev, out_dev, stream)
        assert rc == _lib.QGN_OK
        torch.cuda.synchronize()
        out = out_dev.cpu().numpy()
        assert np.all(np.isfinite(out))
        assert np.all(layer_rel(out, ref) <= RHS_TOL)


def test_rhs_static_rejects_grids_beyond_the_scratch(cuda_ok):
    import torch

    nz = 8
    H, S, U = exponential_stratification(nz)
    params = dict(nx=1024, ny=1024, nz=nz, Lx=2.0e6, Ly=2.0e6, Htot=4000.0)
    g = QGNModule(params, H, S, U)
    q_dev = torch.zeros((nz, 1024, 513), dtype=torch.complex128, device="cuda")
    out_dev = torch.empty_like(q_dev)
    rc = call_static(g, q_dev, out_dev, torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.QGN_ERR_TOO_LARGE


def test_rhs_static_refuses_stream_capture(cuda_ok):
    """The constants are copied from the call's stack, so a capture is refused, not recorded."""
    import torch

    nz = 2
    H, S, U = exponential_stratification(nz)
    params = dict(nx=64, ny=64, nz=nz, Lx=2.0e6, Ly=2.0e6, Htot=4000.0)
    g = QGNModule(params, H, S, U)
    q_dev = torch.zeros((nz, 64, 33), dtype=torch.complex128, device="cuda")
    out_dev = torch.empty_like(q_dev)
    s = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s, capture_error_mode="thread_local"):
        rc = call_static(g, q_dev, out_dev, s.cuda_stream)
        out_dev.zero_()     # one captured node, so the graph is not empty
    assert rc == _lib.QGN_ERR_CONFIG


def test_rhs_static_on_a_second_device(cuda_ok):
    """The scratch array's device address and the kernels' shared-memory opt-in are per device:
    after calls on device 0, calls on device 1 (qgn_rhs_static, then a context there) must give
    the same right-hand side.  Needs two GPUs."""
    import torch

    if torch.cuda.device_count() < 2:
        pytest.skip("one visible GPU")
    nx, ny, nz = 128, 256, 4
    H, S, U = exponential_stratification(nz)
    params = dict(nx=nx, ny=ny, nz=nz, Lx=2.0e6, Ly=4.0e6, Htot=4000.0, beta=2.0e-11, A8=1.0e20, r0=1.0e-7,
                  TOL=1.0e-12)
    outs = []
    for dev in (0, 1):
        with torch.cuda.device(dev):
            g = QGNModule(params, H, S, U, scheme="ark43_qgleith")
            q = g.initialize(seeded_random_pv(nx, ny, nz, 8.0, 1.0e-6, seed=31))
            q_dev = torch.from_numpy(q).to(f"cuda:{dev}")
            out_dev = torch.empty_like(q_dev)
            assert call_static(g, q_dev, out_dev, torch.cuda.current_stream(dev).cuda_stream) == _lib.QGN_OK
            torch.cuda.synchronize(dev)
            out = out_dev.cpu().numpy()
            assert np.all(layer_rel(out, g.get_rhs(q)) <= RHS_TOL)
            outs.append(out)
            g.cleanup()
    assert np.all(layer_rel(outs[1], outs[0]) <= RHS_TOL)
