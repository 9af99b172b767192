"""Mixed precision (QGN_PREC_MIXED): FP32 transforms, Jacobian, RHS and stage storage with
compensated FP32 stage sums; FP64 state, GetPsi, error norm, PI controller and Leith.

Stated error bounds against FP64 (the oracle for one RHS; the FP64 GPU path for trajectories):
one RHS per-layer relative L2 <= 2e-6; 20 fixed-dt ARK43 / ARK43_QGLeith steps: state <= 1e-5.
Adaptive runs are compared by their simulated time only: the FP32 noise in the stage values
raises the floor of the embedded error estimate, so the controller legitimately picks
different dt and the states are at different times.
"""
import math

import numpy as np
import pytest

from oracle.qgn_oracle import Params, QGNOracle
from qgn_fortran_b200 import QGNModule
from qgn_fortran_b200.inputs import exponential_stratification, seeded_random_pv, workload

pytestmark = pytest.mark.gpu


def layer_rel(a, b):
    num = np.sqrt(np.sum(np.abs(a - b) ** 2, axis=(1, 2)))
    den = np.sqrt(np.sum(np.abs(b) ** 2, axis=(1, 2)))
    return num / np.where(den > 0, den, 1.0)


@pytest.mark.parametrize("nx,nz,drag", [(64, 4, False), (128, 3, True), (256, 8, False)])
def test_mixed_rhs_against_oracle(cuda_ok, nx, nz, drag):
    H, S, U = exponential_stratification(nz)
    params = dict(nx=nx, ny=nx, nz=nz, Lx=2.0e6, Ly=2.0e6, Htot=4000.0, beta=2.0e-11, A8=1.0e20,
                  r0=1.0e-7, C_d=1.0e-5 if drag else 0.0, TOL=1.0e-12, dt_max=math.pi / (2.0e-11 * 2.0e6))
    m = QGNOracle(Params(**params), H, S, U)
    g = QGNModule(params, H, S, U, precision="mixed")
    q = m.initialize_spec(seeded_random_pv(nx, nx, nz, 8.0, 1.0e-6, seed=nx + nz))
    err = layer_rel(g.get_rhs(q), m.get_rhs(q))
    assert np.all(err <= 2e-6), err


@pytest.mark.parametrize("scheme", ["ark43_qgleith", "ark43"])
def test_mixed_fixed_dt_trajectory_against_fp64(cuda_ok, scheme):
    w = workload("strat1024x8", nx=256, nz=4)
    p = dict(w.params)
    p.update(TOL=1.0e30, dt_max=2000.0, A8=1.0e20)      # the controller clips to dt_max: fixed dt
    g64 = QGNModule(p, w.H, w.S, w.U, scheme=scheme, precision="fp64")
    g32 = QGNModule(p, w.H, w.S, w.U, scheme=scheme, precision="mixed")
    g64.initialize(w.qp, 0.0, 2000.0)
    g32.initialize(w.qp, 0.0, 2000.0)
    g64.advance_resident(20)
    g32.advance_resident(20)
    a, b = g32.get_state(), g64.get_state()
    assert g32.t == g64.t
    assert np.all(layer_rel(a, b) <= 1e-5), layer_rel(a, b)


def test_mixed_adaptive_run_tracks_fp64_time(cuda_ok):
    w = workload("strat1024x8", nx=256, nz=4)
    g64 = QGNModule(w.params, w.H, w.S, w.U, precision="fp64")
    g32 = QGNModule(w.params, w.H, w.S, w.U, precision="mixed")
    for g in (g64, g32):
        g.initialize(w.qp, 0.0, 750.0)
        g.advance_resident(30)
    assert np.all(np.isfinite(g32.get_state()))
    t32, _ = g32.time()
    t64, _ = g64.time()
    assert t32 == pytest.approx(t64, rel=0.25)


def test_mixed_graph_equals_eager(cuda_ok, monkeypatch):
    w = workload("strat1024x8", nx=128, nz=4)
    ga = QGNModule(w.params, w.H, w.S, w.U, precision="mixed")
    gb = QGNModule(w.params, w.H, w.S, w.U, precision="mixed")
    q = ga.initialize(w.qp, 0.0, 20000.0)
    gb.set_state(q, 0.0, 20000.0)
    ga.advance_resident(6)                # first step eager, then graphs
    q1 = q.copy()
    t, dt = 0.0, 20000.0
    for _ in range(6):                    # one qgn_step per call: eager first call, graphs later
        t, dt = gb.time_step(q1, t, dt)
    assert np.array_equal(ga.get_state(), gb.get_state())
    assert (ga.t, ga.dt) == (gb.t, gb.dt)


def test_mixed_rejected_for_other_schemes(cuda_ok):
    from qgn_fortran_b200._lib import QGNError, QGN_ERR_CONFIG
    w = workload("strat1024x8", nx=64, nz=2, with_ic=False)
    with pytest.raises(QGNError) as ei:
        QGNModule(w.params, w.H, w.S, w.U, scheme="rk4", precision="mixed")
    assert ei.value.code == QGN_ERR_CONFIG


def test_mixed_error_table_strat2048x16(cuda_ok):
    """The 2048^2 x 16 workload in the mixed mode against FP64 (both on the GPU, FP64 checked
    against the oracle in tests/test_gpu_ladder.py): one RHS, 100 fixed-dt ARK43_QGLeith steps
    (dt = 3600 s), layer KE and the isotropic KE spectrum of the final states."""
    from qgn_fortran_b200.mixed_error import error_table
    t = error_table("strat2048x16", steps=100, dt=3600.0)
    print("strat2048x16 mixed vs FP64:", t)
    # measured on B200: rhs 4.3e-6, state 1.9e-7, layer KE 8.0e-9, spectrum 7.7e-7
    assert t["rhs"] <= 1e-5
    assert t["fixed_steps"]["state"] <= 1e-6
    assert t["fixed_steps"]["ke_layer"] <= 1e-7
    assert t["fixed_steps"]["ke_spectrum"] <= 1e-5
