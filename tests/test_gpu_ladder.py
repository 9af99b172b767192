"""GPU parity ladder on the named workloads, against the C/OpenMP FP64 restatement of the reference
(oracle/qgn_ref.c, itself checked against the numpy oracle in tests/test_oracle_c.py).

Rungs (per-layer relative L2 of the spectral state unless stated):
  * one RHS of the 2048^2 x 16 stratified workload                         <= 1e-12
  * 100 fixed-dt ARK43_QGLeith steps of the 1024^2 x 8 stratified workload  <= 1e-12
    (TOL = 1e30, so the PI.3.4 controller always clips dt to dt_max = 7200 s,
    ARK43_QGLeith.f90:135-138; QG-Leith coefficient recomputed every step)
  * 1000 steps of the 2-layer Phillips problem on 256^2 (ARK43, dt = 900 s)  <= 1e-12
Both sides of every rung start from the same seeded initial condition, transformed by each side.
"""
import math

import numpy as np
import pytest

from oracle.qgn_oracle import Params
from oracle.qgn_ref_c import RefC
from qgn_fortran_b200 import QGNModule
from qgn_fortran_b200.inputs import workload

pytestmark = pytest.mark.gpu

TOL = 1e-12


def layer_rel(a, b):
    num = np.sqrt(np.sum(np.abs(a - b) ** 2, axis=(1, 2)))
    den = np.sqrt(np.sum(np.abs(b) ** 2, axis=(1, 2)))
    return num / np.where(den > 0, den, 1.0)


def test_rhs_strat2048x16(cuda_ok):
    """One GetRHS (QGN_Module.f90:258-296) of the 2048^2 x 16 workload."""
    w = workload("strat2048x16")
    c = RefC(Params(**w.params), w.H, w.S, w.U, scheme=w.scheme)
    g = QGNModule(w.params, w.H, w.S, w.U, scheme=w.scheme)
    q = c.initialize_spec(w.qp)
    qg = g.initialize(w.qp)
    assert np.all(layer_rel(qg, q) <= TOL)
    err = layer_rel(g.get_rhs(q), c.get_rhs(q))
    print(f"strat2048x16 one RHS: max per-layer rel L2 {err.max():.3e}")
    assert np.all(err <= TOL)
    g.cleanup()


def test_hundred_fixed_steps_strat1024x8(cuda_ok):
    """100 ARK43_QGLeith steps at fixed dt (ARK43_QGLeith.f90:75-140) on 1024^2 x 8."""
    w = workload("strat1024x8")
    dt_max = 7200.0
    p = dict(w.params, TOL=1.0e30, dt_max=dt_max)
    c = RefC(Params(**p), w.H, w.S, w.U, scheme="ark43_qgleith")
    g = QGNModule(p, w.H, w.S, w.U, scheme="ark43_qgleith")
    q = c.initialize_spec(w.qp)
    g.initialize(w.qp, 0.0, dt_max)
    g.advance_resident(100)
    qg = g.get_state()
    t, dt = 0.0, dt_max
    for _ in range(100):
        t, dt = c.step(q, t, dt)
    assert g.t == pytest.approx(t, rel=1e-14) and g.dt == dt
    err = layer_rel(qg, q)
    print(f"strat1024x8 100 fixed steps: max per-layer rel L2 {err.max():.3e}")
    assert np.all(err <= TOL)
    g.cleanup()


def test_phillips256_thousand_steps(cuda_ok):
    """The 2-layer Phillips problem on 256^2, ARK43 (fixed A8, ARK43.f90:61-125) at dt = 900 s
    (dt_max = 900 with TOL = 1e30), 1000 steps through the drop-in TimeStep."""
    w = workload("phillips256")
    c = RefC(Params(**w.params), w.H, w.S, w.U, scheme="ark43")
    g = QGNModule(w.params, w.H, w.S, w.U, scheme="ark43")
    q = c.initialize_spec(w.qp)
    qg = g.initialize(w.qp, 0.0, 900.0)
    qg = qg.copy()
    t, dt = 0.0, 900.0
    tg, dtg = g.advance(qg, 0.0, 900.0, 1000)
    for _ in range(1000):
        t, dt = c.step(q, t, dt)
    assert tg == pytest.approx(t, rel=1e-14) and dtg == dt == 900.0
    err = layer_rel(qg, q)
    print(f"phillips256 1000 steps: max per-layer rel L2 {err.max():.3e}")
    assert np.all(err <= TOL)
    g.cleanup()
