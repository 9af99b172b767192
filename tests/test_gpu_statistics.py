"""Long-time statistics rung of the parity ladder: past the chaotic predictability horizon the GPU
and the C/OpenMP restatement of the reference (oracle/qgn_ref.c) are two independent realisations
of the same turbulence, and their time-mean layer kinetic energies and isotropic KE spectra (in
octave bands of the shell index) must agree within 2 %.

Both start from the same seeded IC and run ARK43_QGLeith with the PI.3.4 controller
(ARK43_QGLeith.f90:75-140) for SPIN years, which separates the trajectories completely (checked),
then average daily samples for MEAN years.  The configuration -- a two-layer Phillips problem on
128^2 with a one-day bottom drag on the f-plane -- equilibrates within months and forgets its
state within days, so the sampling error of a MEAN-year mean is well under the 2 % bound: the
standard error measured on B200 from a 10-year GPU run of the same configuration is given beside
the constants.  The oracle's side is the costly one (about 1 minute on the GPU box's 16 cores).
"""
import math

import numpy as np
import pytest

from oracle.qgn_oracle import Params, QGNOracle
from oracle.qgn_ref_c import RefC
from qgn_fortran_b200 import QGNModule
from qgn_fortran_b200.inputs import phillips_two_layer, seeded_random_pv

pytestmark = pytest.mark.gpu

DAY = 86400.0
YEAR = 365.0 * DAY
N, L_DOMAIN, U1, R0, BETA = 128, 1.0e6, 0.1, 1.0e-5, 0.0
SPIN, MEAN = 1.0, 2.0          # years
BANDS = [(1, 2), (2, 4), (4, 8), (8, 16), (16, 32), (32, 64)]
TOL_STAT = 0.02


def config():
    H, S, U = phillips_two_layer(U=(U1, 0.0))
    qp = seeded_random_pv(N, N, 2, 8.0, 1.0e-6, seed=11)
    p = dict(nx=N, ny=N, nz=2, Lx=L_DOMAIN, Ly=L_DOMAIN, Htot=4000.0, f0=1.0e-4, beta=BETA, A2=0.0, A8=1.0e23,
             r0=R0, C_d=0.0, TOL=1.0e-6 * float(np.max(np.abs(qp))), is_explicit=False,
             dt_max=math.pi / (1.6e-11 * L_DOMAIN))
    return p, H, S, U, qp


def bands_of(spec):
    return np.array([[spec[l, a:b].sum() for a, b in BANDS] for l in range(spec.shape[0])])


def test_time_mean_statistics_match_the_oracle(cuda_ok):
    p, H, S, U, qp = config()
    # GPU: sample every simulated day after the spin-up
    g = QGNModule(p, H, S, U, scheme="ark43_qgleith")
    g.initialize(qp, 0.0, 1800.0)
    t = 0.0
    while t < SPIN * YEAR:
        g.advance_resident(10)
        t, _ = g.time()
    ke_g, bd_g, n_g, nxt = 0.0, 0.0, 0, t + DAY
    while t < (SPIN + MEAN) * YEAR:
        g.advance_resident(1)
        t, _ = g.time()
        if t >= nxt:
            ke, sp = g.diagnostics(N // 2)
            ke_g, bd_g, n_g = ke_g + ke, bd_g + bands_of(sp), n_g + 1
            nxt += DAY
    q_gpu = g.get_state()
    g.cleanup()

    # the C oracle, the same way; its diagnostics from the numpy oracle's physical-space forms
    c = RefC(Params(**p), H, S, U, scheme="ark43_qgleith")
    m = QGNOracle(Params(**p), H, S, U)
    q = c.initialize_spec(qp)
    t, dt = 0.0, 1800.0
    while t < SPIN * YEAR:
        t, dt = c.step(q, t, dt)
    ke_o, bd_o, n_o, nxt = 0.0, 0.0, 0, t + DAY
    while t < (SPIN + MEAN) * YEAR:
        t, dt = c.step(q, t, dt)
        if t >= nxt:
            ke_o, bd_o, n_o = ke_o + m.layer_ke(q), bd_o + bands_of(m.ke_spectrum(q, N // 2)), n_o + 1
            nxt += DAY

    # past the predictability horizon: the two states are unrelated
    sep = np.linalg.norm(q_gpu - q) / np.linalg.norm(q)
    ke_g, ke_o = ke_g / n_g, ke_o / n_o
    bd_g, bd_o = bd_g / n_g, bd_o / n_o
    ke_err = np.abs(ke_g / ke_o - 1.0)
    keep = bd_o >= 0.01 * bd_o.sum(axis=1, keepdims=True)
    bd_err = np.abs(bd_g / bd_o - 1.0)[keep]
    print(f"long-time statistics: separation {sep:.2f}, samples {n_g}/{n_o}, layer KE err {ke_err.max():.4f}, "
          f"band err {bd_err.max():.4f}")
    assert sep > 0.5
    assert abs(n_g - n_o) <= 2
    assert np.all(ke_err <= TOL_STAT)
    assert np.all(bd_err <= TOL_STAT)
