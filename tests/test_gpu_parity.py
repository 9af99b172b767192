"""GPU parity: the CUDA path (through the C-ABI) against the FP64 oracle.

Tolerances: per-layer relative L2 <= 1e-12 for one RHS, GetPsi and the transforms; fixed-dt
trajectories (ARK43 clipped at dt_max, RK4, AB3) <= 1e-11 after up to 100 steps.  The
adaptive schemes (ARK43_QGLeith, BSRK3) feed the embedded error estimate -- a difference of
stage values that cancels to ~1e-12 of the RHS -- through err^-0.175 into dt, which
amplifies last-bit differences by 1e3..1e7; they are compared from initial steps whose
error estimate is well above roundoff, with t, dt and the state to 1e-9 relative.
"""
import glob
import json
import math
import os

import numpy as np
import pytest

from oracle.qgn_oracle import Params, QGNOracle, SCHEMES
from qgn_fortran_b200 import QGNModule
from qgn_fortran_b200._lib import QGNError, QGN_ERR_NONFINITE, QGN_ERR_REJECT_LIMIT
from qgn_fortran_b200.inputs import exponential_stratification, phillips_two_layer, seeded_random_pv, workload

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
RHS_TOL = 1e-12
FIXED_TOL = 1e-11
ADAPT_TOL = 1e-9
ADAPTIVE = ("ark43_qgleith", "ark43", "bsrk3")


def adaptive(scheme, params):
    """ARK43 with TOL so large that the controller always clips to dt_max runs at fixed dt."""
    return scheme in ADAPTIVE and params["TOL"] < 1e20


def layer_rel(a, b):
    num = np.sqrt(np.sum(np.abs(a - b) ** 2, axis=(1, 2)))
    den = np.sqrt(np.sum(np.abs(b) ** 2, axis=(1, 2)))
    return num / np.where(den > 0, den, 1.0)


def pair(params: dict, H, S, U, scheme="ark43_qgleith", **kw):
    m = QGNOracle(Params(**params), H, S, U)
    g = QGNModule(params, H, S, U, scheme=scheme, **kw)
    return m, g


def strat_params(nx, ny, nz, **kw):
    p = dict(nx=nx, ny=ny, nz=nz, Lx=2.0e6, Ly=2.0e6 * ny / nx, Htot=4000.0, f0=1.0e-4, beta=2.0e-11,
             A2=0.0, A8=1.0e20, r0=1.0e-7, C_d=0.0, TOL=1.0e-12, is_explicit=False,
             dt_max=math.pi / (2.0e-11 * 2.0e6))
    p.update(kw)
    return p


def golden_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_case(path):
    d = np.load(path)
    meta = json.loads(str(d["meta"]))
    return d, meta


# ---------------------------------------------------------------------------------------
@pytest.mark.parametrize("path", golden_cases(), ids=lambda p: os.path.basename(p)[:-4])
def test_rhs_psi_leith_golden(cuda_ok, path):
    d, meta = load_case(path)
    g = QGNModule(meta["params"], d["H"], d["S"], d["U"], scheme=meta["scheme"])
    assert np.all(layer_rel(g.get_rhs(d["q0"]), d["rhs"]) <= RHS_TOL)
    assert np.all(layer_rel(g.get_psi(d["q0"]), d["psi"]) <= RHS_TOL)
    q0 = g.initialize(d["qp"])
    assert np.all(layer_rel(q0, d["q0"]) <= RHS_TOL)
    assert np.allclose(g.leith(), d["a8l"], rtol=1e-12, atol=0)


@pytest.mark.parametrize("path", golden_cases(), ids=lambda p: os.path.basename(p)[:-4])
def test_trajectory_golden(cuda_ok, path):
    d, meta = load_case(path)
    g = QGNModule(meta["params"], d["H"], d["S"], d["U"], scheme=meta["scheme"])
    q = np.ascontiguousarray(d["q0"]).copy()
    t, dt = 0.0, meta["dt0"]
    tol = ADAPT_TOL if adaptive(meta["scheme"], meta["params"]) else FIXED_TOL
    for k in range(meta["nsteps"]):
        t, dt = g.time_step(q, t, dt)
        assert t == pytest.approx(d["t"][k], rel=tol)
        assert dt == pytest.approx(d["dt"][k], rel=tol)
    assert np.all(layer_rel(q, d["qfinal"]) <= tol)
    assert g.rejects() == meta["rejects"]


@pytest.mark.parametrize("nx,ny,nz,drag,expl", [
    (16, 16, 2, False, False), (32, 64, 3, True, False), (64, 32, 2, True, True),
    (128, 128, 4, False, True), (256, 128, 5, True, False), (512, 512, 2, True, False),
    (64, 2048, 2, False, False), (2048, 64, 2, True, False), (128, 128, 16, False, False),
    (64, 64, 32, True, False), (64, 64, 7, False, False)])
def test_rhs_sizes(cuda_ok, nx, ny, nz, drag, expl):
    H, S, U = exponential_stratification(nz)
    params = strat_params(nx, ny, nz, C_d=1.0e-5 if drag else 0.0, is_explicit=expl, A2=3.0 if expl else 0.0)
    m, g = pair(params, H, S, U)
    q = m.initialize_spec(seeded_random_pv(nx, ny, nz, 6.0, 1.0e-6, seed=nx + 7 * ny + nz))
    assert np.all(layer_rel(g.get_rhs(q), m.get_rhs(q)) <= RHS_TOL)
    assert np.all(layer_rel(g.get_psi(q), m.get_psi(q)) <= RHS_TOL)


def test_rhs_strat1024x8(cuda_ok):
    """One RHS of the 1024^2 x 8 stratified workload against the oracle, per-layer L2 <= 1e-12."""
    w = workload("strat1024x8")
    m, g = pair(w.params, w.H, w.S, w.U)
    q = m.initialize_spec(w.qp)
    q_gpu = g.initialize(w.qp)
    assert np.all(layer_rel(q_gpu, q) <= RHS_TOL)
    assert np.all(layer_rel(g.get_rhs(q), m.get_rhs(q)) <= RHS_TOL)
    a8 = g.leith()
    assert np.allclose(a8, m.leith_A8L(q), rtol=1e-12, atol=0)


def test_physical_fields(cuda_ok):
    H, S, U = exponential_stratification(3)
    params = strat_params(64, 128, 3)
    m, g = pair(params, H, S, U)
    q = m.initialize_spec(seeded_random_pv(64, 128, 3, 6.0, 1.0e-6, seed=5))
    qp, pp = g.physical(q)
    assert np.allclose(qp, m.s2g_scaled(q), rtol=0, atol=1e-13 * np.abs(qp).max())
    assert np.allclose(pp, m.s2g_scaled(m.get_psi(q)), rtol=0, atol=1e-13 * np.abs(pp).max())
    g.set_state(q, 0.0, 100.0)
    ke, _ = g.diagnostics()
    assert np.allclose(ke, m.layer_ke(q), rtol=1e-11)


@pytest.mark.parametrize("nx,ny,nz", [(64, 64, 2), (64, 128, 3), (256, 128, 5), (128, 32, 8)])
def test_write_qp_modal(cuda_ok, tmp_path, nx, ny, nz):
    """WriteQPmodal's q_mode, p_mode and J_mode (full undealiased Jacobian) against the oracle."""
    H, S, U = exponential_stratification(nz)
    params = strat_params(nx, ny, nz)
    m, g = pair(params, H, S, U)
    q = m.initialize_spec(seeded_random_pv(nx, ny, nz, 6.0, 1.0e-6, seed=nx + ny + nz))
    want = m.write_qp_modal(q)
    got = g.write_qp_modal(q, 1, 17, directory=str(tmp_path))
    for a, b in zip(got, want):
        assert np.all(layer_rel(a, b) <= RHS_TOL)
    # the files hold the same fields; the resident-state form gives the same result
    back = np.fromfile(tmp_path / "J_mode.000000017.dat", dtype="<f8").reshape(g.physical_shape())
    assert np.array_equal(back, got[2])
    g.set_state(q, 0.0, 100.0)
    again = g.physical_modal()
    for a, b in zip(again, got):
        assert np.array_equal(a, b)
    # stepping afterwards is unaffected by the work buffers the call used
    q1 = q.copy()
    g.time_step(q1, 0.0, 100.0)
    m2, g2 = pair(params, H, S, U)
    q2 = q.copy()
    g2.time_step(q2, 0.0, 100.0)
    assert np.array_equal(q1, q2)


@pytest.mark.parametrize("scheme", ["ark43_qgleith", "ark43", "bsrk3", "rk4", "ab3"])
def test_schemes_short_run(cuda_ok, scheme):
    H, S, U = exponential_stratification(4)
    params = strat_params(128, 128, 4, C_d=1.0e-5, TOL=2.0e-12, is_explicit=scheme in ("bsrk3", "rk4", "ab3"))
    m, g = pair(params, H, S, U, scheme=scheme)
    q = m.initialize_spec(seeded_random_pv(128, 128, 4, 10.0, 1.0e-6, seed=21))
    qg = q.copy()
    st = SCHEMES[scheme](m)
    t = tg = 0.0
    dt = dtg = 20000.0 if adaptive(scheme, params) else 900.0
    tol = ADAPT_TOL if adaptive(scheme, params) else FIXED_TOL
    for _ in range(8):
        q, t, dt = st.step(q, t, dt)
        tg, dtg = g.time_step(qg, tg, dtg)
    assert tg == pytest.approx(t, rel=tol)
    assert dtg == pytest.approx(dt, rel=tol)
    assert np.all(layer_rel(qg, q) <= tol)


def test_hundred_fixed_steps(cuda_ok):
    """100 fixed-dt ARK43 steps (dt_max clip, huge TOL) of the 2-layer Phillips problem."""
    H, S, U = phillips_two_layer()
    n = 128
    A8 = 1.0 / (86400.0 * (math.pi * n / 1.0e6) ** 8)
    params = dict(nx=n, ny=n, nz=2, Lx=1.0e6, Ly=1.0e6, Htot=4000.0, f0=1.0e-4, beta=1.6e-11, A2=0.0, A8=A8,
                  r0=1.0e-7, C_d=0.0, TOL=1.0e30, is_explicit=False, dt_max=900.0)
    m, g = pair(params, H, S, U, scheme="ark43")
    q = m.initialize_spec(seeded_random_pv(n, n, 2, 10.0, 1.0e-6, seed=1))
    g.set_state(q, 0.0, 900.0)
    g.advance_resident(100)
    qg = g.get_state()
    st = SCHEMES["ark43"](m)
    t, dt = 0.0, 900.0
    for _ in range(100):
        q, t, dt = st.step(q, t, dt)
    assert g.t == pytest.approx(t, rel=1e-14)
    assert np.all(layer_rel(qg, q) <= FIXED_TOL)


def test_resident_equals_step_api(cuda_ok):
    w = workload("strat1024x8", nx=128, nz=4)
    g1 = QGNModule(w.params, w.H, w.S, w.U, scheme="ark43_qgleith")
    g2 = QGNModule(w.params, w.H, w.S, w.U, scheme="ark43_qgleith")
    q = g1.initialize(w.qp, 0.0, 750.0)
    q1 = q.copy()
    t, dt = 0.0, 750.0
    for _ in range(4):
        t, dt = g1.time_step(q1, t, dt)
    g2.set_state(q, 0.0, 750.0)
    g2.advance_resident(4)
    q2 = g2.get_state()
    assert np.array_equal(q1, q2)
    assert (g2.t, g2.dt) == (t, dt)


def test_reject_limit_is_reported(cuda_ok):
    H, S, U = exponential_stratification(2)
    params = strat_params(32, 32, 2, TOL=0.0)
    g = QGNModule(params, H, S, U, scheme="ark43_qgleith", max_rejects=3)
    q = g.initialize(seeded_random_pv(32, 32, 2, 4.0, 1.0e-6, seed=3), 0.0, 500.0)
    with pytest.raises(QGNError) as ei:
        g.time_step(q, 0.0, 500.0)
    assert ei.value.code == QGN_ERR_REJECT_LIMIT
    assert g.rejects() == 3
    # the context stays usable after the failure
    assert np.isfinite(g.get_rhs(q)).all()


def test_nonfinite_input_is_reported(cuda_ok):
    H, S, U = exponential_stratification(2)
    params = strat_params(32, 32, 2)
    for scheme in ("ark43_qgleith", "rk4"):
        g = QGNModule(params, H, S, U, scheme=scheme)
        q = g.initialize(seeded_random_pv(32, 32, 2, 4.0, 1.0e-6, seed=3), 0.0, 500.0)
        q[1, 3, 2] = np.nan
        with pytest.raises(QGNError) as ei:
            g.time_step(q, 0.0, 500.0)
        assert ei.value.code == QGN_ERR_NONFINITE


def test_step_output_modes(cuda_ok):
    """qgn_step writes back the kept modes by default (TimeStep's trailing DeAlias,
    QGN_Module.f90:307, zeroes the rest on the host); QGN_OUTPUT_FULL writes zeros there."""
    w = workload("strat1024x8", nx=64, nz=3)
    g1 = QGNModule(w.params, w.H, w.S, w.U, scheme="ark43_qgleith")
    g2 = QGNModule(w.params, w.H, w.S, w.U, scheme="ark43_qgleith")
    q = g1.initialize(w.qp, 0.0, 5000.0)
    band = np.zeros(q.shape, dtype=bool)
    ny, nx = 64, 64
    band[:, ny // 3:2 * (ny // 3) + 1, :] = True
    band[:, :, nx // 3:] = True
    assert np.all(q[band] == 0)
    qa, qb = q.copy(), q.copy()
    marker = complex(3.0, -7.0)
    qa[band] = marker
    qb[band] = marker
    ta = g1.time_step(qa, 0.0, 5000.0)
    g2.set_output("full")
    tb = g2.time_step(qb, 0.0, 5000.0)
    assert ta == tb
    assert np.all(qa[band] == marker)          # kept mode: the band is not written
    assert np.all(qb[band] == 0)               # full mode: zeros, as after DeAlias
    assert np.array_equal(qa[~band], qb[~band])


@pytest.mark.parametrize("nx,ny,nz", [(64, 128, 3), (256, 256, 8), (128, 64, 2)])
def test_energetics_and_spectrum(cuda_ok, nx, ny, nz):
    """Layer KE, APE, enstrophy and the isotropic KE spectrum of the resident state against the
    oracle's physical-space forms (per-layer 1e-12; spectrum per-layer relative L2 1e-12)."""
    H, S, U = exponential_stratification(nz)
    params = strat_params(nx, ny, nz)
    m, g = pair(params, H, S, U)
    q = m.initialize_spec(seeded_random_pv(nx, ny, nz, 6.0, 1.0e-6, seed=3 * nx + nz))
    g.set_state(q, 0.0, 100.0)
    ke, ape, Z = g.energetics()
    assert np.allclose(ke, m.layer_ke(q), rtol=RHS_TOL, atol=0)
    want_ape = m.layer_ape(q)
    assert np.allclose(ape, want_ape, rtol=0, atol=RHS_TOL * np.abs(want_ape).max())
    assert np.allclose(Z, m.layer_enstrophy(q), rtol=RHS_TOL, atol=0)
    nbins = max(nx, ny) // 2
    ke2, spec = g.diagnostics(nbins)
    assert np.allclose(ke2, ke, rtol=1e-13, atol=0)     # two reductions in different orders
    want = m.ke_spectrum(q, nbins)
    num = np.sqrt(np.sum((spec - want) ** 2, axis=1))
    assert np.all(num <= RHS_TOL * np.sqrt(np.sum(want ** 2, axis=1)))
