"""Known-answer tests that pin the FP64 oracle (oracle/qgn_oracle.py).

The reference ships no tests or golden data and cannot be built here (Fortran + MKL), so
the oracle is pinned by mathematics: the FFT conventions against a direct DFT, the
dealias index rule, modal orthonormality and the inversion identity, the exact ARK
tableau identities, linear Rossby/Phillips solutions, inviscid conservation and the
order of accuracy.  The committed golden fixtures are re-derived from the oracle.
"""
import glob
import json
import math
import os
from fractions import Fraction

import numpy as np
import pytest

from oracle.qgn_oracle import (ARK43, RK4, LEITH_13, Params, QGNOracle, SCHEMES, ark43_tableau,
                               dealias_mask)
from qgn_fortran_b200.inputs import exponential_stratification, phillips_two_layer, seeded_random_pv

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def small_model(nx=32, ny=32, nz=3, **kw):
    H, S, U = exponential_stratification(nz)
    p = Params(nx=nx, ny=ny, nz=nz, Lx=1.0e6, Ly=1.0e6, Htot=4000.0, **kw)
    return QGNOracle(p, H, S, U)


# ---------------------------------------------------------------------------------------
# FFT conventions (MKL_DFTI_Setup.f90): unnormalised r2c, c2r with Re of the kx=0 entry
# ---------------------------------------------------------------------------------------
def direct_c2r(spec, nx, ny):
    """Direct y-then-x c2r of a CCE array: complex inverse DFT along y, then a real
    inverse along x that uses Re of the kx=0 (and Nyquist) entries."""
    nxh = nx // 2 + 1
    j = np.arange(ny)
    Ey = np.exp(2j * np.pi * np.outer(j, j) / ny)          # [y, ky]
    half = Ey @ spec                                       # [y, kx]
    x = np.arange(nx)
    out = np.zeros((ny, nx))
    for k in range(nxh):
        c = half[:, k]
        if k == 0 or (nx % 2 == 0 and k == nx // 2):
            out += np.real(c)[:, None] * np.cos(2 * np.pi * k * x / nx)[None, :]
        else:
            ph = np.exp(2j * np.pi * k * x / nx)
            out += 2.0 * np.real(c[:, None] * ph[None, :])
    return out


def test_fft_against_direct_dft():
    rng = np.random.default_rng(0)
    nx, ny = 8, 12
    m = small_model(nx=16, ny=16, nz=2)
    g = rng.standard_normal((2, ny, nx))
    spec = m.g2s(g)
    x = np.arange(nx)
    y = np.arange(ny)
    E = np.exp(-2j * np.pi * np.outer(y, y) / ny)
    F = np.exp(-2j * np.pi * np.outer(x, np.arange(nx // 2 + 1)) / nx)
    direct = np.einsum("ab,zbc,cd->zad", E, g, F)
    assert np.allclose(spec, direct, rtol=0, atol=1e-12)
    # non-Hermitian kx=0 column: c2r is the Hermitian projection (y first, Re at kx=0)
    spec2 = spec.copy()
    spec2[:, 3, 0] += 0.7 + 0.2j
    back = np.fft.irfft2(spec2, s=(ny, nx), axes=(-2, -1)) * (nx * ny)
    for z in range(2):
        assert np.allclose(back[z], direct_c2r(spec2[z], nx, ny), rtol=0, atol=1e-10)


def test_round_trip():
    m = small_model(nx=64, ny=32, nz=2)
    g = np.random.default_rng(1).standard_normal((2, 32, 64))
    assert np.allclose(m.s2g_scaled(m.g2s(g)), g, atol=1e-13)


# ---------------------------------------------------------------------------------------
# DeAlias (QGN_Module.f90:194-204)
# ---------------------------------------------------------------------------------------
@pytest.mark.parametrize("n,lo,hi", [(128, -43, 41), (256, -85, 84), (512, -171, 169),
                                     (1024, -341, 340), (2048, -683, 681), (384, -127, 127)])
def test_dealias_ky_ranges(n, lo, hi):
    keep = dealias_mask(n, n)
    j = np.arange(n)
    jj = np.where(j <= n // 2, j, j - n)
    kept = jj[keep[:, 1]]
    assert kept.min() == lo and kept.max() == hi
    assert keep[:, : n // 3].any() and not keep[:, n // 3:].any()
    assert not keep[0, 0]


def test_dealias_idempotent_and_index_rule():
    m = small_model(nx=48, ny=30, nz=2)
    f = np.random.default_rng(2).standard_normal((2, 30, 25)) + 1j
    d = m.dealias(f)
    assert np.array_equal(m.dealias(d), d)
    for i in range(25):
        for j in range(30):
            zero = (i >= 48 // 3) or (30 // 3 <= j <= 2 * (30 // 3)) or (i == 0 and j == 0)
            assert (np.all(d[:, j, i] == 0)) == zero or np.all(f[:, j, i] == 0)


# ---------------------------------------------------------------------------------------
# Vertical modes (QGN_Module.f90:102-141) and GetPsi (QGN_Module.f90:315-341)
# ---------------------------------------------------------------------------------------
@pytest.mark.parametrize("nz", [2, 3, 8, 16])
def test_modes_orthonormal(nz):
    m = small_model(nz=nz)
    G = (m.Modes.T * m.H) @ m.Modes / m.p.Htot
    assert np.allclose(G, np.eye(nz), atol=1e-10)
    assert np.all(m.Modes[0] > 0)
    assert np.max(m.EVals) == pytest.approx(0.0, abs=1e-12 * np.max(np.abs(m.EVals)))
    assert np.allclose(m.L @ m.Modes, m.Modes * m.EVals[None, :], atol=1e-12 * np.abs(m.L).max())


def test_getpsi_inverts_stretching():
    m = small_model(nz=4)
    rng = np.random.default_rng(3)
    q = m.dealias(rng.standard_normal((4, 32, 17)) + 1j * rng.standard_normal((4, 32, 17)))
    psi = m.get_psi(q)
    lhs = -m.k2[None] * psi + np.einsum("ab,byx->ayx", m.L, psi)
    mask = m.keep
    assert np.allclose(lhs[:, mask], q[:, mask], rtol=1e-10, atol=1e-12 * np.abs(q).max())


# ---------------------------------------------------------------------------------------
# ARK4(3)6L[2]SA tableau (ARK43_QGLeith.f90:15-58) in exact rationals
# ---------------------------------------------------------------------------------------
def test_tableau_identities():
    F = Fraction
    ae = {(2, 1): F(1, 2), (3, 1): F(13861, 62500), (3, 2): F(6889, 62500),
          (4, 1): F(-116923316275, 2393684061468), (4, 2): F(-2731218467317, 15368042101831),
          (4, 3): F(9408046702089, 11113171139209),
          (5, 1): F(-451086348788, 2902428689909), (5, 2): F(-2682348792572, 7519795681897),
          (5, 3): F(12662868775082, 11960479115383), (5, 4): F(3355817975965, 11060851509271),
          (6, 1): F(647845179188, 3216320057751), (6, 2): F(73281519250, 8382639484533),
          (6, 3): F(552539513391, 3454668386233), (6, 4): F(3354512671639, 8306763924573),
          (6, 5): F(4040, 17871)}
    b = [F(82889, 524892), F(0), F(15625, 83664), F(69875, 102672), F(-2260, 8211), F(1, 4)]
    ai = {(2, 1): F(1, 4), (3, 1): F(8611, 62500), (3, 2): F(-1743, 31250),
          (4, 1): F(5012029, 34652500), (4, 2): F(-654441, 2922500), (4, 3): F(174375, 388108),
          (5, 1): F(15267082809, 155376265600), (5, 2): F(-71443401, 120774400),
          (5, 3): F(730878875, 902184768), (5, 4): F(2285395, 8070912)}
    for j in range(1, 6):
        ai[(6, j)] = b[j - 1]
    be = [F(31666707, 9881966720), F(0), F(-256875, 105007616), F(-2768025, 128864768),
          F(169839, 3864644), F(-5247, 225920)]
    c_e = [sum(ae.get((i, j), 0) for j in range(1, 7)) for i in range(1, 7)]
    c_i = [sum(ai.get((i, j), 0) for j in range(1, 7)) + (F(1, 4) if i > 1 else 0) for i in range(1, 7)]
    # the implicit rows sum exactly to c; the published explicit coefficients are rational
    # approximations whose row sums agree to ~1e-13
    assert c_i[:3] == c_e[:3]
    assert all(abs(float(a - b)) < 1e-12 for a, b in zip(c_e, c_i))
    assert [float(c) for c in c_i] == pytest.approx([0, 0.5, 0.332, 0.62, 0.85, 1.0])
    assert sum(b) == 1
    assert sum(be) == 0
    ae_f, ai_f, b_f, be_f = ark43_tableau()
    for (i, j), v in ae.items():
        assert ae_f[i - 1, j - 1] == float(v)
    for (i, j), v in ai.items():
        assert ai_f[i - 1, j - 1] == float(v)
    assert list(b_f) == [float(x) for x in b]
    assert list(be_f) == [float(x) for x in be]


# ---------------------------------------------------------------------------------------
# Linear physics
# ---------------------------------------------------------------------------------------
def test_single_mode_has_zero_jacobian():
    m = small_model(nz=3, C_d=0.0)   # quadratic drag is nonlinear even for one mode
    q = np.zeros((3, 32, 17), dtype=complex)
    q[:, 5, 3] = [1e-6, -2e-6, 0.5e-6]
    rhs = m.get_rhs(q)
    psi = m.get_psi(q)
    p = m.p
    expect = -(1j * m.kx)[None] * (m.uBar[:, None, None] * q + (p.beta + m.qyBar)[:, None, None] * psi)
    expect[-1] += (p.r0 * p.Htot / m.H[-1]) * m.k2 * psi[-1]
    assert np.allclose(rhs, m.dealias(expect), rtol=1e-12, atol=1e-12 * np.abs(expect).max())


def test_phillips_growth_rate():
    """2-layer Phillips problem: a single unstable mode grows at the rate of the linear
    operator's most unstable eigenvalue (RK4, small amplitude, no dissipation)."""
    H, S, U = phillips_two_layer()
    p = Params(nx=32, ny=32, nz=2, Lx=1.0e6, Ly=1.0e6, Htot=4000.0, beta=1.6e-11, A8=0.0, r0=0.0, C_d=0.0)
    m = QGNOracle(p, H, S, U)
    i, j = 4, 0
    kx, ky = m.kx[j, i], m.ky[j, i]
    k2 = kx * kx + ky * ky
    Minv = np.linalg.inv(-k2 * np.eye(2) + m.L)
    A = -1j * kx * (np.diag(m.uBar) + np.diag(p.beta + m.qyBar) @ Minv)
    w, V = np.linalg.eig(A)
    sigma = np.max(w.real)
    assert sigma > 0
    v = V[:, np.argmax(w.real)]
    q = np.zeros((2, 32, 17), dtype=complex)
    q[:, j, i] = 1e-12 * v / np.abs(v).max()
    st = RK4(m)
    dt = 1800.0
    t = 0.0
    n0 = np.linalg.norm(q)
    for _ in range(200):
        q, t, dt = st.step(q, t, dt)
    rate = math.log(np.linalg.norm(q) / n0) / t
    assert rate == pytest.approx(sigma, rel=1e-6)


def total_energy(m, q):
    psi = m.get_psi(q)
    w = np.full(q.shape[-1], 2.0)
    w[0] = 1.0
    return -0.5 * np.sum((m.H / m.p.Htot)[:, None, None] * w[None, None, :] * (np.conj(psi) * q).real)


def test_inviscid_conservation_and_order():
    H, S, U = exponential_stratification(2)
    p = Params(nx=32, ny=32, nz=2, Lx=1.0e6, Ly=1.0e6, Htot=4000.0, beta=0.0, A2=0.0, A8=0.0, r0=0.0, C_d=0.0,
               dt_max=1.0e9)
    m = QGNOracle(p, H, S, np.zeros(2))
    q0 = m.initialize_spec(seeded_random_pv(32, 32, 2, 4.0, 1.0e-5, seed=7))
    E0 = total_energy(m, q0)
    w = np.full(q0.shape[-1], 2.0)
    w[0] = 1.0
    Z0 = np.sum(w * np.abs(q0) ** 2, axis=(1, 2))    # per-layer enstrophy (Parseval weights)
    errs = []
    for dt in (8000.0, 4000.0):
        q = q0.copy()
        st = RK4(m)
        t = 0.0
        for _ in range(int(64000 / dt)):
            q, t, _ = st.step(q, t, dt)
        errs.append(abs(total_energy(m, q) - E0) / abs(E0))
    assert errs[0] < 1e-5
    order = math.log(errs[0] / errs[1], 2)
    assert order > 3.5
    # ARK43 with zero hyperviscosity is explicit RK too: enstrophy drift small
    st = ARK43(m.__class__(p.copy(TOL=1e30, dt_max=2000.0), H, S, np.zeros(2)))
    q = q0.copy()
    t, dt = 0.0, 2000.0
    for _ in range(10):
        q, t, dt = st.step(q, t, dt)
    assert np.all(np.abs(np.sum(w * np.abs(q) ** 2, axis=(1, 2)) - Z0) / Z0 < 1e-6)


def test_leith_parseval_matches_physical():
    m = small_model(nx=64, ny=64, nz=3)
    q = m.initialize_spec(seeded_random_pv(64, 64, 3, 8.0, 1e-6, seed=11))
    a = m.leith_A8L(q)
    b = m.leith_A8L_parseval(q)
    assert np.allclose(a, b, rtol=1e-12)
    assert LEITH_13 == 1.2999999523162842


@pytest.mark.parametrize("nx,ny,nz", [(64, 64, 3), (32, 64, 5), (64, 32, 2)])
def test_energetics_identities(nx, ny, nz):
    """KE from the spectrum shells, KE + APE = -0.5 sum_k w_k mean(psi q), APE in its interface
    form sum_i S_i/(Htot (H_i + H_i+1)) mean((psi_i+1 - psi_i)^2) (from QGN_Module.f90:100-112)."""
    m = small_model(nx=nx, ny=ny, nz=nz)
    q = m.initialize_spec(seeded_random_pv(nx, ny, nz, 6.0, 1e-6, seed=nx + nz))
    ke = m.layer_ke(q)
    spec = m.ke_spectrum(q, nbins=max(nx, ny))
    assert np.allclose(spec.sum(axis=1), ke, rtol=1e-12)
    ape = m.layer_ape(q)
    psi = m.s2g_scaled(m.get_psi(q))
    qp = m.s2g_scaled(q)
    w = m.H / m.p.Htot
    assert np.sum(ke) + np.sum(ape) == pytest.approx(-0.5 * np.sum(w * np.mean(psi * qp, axis=(1, 2))), rel=1e-12)
    iface = sum(m.S[i + 1] / (m.p.Htot * (m.H[i] + m.H[i + 1])) * np.mean((psi[i + 1] - psi[i]) ** 2)
                for i in range(nz - 1))
    assert np.sum(ape) == pytest.approx(iface, rel=1e-12)
    assert np.sum(ape) > 0
    Z = m.layer_enstrophy(q)
    assert np.allclose(Z, 0.5 * np.mean(qp ** 2, axis=(1, 2)) * w, rtol=1e-14)


def test_notebook_profiles_against_the_reference_notebook():
    """inputs.notebook_profiles against set_background_profiles.ipynb's own computation (its code
    cells run by tests/golden/notebook/make_notebook_golden.py, nz = 32, alpha = 1), and the deformation
    radii of the QGN stretching matrix (QGN_Module.f90:100-112, built from those H and S) against
    the radii the notebook printed in its stored output (cell 9, 8 decimals, H_tot = 4800 m)."""
    from oracle.qgn_oracle import stretching_matrix
    from qgn_fortran_b200.inputs import notebook_profiles
    d = np.load(os.path.join(GOLDEN, "notebook", "notebook_profiles_nz32.npz"))
    H, S, U, zc = notebook_profiles(nz=int(d["nz"]), alpha=float(d["alpha"]))
    assert np.allclose(H, d["H"], rtol=1e-12, atol=0)
    assert np.allclose(S, d["S"], rtol=1e-12, atol=0)
    assert np.allclose(U, d["UBar"], rtol=1e-12, atol=1e-15)
    assert np.allclose(zc, d["zc"], rtol=1e-12, atol=0)
    L = stretching_matrix(H, S)       # depth 1 (sum(h) = 1), f = 1: the notebook's units
    from qgn_fortran_b200 import model
    assert np.array_equal(model.stretching_matrix(H, S), L)     # the GPU host set-up builds the same L
    vals = np.linalg.eigvals(L).real
    with np.errstate(invalid="ignore", divide="ignore"):
        radii = float(d["H_tot"]) * np.sort(1.0 / np.sqrt(-vals)) / 1e3
    want = d["radii_printed"]
    n = int(np.sum(np.isfinite(want)))            # the barotropic mode prints as nan
    assert n == int(d["nz"]) - 1
    assert np.allclose(radii[:n], want[:n], rtol=0, atol=6e-9)


def test_write_qp_modal_identities():
    """WriteQPmodal: the modes back-project onto q, psi and the full Jacobian; a single
    Fourier mode in one vertical mode gives that mode alone, psi_mode = q_mode/(-k^2+EVals),
    and a zero Jacobian."""
    nx, ny, nz = 32, 64, 3
    m = small_model(nx=nx, ny=ny, nz=nz)
    q = m.initialize_spec(seeded_random_pv(nx, ny, nz, 6.0, 1e-6, seed=2))
    qm, pm, jm = m.write_qp_modal(q)
    back = lambda f: np.einsum("ab,byx->ayx", m.Modes, f)
    tol = 1e-12
    assert np.allclose(back(qm), m.s2g_scaled(q), rtol=0, atol=tol * np.abs(qm).max())
    assert np.allclose(back(pm), m.s2g_scaled(m.get_psi(q)), rtol=0, atol=tol * np.abs(pm).max())
    assert np.allclose(back(jm), m.s2g_scaled(m.jacobian(q)), rtol=0, atol=tol * np.abs(jm).max())
    # one Fourier mode (kx = 3, ky = 2) carried by vertical mode 1
    x = np.arange(nx) * m.p.Lx / nx
    y = np.arange(ny) * m.p.Ly / ny
    kx, ky = 3 * 2 * np.pi / m.p.Lx, 2 * 2 * np.pi / m.p.Ly
    f = np.cos(kx * x[None, :] + ky * y[:, None])
    qp = 1e-5 * m.Modes[:, 1][:, None, None] * f[None]
    qm, pm, jm = m.write_qp_modal(m.initialize_spec(qp))
    assert np.allclose(qm[1], 1e-5 * f, atol=1e-18)
    assert np.allclose(qm[[0, 2]], 0.0, atol=1e-18)
    p1 = 1e-5 * f / (-(kx * kx + ky * ky) + m.EVals[1])
    assert np.allclose(pm[1], p1, rtol=0, atol=1e-12 * np.abs(p1).max())
    assert np.abs(jm).max() <= 1e-12 * (kx * kx + ky * ky) * np.abs(p1).max() * 1e-5


# ---------------------------------------------------------------------------------------
# Golden fixtures are reproduced by the oracle
# ---------------------------------------------------------------------------------------
@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))))
def test_golden_reproduced(path):
    d = np.load(path)
    meta = json.loads(str(d["meta"]))
    p = Params(**meta["params"])
    m = QGNOracle(p, d["H"], d["S"], d["U"])
    q0 = m.initialize_spec(d["qp"])
    assert np.array_equal(q0, d["q0"]) or np.allclose(q0, d["q0"], rtol=0, atol=1e-15 * np.abs(q0).max())
    assert np.allclose(m.get_rhs(q0), d["rhs"], rtol=0, atol=1e-14 * np.abs(d["rhs"]).max())
    st = SCHEMES[meta["scheme"]](m)
    q, t, dt = q0.copy(), 0.0, meta["dt0"]
    for k in range(meta["nsteps"]):
        q, t, dt = st.step(q, t, dt)
        assert t == pytest.approx(d["t"][k], rel=1e-13)
        assert dt == pytest.approx(d["dt"][k], rel=1e-12)
    assert np.allclose(q, d["qfinal"], rtol=0, atol=1e-13 * np.abs(q).max())
