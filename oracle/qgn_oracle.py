"""CPU FP64 restatement of QGN's pseudo-spectral right-hand side and time steppers.

TEST INFRASTRUCTURE ONLY.  This module is the parity oracle for the CUDA path of
``qgn_fortran_b200``.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it, and
only as the checker or the timed CPU baseline -- never as the product path.

Parity status: UNPINNED.  The reference (iangrooms/QGN_Fortran) is Fortran 90 whose
arithmetic lives in Intel MKL (DFTI FFTs and LAPACK DGEEV); no Fortran compiler and no
MKL exist where this project is built, and the reference ships no tests, golden vectors
or fixtures.  This restatement is therefore pinned only by the known-answer tests in
``tests/test_oracle.py`` (FFT against numpy's pocketfft, modal orthonormality, the
inversion identity, the dealias index rule, exact tableau identities, linear Rossby /
Phillips solutions, inviscid energy/enstrophy conservation and 4th-order convergence).

Every function cites the reference file:line it follows.  Array layout mirrors the
reference's Fortran storage exactly: the Fortran ``complex(dp) q_hat(nx/2+1,ny,nz)``
is the C-order numpy array ``q_hat[nz, ny, nx//2+1]`` and the physical
``real(dp) q(nx,ny,nz)`` is ``q[nz, ny, nx]``.

FFT conventions follow ``MKL_DFTI_Setup.f90:1-52``: out-of-place, unnormalised,
batched over ``nz`` 2-D transforms, conjugate-even (CCE) storage.  numpy's
``rfft2`` / ``irfft2`` implement the same transforms; ``irfft2`` divides by
``nx*ny`` which is exactly the reference's ``grid/real(nx*ny,dp)``.  For a kx=0
column that is not Hermitian in ky (asymmetric dealiasing when ``n mod 3 != 0``)
``irfft2`` performs the y transform first and keeps Re of the kx=0 entry -- the
Hermitian projection that a y-then-x c2r performs.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace

import numpy as np
from scipy.linalg import lapack

# Fortran default-REAL literal 1.3 promoted to double (ARK43_QGLeith.f90:72).
LEITH_13 = float(np.float32(1.3))

# FFT backend: numpy's pocketfft (default, single thread) or scipy.fft with worker threads
# (used when the oracle is timed as the CPU baseline).
_FFT_WORKERS = None


def set_fft_workers(n):
    """Use scipy.fft with n worker threads (None restores numpy.fft)."""
    global _FFT_WORKERS
    _FFT_WORKERS = n


def _rfft2(a):
    if _FFT_WORKERS:
        import scipy.fft as sfft
        return sfft.rfft2(a, axes=(-2, -1), workers=_FFT_WORKERS)
    return np.fft.rfft2(a, axes=(-2, -1))


def _irfft2(a, s):
    if _FFT_WORKERS:
        import scipy.fft as sfft
        return sfft.irfft2(a, s=s, axes=(-2, -1), workers=_FFT_WORKERS)
    return np.fft.irfft2(a, s=s, axes=(-2, -1))


@dataclass
class Params:
    """Compile-time constants of ``parameters.f90:1-31`` as a runtime record."""
    nx: int = 384
    ny: int = 384
    nz: int = 32
    Lx: float = 1.3824e6
    Ly: float = 1.3824e6
    Htot: float = 4800.0
    f0: float = 1.0e-4
    beta: float = 2.0e-11
    A2: float = 0.0
    A8: float = 1.0e23
    r0: float = 1.0e-7
    C_d: float = 1.0e-5
    TOL: float = 1.0e-10
    is_explicit: bool = False
    dt_max: float = float("nan")  # NaN -> reference default pi/(beta*Lx)

    def __post_init__(self):
        if not (self.dt_max == self.dt_max):
            self.dt_max = math.pi / (self.beta * self.Lx)

    def copy(self, **kw):
        return replace(self, **kw)


# ---------------------------------------------------------------------------
# Initialize math (QGN_Module.f90:53-188)
# ---------------------------------------------------------------------------
def stretching_matrix(H: np.ndarray, S: np.ndarray) -> np.ndarray:
    """Tridiagonal L of ([Del+L]psi=q), QGN_Module.f90:102-113.  S has nz+1 entries S(0:nz)."""
    nz = H.shape[0]
    L = np.zeros((nz, nz))
    # Fortran 1-based k maps to python k-1; S(k) maps to S[k].
    L[0, 1] = 2.0 * S[1] / (H[0] * (H[0] + H[1]))
    L[0, 0] = -L[0, 1]
    for k in range(2, nz):  # Fortran k=2..nz-1
        L[k - 1, k - 2] = 2.0 * S[k - 1] / (H[k - 1] * (H[k - 1] + H[k - 2]))
        L[k - 1, k] = 2.0 * S[k] / (H[k - 1] * (H[k - 1] + H[k]))
        L[k - 1, k - 1] = -(L[k - 1, k - 2] + L[k - 1, k])
    L[nz - 1, nz - 2] = 2.0 * S[nz - 1] / (H[nz - 1] * (H[nz - 1] + H[nz - 2]))
    L[nz - 1, nz - 1] = -L[nz - 1, nz - 2]
    return L


def vertical_modes(L: np.ndarray, H: np.ndarray, Htot: float):
    """DGEEV('N','V') + normalisation, QGN_Module.f90:119-127.

    Returns (Modes, EVals, info).  Modes[kk, k] is Fortran Modes(kk,k): layer kk of mode k.
    """
    wr, wi, vl, vr, info = lapack.dgeev(L.copy(), compute_vl=0, compute_vr=1)
    Modes = np.array(vr, dtype=np.float64)
    for k in range(L.shape[0]):
        sgn = -1.0 if Modes[0, k] < 0 or (Modes[0, k] == 0 and math.copysign(1.0, Modes[0, k]) < 0) else 1.0
        Modes[:, k] = sgn * Modes[:, k] / np.sqrt(np.sum(H * Modes[:, k] ** 2) / Htot)
    return Modes, np.array(wr, dtype=np.float64), int(info)


def wavenumbers(p: Params):
    """kx, ky, k2 on the CCE grid, QGN_Module.f90:161-172.  Shapes (ny, nx//2+1)."""
    nxh = p.nx // 2 + 1
    i = np.arange(nxh, dtype=np.float64)
    kx1 = (2.0 * math.pi / p.Lx) * i
    j = np.arange(p.ny)
    jj = np.where(j <= p.ny // 2, j, j - p.ny).astype(np.float64)
    ky1 = (2.0 * math.pi / p.Ly) * jj
    kx = np.broadcast_to(kx1[None, :], (p.ny, nxh)).copy()
    ky = np.broadcast_to(ky1[:, None], (p.ny, nxh)).copy()
    k2 = kx ** 2 + ky ** 2
    return kx, ky, k2


def dealias_mask(nx: int, ny: int) -> np.ndarray:
    """Boolean keep-mask of DeAlias, QGN_Module.f90:194-204 (True = kept)."""
    nxh = nx // 2 + 1
    keep = np.ones((ny, nxh), dtype=bool)
    keep[:, nx // 3: nx // 2 + 1] = False          # i = nx/3+1 .. nx/2+1 (1-based)
    keep[ny // 3: 2 * (ny // 3) + 1, :] = False     # j = ny/3+1 .. 2*(ny/3)+1 (1-based)
    keep[0, 0] = False
    return keep


class QGNOracle:
    """Module state of QGN_Module plus its private subroutines."""

    def __init__(self, p: Params, H_raw, S, uBar):
        self.p = p
        H_raw = np.asarray(H_raw, dtype=np.float64)
        self.S = np.asarray(S, dtype=np.float64)
        self.H = p.Htot * H_raw / np.sum(H_raw)                     # QGN_Module.f90:87
        self.L = stretching_matrix(self.H, self.S)
        self.Modes, self.EVals, self.info = vertical_modes(self.L, self.H, p.Htot)
        self.uBar = np.asarray(uBar, dtype=np.float64)
        self.qyBar = self.L @ (-self.uBar)                             # QGN_Module.f90:148
        self.kx, self.ky, self.k2 = wavenumbers(p)
        self.keep = dealias_mask(p.nx, p.ny)
        self.k8 = self.k2 ** 4
        # side-effect module arrays (QGN_Module.f90:40-41)
        self.psi_hat = None
        self.u_hat = None
        self.v_hat = None
        self.u_phys = None
        self.v_phys = None
        self.q_phys = None

    # -- transforms (MKL_DFTI_Setup.f90) --------------------------------------
    def g2s(self, grid):
        """Unnormalised batched r2c, DftiComputeForward(g2s_q, gridE, specE)."""
        return _rfft2(grid)

    def s2g_scaled(self, spec):
        """DftiComputeBackward(s2g_q, ...) followed by grid/real(nx*ny,dp)."""
        return _irfft2(spec, (self.p.ny, self.p.nx))

    def initialize_spec(self, qp):
        """Forward transform and dealias of the physical IC, QGN_Module.f90:179-183."""
        q_hat = self.g2s(np.asarray(qp, dtype=np.float64))
        return self.dealias(q_hat)

    # -- DeAlias (QGN_Module.f90:194-204) -------------------------------------
    def dealias(self, field):
        p = self.p
        f = np.array(field, dtype=np.complex128, copy=True)
        f[..., :, p.nx // 3: p.nx // 2 + 1] = 0.0
        f[..., p.ny // 3: 2 * (p.ny // 3) + 1, :] = 0.0
        f[..., 0, 0] = 0.0
        return f

    # -- GetPsi (QGN_Module.f90:315-341) --------------------------------------
    def get_psi(self, q_hat):
        p = self.p
        nz = p.nz
        H, Modes, EVals = self.H, self.Modes, self.EVals
        q_mode = np.zeros_like(q_hat)
        psi_mode = np.empty_like(q_hat)
        with np.errstate(divide="ignore", invalid="ignore"):
            for k in range(nz):
                acc = np.zeros(q_hat.shape[1:], dtype=np.complex128)
                for kk in range(nz):
                    acc = acc + (H[kk] * Modes[kk, k]) * q_hat[kk]
                q_mode[k] = acc / p.Htot
                psi_mode[k] = q_mode[k] / (-self.k2 + EVals[k])
                psi_mode[k, 0, 0] = 0.0
        psi = np.zeros_like(q_hat)
        for k in range(nz):
            acc = np.zeros(q_hat.shape[1:], dtype=np.complex128)
            for kk in range(nz):
                acc = acc + psi_mode[kk] * Modes[k, kk]
            psi[k] = acc
        self.psi_hat = psi
        return psi

    # -- Jacobian (QGN_Module.f90:215-249) ------------------------------------
    def jacobian(self, q_hat):
        psi = self.get_psi(q_hat)
        I = 1j
        self.u_hat = -(I * self.ky)[None] * psi
        self.v_hat = (I * self.kx)[None] * psi
        self.q_phys = self.s2g_scaled(q_hat)
        self.u_phys = self.s2g_scaled(self.u_hat)
        self.v_phys = self.s2g_scaled(self.v_hat)
        uq_hat = self.g2s(self.u_phys * self.q_phys)
        vq_hat = self.g2s(self.v_phys * self.q_phys)
        return (I * self.kx)[None] * uq_hat + (I * self.ky)[None] * vq_hat

    # -- GetRHS (QGN_Module.f90:258-296) --------------------------------------
    def get_rhs(self, q_hat):
        p = self.p
        nz = p.nz
        jaco = self.jacobian(q_hat)
        rhs = -jaco
        I = 1j
        for k in range(nz):
            rhs[k] = rhs[k] - self.uBar[k] * (I * self.kx) * q_hat[k] \
                - (p.beta + self.qyBar[k]) * self.v_hat[k]
        if p.is_explicit:
            for k in range(nz):
                rhs[k] = rhs[k] - (p.A2 * self.k2 + p.A8 * self.k8) * q_hat[k]
        rhs[nz - 1] = rhs[nz - 1] + (p.r0 * p.Htot / self.H[nz - 1]) * self.k2 * self.psi_hat[nz - 1]
        urms = np.sqrt(self.u_phys ** 2 + self.v_phys ** 2)
        spec = self.g2s(urms * self.u_phys)
        drag = (I * self.ky) * spec[nz - 1]
        spec = self.g2s(urms * self.v_phys)
        drag = drag - (I * self.kx) * spec[nz - 1]
        rhs[nz - 1] = rhs[nz - 1] + (p.C_d * p.Htot / self.H[nz - 1]) * drag
        return self.dealias(rhs)

    # -- QG-Leith coefficient (ARK43_QGLeith.f90:62-73) -----------------------
    def leith_A8L(self, q_hat):
        p = self.p
        d_phys = self.s2g_scaled(self.k8[None] * q_hat)
        q_phys = self.s2g_scaled(q_hat)
        fac = (LEITH_13 * p.Lx / (p.nx * math.pi)) ** 12
        return np.array([fac * math.sqrt(np.sum(q_phys[k] * d_phys[k]) / float(p.nx * p.ny))
                         for k in range(p.nz)])

    def leith_A8L_parseval(self, q_hat):
        """Spectral (Parseval) form of leith_A8L, the form the CUDA path computes."""
        p = self.p
        N = float(p.nx * p.ny)
        w = np.full(q_hat.shape[-1], 2.0)
        w[0] = 0.0
        tot = np.sum(w[None, None, :] * self.k8[None] * np.abs(q_hat) ** 2, axis=(1, 2))
        col = q_hat[:, :, 0]
        neg = np.roll(col[:, ::-1], 1, axis=1)          # f(-ky)
        h = 0.5 * (col + np.conj(neg))
        k8c = self.k8[:, 0]
        tot = tot + np.sum(k8c[None] * np.abs(h) ** 2, axis=1)
        fac = (LEITH_13 * p.Lx / (p.nx * math.pi)) ** 12
        return fac * np.sqrt(tot / (N * N))

    # -- diagnostics ------------------------------------------------------------
    def layer_ke(self, q_hat):
        """Layer kinetic energy 0.5*mean(u^2+v^2)*H_k/Htot from the physical velocities."""
        p = self.p
        psi = self.get_psi(q_hat)
        u = self.s2g_scaled(-(1j * self.ky)[None] * psi)
        v = self.s2g_scaled((1j * self.kx)[None] * psi)
        return 0.5 * np.mean(u ** 2 + v ** 2, axis=(1, 2)) * self.H / p.Htot

    def layer_ape(self, q_hat):
        """Layer share of the available potential energy, -0.5*mean(psi_k (L psi)_k)*H_k/Htot,
        with the stretching matrix L of QGN_Module.f90:100-112 applied to the physical psi.
        The layers sum to sum_i S_i/(Htot (H_i+H_{i+1})) mean((psi_{i+1}-psi_i)^2) >= 0."""
        p = self.p
        psi = self.s2g_scaled(self.get_psi(q_hat))
        Lpsi = np.einsum("kj,jyx->kyx", self.L, psi)
        return -0.5 * np.mean(psi * Lpsi, axis=(1, 2)) * self.H / p.Htot

    def layer_enstrophy(self, q_hat):
        """Layer enstrophy 0.5*mean(q^2)*H_k/Htot from the physical PV."""
        p = self.p
        q = self.s2g_scaled(q_hat)
        return 0.5 * np.mean(q ** 2, axis=(1, 2)) * self.H / p.Htot

    def ke_spectrum(self, q_hat, nbins):
        """Isotropic KE spectrum per layer: shell round(sqrt(i^2 + j^2)) (integer wavenumber
        indices) of 0.5*k^2|psi_hat|^2/(nx ny)^2 * H_k/Htot over the full FFT plane of the
        physical psi, so that sum over shells (nbins large enough) equals layer_ke."""
        p = self.p
        psi = self.s2g_scaled(self.get_psi(q_hat))
        full = np.fft.fft2(psi, axes=(-2, -1))
        i = np.fft.fftfreq(p.nx, d=1.0 / p.nx)
        j = np.fft.fftfreq(p.ny, d=1.0 / p.ny)
        kx = (2.0 * math.pi / p.Lx) * i
        ky = (2.0 * math.pi / p.Ly) * j
        k2 = kx[None, :] ** 2 + ky[:, None] ** 2
        shell = np.floor(np.sqrt(i[None, :] ** 2 + j[:, None] ** 2) + 0.5).astype(np.int64)
        N = float(p.nx * p.ny)
        out = np.zeros((p.nz, nbins))
        ok = shell < nbins
        for k in range(p.nz):
            dens = 0.5 * k2 * np.abs(full[k]) ** 2 / N / N * self.H[k] / p.Htot
            out[k] = np.bincount(shell[ok], weights=dens[ok], minlength=nbins)[:nbins]
        return out

    # -- WriteQPmodal (QGN_Module.f90:381-440) -----------------------------------
    def write_qp_modal(self, q_hat):
        """The three physical fields WriteQPmodal writes: q_mode, p_mode, J_mode, each (nz, ny, nx).

        The Jacobian is the full undealiased spectrum of i kx (uq)^ + i ky (vq)^
        (QGN_Module.f90:388), projected on the vertical modes like q_hat (lines 392-398);
        psi_mode = q_mode / (-k2 + EVals) with the (0,0) mode zero (lines 399-400).
        """
        p = self.p
        nz = p.nz
        H, Modes, EVals = self.H, self.Modes, self.EVals
        jaco = self.jacobian(q_hat)
        q_mode = np.zeros_like(q_hat)
        j_mode = np.zeros_like(q_hat)
        psi_mode = np.empty_like(q_hat)
        with np.errstate(divide="ignore", invalid="ignore"):
            for k in range(nz):
                for kk in range(nz):
                    q_mode[k] = q_mode[k] + (H[kk] * Modes[kk, k]) * q_hat[kk]
                    j_mode[k] = j_mode[k] + (H[kk] * Modes[kk, k]) * jaco[kk]
                q_mode[k] = q_mode[k] / p.Htot
                j_mode[k] = j_mode[k] / p.Htot
                psi_mode[k] = q_mode[k] / (-self.k2 + EVals[k])
                psi_mode[k, 0, 0] = 0.0
        shape = (p.ny, p.nx)
        return _irfft2(q_mode, shape), _irfft2(psi_mode, shape), _irfft2(j_mode, shape)


# ---------------------------------------------------------------------------
# Time steppers (the include files selected at QGN_Module.f90:306)
# ---------------------------------------------------------------------------
def ark43_tableau():
    """ARK4(3)6L[2]SA coefficients, ARK43_QGLeith.f90:15-58 / ARK43.f90:15-58."""
    ae = np.zeros((6, 6))
    ae[1, 0] = 0.5
    ae[2, 0] = 13861.0 / 62500.0
    ae[2, 1] = 6889.0 / 62500.0
    ae[3, 0] = -116923316275.0 / 2393684061468.0
    ae[3, 1] = -2731218467317.0 / 15368042101831.0
    ae[3, 2] = 9408046702089.0 / 11113171139209.0
    ae[4, 0] = -451086348788.0 / 2902428689909.0
    ae[4, 1] = -2682348792572.0 / 7519795681897.0
    ae[4, 2] = 12662868775082.0 / 11960479115383.0
    ae[4, 3] = 3355817975965.0 / 11060851509271.0
    ae[5, 0] = 647845179188.0 / 3216320057751.0
    ae[5, 1] = 73281519250.0 / 8382639484533.0
    ae[5, 2] = 552539513391.0 / 3454668386233.0
    ae[5, 3] = 3354512671639.0 / 8306763924573.0
    ae[5, 4] = 4040.0 / 17871.0
    b = np.array([82889.0 / 524892.0, 0.0, 15625.0 / 83664.0, 69875.0 / 102672.0,
                  -2260.0 / 8211.0, 0.25])
    ai = np.zeros((6, 6))
    ai[1, 0] = 0.25
    ai[1, 1] = 0.25
    ai[2, 0] = 8611.0 / 62500.0
    ai[2, 1] = -1743.0 / 31250.0
    ai[3, 0] = 5012029.0 / 34652500.0
    ai[3, 1] = -654441.0 / 2922500.0
    ai[3, 2] = 174375.0 / 388108.0
    ai[4, 0] = 15267082809.0 / 155376265600.0
    ai[4, 1] = -71443401.0 / 120774400.0
    ai[4, 2] = 730878875.0 / 902184768.0
    ai[4, 3] = 2285395.0 / 8070912.0
    ai[5, :] = b
    be = np.array([31666707.0 / 9881966720.0, 0.0, -256875.0 / 105007616.0,
                   -2768025.0 / 128864768.0, 169839.0 / 3864644.0, -5247.0 / 225920.0])
    return ae, ai, b, be


class _ARK43Base:
    """Shared body of ARK43_QGLeith.f90 and ARK43.f90 (identical tableau and stage loop)."""
    leith = False
    reject_fac = 0.75
    pi_safety = 0.75

    def __init__(self, m: QGNOracle):
        self.m = m
        self.ae, self.ai, self.b, self.be = ark43_tableau()
        self.err0 = m.p.TOL           # FirstCall, :17
        self.err1 = None
        self.rejects = 0

    def hypervisc(self, q_hat):
        p = self.m.p
        if self.leith:
            return self.m.leith_A8L(q_hat)
        return np.full(p.nz, p.A8)

    def step(self, q_hat, t, dt, max_rejects=10_000):
        m, p = self.m, self.m.p
        ae, ai, b, be = self.ae, self.ai, self.b, self.be
        A8L = self.hypervisc(q_hat)
        D = np.stack([p.A2 * m.k2 + A8L[k] * m.k8 for k in range(p.nz)])   # (A2*k2+A8L(k)*k8)
        Nn = [None] * 6
        Ll = [None] * 6
        Nn[0] = m.get_rhs(q_hat)
        Ll[0] = -D * q_hat
        nrej = 0
        while True:
            Mq = 1.0 / (1.0 + 0.25 * dt * D)
            for s in range(1, 6):
                acc = ae[s, 0] * Nn[0]
                for j in range(1, s):
                    acc = acc + ae[s, j] * Nn[j]
                for j in range(0, s):
                    acc = acc + ai[s, j] * Ll[j]
                q_tmp = Mq * (q_hat + dt * acc)
                Nn[s] = m.get_rhs(q_tmp)
                Ll[s] = -D * q_tmp
            spec = be[0] * (Nn[0] + Ll[0])
            for i in (2, 3, 4, 5):
                spec = spec + be[i] * (Nn[i] + Ll[i])
            grid = _irfft2(spec, (p.ny, p.nx)) * float(p.nx * p.ny)
            err1 = dt * np.max(np.abs(grid)) / float(p.nx * p.ny)
            self.err1 = err1
            if err1 > p.TOL:
                dt = self.reject_fac * dt
                nrej += 1
                self.rejects += 1
                if nrej > max_rejects:
                    raise RuntimeError("reject limit")
                continue
            upd = b[0] * (Nn[0] + Ll[0])
            for i in (2, 3, 4, 5):
                upd = upd + b[i] * (Nn[i] + Ll[i])
            q_new = q_hat + dt * upd
            q_new[:, 0, 0] = 0.0
            t = t + dt
            dt = min(dt * ((self.pi_safety * p.TOL / err1) ** 0.075) * ((self.err0 / err1) ** 0.1), p.dt_max)
            self.err0 = err1
            return m.dealias(q_new), t, dt         # TimeStep's DeAlias, QGN_Module.f90:307


class ARK43QGLeith(_ARK43Base):
    """ARK43_QGLeith.f90:1-141 (the reference default)."""
    leith = True
    reject_fac = 0.5
    pi_safety = 0.2


class ARK43(_ARK43Base):
    """ARK43.f90:1-126 (fixed hyperviscosity A8)."""
    leith = False
    reject_fac = 0.75
    pi_safety = 0.75


class BSRK3:
    """Bogacki-Shampine 3(2) FSAL with PI control, BSRK3.f90:1-50."""

    def __init__(self, m: QGNOracle):
        self.m = m
        self.first = True
        self.RHS0 = None
        self.r0 = None
        self.rejects = 0

    def step(self, q_hat, t, dt, max_rejects=10_000):
        m, p = self.m, self.m.p
        if self.first:
            self.RHS0 = m.get_rhs(q_hat)
            self.r0 = p.TOL
            self.first = False
        nrej = 0
        while True:
            q_tmp = q_hat + 0.5 * dt * self.RHS0
            RHS1 = m.get_rhs(q_tmp)
            q_tmp = q_hat + 0.75 * dt * RHS1
            RHS2 = m.get_rhs(q_tmp)
            q_tmp = q_hat + (2.0 * dt / 9.0) * self.RHS0 + (1.0 * dt / 3.0) * RHS1 + (4.0 * dt / 9.0) * RHS2
            RHS3 = m.get_rhs(q_tmp)
            err_spec = (5.0 / 72.0) * self.RHS0 - (1.0 / 12.0) * RHS1 - (1.0 / 9.0) * RHS2 + (1.0 / 8.0) * RHS3
            err_phys = _irfft2(err_spec, (p.ny, p.nx))
            r1 = dt * np.max(np.abs(err_phys))
            if r1 > p.TOL:
                dt = 0.75 * dt
                nrej += 1
                self.rejects += 1
                if nrej > max_rejects:
                    raise RuntimeError("reject limit")
                continue
            q_new = q_tmp
            t = t + dt
            self.RHS0 = RHS3
            dt = min(dt * ((0.75 * p.TOL / r1) ** 0.1) * ((self.r0 / r1) ** (0.4 / 3.0)), p.dt_max)
            self.r0 = r1
            return m.dealias(q_new), t, dt


class RK4:
    """Classic RK4, RK4.f90:1-18."""

    def __init__(self, m: QGNOracle):
        self.m = m

    def step(self, q_hat, t, dt):
        m = self.m
        R0 = m.get_rhs(q_hat)
        R1 = m.get_rhs(q_hat + (0.5 * dt) * R0)
        R2 = m.get_rhs(q_hat + (0.5 * dt) * R1)
        R3 = m.get_rhs(q_hat + dt * R2)
        q_new = q_hat + (dt / 6.0) * (R0 + 2.0 * R1 + 2.0 * R2 + R3)
        return m.dealias(q_new), t + dt, dt


class AB3:
    """AB3 with forward-Euler and AB2 start-up, AB3.f90:1-23."""

    def __init__(self, m: QGNOracle):
        self.m = m
        self.calls = 0
        self.R0 = self.R1 = None

    def step(self, q_hat, t, dt):
        m = self.m
        if self.calls == 0:
            self.R0 = m.get_rhs(q_hat)
            q_new = q_hat + dt * self.R0
        elif self.calls == 1:
            self.R1 = m.get_rhs(q_hat)
            q_new = q_hat + dt * (1.5 * self.R1 - 0.5 * self.R0)
        else:
            R2 = m.get_rhs(q_hat)
            q_new = q_hat + (dt / 12.0) * (23.0 * R2 - 16.0 * self.R1 + 5.0 * self.R0)
            self.R0 = self.R1
            self.R1 = R2
        self.calls += 1
        return m.dealias(q_new), t + dt, dt


SCHEMES = {
    "ark43_qgleith": ARK43QGLeith,
    "ark43": ARK43,
    "bsrk3": BSRK3,
    "rk4": RK4,
    "ab3": AB3,
}
