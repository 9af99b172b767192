"""Background profiles, initial conditions and the reference's binary file formats.

The reference reads three raw float64 stream files in ``Initialize``
(``QGN_Module.f90:84-90,145-147``): ``H.dat`` (nz layer thicknesses, top first,
rescaled to Htot on read), ``S.dat`` (nz+1 values of f0^2/N^2 at the interfaces
S(0:nz), top first) and ``UBar.dat`` (nz mean zonal velocities).  Restarts read
``q.%09d.dat``: the physical PV as ``real(dp) q(nx,ny,nz)`` in Fortran order
(``QGN_Driver.f90:21-30``), i.e. C-order ``[nz][ny][nx]``.

The generators below write the same formats.  ``notebook_profiles`` restates the
stretched-grid / first-baroclinic / ocean-Charney construction of
``set_background_profiles.ipynb`` (cells 2-15); the other generators build the
named workloads (2-layer Phillips problem; exponential N^2(z) with a
surface-intensified mean flow).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass

import numpy as np


# ---------------------------------------------------------------------------
# Binary formats
# ---------------------------------------------------------------------------
def write_profiles(directory, H, S, UBar):
    os.makedirs(directory, exist_ok=True)
    np.asarray(H, dtype="<f8").tofile(os.path.join(directory, "H.dat"))
    np.asarray(S, dtype="<f8").tofile(os.path.join(directory, "S.dat"))
    np.asarray(UBar, dtype="<f8").tofile(os.path.join(directory, "UBar.dat"))


def read_profiles(directory, nz):
    """Read H.dat, S.dat, UBar.dat; rejects short or long files (the reference does not check)."""
    out = []
    for name, n in (("H.dat", nz), ("S.dat", nz + 1), ("UBar.dat", nz)):
        path = os.path.join(directory, name)
        a = np.fromfile(path, dtype="<f8")
        if a.size != n:
            raise ValueError(f"{name}: expected {n} float64 values for nz={nz}, found {a.size}")
        if not np.all(np.isfinite(a)):
            raise ValueError(f"{name}: non-finite values")
        out.append(a)
    H, S, U = out
    if np.any(H <= 0):
        raise ValueError("H.dat: layer thicknesses must be positive")
    return H, S, U


def qp_filename(step: int, prefix: str = "q") -> str:
    """File name pattern '(A2,I0.9,A4)' of QGN_Driver.f90:22 and QGN_Module.f90:364."""
    return f"{prefix}.{step:09d}.dat"


def write_physical(path, field):
    """Raw float64 stream of a C-order [nz][ny][nx] array == Fortran (nx,ny,nz)."""
    np.ascontiguousarray(field, dtype="<f8").tofile(path)


def read_physical(path, nx, ny, nz):
    a = np.fromfile(path, dtype="<f8")
    if a.size != nx * ny * nz:
        raise ValueError(f"{path}: expected {nx * ny * nz} float64 values, found {a.size}")
    return a.reshape(nz, ny, nx)


# ---------------------------------------------------------------------------
# Profile generators
# ---------------------------------------------------------------------------
def phillips_two_layer(H1=1000.0, H2=3000.0, f0=1.0e-4, gprime=0.02, U=(0.05, 0.0)):
    """Two-layer Phillips problem.  S(1)=f0^2 (H1+H2)/(2 g') makes L(1,2)=f0^2/(g' H1)."""
    s1 = f0 * f0 * (H1 + H2) / (2.0 * gprime)
    H = np.array([H1, H2])
    S = np.array([s1, s1, s1])
    return H, S, np.array(U, dtype=np.float64)


def exponential_stratification(nz, Htot=4000.0, ratio=1.4, f0=1.0e-4, N0=5.0e-3,
                               N_efold=1000.0, U0=0.1, U_efold=1000.0):
    """Geometric layers (thinnest on top, each ``ratio`` x the one above);
    N^2(z) = N0^2 exp(z/N_efold) with z<=0 upward-positive; U(z) = U0 exp(z/U_efold) at layer centres.
    S(k) = f0^2/N^2 at interface k (k=0 surface, k=nz bottom)."""
    w = ratio ** np.arange(nz, dtype=np.float64)
    H = Htot * w / w.sum()
    zi = -np.concatenate(([0.0], np.cumsum(H)))              # interface heights, top first
    S = f0 * f0 / (N0 * N0 * np.exp(zi / N_efold))
    zc = 0.5 * (zi[:-1] + zi[1:])
    U = U0 * np.exp(zc / U_efold)
    return H, S, U


def notebook_profiles(nz=32, alpha=1.0):
    """Stretched grid + mean flow of set_background_profiles.ipynb (cells 2-15).

    N^2(t)/f^2 = (1 + 9t + 50 exp(-75 (t-0.8)^2))^2 on t in [0,1] (bottom to top);
    interfaces equally spaced in int sqrt(N^2)^alpha; mean flow
    0.22 * first baroclinic mode - 0.08 * ocean-Charney profile.
    Returns (H, S, UBar, zc) top first (H relative; QGN rescales to Htot)."""
    from scipy import integrate, optimize

    def N2(t):
        return (1.0 + 9.0 * t + 50.0 * np.exp(-75.0 * (t - 0.8) ** 2)) ** 2

    def SS(t):
        return np.sqrt(N2(t)) ** alpha

    norm = integrate.quad(SS, 0, 1)[0]
    z = np.zeros(nz + 1)
    z[nz] = 1.0
    for i in range(1, nz):
        z[i] = optimize.fsolve(lambda t: integrate.quad(SS, 0, t)[0] - norm * i / nz, i / nz)[0]
    h = z[1:] - z[:-1]
    zc = 0.5 * (z[:-1] + z[1:])
    DS = np.diag(1.0 / N2(z[1:-1]))
    D0 = np.zeros((nz - 1, nz))
    D0[:, :-1] = 2.0 * np.diag(1.0 / (h[:-1] + h[1:]))
    D0[:, 1:] = D0[:, 1:] - 2.0 * np.diag(1.0 / (h[:-1] + h[1:]))
    D = DS @ D0
    L = (1.0 / h) * (np.vstack((np.zeros((1, nz)), D)) - np.vstack((D, np.zeros((1, nz)))))
    L = L.T
    vals, vecs = np.linalg.eig(L)
    vals = vals.real
    vecs = vecs.real
    ind = np.argsort(-vals)
    bc1 = vecs[:, ind[1]] / vecs[-1, ind[1]]
    L_oc = L[:-1, 1:]
    oc = np.concatenate((np.zeros(1), np.linalg.solve(L_oc, np.ones(nz - 1))))
    oc = oc / oc[-1]
    u_bar = 0.22 * bc1 - 0.08 * oc
    S = np.zeros(nz + 1)
    for i in range(nz + 1):
        S[nz - i] = 1.0 / N2(z[i])
    return np.flip(h).copy(), S, np.flip(u_bar).copy(), np.flip(zc).copy()


# ---------------------------------------------------------------------------
# Initial conditions
# ---------------------------------------------------------------------------
def seeded_random_pv(nx, ny, nz, k0, rms, seed, Lx=None, Ly=None):
    """Seeded Gaussian random PV field, physical C-order [nz][ny][nx].

    Real white noise is forward transformed (so the spectrum is Hermitian), shaped by
    (|k|/k0) exp(-(|k|/k0)^2/2) with |k| in integer wavenumbers, transformed back and
    scaled to the requested rms in every layer."""
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal((nz, ny, nx))
    spec = np.fft.rfft2(noise, axes=(-2, -1))
    kx = np.arange(nx // 2 + 1, dtype=np.float64)
    ky = np.fft.fftfreq(ny, d=1.0 / ny)
    kk = np.sqrt(kx[None, :] ** 2 + ky[:, None] ** 2)
    amp = (kk / k0) * np.exp(-0.5 * (kk / k0) ** 2)
    q = np.fft.irfft2(spec * amp[None], s=(ny, nx), axes=(-2, -1))
    q -= q.mean(axis=(1, 2), keepdims=True)
    q *= rms / np.sqrt(np.mean(q ** 2, axis=(1, 2), keepdims=True))
    return q


def driver_sinusoid_ic(nx, ny, nz):
    """The hard-coded IC of QGN_Driver.f90:38-43."""
    i = np.arange(nx, dtype=np.float64)
    j = np.arange(ny, dtype=np.float64)
    q = 1.0e-5 * np.sin(48.0 * math.pi * i / nx)[None, :] + 2.0e-5 * np.cos(32.0 * math.pi * j / ny)[:, None]
    return np.broadcast_to(q, (nz, ny, nx)).copy()


# ---------------------------------------------------------------------------
# Named workloads
# ---------------------------------------------------------------------------
@dataclass
class Workload:
    name: str
    params: dict
    H: np.ndarray
    S: np.ndarray
    U: np.ndarray
    qp: np.ndarray
    scheme: str
    dt0: float
    t0: float = 0.0
    ic: str = "seeded"


DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


def spinup_path(name: str) -> str:
    return os.path.join(DATA, f"{name}_spinup.npz")


def spunup_pv(name: str, path: str | None = None):
    """The spun-up state of a named workload (written by ``qgn_fortran_b200.spinup``) as a physical
    PV field C-order [nz][ny][nx], with its metadata (simulated time t, last dt, TOL, ...).  The
    fixture holds the modes DeAlias keeps at bfloat16 precision; the field is their c2r/(nx ny)
    (MKL_DFTI_Setup.f90 backward transform, QGN_Module.f90:348-377 scaling)."""
    import json
    d = np.load(path or spinup_path(name))
    meta = json.loads(str(d["meta"]))
    nx, ny, nz = meta["nx"], meta["ny"], meta["nz"]

    def f32(bits):
        return (np.asarray(bits, dtype=np.uint32) << 16).view(np.float32).astype(np.float64)

    full = np.zeros((nz, ny, nx // 2 + 1), dtype=np.complex128)
    rows = np.r_[0:ny // 3, 2 * (ny // 3) + 1:ny]
    full[:, rows, :nx // 3] = f32(d["re"]) + 1j * f32(d["im"])
    full[:, 0, 0] = 0.0
    return np.fft.irfft2(full, s=(ny, nx), axes=(-2, -1)), meta


def ensemble_members(n=64, seed0=1000, sizes=(128, 256, 512), layers=(2, 4, 8), Lx=2.0e6, with_ic=True):
    """Members of the batched-ensemble workload: grid n^2 drawn uniformly from ``sizes``, layer
    count from ``layers``; each member's exponential stratification has its own e-folding
    depth in [500, 1500] m (for N^2 and for the mean flow) and surface flow in
    [0.02, 0.15] m/s.  BSRK3 with PI.3.4 adaptive dt, absolute TOL = 1e-6 x max|q_IC|,
    explicit hyperviscosity with a 1-day grid-scale e-folding, C_d = 0.  The IC of member m
    is the seeded random PV field (peak wavenumber 8, rms 1e-6) with seed ``seed0 + m``.
    Returns a list of ``Workload``."""
    out = []
    for m in range(n):
        rng = np.random.default_rng(seed0 + m)
        nxy = int(rng.choice(sizes))
        nz = int(rng.choice(layers))
        efold = float(rng.uniform(500.0, 1500.0))
        U0 = float(rng.uniform(0.02, 0.15))
        H, S, U = exponential_stratification(nz, N_efold=efold, U0=U0, U_efold=efold)
        qp = seeded_random_pv(nxy, nxy, nz, 8.0, 1.0e-6, seed0 + m) if with_ic else None
        tol = 1.0e-6 * (float(np.max(np.abs(qp))) if qp is not None else 4.0e-6)
        beta = 2.0e-11
        A8 = 1.0 / (86400.0 * (math.pi * nxy / Lx) ** 8)
        p = dict(nx=nxy, ny=nxy, nz=nz, Lx=Lx, Ly=Lx, Htot=4000.0, f0=1.0e-4, beta=beta,
                 A2=0.0, A8=A8, r0=1.0e-7, C_d=0.0, TOL=tol, is_explicit=True,
                 dt_max=math.pi / (beta * Lx))
        out.append(Workload(f"member{m}_{nxy}x{nz}", p, H, S, U, qp, "bsrk3", 1800.0))
    return out


def workload(name: str, nx=None, nz=None, seed=None, with_ic=True, ic: str = "seeded") -> Workload:
    """Named synthetic workloads.

    * ``phillips256``: 2-layer Phillips problem, 256^2, L=1000 km, H=[1000,3000] m,
      f0=1e-4, beta=1.6e-11, g'=0.02, U=[0.05,0], r0=1e-7, A8 for a 1-day grid-scale
      e-folding, ARK43 (fixed A8) at dt=900 s (dt_max=900, TOL=1e30 so the PI
      controller is always clipped to dt_max).  IC peak wavenumber 10, rms 1e-6, seed 1.
    * ``strat1024x8``: 8 geometric layers (ratio 1.4) over 4000 m on 1024^2, L=2000 km,
      N^2=(5e-3)^2 exp(z/1000), U=0.1 exp(z/1000), ARK43_QGLeith with PI.3.4 and an
      absolute TOL of 1e-6 x max|q_IC|; f0, beta, A2, r0 from parameters.f90 defaults,
      C_d=0.  IC peak wavenumber 16, rms 1e-6, seed 2.
    * ``strat2048x16``: the same stratification on 2048^2 x 16 layers (seed 3).
    ``nx``/``nz`` override the grid for reduced-size parity cases.
    ``ic="spinup"`` starts from the committed spun-up state of the full-size workload instead
    (``spunup_pv``): t0 and dt0 are the spin-up's final t and dt, TOL stays the configured one.
    """
    if ic == "spinup":
        if nx or nz or seed is not None:
            raise ValueError("the spun-up state exists for the full-size workload only")
        w = workload(name, with_ic=False)
        qp, meta = spunup_pv(name)
        w.params["TOL"] = meta["TOL"]
        return Workload(name, w.params, w.H, w.S, w.U, qp, w.scheme, meta["dt"], meta["t"], "spinup")
    if name == "phillips256":
        n = nx or 256
        Lx = 1.0e6
        H, S, U = phillips_two_layer()
        A8 = 1.0 / (86400.0 * (math.pi * n / Lx) ** 8)
        p = dict(nx=n, ny=n, nz=2, Lx=Lx, Ly=Lx, Htot=4000.0, f0=1.0e-4, beta=1.6e-11,
                 A2=0.0, A8=A8, r0=1.0e-7, C_d=0.0, TOL=1.0e30, is_explicit=False, dt_max=900.0)
        qp = seeded_random_pv(n, n, 2, 10.0, 1.0e-6, 1 if seed is None else seed) if with_ic else None
        return Workload(name, p, H, S, U, qp, "ark43", 900.0)
    if name in ("strat1024x8", "strat2048x16"):
        n = nx or (1024 if name == "strat1024x8" else 2048)
        z = nz or (8 if name == "strat1024x8" else 16)
        Lx = 2.0e6
        H, S, U = exponential_stratification(z)
        qp = seeded_random_pv(n, n, z, 16.0, 1.0e-6,
                              (2 if name == "strat1024x8" else 3) if seed is None else seed) if with_ic else None
        tol = 1.0e-6 * (float(np.max(np.abs(qp))) if qp is not None else 4.0e-6)
        beta = 2.0e-11
        p = dict(nx=n, ny=n, nz=z, Lx=Lx, Ly=Lx, Htot=4000.0, f0=1.0e-4, beta=beta,
                 A2=0.0, A8=1.0e23, r0=1.0e-7, C_d=0.0, TOL=tol, is_explicit=False,
                 dt_max=math.pi / (beta * Lx))
        return Workload(name, p, H, S, U, qp, "ark43_qgleith", 750.0)
    raise KeyError(name)
