"""Host-side mirror of the reference's QGN_Module public API over the CUDA C-ABI.

``QGNModule`` plays the role of ``module QGN_Module`` (QGN_Module.f90:1-460):

* ``__init__`` + ``initialize(qp)``  -> ``Initialize(qp, q_hat)`` (QGN_Module.f90:53-188):
  H rescale, stretching matrix, LAPACK DGEEV('N','V') eigen-decomposition and mode
  normalisation, qyBar = L(-uBar) stay on the host in FP64 (as in the reference); the
  forward transform and DeAlias of the IC run on the GPU.
* ``time_step(q_hat, t, dt)``         -> ``TimeStep(q_hat, t, dt)`` (QGN_Module.f90:302-309)
* ``write_qp(q_hat, rec_no, nt)``     -> ``WriteQP`` (QGN_Module.f90:348-377)
* ``cleanup()``                       -> ``Cleanup`` (QGN_Module.f90:448-458)

plus device-resident helpers (``set_state``/``get_state``/``advance_resident``), the
``get_rhs`` parity hook and FP64 diagnostics.  Every call goes through
``libqgn_b200.so``; there is no CPU compute path, and construction fails with
``QGN_ERR_NO_DEVICE`` when no B200 is present.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

from . import _lib
from ._lib import QGNError, dptr

PARAM_DEFAULTS = dict(nx=384, ny=384, nz=32, Lx=1.3824e6, Ly=1.3824e6, Htot=4800.0, f0=1.0e-4,
                      beta=2.0e-11, A2=0.0, A8=1.0e23, r0=1.0e-7, C_d=1.0e-5, TOL=1.0e-10,
                      is_explicit=False, dt_max=None)


def full_params(**kw) -> dict:
    """parameters.f90:1-31 with overrides; dt_max defaults to pi/(beta*Lx) (parameters.f90:31)."""
    p = dict(PARAM_DEFAULTS)
    unknown = set(kw) - set(p)
    if unknown:
        raise KeyError(f"unknown parameters {sorted(unknown)}")
    p.update(kw)
    if p["dt_max"] is None:
        p["dt_max"] = (4.0 * math.atan(1.0)) / (p["beta"] * p["Lx"])
    return p


def stretching_matrix(H, S):
    """L of ([Del+L]psi = q), QGN_Module.f90:102-113 (S holds S(0:nz))."""
    nz = len(H)
    L = np.zeros((nz, nz))
    L[0, 1] = 2.0 * S[1] / (H[0] * (H[0] + H[1]))
    L[0, 0] = -L[0, 1]
    for k in range(1, nz - 1):
        L[k, k - 1] = 2.0 * S[k] / (H[k] * (H[k] + H[k - 1]))
        L[k, k + 1] = 2.0 * S[k + 1] / (H[k] * (H[k] + H[k + 1]))
        L[k, k] = -(L[k, k - 1] + L[k, k + 1])
    L[nz - 1, nz - 2] = 2.0 * S[nz - 1] / (H[nz - 1] * (H[nz - 1] + H[nz - 2]))
    L[nz - 1, nz - 1] = -L[nz - 1, nz - 2]
    return L


def host_initialize(p: dict, H_raw, S, uBar):
    """Host FP64 part of Initialize (QGN_Module.f90:84-148): returns H, L, Modes, EVals, qyBar, info."""
    from scipy.linalg import lapack

    H_raw = np.asarray(H_raw, dtype=np.float64)
    S = np.asarray(S, dtype=np.float64)
    uBar = np.asarray(uBar, dtype=np.float64)
    nz = p["nz"]
    if H_raw.size != nz or S.size != nz + 1 or uBar.size != nz:
        raise ValueError(f"profile sizes {H_raw.size}/{S.size}/{uBar.size} do not match nz={nz}")
    H = p["Htot"] * H_raw / np.sum(H_raw)
    L = stretching_matrix(H, S)
    wr, wi, vl, vr, info = lapack.dgeev(L.copy(), compute_vl=0, compute_vr=1)
    if info != 0:
        raise RuntimeError(f"DGEEV failed, INFO={info}")
    Modes = np.array(vr, dtype=np.float64)
    for k in range(nz):
        sgn = -1.0 if math.copysign(1.0, Modes[0, k]) < 0 else 1.0
        Modes[:, k] = sgn * Modes[:, k] / np.sqrt(np.sum(H * Modes[:, k] ** 2) / p["Htot"])
    qyBar = L @ (-uBar)
    return H, L, Modes, np.asarray(wr, dtype=np.float64), qyBar, int(info)


class QGNModule:
    """One QGN model instance on one GPU (the module state of QGN_Module)."""

    def __init__(self, params: dict, H_raw, S, uBar, scheme: str = "ark43_qgleith",
                 precision: str = "fp64", max_rejects: int = 0):
        self.lib = _lib.load()
        self.p = full_params(**params)
        p = self.p
        self.nx, self.ny, self.nz = p["nx"], p["ny"], p["nz"]
        self.nxh = self.nx // 2 + 1
        self.H, self.L, self.Modes, self.EVals, self.qyBar, self.info = host_initialize(p, H_raw, S, uBar)
        self.S = np.asarray(S, dtype=np.float64)
        self.uBar = np.asarray(uBar, dtype=np.float64)
        cp = _lib.qgn_params(nx=self.nx, ny=self.ny, nz=self.nz, is_explicit=int(bool(p["is_explicit"])),
                             Lx=p["Lx"], Ly=p["Ly"], Htot=p["Htot"], f0=p["f0"], beta=p["beta"],
                             A2=p["A2"], A8=p["A8"], r0=p["r0"], C_d=p["C_d"], TOL=p["TOL"],
                             dt_max=p["dt_max"], max_rejects=int(max_rejects), reserved=0)
        self._cp = cp
        modes_f = np.asfortranarray(self.Modes)
        ctx = C.c_void_p()
        rc = self.lib.qgn_create(C.byref(cp), dptr(np.ascontiguousarray(self.H)), dptr(self.S),
                                 dptr(self.uBar), dptr(np.ascontiguousarray(self.qyBar)),
                                 modes_f.ctypes.data_as(C.POINTER(C.c_double)),
                                 dptr(np.ascontiguousarray(self.EVals)),
                                 _lib.SCHEMES[scheme], _lib.PRECISIONS[precision], C.byref(ctx))
        if rc != 0:
            raise QGNError(rc, f"qgn_create(nx={self.nx}, ny={self.ny}, nz={self.nz}, scheme={scheme})")
        self.ctx = ctx
        self.scheme = scheme
        self.t = 0.0
        self.dt = 0.0

    # -- helpers ---------------------------------------------------------------------
    def _check(self, rc, what):
        if rc != 0:
            msg = self.lib.qgn_last_error(self.ctx)
            raise QGNError(rc, f"{what}: {msg.decode() if msg else ''}")

    def spectral_shape(self):
        return (self.nz, self.ny, self.nxh)

    def physical_shape(self):
        return (self.nz, self.ny, self.nx)

    def _spec(self, a, writable=False):
        a = np.asarray(a)
        if a.shape != self.spectral_shape() or a.dtype != np.complex128 or not a.flags.c_contiguous:
            if writable:
                raise ValueError(f"q_hat must be C-contiguous complex128 of shape {self.spectral_shape()}")
            a = np.ascontiguousarray(a, dtype=np.complex128).reshape(self.spectral_shape())
        return a

    # -- reference API ----------------------------------------------------------------
    def initialize(self, qp, t: float = 0.0, dt: float = 750.0):
        """Initialize's IC transform (QGN_Module.f90:179-183); returns the dealiased q_hat."""
        qp = np.ascontiguousarray(qp, dtype=np.float64).reshape(self.physical_shape())
        self._check(self.lib.qgn_set_state_physical(self.ctx, dptr(qp), t, dt), "qgn_set_state_physical")
        q_hat = np.empty(self.spectral_shape(), dtype=np.complex128)
        self.get_state(q_hat)
        return q_hat

    def time_step(self, q_hat, t: float, dt: float):
        """TimeStep(q_hat, t, dt): advances q_hat in place; returns the new (t, dt)."""
        q_hat = self._spec(q_hat, writable=True)
        tt, dd = C.c_double(t), C.c_double(dt)
        # qgn_step writes back the kept modes; the entries TimeStep's trailing DeAlias
        # (QGN_Module.f90:307) zeroes keep their input values, zero for a dealiased q_hat
        # (set_output("full") writes them as zeros)
        self._check(self.lib.qgn_step(self.ctx, dptr(q_hat), C.byref(tt), C.byref(dd)), "qgn_step")
        self.t, self.dt = tt.value, dd.value
        return tt.value, dd.value

    def set_output(self, mode: str):
        """What time_step/advance write back: "kept" (the kept modes, default) or "full"."""
        code = {"kept": _lib.QGN_OUTPUT_KEPT, "full": _lib.QGN_OUTPUT_FULL}[mode]
        self._check(self.lib.qgn_set_output(self.ctx, code), "qgn_set_output")

    def advance(self, q_hat, t: float, dt: float, nsteps: int):
        q_hat = self._spec(q_hat, writable=True)
        tt, dd = C.c_double(t), C.c_double(dt)
        self._check(self.lib.qgn_advance(self.ctx, dptr(q_hat), C.byref(tt), C.byref(dd), int(nsteps)),
                    "qgn_advance")
        self.t, self.dt = tt.value, dd.value
        return tt.value, dd.value

    def write_qp(self, q_hat, rec_no: int, nt: int, directory: str = "."):
        """WriteQP: q.%09d.dat and p.%09d.dat raw float64 physical fields (QGN_Module.f90:348-377)."""
        qphys, pphys = self.physical(q_hat)
        os.makedirs(directory, exist_ok=True)
        for prefix, arr in (("q", qphys), ("p", pphys)):
            path = os.path.join(directory, f"{prefix}.{nt:09d}.dat")
            np.ascontiguousarray(arr, dtype="<f8").tofile(path)
        return qphys, pphys

    def physical_modal(self, q_hat=None):
        """The physical q_mode, p_mode and J_mode fields of WriteQPmodal (QGN_Module.f90:381-440)."""
        out = [np.empty(self.physical_shape()) for _ in range(3)]
        src = None if q_hat is None else dptr(self._spec(q_hat))
        self._check(self.lib.qgn_physical_modal(self.ctx, src, *(dptr(a) for a in out)), "qgn_physical_modal")
        return tuple(out)

    def write_qp_modal(self, q_hat, rec_no: int, nt: int, directory: str = "."):
        """WriteQPmodal: q_mode/p_mode/J_mode.%09d.dat raw float64 physical fields (QGN_Module.f90:381-440)."""
        fields = self.physical_modal(q_hat)
        os.makedirs(directory, exist_ok=True)
        for prefix, arr in zip(("q_mode", "p_mode", "J_mode"), fields):
            path = os.path.join(directory, f"{prefix}.{nt:09d}.dat")
            np.ascontiguousarray(arr, dtype="<f8").tofile(path)
        return fields

    def cleanup(self):
        if getattr(self, "ctx", None):
            self.lib.qgn_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.cleanup()
        except Exception:
            pass

    # -- device-resident state ----------------------------------------------------------
    def set_state(self, q_hat, t: float, dt: float):
        q_hat = self._spec(q_hat)
        self._check(self.lib.qgn_set_state(self.ctx, dptr(q_hat), t, dt), "qgn_set_state")

    def get_state(self, q_hat=None):
        if q_hat is None:
            q_hat = np.empty(self.spectral_shape(), dtype=np.complex128)
        q_hat = self._spec(q_hat, writable=True)
        tt, dd = C.c_double(), C.c_double()
        self._check(self.lib.qgn_get_state(self.ctx, dptr(q_hat), C.byref(tt), C.byref(dd)), "qgn_get_state")
        self.t, self.dt = tt.value, dd.value
        return q_hat

    def advance_resident(self, nsteps: int):
        self._check(self.lib.qgn_advance_resident(self.ctx, int(nsteps)), "qgn_advance_resident")

    def time(self):
        tt, dd = C.c_double(), C.c_double()
        self._check(self.lib.qgn_get_time(self.ctx, C.byref(tt), C.byref(dd)), "qgn_get_time")
        return tt.value, dd.value

    # -- parity hooks and diagnostics ---------------------------------------------------
    def get_rhs(self, q_hat):
        q_hat = self._spec(q_hat)
        out = np.empty(self.spectral_shape(), dtype=np.complex128)
        self._check(self.lib.qgn_rhs(self.ctx, dptr(q_hat), dptr(out)), "qgn_rhs")
        return out

    def get_psi(self, q_hat):
        q_hat = self._spec(q_hat)
        out = np.empty(self.spectral_shape(), dtype=np.complex128)
        self._check(self.lib.qgn_psi(self.ctx, dptr(q_hat), dptr(out)), "qgn_psi")
        return out

    def leith(self):
        out = np.empty(self.nz)
        self._check(self.lib.qgn_leith(self.ctx, dptr(out)), "qgn_leith")
        return out

    def physical(self, q_hat=None):
        qp = np.empty(self.physical_shape())
        pp = np.empty(self.physical_shape())
        src = None if q_hat is None else dptr(self._spec(q_hat))
        self._check(self.lib.qgn_physical(self.ctx, src, dptr(qp), dptr(pp)), "qgn_physical")
        return qp, pp

    def diagnostics(self, nbins: int = 0):
        ke = np.empty(self.nz)
        spec = np.empty((self.nz, nbins)) if nbins > 0 else None
        self._check(self.lib.qgn_diagnostics(self.ctx, dptr(ke), None if spec is None else dptr(spec), int(nbins)),
                    "qgn_diagnostics")
        return ke, spec

    def energetics(self):
        """Per-layer (KE, APE, enstrophy) of the resident state, each weighted by H_k/Htot."""
        out = [np.empty(self.nz) for _ in range(3)]
        self._check(self.lib.qgn_energetics(self.ctx, *(dptr(a) for a in out)), "qgn_energetics")
        return tuple(out)

    def rejects(self):
        n = C.c_longlong()
        self._check(self.lib.qgn_rejects(self.ctx, C.byref(n)), "qgn_rejects")
        return n.value


class QGNEnsemble:
    """Independent members advanced together with BSRK3 (BSRK3.f90), one launch per pass.

    ``members`` are ``QGNModule`` instances made with ``scheme="bsrk3"`` (FP64 contexts;
    nx, ny in {128, 256, 512}, nz in 2..8 or 16, C_d = 0).  The ensemble borrows their
    device state: load states with ``member.set_state`` and read them with
    ``member.get_state``.  ``precision="mixed"`` runs transforms, stage right-hand sides
    and stage inputs in FP32 with FP64 state, stage sums, GetPsi, error norm and controller.
    """

    PASSES = ("yinv", "xpass", "yfwd")

    def __init__(self, members, precision: str = "mixed"):
        self.lib = _lib.load()
        self.members = list(members)
        n = len(self.members)
        arr = (C.c_void_p * n)(*[m.ctx.value for m in self.members])
        ens = C.c_void_p()
        rc = self.lib.qgn_ens_create(arr, n, _lib.PRECISIONS[precision], C.byref(ens))
        if rc != 0:
            raise QGNError(rc, f"qgn_ens_create({n} members, precision={precision})")
        self.ens = ens
        self.precision = precision

    def _check(self, rc, what):
        if rc != 0:
            msg = self.lib.qgn_ens_last_error(self.ens)
            raise QGNError(rc, f"{what}: {msg.decode() if msg else ''}")

    def advance(self, nsteps: int):
        """Every member takes ``nsteps`` accepted steps."""
        self._check(self.lib.qgn_ens_advance(self.ens, int(nsteps)), "qgn_ens_advance")

    def stream(self):
        """The ensemble's cudaStream_t (as an integer handle)."""
        sp = C.c_void_p()
        self._check(self.lib.qgn_ens_stream(self.ens, C.byref(sp)), "qgn_ens_stream")
        return sp.value

    def tuning(self):
        """The autotuner's choice per right-hand-side pass."""
        out = {}
        for i, name in enumerate(self.PASSES):
            th, cps, ms = C.c_int(), C.c_int(), C.c_float()
            self._check(self.lib.qgn_ens_tuning(self.ens, i, C.byref(th), C.byref(cps), C.byref(ms)),
                        "qgn_ens_tuning")
            rad = C.c_int()
            self._check(self.lib.qgn_ens_fft_radix(self.ens, i, C.byref(rad)), "qgn_ens_fft_radix")
            out[name] = {"threads": th.value, "ctas_per_sm": cps.value, "ms": ms.value,
                         "elements_per_thread": rad.value}
        return out

    def set_tiles(self, pass_name: str, threads: int, elements_per_thread: int, ctas_per_sm: int = 0):
        """Pin a right-hand-side pass to one tile variant (the autotuner then leaves it alone)."""
        i = self.PASSES.index(pass_name)
        self._check(self.lib.qgn_ens_set_tiles(self.ens, i, int(threads), int(elements_per_thread),
                                               int(ctas_per_sm)), "qgn_ens_set_tiles")

    def profile_enable(self, on: bool = True):
        self._check(self.lib.qgn_ens_profile_enable(self.ens, int(bool(on))), "qgn_ens_profile_enable")

    def profile_read(self):
        out = {}
        for k in range(_lib.QGN_KERNEL_FAMILIES):
            ms, nb = C.c_double(), C.c_double()
            timed, launches = C.c_longlong(), C.c_longlong()
            self._check(self.lib.qgn_ens_profile_read(self.ens, k, C.byref(ms), C.byref(nb), C.byref(timed),
                                                      C.byref(launches)), "qgn_ens_profile_read")
            if launches.value:
                out[self.lib.qgn_kernel_name(k).decode()] = {"ms": ms.value, "bytes": nb.value,
                                                            "timed": timed.value, "launches": launches.value}
        return out

    def close(self):
        if getattr(self, "ens", None):
            self.lib.qgn_ens_destroy(self.ens)
            self.ens = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
