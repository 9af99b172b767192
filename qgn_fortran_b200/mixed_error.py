"""Per-field error of the mixed-precision mode against the FP64 path, for one named workload.

    python -m qgn_fortran_b200.mixed_error --workload strat2048x16 [--steps 100] [--years 1]

Both modes start from the same seeded initial condition (transformed and dealiased on the GPU in
FP64).  Reported, each as the largest per-layer relative L2 (or relative difference) over layers:

* ``rhs``: one GetRHS (QGN_Module.f90:258-296) of the initial state;
* ``fixed_steps``: the spectral state after ``--steps`` ARK43_QGLeith steps at a fixed dt
  (TOL = 1e30, so the PI.3.4 controller clips every step to dt_max = ``--dt``);
* ``ke_layer`` and ``ke_spectrum``: layer kinetic energy and the isotropic KE spectrum (shells
  with at least 1e-6 of the layer's energy) of those two states;
* with ``--years`` > 0, ``time_mean``: the same two diagnostics averaged over daily samples of
  adaptive runs (PI.3.4, the workload's TOL) of that length.  The runs separate after the
  predictability horizon, so this compares statistics, not states.

The FP64 path's own error against the reference's arithmetic is the parity suite's business
(tests/); this module needs only the GPU library.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import QGNModule
from .inputs import workload

DAY = 86400.0


def layer_rel(a, b):
    num = np.sqrt(np.sum(np.abs(a - b) ** 2, axis=(1, 2)))
    den = np.sqrt(np.sum(np.abs(b) ** 2, axis=(1, 2)))
    return num / np.where(den > 0, den, 1.0)


def spectrum_rel(a, b, floor=1e-6):
    """Largest relative difference over the shells that hold at least `floor` of a layer's KE."""
    keep = b >= floor * b.sum(axis=1, keepdims=True)
    return float(np.max(np.abs(a - b)[keep] / b[keep]))


def _pair(w, params):
    return (QGNModule(params, w.H, w.S, w.U, scheme=w.scheme, precision="fp64"),
            QGNModule(params, w.H, w.S, w.U, scheme=w.scheme, precision="mixed"))


def error_table(name="strat2048x16", steps=100, dt=3600.0, years=0.0, nbins=None):
    w = workload(name)
    nb = nbins or w.params["nx"] // 2
    out = {"workload": name, "grid": [w.params["nx"], w.params["ny"], w.params["nz"]]}

    g64, g32 = _pair(w, w.params)
    q = g64.initialize(w.qp, 0.0, w.dt0)
    out["rhs"] = float(np.max(layer_rel(g32.get_rhs(q), g64.get_rhs(q))))
    g64.cleanup()
    g32.cleanup()

    fixed = dict(w.params, TOL=1.0e30, dt_max=dt)
    g64, g32 = _pair(w, fixed)
    for g in (g64, g32):
        g.initialize(w.qp, 0.0, dt)
        g.advance_resident(steps)
    a, b = g32.get_state(), g64.get_state()
    out["fixed_steps"] = {"steps": steps, "dt_s": dt, "state": float(np.max(layer_rel(a, b)))}
    ke32, sp32 = g32.diagnostics(nb)
    ke64, sp64 = g64.diagnostics(nb)
    out["fixed_steps"]["ke_layer"] = float(np.max(np.abs(ke32 - ke64) / ke64))
    out["fixed_steps"]["ke_spectrum"] = spectrum_rel(sp32, sp64)
    g64.cleanup()
    g32.cleanup()

    if years > 0:
        res = {}
        for prec in ("fp64", "mixed"):
            g = QGNModule(w.params, w.H, w.S, w.U, scheme=w.scheme, precision=prec)
            g.initialize(w.qp, 0.0, w.dt0)
            t_end = years * 365.0 * DAY
            ke_sum, sp_sum, n = 0.0, 0.0, 0
            t, nxt = 0.0, DAY
            c0 = time.perf_counter()
            while t < t_end:
                g.advance_resident(10)
                t, _ = g.time()
                if t >= nxt:
                    ke, sp = g.diagnostics(nb)
                    ke_sum, sp_sum, n = ke_sum + ke, sp_sum + sp, n + 1
                    nxt += DAY
            res[prec] = (ke_sum / n, sp_sum / n, n, time.perf_counter() - c0)
            g.cleanup()
        (k64, s64, n64, w64), (k32, s32, n32, w32) = res["fp64"], res["mixed"]
        out["time_mean"] = {"years": years, "samples": [n64, n32], "wall_s": [w64, w32],
                            "ke_layer": float(np.max(np.abs(k32 - k64) / k64)),
                            "ke_spectrum": spectrum_rel(s32, s64)}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="strat2048x16")
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--dt", type=float, default=3600.0)
    ap.add_argument("--years", type=float, default=0.0)
    a = ap.parse_args()
    print(json.dumps(error_table(a.workload, a.steps, a.dt, a.years)), flush=True)


if __name__ == "__main__":
    main()
