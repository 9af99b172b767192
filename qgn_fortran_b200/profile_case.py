"""Small fixed workload for profiler captures (ncu) and quick timing.

    python -m qgn_fortran_b200.profile_case --workload strat1024x8 --steps 1

Builds the named workload, sets the seeded IC on the GPU and advances ``--steps``
device-resident TimeSteps, then prints the per-kernel-family launch counts and CUDA-event
times of those steps.  Device memory held: the model's working set only (about 0.7 GB for
strat1024x8).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time

from . import QGNModule, _lib
from .inputs import workload


def kernel_table(g):
    out = {}
    for k in range(_lib.QGN_KERNEL_FAMILIES):
        tot, nb = C.c_double(), C.c_double()
        nt, nl = C.c_longlong(), C.c_longlong()
        g.lib.qgn_profile_read(g.ctx, k, C.byref(tot), C.byref(nb), C.byref(nt), C.byref(nl))
        if nl.value:
            name = g.lib.qgn_kernel_name(k).decode()
            gbs = (nb.value / (tot.value / 1000.0) / 1e9) if tot.value > 0 else None
            out[name] = {"launches": nl.value, "ms": round(tot.value, 4),
                         "algorithmic_GBps": round(gbs, 1) if gbs else None}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="strat1024x8")
    ap.add_argument("--nx", type=int, default=None)
    ap.add_argument("--nz", type=int, default=None)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--precision", default="fp64")
    a = ap.parse_args()
    w = workload(a.workload, nx=a.nx, nz=a.nz)
    g = QGNModule(w.params, w.H, w.S, w.U, scheme=w.scheme, precision=a.precision)
    g.initialize(w.qp, 0.0, w.dt0)
    g.lib.qgn_profile_enable(g.ctx, 1)
    t0 = time.perf_counter()
    g.advance_resident(a.steps)
    wall = time.perf_counter() - t0
    t, dt = g.time()
    print(json.dumps({"workload": a.workload, "steps": a.steps, "wall_ms": 1000 * wall, "t": t, "dt": dt,
                      "kernels": kernel_table(g)}))
    g.cleanup()


if __name__ == "__main__":
    main()
