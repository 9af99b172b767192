"""Spin a named workload up on the GPU and save the equilibrated state.

    python -m qgn_fortran_b200.spinup --workload strat1024x8 --years 10 --out DIR

The named workload's seeded initial condition is advanced with its own scheme and PI.3.4
controller (device-resident graph steps) for ``--years`` model years.  Written to DIR:

* ``q.%09d.dat`` -- the physical PV field real(dp) q(nx,ny,nz), the reference's restart file
  (QGN_Driver.f90:21-30; the step number is the number of steps taken);
* ``<workload>_spinup.npz`` -- the same state as the modes DeAlias keeps (QGN_Module.f90:194-204),
  stored compactly for a fixture: the top 16 bits of each FP32 real and imaginary part
  (bfloat16 rounding), with the simulated time, the last dt and the step count.
  ``inputs.spunup_pv`` turns it back into a physical field.

The configuration being spun up (BASELINE config "strat1024x8": 10 model years of spin-up) is
what the benchmark's timing window starts from.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import QGNModule
from .inputs import qp_filename, workload

YEAR = 365.0 * 86400.0


def to_bf16_bits(a: np.ndarray) -> np.ndarray:
    """float32 -> upper 16 bits, rounded to nearest even (bfloat16 as uint16)."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return r.astype(np.uint16)


def kept_modes(q_hat: np.ndarray, nx: int, ny: int) -> np.ndarray:
    """The modes DeAlias keeps, [nz][nky][nkx] with nky rows ky index < ny/3 then > 2(ny/3)."""
    nkx = nx // 3
    rows = np.r_[0:ny // 3, 2 * (ny // 3) + 1:ny]
    return q_hat[:, rows, :nkx]


def run(name: str, years: float, out: str, chunk: int = 200) -> dict:
    w = workload(name)
    g = QGNModule(w.params, w.H, w.S, w.U, scheme=w.scheme)
    g.initialize(w.qp, 0.0, w.dt0)
    steps = 0
    c0 = time.perf_counter()
    t, dt = 0.0, w.dt0
    while t < years * YEAR:
        g.advance_resident(chunk)
        steps += chunk
        t, dt = g.time()
    wall = time.perf_counter() - c0
    q_hat = g.get_state()
    qp, _ = g.physical()
    ke = g.energetics()[0]
    g.cleanup()
    os.makedirs(out, exist_ok=True)
    np.ascontiguousarray(qp, dtype="<f8").tofile(os.path.join(out, qp_filename(steps)))
    k = kept_modes(q_hat, w.params["nx"], w.params["ny"])
    np.savez_compressed(os.path.join(out, f"{name}_spinup.npz"),
                        re=to_bf16_bits(k.real), im=to_bf16_bits(k.imag),
                        meta=json.dumps({"workload": name, "years": years, "t": t, "dt": dt, "steps": steps,
                                         "nx": w.params["nx"], "ny": w.params["ny"], "nz": w.params["nz"],
                                         "TOL": w.params["TOL"],
                                         "ke_layer": [float(x) for x in ke]}))
    return {"workload": name, "years": years, "t": t, "dt": dt, "steps": steps, "wall_s": wall,
            "ke_layer": [float(x) for x in ke]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="strat1024x8")
    ap.add_argument("--years", type=float, default=10.0)
    ap.add_argument("--out", default=".")
    a = ap.parse_args()
    print(json.dumps(run(a.workload, a.years, a.out)), flush=True)


if __name__ == "__main__":
    main()
