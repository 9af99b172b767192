"""Generate the committed golden fixtures from the FP64 oracle (oracle/qgn_oracle.py).

Run from the repository root:  python tests/golden/make_golden.py
Each case stores its inputs (parameters, profiles, the spectral state) and the oracle's
outputs: one GetRHS, GetPsi, the QG-Leith coefficients and a short trajectory of one
scheme with its (t, dt) sequence.
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.qgn_oracle import Params, QGNOracle, SCHEMES  # noqa: E402
from qgn_fortran_b200.inputs import exponential_stratification, phillips_two_layer, seeded_random_pv  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

CASES = [
    # name, nx, ny, nz, Lx, Ly, profile, extra params, scheme, dt0, nsteps
    ("phillips32_ark43", 32, 32, 2, 1.0e6, 1.0e6, "phillips",
     dict(beta=1.6e-11, A8=1.0 / (86400.0 * (np.pi * 32 / 1.0e6) ** 8), C_d=0.0, TOL=1e30, dt_max=900.0),
     "ark43", 900.0, 5),
    ("strat64x4_qgleith", 64, 64, 4, 2.0e6, 2.0e6, "strat",
     dict(C_d=1.0e-5, TOL=4.0e-13), "ark43_qgleith", 60000.0, 5),
    ("rect64x32x3_bsrk3", 64, 32, 3, 2.0e6, 1.0e6, "strat",
     dict(C_d=2.0e-5, TOL=1.0e-12, is_explicit=True, A8=1.0e20, A2=5.0), "bsrk3", 30000.0, 5),
    ("strat32x2_rk4", 32, 32, 2, 1.0e6, 1.0e6, "strat", dict(C_d=0.0), "rk4", 1200.0, 4),
    ("rect32x64x5_ab3", 32, 64, 5, 1.5e6, 3.0e6, "strat",
     dict(C_d=1.0e-5, is_explicit=True, A8=5.0e19), "ab3", 900.0, 5),
]


def build_case(name, nx, ny, nz, Lx, Ly, prof, extra, scheme, dt0, nsteps):
    if prof == "phillips":
        H, S, U = phillips_two_layer()
        Htot = 4000.0
    else:
        H, S, U = exponential_stratification(nz)
        Htot = 4000.0
    p = Params(nx=nx, ny=ny, nz=nz, Lx=Lx, Ly=Ly, Htot=Htot, **extra)
    m = QGNOracle(p, H, S, U)
    qp = seeded_random_pv(nx, ny, nz, 6.0, 1.0e-6, seed=sum(map(ord, name)))
    q0 = m.initialize_spec(qp)
    rhs = m.get_rhs(q0)
    psi = m.get_psi(q0)
    a8l = m.leith_A8L(q0)
    st = SCHEMES[scheme](m)
    q = q0.copy()
    t, dt = 0.0, dt0
    ts, dts = [], []
    for _ in range(nsteps):
        q, t, dt = st.step(q, t, dt)
        ts.append(t)
        dts.append(dt)
    rejects = int(getattr(st, "rejects", 0))
    meta = dict(name=name, params=p.__dict__, scheme=scheme, dt0=dt0, nsteps=nsteps, rejects=rejects)
    return dict(meta=np.array(json.dumps(meta)), H=np.asarray(H, float), S=np.asarray(S, float),
                U=np.asarray(U, float), qp=qp, q0=q0, rhs=rhs, psi=psi, a8l=a8l,
                qfinal=q, t=np.array(ts), dt=np.array(dts))


def main():
    for c in CASES:
        d = build_case(*c)
        np.savez_compressed(os.path.join(HERE, c[0] + ".npz"), **d)
        print("wrote", c[0], json.loads(str(d["meta"]))["rejects"], "rejects", d["dt"])


if __name__ == "__main__":
    main()
