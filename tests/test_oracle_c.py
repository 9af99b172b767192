"""The C / OpenMP restatement (oracle/qgn_ref.c) agrees with the numpy restatement."""
import json
import glob
import os

import numpy as np
import pytest

from oracle.qgn_oracle import Params, QGNOracle, SCHEMES
from oracle.qgn_ref_c import RefC
from qgn_fortran_b200.inputs import exponential_stratification, seeded_random_pv

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def layer_rel(a, b):
    num = np.sqrt(np.sum(np.abs(a - b) ** 2, axis=(1, 2)))
    den = np.sqrt(np.sum(np.abs(b) ** 2, axis=(1, 2)))
    return num / np.where(den > 0, den, 1.0)


@pytest.mark.parametrize("nx,ny,nz,drag,expl", [(32, 32, 2, False, False), (64, 32, 3, True, True),
                                               (128, 128, 4, True, False)])
def test_c_rhs_matches_numpy(nx, ny, nz, drag, expl):
    H, S, U = exponential_stratification(nz)
    p = Params(nx=nx, ny=ny, nz=nz, Lx=2.0e6, Ly=2.0e6 * ny / nx, Htot=4000.0, C_d=1e-5 if drag else 0.0,
               is_explicit=expl, A2=3.0 if expl else 0.0, A8=1e20)
    m = QGNOracle(p, H, S, U)
    c = RefC(p, H, S, U)
    qp = seeded_random_pv(nx, ny, nz, 6.0, 1e-6, seed=4)
    q = m.initialize_spec(qp)
    assert np.all(layer_rel(c.initialize_spec(qp), q) <= 1e-14)
    assert np.all(layer_rel(c.get_rhs(q), m.get_rhs(q)) <= 1e-13)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))),
                         ids=lambda p: os.path.basename(p)[:-4])
def test_c_trajectory_matches_golden(path):
    d = np.load(path)
    meta = json.loads(str(d["meta"]))
    p = Params(**meta["params"])
    c = RefC(p, d["H"], d["S"], d["U"], scheme=meta["scheme"])
    q = np.ascontiguousarray(d["q0"]).copy()
    t, dt = 0.0, meta["dt0"]
    adaptive = meta["scheme"] in ("ark43_qgleith", "ark43", "bsrk3") and p.TOL < 1e20
    tol = 1e-9 if adaptive else 1e-11
    for k in range(meta["nsteps"]):
        t, dt = c.step(q, t, dt)
        assert t == pytest.approx(d["t"][k], rel=tol)
    assert np.all(layer_rel(q, d["qfinal"]) <= tol)
    assert c.rejects() == meta["rejects"]
