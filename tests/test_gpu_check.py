"""The bounds-checked debug build (libqgn_b200_check.so, -DQGN_CHECK).

Every index of the right-hand-side transforms and of GetPsi is tested against the length of the
array it addresses; an index out of range is skipped and counted (qgn_check_failures), nothing
traps.  This test runs small grids of every scheme, both precisions, drag and explicit
dissipation, WriteQPmodal's full-spectrum geometry and a two-member ensemble through the checked
build in a child process (a process loads one build of the library), asserts that no check failed
and that the checked build computes what the normal build computes in this process.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from qgn_fortran_b200 import QGNModule, _lib
from qgn_fortran_b200.inputs import exponential_stratification, seeded_random_pv

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = [  # nx, ny, nz, C_d, explicit, scheme, precision
    (64, 128, 3, 1.0e-5, True, "ark43_qgleith", "fp64"),
    (128, 128, 4, 0.0, False, "ark43_qgleith", "mixed"),
    (256, 256, 2, 1.0e-5, False, "rk4", "fp64"),
    (32, 64, 5, 0.0, True, "ab3", "fp64"),
    (512, 256, 2, 0.0, True, "bsrk3", "fp64"),
    (1024, 1024, 2, 1.0e-5, False, "ark43", "fp64"),
]

RUNNER = r'''
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from qgn_fortran_b200 import _lib
_lib.load(_lib.CHECK_LIB_PATH)
sys.path.insert(0, sys.argv[1] + "/tests")
from test_gpu_check import CASES, run_case, run_ensemble
out = [run_case(*c) for c in CASES] + [run_ensemble()]
json.dump(out, open(sys.argv[2], "w"))
'''


def _model(nx, ny, nz, C_d, expl, scheme, prec):
    H, S, U = exponential_stratification(nz)
    p = dict(nx=nx, ny=ny, nz=nz, Lx=2.0e6, Ly=2.0e6 * ny / nx, Htot=4000.0, beta=2.0e-11, A2=1.0 if expl else 0.0,
             A8=1.0e20, r0=1.0e-7, C_d=C_d, TOL=1.0e-12, is_explicit=expl, dt_max=2.0e4)
    g = QGNModule(p, H, S, U, scheme=scheme, precision=prec)
    q = g.initialize(seeded_random_pv(nx, ny, nz, 6.0, 1.0e-6, seed=nx + ny + nz), 0.0, 5000.0)
    return g, q


def run_case(nx, ny, nz, C_d, expl, scheme, prec):
    """RHS, three TimeSteps, diagnostics and (FP64) WriteQPmodal's fields of one small model."""
    g, q = _model(nx, ny, nz, C_d, expl, scheme, prec)
    rhs = g.get_rhs(q)
    t, dt = 0.0, 5000.0
    for _ in range(3):
        t, dt = g.time_step(q, t, dt)
    ke, spec = g.diagnostics(8)
    res = {"rhs_norm": float(np.linalg.norm(rhs)), "rhs_sum": complex(rhs.sum()).__repr__(),
           "q_norm": float(np.linalg.norm(q)), "t": t, "dt": dt, "ke": ke.tolist()}
    if prec == "fp64":
        res["jmode_norm"] = float(np.linalg.norm(g.physical_modal(q)[2]))
    n = _lib.C.c_longlong()
    assert g.lib.qgn_check_failures(g.ctx, _lib.C.byref(n)) == 0
    res["failures"] = n.value
    g.cleanup()
    return res


def run_ensemble():
    from qgn_fortran_b200 import QGNEnsemble
    gs = [_model(128, 128, 2, 0.0, True, "bsrk3", "fp64")[0], _model(256, 256, 4, 0.0, True, "bsrk3", "fp64")[0]]
    ens = QGNEnsemble(gs, precision="mixed")
    ens.advance(2)
    ens.close()
    fails = []
    for g in gs:
        n = _lib.C.c_longlong()
        assert g.lib.qgn_check_failures(g.ctx, _lib.C.byref(n)) == 0
        fails.append(n.value)
        g.cleanup()
    return {"ensemble_failures": fails}


def test_checked_build_finds_no_out_of_range_index(cuda_ok, tmp_path):
    assert os.path.exists(_lib.CHECK_LIB_PATH), "build the checked library: python -m qgn_fortran_b200.build --check"
    out = tmp_path / "checked.json"
    r = subprocess.run([sys.executable, "-c", RUNNER, ROOT, str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    checked = json.load(open(out))
    for c, res in zip(CASES, checked[:-1]):
        assert res["failures"] == 0, (c, res)
        want = run_case(*c)          # the normal build, in this process
        assert want["failures"] == -1
        for key in ("rhs_norm", "q_norm", "jmode_norm"):
            if key in want:
                assert res[key] == pytest.approx(want[key], rel=1e-13), (c, key)
        assert (res["t"], res["dt"]) == pytest.approx((want["t"], want["dt"]), rel=1e-12)
        assert np.allclose(res["ke"], want["ke"], rtol=1e-12)
    assert checked[-1]["ensemble_failures"] == [0, 0]
