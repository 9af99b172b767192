"""Programmatic dependent launch changes when kernels are scheduled, never what they compute.

Each case runs the same steps twice, with the programmatic-serialization launch attribute
(the default) and with QGN_NO_PDL=1, and requires bit-identical states and times.  A kernel
that read its predecessor's output before griddepcontrol.wait would race and differ.
"""
import numpy as np
import pytest

from qgn_fortran_b200 import QGNEnsemble, QGNModule
from qgn_fortran_b200 import closure as cl
from qgn_fortran_b200.inputs import ensemble_members, workload

pytestmark = pytest.mark.gpu


def run_model(n, nz, scheme, precision, steps, closure=False):
    w = workload("strat1024x8", nx=n, nz=nz)
    g = QGNModule(w.params, w.H, w.S, w.U, scheme=scheme, precision=precision)
    g.initialize(w.qp, 0.0, 3000.0)
    if closure:
        net = cl.ClosureNet(nz=nz, H=n, W=n, layers=3, max_batch=1, seed=5)
        rng = np.random.default_rng(5)
        net.set_weights([(1e-3 * rng.standard_normal(a.shape).astype(np.float32), b)
                         for a, b in net.get_weights()])
        cl.attach(g, net, np.ones(2 * nz), np.full(nz, 1e9), A8_background=w.params["A8"], energy_limit=1.0)
    g.advance_resident(steps)
    out = g.get_state(), g.time()
    g.cleanup()
    return out


@pytest.mark.parametrize("n,nz,scheme,precision,closure", [
    (128, 4, "ark43_qgleith", "fp64", False),
    (256, 3, "ark43_qgleith", "mixed", False),
    (128, 4, "ark43_qgleith", "fp64", True),
    (128, 2, "bsrk3", "fp64", False),
    (128, 2, "rk4", "fp64", False),
])
def test_pdl_is_bit_identical(cuda_ok, monkeypatch, n, nz, scheme, precision, closure):
    qa, ta = run_model(n, nz, scheme, precision, 6, closure)
    monkeypatch.setenv("QGN_NO_PDL", "1")
    qb, tb = run_model(n, nz, scheme, precision, 6, closure)
    assert ta == tb
    assert np.array_equal(qa, qb)


def test_pdl_ensemble_is_bit_identical(cuda_ok, monkeypatch):
    monkeypatch.setenv("QGN_NO_AUTOTUNE", "1")   # the same tile widths in both runs

    def go():
        ws = ensemble_members(4, sizes=(128, 256), layers=(2, 3))
        gs = [QGNModule(w.params, w.H, w.S, w.U, scheme="bsrk3") for w in ws]
        for g, w in zip(gs, ws):
            g.initialize(w.qp, 0.0, w.dt0)
        QGNEnsemble(gs, precision="mixed").advance(5)
        return [(g.get_state(), g.time()) for g in gs]

    a = go()
    monkeypatch.setenv("QGN_NO_PDL", "1")
    b = go()
    for (qa, ta), (qb, tb) in zip(a, b):
        assert ta == tb
        assert np.array_equal(qa, qb)
