"""Small-grid ARK43 steps with the column kernels against the separate kernels.

On grids of at most 2^17 kept mode-layers an attempt runs stage s, GetPsi and the y-inverse of
its RHS in one launch per kx column, and (without quadratic drag) the y-forward pass of the
previous RHS in the same launch.  The formulas are those of the separate kernels, but the
compiler is free to contract them into fused multiply-adds differently, so the two paths agree
to roundoff (about 1e-17 relative per step), which the adaptive controller carries into dt:
the comparison uses the adaptive tolerance of the oracle tests.
"""
import numpy as np
import pytest

from qgn_fortran_b200 import QGNModule
from qgn_fortran_b200 import closure as cl
from qgn_fortran_b200.inputs import workload

pytestmark = pytest.mark.gpu


def run(n, nz, scheme, steps, drag=False, closure=False):
    w = workload("strat1024x8", nx=n, nz=nz)
    params = dict(w.params)
    if drag:
        params["C_d"] = 1.0e-5
    g = QGNModule(params, w.H, w.S, w.U, scheme=scheme)
    g.initialize(w.qp, 0.0, 3000.0)
    if closure:
        net = cl.ClosureNet(nz=nz, H=n, W=n, layers=3, max_batch=1, seed=5)
        rng = np.random.default_rng(5)
        net.set_weights([(1e-3 * rng.standard_normal(a.shape).astype(np.float32), b)
                         for a, b in net.get_weights()])
        cl.attach(g, net, np.ones(2 * nz), np.full(nz, 1e9), A8_background=w.params["A8"], energy_limit=1.0)
    g.advance_resident(steps)
    out = g.get_state(), g.time(), g.rejects()
    g.cleanup()
    return out


@pytest.mark.parametrize("n,nz,scheme,drag,closure", [
    (128, 4, "ark43_qgleith", False, False),
    (128, 8, "ark43", False, False),
    (256, 2, "ark43_qgleith", False, False),
    (128, 4, "ark43_qgleith", True, False),
    (128, 4, "ark43_qgleith", False, True),
])
def test_fused_stage_matches_separate_kernels(cuda_ok, monkeypatch, n, nz, scheme, drag, closure):
    qa, ta, ra = run(n, nz, scheme, 8, drag, closure)
    monkeypatch.setenv("QGN_NO_FUSED_STAGE", "1")
    qb, tb, rb = run(n, nz, scheme, 8, drag, closure)
    assert ra == rb
    assert ta[0] == pytest.approx(tb[0], rel=1e-9) and ta[1] == pytest.approx(tb[1], rel=1e-9)
    num = np.sqrt(np.sum(np.abs(qa - qb) ** 2, axis=(1, 2)))
    den = np.sqrt(np.sum(np.abs(qb) ** 2, axis=(1, 2)))
    assert np.all(num <= 1e-9 * den)
