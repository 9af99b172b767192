"""Ensembles of heterogeneous members (BSRK3) on the GPU.

The FP64 ensemble runs each member through the same arithmetic as a single context's
BSRK3 step, so its trajectories must equal single-context runs (which the parity suite ties
to the oracle); the mixed ensemble is checked against the FP64 oracle at fixed dt and
against the FP64 ensemble with adaptive dt.
"""
import math
import os

import numpy as np
import pytest

from oracle.qgn_oracle import BSRK3, Params, QGNOracle
from qgn_fortran_b200 import QGNEnsemble, QGNModule
from qgn_fortran_b200._lib import QGN_ERR_ARG, QGN_ERR_CONFIG, QGN_ERR_NONFINITE, QGNError
from qgn_fortran_b200.inputs import Workload, ensemble_members, exponential_stratification, seeded_random_pv

pytestmark = pytest.mark.gpu


def layer_rel(a, b):
    num = np.sqrt(np.sum(np.abs(a - b) ** 2, axis=(1, 2)))
    den = np.sqrt(np.sum(np.abs(b) ** 2, axis=(1, 2)))
    return num / np.where(den > 0, den, 1.0)


def rect_member(nx, ny, nz, seed, **kw):
    """A member with nx != ny (Ly scaled with ny/nx)."""
    H, S, U = exponential_stratification(nz, N_efold=800.0, U0=0.08, U_efold=800.0)
    Lx = 2.0e6
    qp = seeded_random_pv(nx, ny, nz, 8.0, 1.0e-6, seed)
    p = dict(nx=nx, ny=ny, nz=nz, Lx=Lx, Ly=Lx * ny / nx, Htot=4000.0, f0=1.0e-4, beta=2.0e-11, A2=0.0,
             A8=1.0 / (86400.0 * (math.pi * nx / Lx) ** 8), r0=1.0e-7, C_d=0.0,
             TOL=1.0e-6 * float(np.max(np.abs(qp))), is_explicit=True, dt_max=math.pi / (2.0e-11 * Lx))
    p.update(kw)
    return Workload(f"rect{nx}x{ny}x{nz}", p, H, S, U, qp, "bsrk3", 1800.0)


def small_set(fixed_dt=False):
    ws = ensemble_members(5, sizes=(128, 256), layers=(2, 3, 4))
    ws.append(rect_member(256, 128, 3, 77))
    ws.append(rect_member(128, 512, 2, 78))
    if fixed_dt:
        for w in ws:
            w.params["TOL"] = 1.0e30
            w.params["dt_max"] = 1800.0
    return ws


def contexts(ws):
    gs = [QGNModule(w.params, w.H, w.S, w.U, scheme="bsrk3") for w in ws]
    q0 = [g.initialize(w.qp, 0.0, w.dt0) for g, w in zip(gs, ws)]
    return gs, q0


def single_run(w, q0, nsteps):
    g = QGNModule(w.params, w.H, w.S, w.U, scheme="bsrk3")
    q = q0.copy()
    t, dt = 0.0, w.dt0
    for _ in range(nsteps):
        t, dt = g.time_step(q, t, dt)
    return q, t, dt


def test_fp64_ensemble_equals_single_contexts(cuda_ok):
    ws = small_set()
    gs, q0 = contexts(ws)
    ens = QGNEnsemble(gs, precision="fp64")
    ens.advance(4)
    ens.advance(3)      # the FSAL RHS0 and the captured graph carry over between calls
    tune = ens.tuning()
    radix16 = all(v["elements_per_thread"] == 16 for v in tune.values())
    for w, g, q in zip(ws, gs, q0):
        got = g.get_state()
        t, dt = g.time()
        ref, tr, dr = single_run(w, q, 7)
        # a single context transforms 512- and 1024-point y columns with 8 elements per thread
        # and rows with 32, the ensemble's tiles with 16 unless the autotuner chose 8 or 32: the
        # same transform with another radix schedule, whose roundoff the adaptive dt carries
        # along (the adaptive tolerance of the oracle comparisons)
        if max(w.params["nx"], w.params["ny"]) >= 512:
            tol = 1e-9
        else:
            tol = 1e-13 if radix16 else 1e-11
        assert np.all(layer_rel(got, ref) <= tol), w.name
        assert t == pytest.approx(tr, rel=tol) and dt == pytest.approx(dr, rel=tol), w.name
    assert tune["yinv"]["threads"] in (64, 128, 256)
    assert tune["xpass"]["threads"] in (96, 192, 384)
    assert tune["yfwd"]["threads"] in (64, 128, 256)


def test_fp64_ensemble_member_against_oracle(cuda_ok):
    w = rect_member(128, 256, 3, 91)
    gs, q0 = contexts([w])
    QGNEnsemble(gs, precision="fp64").advance(3)
    m = QGNOracle(Params(**w.params), w.H, w.S, w.U)
    st = BSRK3(m)
    q, t, dt = q0[0].copy(), 0.0, w.dt0
    for _ in range(3):
        q, t, dt = st.step(q, t, dt)
    assert np.all(layer_rel(gs[0].get_state(), q) <= 1e-9)
    assert gs[0].time()[0] == pytest.approx(t, rel=1e-9)


def test_mixed_ensemble_fixed_dt_against_oracle(cuda_ok):
    """FP32 transforms and stage storage, FP64 state and stage sums: 10 fixed-dt steps."""
    ws = small_set(fixed_dt=True)[:4]
    gs, q0 = contexts(ws)
    QGNEnsemble(gs, precision="mixed").advance(10)
    for w, g, q in zip(ws, gs, q0):
        m = QGNOracle(Params(**w.params), w.H, w.S, w.U)
        st = BSRK3(m)
        qq, t, dt = q.copy(), 0.0, w.dt0
        for _ in range(10):
            qq, t, dt = st.step(qq, t, dt)
        err = layer_rel(g.get_state(), qq)
        assert np.all(err <= 2e-5), (w.name, err)
        assert g.time()[0] == pytest.approx(t, rel=1e-12)


def test_mixed_ensemble_adaptive_against_fp64(cuda_ok):
    ws = small_set()
    g64, q0 = contexts(ws)
    g32, _ = contexts(ws)
    QGNEnsemble(g64, precision="fp64").advance(6)
    QGNEnsemble(g32, precision="mixed").advance(6)
    for w, a, b in zip(ws, g32, g64):
        ta, tb = a.time()[0], b.time()[0]
        assert ta == pytest.approx(tb, rel=0.05), w.name
        assert np.all(layer_rel(a.get_state(), b.get_state()) <= 5e-2), w.name


def test_graph_equals_eager(cuda_ok, monkeypatch):
    ws = small_set()[:4]
    ga, q0 = contexts(ws)
    QGNEnsemble(ga, precision="mixed").advance(4)
    monkeypatch.setenv("QGN_NO_GRAPHS", "1")
    gb, _ = contexts(ws)
    eb = QGNEnsemble(gb, precision="mixed")
    eb.profile_enable(True)
    eb.advance(4)
    prof = eb.profile_read()
    monkeypatch.delenv("QGN_NO_GRAPHS")
    for a, b in zip(ga, gb):
        assert np.array_equal(a.get_state(), b.get_state())
        assert a.time() == b.time()
    for fam in ("yinv", "xpass", "yfwd", "ark_stage"):
        assert prof[fam]["launches"] > 0 and prof[fam]["timed"] > 0


def test_halted_member_does_not_stop_the_others(cuda_ok):
    ws = small_set()[:3]
    gs, q0 = contexts(ws)
    bad = q0[1].copy()
    bad[0, 3, 2] = np.nan
    gs[1].set_state(bad, 0.0, ws[1].dt0)
    ens = QGNEnsemble(gs, precision="mixed")
    with pytest.raises(QGNError) as ei:
        ens.advance(3)
    assert ei.value.code == QGN_ERR_NONFINITE and "member 1" in str(ei.value)
    for i in (0, 2):
        t, dt = gs[i].time()
        assert t > 0 and math.isfinite(t)
        assert np.all(np.isfinite(gs[i].get_state()))


def test_create_rejects_unsupported_members(cuda_ok):
    w = small_set()[0]
    rk4 = QGNModule(w.params, w.H, w.S, w.U, scheme="rk4")
    with pytest.raises(QGNError) as ei:
        QGNEnsemble([rk4])
    assert ei.value.code == QGN_ERR_CONFIG
    small = rect_member(64, 64, 2, 5)
    g64 = QGNModule(small.params, small.H, small.S, small.U, scheme="bsrk3")
    with pytest.raises(QGNError) as ei:
        QGNEnsemble([g64])
    assert ei.value.code == QGN_ERR_CONFIG
    g = QGNModule(w.params, w.H, w.S, w.U, scheme="bsrk3")
    with pytest.raises(QGNError) as ei:
        QGNEnsemble([g, g])
    assert ei.value.code == QGN_ERR_ARG


# every tile variant the autotuner can choose (qgn_ens_set_tiles): CTA threads, elements per thread
VARIANTS = {
    "fp64": {"yinv": [(64, 16), (128, 16), (256, 16), (64, 8), (128, 8), (256, 8)],
             "xpass": [(96, 16), (192, 16), (384, 16), (192, 8), (384, 8)],
             "yfwd": [(64, 16), (128, 16), (256, 16), (128, 8), (256, 8)]},
    "mixed": {"yinv": [(64, 16), (128, 16), (256, 16), (64, 8), (128, 8), (256, 8), (64, 32), (128, 32),
                       (256, 32)],
              "xpass": [(96, 16), (192, 16), (384, 16), (192, 8), (384, 8), (96, 32), (192, 32), (384, 32)],
              "yfwd": [(64, 16), (128, 16), (256, 16), (128, 8), (256, 8), (64, 32), (128, 32)]},
}


def variant_set():
    """128-, 256- and 512-point transforms along both x and y, fixed dt."""
    ws = [rect_member(128, 128, 2, 81), rect_member(512, 128, 2, 82), rect_member(128, 512, 3, 83),
          rect_member(256, 256, 2, 84)]
    for w in ws:
        w.params["TOL"] = 1.0e30
        w.params["dt_max"] = 1800.0
    return ws


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_every_tile_variant_matches(cuda_ok, monkeypatch, precision):
    """Each pass pinned to each of its tile variants (the others at their defaults, no tuning):
    FP64 equals single-context runs within the roundoff of another radix schedule, and the mixed
    ensemble its own default variant within FP32 roundoff; the pinned choice is reported back."""
    monkeypatch.setenv("QGN_NO_AUTOTUNE", "1")
    ws = variant_set()
    nsteps = 2
    if precision == "fp64":
        _, q0 = contexts(ws)
        refs = [single_run(w, q, nsteps)[0] for w, q in zip(ws, q0)]
        tol = 1e-12
    else:
        gs, _ = contexts(ws)
        QGNEnsemble(gs, precision="mixed").advance(nsteps)
        refs = [g.get_state() for g in gs]
        tol = 1e-5
    for pname, variants in VARIANTS[precision].items():
        for threads, ept in variants:
            gs, _ = contexts(ws)
            ens = QGNEnsemble(gs, precision=precision)
            ens.set_tiles(pname, threads, ept)
            ens.advance(nsteps)
            tune = ens.tuning()[pname]
            assert (tune["threads"], tune["elements_per_thread"]) == (threads, ept)
            for w, g, ref in zip(ws, gs, refs):
                err = layer_rel(g.get_state(), ref)
                assert np.all(err <= tol), (pname, threads, ept, w.name, err)
    gs, _ = contexts(ws)
    ens = QGNEnsemble(gs, precision=precision)
    with pytest.raises(QGNError) as ei:
        ens.set_tiles("yfwd", 64, 8)          # two 512-point transforms need 128 threads
    assert ei.value.code == QGN_ERR_CONFIG
