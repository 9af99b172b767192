"""The learned-closure experiment: a 1024^2 x 4 truth run, its coarse-grained training data at
128^2, the network trained on the GPU, and 128^2 runs with QG-Leith and with the learned
closure compared against the coarse-grained truth on the KE spectrum and on days/s.

Inputs are synthetic: the exponential stratification restricted to 4 layers on a 2000 km
square, the seeded random PV initial condition (peak wavenumber 16, rms 1e-6, seed 5),
ARK43_QGLeith with PI.3.4 adaptive dt.  Every truth run is spun up for a model year before
any sample is taken: while the initial condition decays, the subgrid statistics drift and a
network trained on earlier samples does not carry to later ones.  The training samples come
from separate truth runs (other seeds of the same initial-condition generator), the 60-day
evaluation from the seed-5 truth: the network is scored on a trajectory it never saw.  Sizes
(spin-up, samples, training steps, evaluation window) are arguments, so the experiment runs at
benchmark length (1024 samples from one run, 3000 Adam steps) or with the named
configuration's 20 000 samples (five runs, 6000 Adam steps, a 12-day background:
``--samples 20000 --every 2 --iters 6000 --train-seeds 6,7,8,9,10 --background-days 12``).

``python -m qgn_fortran_b200.closure_experiment`` prints the result as one JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

DAY = 86400.0


def _params(n, nz, tol):
    beta, Lx = 2.0e-11, 2.0e6
    return dict(nx=n, ny=n, nz=nz, Lx=Lx, Ly=Lx, Htot=4000.0, f0=1.0e-4, beta=beta, A2=0.0, A8=1.0e23,
                r0=1.0e-7, C_d=0.0, TOL=tol, is_explicit=False, dt_max=math.pi / (beta * Lx))


def _advance_to(model, t_target, chunk=8, max_steps=1_000_000):
    steps = 0
    while model.time()[0] < t_target and steps < max_steps:
        model.advance_resident(chunk)
        steps += chunk
    return steps


def _timed_days_per_s(model, nsteps):
    """Device-timed days/s of nsteps resident steps (CUDA events on the model's stream)."""
    import torch
    from . import _lib

    sp = _lib.C.c_void_p()
    model.lib.qgn_stream(model.ctx, _lib.C.byref(sp))
    st = torch.cuda.ExternalStream(sp.value)
    t0 = model.time()[0]
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(st)
    model.advance_resident(nsteps)
    b.record(st)
    b.synchronize()
    ms = a.elapsed_time(b)
    return (model.time()[0] - t0) / DAY / (ms / 1000.0), ms / nsteps


def _spectrum(model, nbins):
    _, spec = model.diagnostics(nbins)
    return np.sum(spec, axis=0)        # column-summed over layers (H-weighted KE per bin)


def _spec_err(e_model, e_truth):
    k = np.arange(1, len(e_truth))      # skip the k=0 bin
    r = e_model[k] / np.maximum(e_truth[k], 1e-300) - 1.0
    return {"mean_abs_rel": float(np.mean(np.abs(r))), "max_abs_rel": float(np.max(np.abs(r))),
            "total_ke_rel": float(np.sum(e_model[k]) / np.sum(e_truth[k]) - 1.0)}


def _conv_tflops(net, batch):
    """Achieved TFLOP/s of the network's forward (6 convolutions) at `batch`, event-timed."""
    import torch

    x = torch.zeros((batch, net.H, net.W, net.cin_p), dtype=torch.bfloat16, device="cuda")
    y = torch.zeros((batch, net.H, net.W, net.cout_p), dtype=torch.float32, device="cuda")
    st = torch.cuda.ExternalStream(net.stream())
    for _ in range(3):
        net.forward(x, y, batch)
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    reps = 10
    a.record(st)
    for _ in range(reps):
        net.lib.qgn_cnn_forward(net.net, x.data_ptr(), y.data_ptr(), batch, None)
    b.record(st)
    b.synchronize()
    ms = a.elapsed_time(b) / reps
    flop = 0.0
    for cop, cip in net.shapes:
        flop += 2.0 * batch * net.H * net.W * 9 * cip * cop      # padded channels, as computed
    return flop / (ms / 1000.0) / 1e12, ms


def run(truth_n=1024, coarse_n=128, nz=4, spinup_days=365.0, nsnap=1024, every=8, iters=3000, batch=32,
        lr=1e-3, eval_days=60.0, sample_days=1.0, A8_background=None, energy_limit=1.0, seed=5, log=None,
        train_seed=(6,), window_samples=1024, window_every=8, background_days=3.0):
    """By default the network trains on samples of a separate truth run (train_seed: the
    initial condition of seed 6, the same spin-up; several seeds split the samples evenly), and
    the evaluated truth (seed) takes the steps of the default sampling (window_samples every
    window_every steps, discarded): the 60-day window is the same whatever the size of the
    training set, and it lies on a trajectory the network never saw.  With train_seed None the
    network trains on the evaluated truth itself, and the window starts where the sampling ends.
    background_days: grid-scale e-folding time of the hyperviscosity kept under the network
    (A8_background overrides it)."""
    import torch

    from . import QGNModule
    from . import closure as cl
    from .inputs import exponential_stratification, seeded_random_pv

    def say(*a):
        if log:
            print(*a, file=log, flush=True)

    H, S, U = exponential_stratification(nz)
    qp = seeded_random_pv(truth_n, truth_n, nz, 16.0, 1.0e-6, seed)
    tol = 1.0e-6 * float(np.max(np.abs(qp)))
    out = {"truth": f"{truth_n}^2x{nz}", "coarse": f"{coarse_n}^2x{nz}", "scheme": "ark43_qgleith",
           "samples": nsnap, "every_steps": every, "train_iters": iters, "batch": batch,
           "spinup_days": spinup_days, "eval_days": eval_days, "background_days": background_days,
           "training_truth": "the evaluated truth"}
    truth = QGNModule(_params(truth_n, nz, tol), H, S, U)
    truth.initialize(qp, 0.0, 750.0)
    t_wall = time.perf_counter()
    _advance_to(truth, spinup_days * DAY, chunk=100)
    truth_dps, truth_ms = _timed_days_per_s(truth, 200)
    out["truth_days_per_s"] = truth_dps
    out["truth_ms_per_step"] = truth_ms
    say("spin-up", time.perf_counter() - t_wall, "s; truth days/s", truth_dps)

    pc = _params(coarse_n, nz, tol)
    helper = QGNModule(pc, H, S, U)
    net = cl.ClosureNet(nz=nz, H=coarse_n, W=coarse_n, layers=6, max_batch=batch, seed=seed)
    t_wall = time.perf_counter()
    if train_seed is None:
        x, y, isc, osc = cl.make_dataset(truth, helper, nsnap, every, net.cin_p, net.cout_p)
    else:
        seeds = [train_seed] if isinstance(train_seed, int) else list(train_seed)
        out["training_truth"] = f"separate truth runs, seeds {seeds}"
        xs, ys, isc, osc = [], [], None, None
        for i, sd in enumerate(seeds):   # nsnap samples split evenly over the training runs
            ni = nsnap // len(seeds) + (1 if i < nsnap % len(seeds) else 0)
            src = QGNModule(_params(truth_n, nz, tol), H, S, U)
            src.initialize(seeded_random_pv(truth_n, truth_n, nz, 16.0, 1.0e-6, sd), 0.0, 750.0)
            _advance_to(src, spinup_days * DAY, chunk=100)
            _timed_days_per_s(src, 200)      # the same path as the evaluated truth's
            xi, yi, isc, osc = cl.make_dataset(src, helper, ni, every, net.cin_p, net.cout_p, isc, osc)
            src.cleanup()
            xs.append(xi)
            ys.append(yi)
        x, y = (xs[0], ys[0]) if len(xs) == 1 else (torch.cat(xs), torch.cat(ys))
        del xs, ys
        xw, yw, _, _ = cl.make_dataset(truth, helper, window_samples, window_every, net.cin_p, net.cout_p)
        del xw, yw
    out["dataset_s"] = time.perf_counter() - t_wall
    ntr = int(0.9 * nsnap)
    t_wall = time.perf_counter()
    hist = cl.train(net, x[:ntr], y[:ntr], int(0.75 * iters), batch, lr, seed=seed, log_every=max(1, iters // 10))
    hist += cl.train(net, x[:ntr], y[:ntr], iters - int(0.75 * iters), batch, lr / 3, seed=seed + 1,
                     log_every=max(1, iters // 10))
    torch.cuda.synchronize()
    out["train_s"] = time.perf_counter() - t_wall
    out["train_loss_first_last"] = [hist[0][1], hist[-1][1]]
    # offline skill on the held-out samples
    nte = nsnap - ntr
    pred = torch.zeros((nte,) + tuple(y.shape[1:]), dtype=torch.float32, device="cuda")
    for i in range(0, nte, batch):
        j = min(nte, i + batch)
        net.forward(x[ntr + i:ntr + j], pred[i:j], j - i)
    torch.cuda.synchronize()
    yt = y[ntr:, ..., :nz].cpu().numpy()
    yp = pred[..., :nz].cpu().numpy()
    out["offline_r2"] = float(1.0 - np.sum((yp - yt) ** 2) / np.sum((yt - yt.mean(axis=(0, 1, 2))) ** 2))
    tf, fms = _conv_tflops(net, batch)
    out["cnn_forward"] = {"batch": batch, "ms": fms, "tflops": tf}
    say("offline r2", out["offline_r2"], "cnn TF/s", tf)

    # online: both coarse models start from the coarse-grained truth
    leith = QGNModule(pc, H, S, U)
    learned = QGNModule(pc, H, S, U)
    cl.coarse_grain(truth, leith)
    cl.coarse_grain(truth, learned)
    if A8_background is None:
        # background hyperviscosity under the network, a grid-scale e-folding time on the coarse
        # grid.  The better the network, the less it needs (B200, the same 60-day window, QG-Leith
        # 4.4 % mean spectrum error): 1024 samples, 3 / 5 / 8 days -> 2.7 / 4.1 / 5.5 %; 20 000
        # samples from five runs, 3 / 8 / 12 / 20 days -> 5.0 / 2.6 / 2.3 / 2.3 %
        A8_background = 1.0 / (background_days * DAY * (math.pi * coarse_n / pc["Lx"]) ** 8)
    cl.attach(learned, net, isc, osc, A8_background=A8_background, energy_limit=energy_limit)
    nbins = coarse_n // 3
    t0 = truth.time()[0]
    acc = {"truth": np.zeros(nbins), "leith": np.zeros(nbins), "closure": np.zeros(nbins)}
    nsamp = 0
    status = "ok"
    t_wall = time.perf_counter()
    try:
        for k in range(1, int(eval_days / sample_days) + 1):
            tk = t0 + k * sample_days * DAY
            _advance_to(truth, tk, chunk=4)
            _advance_to(leith, tk, chunk=1)
            _advance_to(learned, tk, chunk=1)
            cl.coarse_grain(truth, helper)
            acc["truth"] += _spectrum(helper, nbins)
            acc["leith"] += _spectrum(leith, nbins)
            acc["closure"] += _spectrum(learned, nbins)
            nsamp += 1
    except Exception as exc:     # a coarse run that blows up halts with a status
        status = f"stopped: {exc}"
    out["online_s"] = time.perf_counter() - t_wall
    out["online_status"] = status
    out["online_samples"] = nsamp
    if nsamp:
        spec = {k: v / nsamp for k, v in acc.items()}
        out["ke_spectrum_err_closure"] = _spec_err(spec["closure"], spec["truth"])
        out["ke_spectrum_err_leith"] = _spec_err(spec["leith"], spec["truth"])
        out["ke_spectra"] = {k: [float(x) for x in v] for k, v in spec.items()}
    out["closure_stats"] = cl.stats(learned) if status == "ok" else None
    if status == "ok":
        cdps, cms = _timed_days_per_s(learned, 200)
        ldps, lms = _timed_days_per_s(leith, 200)
        out["closure_days_per_s"] = cdps
        out["closure_ms_per_step"] = cms
        out["leith_days_per_s"] = ldps
        out["leith_ms_per_step"] = lms
        out["closure_speedup_vs_truth"] = cdps / truth_dps
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--truth", type=int, default=1024)
    ap.add_argument("--coarse", type=int, default=128)
    ap.add_argument("--nz", type=int, default=4)
    ap.add_argument("--spinup-days", type=float, default=365.0)
    ap.add_argument("--samples", type=int, default=1024)
    ap.add_argument("--every", type=int, default=8)
    ap.add_argument("--iters", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--eval-days", type=float, default=60.0)
    ap.add_argument("--train-seeds", type=str, default="6",
                    help="comma-separated seeds: train on separate truth runs from these initial conditions "
                         "(the samples split evenly); evaluate on the default window; 'none': train on the "
                         "evaluated truth")
    ap.add_argument("--background-days", type=float, default=3.0,
                    help="grid-scale e-folding time of the background hyperviscosity under the network")
    args = ap.parse_args()
    import sys
    res = run(args.truth, args.coarse, args.nz, args.spinup_days, args.samples, args.every, args.iters, args.batch,
              eval_days=args.eval_days, log=sys.stderr,
              train_seed=None if args.train_seeds == "none" else [int(v) for v in args.train_seeds.split(",")],
              background_days=args.background_days)
    res.pop("ke_spectra", None)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
