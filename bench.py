"""Benchmark: simulated model days per wall second of the QGN time stepper on B200.

Workload (default ``strat1024x8``): 8 geometric layers on a 1024^2 doubly periodic grid,
L = 2000 km, N^2 = (5e-3)^2 exp(z/1000 m), U = 0.1 exp(z/1000 m), ARK43_QGLeith with the
PI.3.4 controller and TOL = 1e-6 x max|q_IC| of the seeded random PV field (seed 2, peak
wavenumber 16, rms 1e-6 s^-1), FP64.  A step is one accepted TimeStep (6 RHS evaluations plus
any rejected attempts).  Data are synthetic.  The window starts from the configuration's
10-year spun-up state (qgn_fortran_b200/data/strat1024x8_spinup.npz, made on the GPU by
qgn_fortran_b200.spinup from the seeded IC; kept modes at bfloat16 precision), the regime the
configuration's statistics year runs in; both arms start there, W untimed steps, K timed.

``value``: device-resident stepping (qgn_advance_resident, graph-launched steps), CUDA
events on the library's stream.  ``e2e``: the drop-in path TimeStep (QGNModule.time_step ->
qgn_step) with the host q_hat in pinned memory: every step copies the kept modes host->device
and back.  ``mixed``: the same workload in the mixed-precision mode.
``cpu_baseline`` and ``--impl reference`` time the FP64 C/OpenMP restatement of the reference
(oracle/qgn_ref.c) on all host threads.

Multi-GPU (torchrun): the path does not shard -- each rank advances an independent replica
("replicas only"); value = total simulated days of all ranks / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "simulated days/s, 1024^2 x 8 layers, ARK43_QGLeith PI.3.4, FP64"
UNIT = "simulated days/s"
DAY = 86400.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="strat1024x8")
    ap.add_argument("--ic", choices=["spinup", "seeded"], default=None,
                    help="window start: the committed 10-year spun-up state (default when the workload "
                         "has one) or the seeded initial condition")
    ap.add_argument("--cpu-sample-steps", type=int, default=6)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-closure", action="store_true")
    ap.add_argument("--no-c3", action="store_true", help="skip the 2048^2 x 16 FP64/mixed leg")
    ap.add_argument("--c3-steps", type=int, default=10)
    ap.add_argument("--ens-members", type=int, default=64)
    ap.add_argument("--ens-steps", type=int, default=20)
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def reduce_over_ranks(ms, units, ws, device="cuda"):
    """Whole-job numbers of the replicas: the slowest rank's time and the sum of the units
    (simulated days) of all ranks.  ws == 1 returns the inputs."""
    if ws <= 1:
        return ms, units
    import torch
    import torch.distributed as dist
    tt = torch.tensor([ms, units], dtype=torch.float64, device=device)
    mx = tt.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    sm = tt.clone()
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return float(mx[0]), float(sm[1])


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.proc = None
        self.gpu = gpu_index
        self.out = os.path.join("/tmp", f"qgn_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.out, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # nvidia-smi takes a moment to start: wait (bounded) for its first sample so the
        # samples cover the timed region
        t0 = time.time()
        while time.time() - t0 < 3.0 and self.proc.poll() is None:
            if os.path.getsize(self.out) > 0:
                break
            time.sleep(0.02)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.out):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.out)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def bench_workload(args):
    """The named workload, starting from its spun-up state when one is committed (or --ic)."""
    from qgn_fortran_b200.inputs import spinup_path, workload
    ic = args.ic or ("spinup" if os.path.exists(spinup_path(args.workload)) else "seeded")
    return workload(args.workload, ic=ic)


def bench_config(args, w, ws):
    """The config keys both arms print (same workload, grid, scheme and step window)."""
    start = ("the committed state after 10 model years of spin-up (qgn_fortran_b200.spinup; t0 = "
             f"{w.t0 / 86400.0 / 365.0:.2f} years, dt0 = {w.dt0:.0f} s)" if w.ic == "spinup" else "the seeded IC")
    return {"workload": args.workload, "grid": f"{w.params['nx']}x{w.params['ny']}x{w.params['nz']}",
            "scheme": w.scheme, "parallelism": "replicas" if ws > 1 else "single",
            "l2": "working set ~0.7 GB > 126 MB L2 (no flush needed)",
            "window": f"steps {args.warmup + 1}..{args.warmup + args.steps} from {start}"}


def run_oracle(w, warmup, steps):
    """Time the FP64 C/OpenMP restatement of the reference (oracle/qgn_ref.c) on the host cores."""
    from oracle.qgn_oracle import Params
    from oracle.qgn_ref_c import RefC

    c = RefC(Params(**w.params), w.H, w.S, w.U, scheme=w.scheme)
    q = c.initialize_spec(w.qp)
    t, dt = w.t0, w.dt0
    for _ in range(warmup):
        t, dt = c.step(q, t, dt)
    t0 = t
    c0 = time.perf_counter()
    for _ in range(steps):
        t, dt = c.step(q, t, dt)
    sec = time.perf_counter() - c0
    return (t - t0) / DAY / sec, sec, steps, c.threads()


def reference_arm(args):
    """The reference algorithm on the host cores over the same step window as our arm: from the
    same start state, W untimed steps, then K timed steps, so both arms simulate the same days."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    w = bench_workload(args)
    warm = max(0, args.warmup)
    steps = max(1, args.steps)
    val, sec, n, nthr = run_oracle(w, warm, steps)
    cfg = bench_config(args, w, ws)
    sample = (f"{cfg['window']} of {w.scheme} on {args.workload} (the window our arm times), FP64 C/OpenMP "
              f"restatement of the reference (oracle/qgn_ref.c), {nthr} threads, {sec:.1f} s timed")
    line = {"metric": METRIC, "value": val, "unit": UNIT, "impl": "reference", "n_gpus": ws, "steps": n,
            "warmup": warm, "ms_per_step": 1000.0 * sec / n, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": cfg,
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": nthr, "kind": "port", "sample": sample},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def ours_arm(args):
    import torch

    ws, rank, local = dist_env()
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)

    from qgn_fortran_b200 import QGNModule, _lib
    from qgn_fortran_b200.inputs import workload

    w = bench_workload(args)
    g = QGNModule(w.params, w.H, w.S, w.U, scheme=w.scheme)
    q = g.initialize(w.qp, w.t0, w.dt0)
    sptr = _lib.C.c_void_p()
    g.lib.qgn_stream(g.ctx, _lib.C.byref(sptr))
    stream = torch.cuda.ExternalStream(sptr.value)

    if args.warmup > 0:
        g.advance_resident(args.warmup)      # the first call also records the step graphs

    def barrier():
        if ws > 1:
            torch.distributed.barrier()

    def kernel_families():
        fam = []
        for k in range(_lib.QGN_KERNEL_FAMILIES):
            tot, nb = _lib.C.c_double(), _lib.C.c_double()
            nt, nl = _lib.C.c_longlong(), _lib.C.c_longlong()
            g.lib.qgn_profile_read(g.ctx, k, _lib.C.byref(tot), _lib.C.byref(nb), _lib.C.byref(nt),
                                   _lib.C.byref(nl))
            fam.append((tot.value, nb.value, nt.value, nl.value, g.lib.qgn_kernel_name(k).decode()))
        return fam

    # ---- timed region: graph-launched steps, launch counting only
    clocks = ClockSampler(local) if rank == 0 else None
    g.lib.qgn_profile_enable(g.ctx, 0)
    t0, _ = g.time()
    barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
        time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    g.advance_resident(args.steps)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop() if clocks else None
    t1, dt1 = g.time()
    days = (t1 - t0) / DAY
    launches = sum(f[3] for f in kernel_families())

    # ---- per-kernel CUDA-event timing of the same kind of steps (eager launches)
    nroof = max(1, min(args.steps, 10))
    g.lib.qgn_profile_enable(g.ctx, 1)
    g.advance_resident(nroof)
    fam = kernel_families()
    g.lib.qgn_profile_enable(g.ctx, 0)
    roof_ms = sum(f[0] for f in fam)

    ms_all, days_all = reduce_over_ranks(ms, days, ws)

    # end-to-end through the drop-in TimeStep (qgn_step) with pinned host q_hat, over the same
    # step window from the IC in a fresh context (the controller's err0 starts at TOL again)
    e2e = None
    if not args.no_e2e:
        gE = QGNModule(w.params, w.H, w.S, w.U, scheme=w.scheme)
        q0 = gE.initialize(w.qp, w.t0, w.dt0)
        qh = torch.empty(q0.shape, dtype=torch.complex128, pin_memory=True).numpy()
        qh[...] = q0
        sE = _lib.C.c_void_p()
        gE.lib.qgn_stream(gE.ctx, _lib.C.byref(sE))
        estream = torch.cuda.ExternalStream(sE.value)
        t, dt = w.t0, w.dt0
        for _ in range(args.warmup):
            t, dt = gE.time_step(qh, t, dt)
        te0 = t
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(estream)
        for _ in range(args.steps):
            t, dt = gE.time_step(qh, t, dt)
        e1.record(estream)
        e1.synchronize()
        ems = e0.elapsed_time(e1)
        edays = (t - te0) / DAY
        ems, edays = reduce_over_ranks(ems, edays, ws)
        # both directions move the kept modes only (two pitched copies each); TimeStep's
        # trailing DeAlias (QGN_Module.f90:307) zeroes the rest of q_hat on the host
        kept = 16 * (w.params["nx"] // 3) * (w.params["ny"] - w.params["ny"] // 3 - 1) * w.params["nz"]
        e2e = {"value": edays / (ems / 1000.0), "unit": UNIT, "h2d_bytes_per_step": kept,
               "d2h_bytes_per_step": kept, "ms_per_step": ems / args.steps,
               "window": bench_config(args, w, ws)["window"]}
        gE.cleanup()

    # ---- the same workload in the mixed mode (FP32 transforms/RHS/stages, FP64 state and control)
    mixed = None
    if not args.no_mixed:
        gm = QGNModule(w.params, w.H, w.S, w.U, scheme=w.scheme, precision="mixed")
        gm.initialize(w.qp, w.t0, w.dt0)
        if args.warmup > 0:
            gm.advance_resident(args.warmup)
        smp = _lib.C.c_void_p()
        gm.lib.qgn_stream(gm.ctx, _lib.C.byref(smp))
        mstream = torch.cuda.ExternalStream(smp.value)
        tm0, _ = gm.time()
        barrier()
        torch.cuda.synchronize()
        m0 = torch.cuda.Event(enable_timing=True)
        m1 = torch.cuda.Event(enable_timing=True)
        m0.record(mstream)
        gm.advance_resident(args.steps)
        m1.record(mstream)
        m1.synchronize()
        mms = m0.elapsed_time(m1)
        tm1, _ = gm.time()
        mdays = (tm1 - tm0) / DAY
        mms, mdays = reduce_over_ranks(mms, mdays, ws)
        mixed = {"value": mdays / (mms / 1000.0), "unit": UNIT, "ms_per_step": mms / args.steps,
                 "ms_per_step_vs_fp64": (ms_all / args.steps) / (mms / args.steps),
                 "dtype": "f32 transforms/RHS/stage storage/error spectrum and norm, f64 state/GetPsi/update/controller"}
        gm.cleanup()

    c3 = None
    if not args.no_c3:
        c3 = c3_bench(args, ws)

    ensemble = None
    if not args.no_ensemble:
        ensemble = ensemble_bench(args, ws)

    # learned closure: a 1024^2 x 4 truth run -> 128^2 training data -> trained network -> 128^2
    # runs with QG-Leith and with the closure against the coarse-grained truth of a second 1024^2
    # x 4 run the network never saw (KE spectrum, days/s)
    closure = None
    if not args.no_closure:
        from qgn_fortran_b200.closure_experiment import run as run_closure
        res = run_closure()
        res.pop("ke_spectra", None)
        closure = res

    if rank != 0:
        g.cleanup()
        if ws > 1:
            torch.distributed.destroy_process_group()
        return

    peak, peak_kind = measured_peaks()
    top = max(fam, key=lambda f: f[0])
    achieved = (top[1] / top[2]) / ((top[0] / top[2]) / 1000.0) / 1e9 if top[2] else None
    traffic = read_traffic(args.workload, top[4])
    roofline = {"bound": "hbm", "kernel": top[4], "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                "traffic": traffic, "algorithmic_bytes_per_launch": top[1] / top[2] if top[2] else None,
                "ms_per_launch": top[0] / top[2] if top[2] else None,
                "share_of_kernel_time": top[0] / roof_ms if roof_ms else None,
                "timed_steps": nroof}
    roofline["fp64"] = fp64_roofline(g, w, fam, ms_all / args.steps)
    kernels = {f[4]: {"ms": round(f[0], 4), "launches": f[3]} for f in fam if f[3]}

    cpu = None
    if ws == 1 and not args.no_cpu_baseline:
        # a bounded sample: seconds per step of the reference algorithm on the host cores, turned
        # into days/s with the mean dt of the timed GPU window (both compute the same trajectory)
        _, sec, n, nthr = run_oracle(w, 1, args.cpu_sample_steps)
        cpu_val = (days_all / args.steps) / (sec / n)
        cpu = {"value": cpu_val, "unit": UNIT, "cores": nthr, "kind": "port", "ms_per_step": 1000.0 * sec / n,
               "sample": f"{n} {w.scheme} steps of {args.workload} after 1 warm-up step from the window's start, "
                         f"FP64 C/OpenMP restatement of the reference (oracle/qgn_ref.c), {nthr} threads, "
                         f"{sec:.1f} s; days/s = mean dt of the timed window / CPU s per step"}

    line = {"metric": METRIC, "value": days_all / (ms_all / 1000.0), "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_all / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": bench_config(args, w, ws),
            "window_stats": {"sim_days": days, "final_dt_s": dt1, "rejects": g.rejects()},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "mixed": mixed, "mixed_2048x16": c3, "ensemble": ensemble, "closure": closure, "gpu_launches": launches,
            "clocks": clk, "kernels": kernels}
    print(json.dumps(line), flush=True)
    g.cleanup()
    if ws > 1:
        torch.distributed.destroy_process_group()


def c3_bench(args, ws):
    """The mixed-precision configuration, 16 layers on 2048^2 (same stratification and mean flow,
    ARK43_QGLeith with PI.3.4, seed 3): FP64 and mixed on the same window of steps from the
    seeded IC, state resident in HBM, graph-launched steps, CUDA events on the library's stream."""
    import torch

    from qgn_fortran_b200 import QGNModule, _lib
    from qgn_fortran_b200.inputs import workload

    w = workload("strat2048x16")
    out = {"workload": "strat2048x16", "grid": "2048x2048x16", "scheme": w.scheme, "steps": args.c3_steps,
           "window": f"steps {args.warmup + 1}..{args.warmup + args.c3_steps} from the seeded IC"}
    for prec in ("fp64", "mixed"):
        g = QGNModule(w.params, w.H, w.S, w.U, scheme=w.scheme, precision=prec)
        g.initialize(w.qp, 0.0, w.dt0)
        g.advance_resident(max(args.warmup, 1))
        sp = _lib.C.c_void_p()
        g.lib.qgn_stream(g.ctx, _lib.C.byref(sp))
        st = torch.cuda.ExternalStream(sp.value)
        t0, _ = g.time()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        g.advance_resident(args.c3_steps)
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        t1, dt1 = g.time()
        ms, days = reduce_over_ranks(ms, (t1 - t0) / DAY, ws)
        out[prec] = {"ms_per_step": ms / args.c3_steps, "days_per_s": days / (ms / 1000.0), "final_dt_s": dt1}
        g.cleanup()
    out["ms_per_step_fp64_vs_mixed"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    return out


def ensemble_bench(args, ws):
    """Batched heterogeneous ensemble: members of 128^2/256^2/512^2 x 2/4/8 layers, BSRK3 with
    adaptive dt, one launch per pass for all members (mixed and FP64), against the same members
    stepped one after another through their own contexts (FP64 BSRK3)."""
    import torch

    from qgn_fortran_b200 import QGNEnsemble, QGNModule
    from qgn_fortran_b200.inputs import ensemble_members

    members = ensemble_members(args.ens_members)
    gs = [QGNModule(w.params, w.H, w.S, w.U, scheme="bsrk3") for w in members]
    K = args.ens_steps
    out = {"members": len(members), "steps": K,
           "sizes": {f"{n}^2x{z}": sum(1 for w in members if w.params["nx"] == n and w.params["nz"] == z)
                     for n in (128, 256, 512) for z in (2, 4, 8)},
           "scheme": "bsrk3 (PI.3.4 adaptive dt)"}

    def reset():
        for g, w in zip(gs, members):
            g.initialize(w.qp, 0.0, w.dt0)

    for prec in ("mixed", "fp64"):
        reset()
        ens = QGNEnsemble(gs, precision=prec)
        ens.advance(max(args.warmup, 1))          # first call: FSAL, autotune, graph capture
        st = torch.cuda.ExternalStream(ens.stream())
        t0 = [g.time()[0] for g in gs]
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        ens.advance(K)
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        days = sum(g.time()[0] - a for g, a in zip(gs, t0)) / DAY
        ms, days = reduce_over_ranks(ms, days, ws)
        out[prec] = {"member_days_per_s": days / (ms / 1000.0), "member_steps_per_s": len(gs) * K / (ms / 1000.0),
                     "ms_per_ensemble_step": ms / K, "tuning": ens.tuning()}
        ens.close()
    # the same members one after another, each through its own context (FP64 BSRK3, qgn_advance_resident)
    reset()
    for g in gs:
        g.advance_resident(max(args.warmup, 1))
    t0 = [g.time()[0] for g in gs]
    torch.cuda.synchronize()
    s = time.perf_counter()
    for g in gs:
        g.advance_resident(K)
    torch.cuda.synchronize()
    sec = time.perf_counter() - s
    days = sum(g.time()[0] - a for g, a in zip(gs, t0)) / DAY
    out["sequential_fp64"] = {"member_days_per_s": days / sec, "member_steps_per_s": len(gs) * K / sec,
                              "timing": "host wall clock around synchronous per-member calls"}
    out["speedup_mixed_vs_sequential"] = out["mixed"]["member_days_per_s"] / out["sequential_fp64"]["member_days_per_s"]
    for g in gs:
        g.cleanup()
    return out


def read_traffic(workload, kernel):
    """DRAM bytes per launch of a kernel from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", f"traffic_{workload}.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        parts = line.split()
        if len(parts) >= 2 and parts[0] == kernel:
            try:
                return float(parts[1])
            except ValueError:
                return None
    return None


def fp64_roofline(g, w, fam, ms_step):
    """FLOP fraction of the x pass and of the step against the FP64 FMA peak measured here.

    Algorithmic FLOPs: 5 N log2 N per complex N-point FFT, i.e. 2.5 nx ny log2(nx) for the x part
    of one real 2-D transform (five per layer: q, u, v inverse and uq, vq forward; two more on
    the bottom layer with quadratic drag) plus 5 nx ny per layer for the scalings and products;
    per RHS 2.5 nx ny log2(nx ny) per real 2-D transform plus 4 nz^2 per kept spectral mode for
    GetPsi (to modes and back); six RHS per ARK43_QGLeith step (stage combinations, update, error
    norm and controller not counted)."""
    tf, pms = ctypes.c_double(), ctypes.c_double()
    rc = g.lib.qgn_probe_fp64_fma(5, ctypes.byref(tf), ctypes.byref(pms))
    if rc != 0:
        return {"unavailable": f"FP64 probe returned {rc}"}
    p = w.params
    nx, ny, nz = p["nx"], p["ny"], p["nz"]
    nkx = nx // 3
    nky = ny - ny // 3 - 1
    drag = p.get("C_d", 0.0) != 0.0
    ntr = 5 * nz + (2 if drag else 0)
    x_flops_layer = 2.5 * nx * ny * math.log2(nx) * 5 + 5.0 * nx * ny
    x_bytes_layer = 5 * ny * nkx * 16
    peak = tf.value
    out = {"unit": "TFLOP/s", "peak": peak, "peak_source": "FP64 FMA probe (qgn_probe_fp64_fma: 32 chains per "
           "thread, 8 CTAs of 256 per SM, best of 5 launches) on this GPU", "probe_ms": pms.value}
    xp = [f for f in fam if f[4] == "xpass" and f[2]]
    if xp and not drag:
        f = xp[0]
        flops = (f[1] / f[2]) / x_bytes_layer * x_flops_layer   # layers per launch x FLOPs per layer
        ach = flops / ((f[0] / f[2]) / 1000.0) / 1e12
        out.update({"kernel": "xpass", "flops_per_launch": flops, "achieved": ach, "frac": ach / peak})
    rhs = 2.5 * nx * ny * math.log2(nx * ny) * ntr + 4.0 * nz * nz * nkx * nky
    step_ach = 6 * rhs / (ms_step / 1000.0) / 1e12
    out.update({"step_flops": 6 * rhs, "step_achieved": step_ach, "step_frac": step_ach / peak})
    return out


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    else:
        ours_arm(args)


if __name__ == "__main__":
    main()
