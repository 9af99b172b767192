"""Small fixed workloads for profiler captures (ncu) and quick timing.

    python -m qgn_fortran_b200.profile_case --workload strat1024x8 --steps 1
    python -m qgn_fortran_b200.profile_case --workload strat1024x8 --nx 128 --nz 4 --steps 3 --closure
    python -m qgn_fortran_b200.profile_case --cnn-batch 8
    python -m qgn_fortran_b200.profile_case --cnn-batch 32 --cnn-train 2
    python -m qgn_fortran_b200.profile_case --ensemble 8 --steps 2

The first two build the named workload (optionally at another grid, optionally with a
closure network of zero weights attached, which always passes the budget check and so runs
the whole closure path), set the seeded IC on the GPU and advance ``--steps`` device-resident
TimeSteps, then print the per-kernel-family launch counts and CUDA-event times of those steps.
``--cnn-batch`` runs two forwards of the 6-layer closure network (128^2, 4 layers of q and
psi in, BF16, tcgen05); with ``--cnn-train`` it instead takes that many Adam steps on seeded
data of that batch (forward, backward-data and weight gradients on tcgen05, the six layers'
weight gradients last layer first).  ``--ensemble`` advances that many members of the batched-ensemble
workload (mixed precision).  Device memory held: the working set only (about 0.7 GB for
strat1024x8, well under 1 GB for the others).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time

import numpy as np

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


def run_model(a):
    w = workload(a.workload, nx=a.nx, nz=a.nz)
    g = QGNModule(w.params, w.H, w.S, w.U, scheme=w.scheme, precision=a.precision)
    g.initialize(w.qp, 0.0, w.dt0)
    net = None
    if a.closure:
        from . import closure as cl
        net = cl.ClosureNet(nz=g.nz, H=g.ny, W=g.nx, layers=6, max_batch=1, seed=1)
        net.set_weights([(np.zeros_like(x), np.zeros_like(b)) for x, b in net.get_weights()])
        cl.attach(g, net, np.ones(2 * g.nz), np.ones(g.nz), A8_background=w.params["A8"], energy_limit=1.0)
    g.lib.qgn_profile_enable(g.ctx, 1)
    t0 = time.perf_counter()
    g.advance_resident(a.steps)
    wall = time.perf_counter() - t0
    t, dt = g.time()
    print(json.dumps({"workload": a.workload, "grid": [g.nx, g.ny, g.nz], "closure": bool(a.closure),
                      "steps": a.steps, "wall_ms": 1000 * wall, "t": t, "dt": dt, "kernels": kernel_table(g)}))
    g.cleanup()


def run_cnn(a):
    import torch

    from . import closure as cl
    net = cl.ClosureNet(nz=4, H=128, W=128, layers=6, max_batch=a.cnn_batch, seed=3)
    if a.cnn_train:
        gen = torch.Generator(device="cpu").manual_seed(3)
        n = 2 * a.cnn_batch
        xd = torch.randn((n, 128, 128, net.cin_p), generator=gen).to(torch.bfloat16).cuda()
        yd = torch.randn((n, 128, 128, net.cout_p), generator=gen).cuda()
        idx = torch.arange(a.cnn_batch, dtype=torch.int32).cuda()
        torch.cuda.synchronize()
        for _ in range(a.cnn_train):
            net.train_step(xd, yd, idx, a.cnn_batch, 1e-4, want_loss=False)
        net.check()
        print(json.dumps({"cnn_batch": a.cnn_batch, "train_steps": a.cnn_train, "ok": True}))
        return
    x = torch.zeros((a.cnn_batch, 128, 128, net.cin_p), dtype=torch.bfloat16, device="cuda")
    y = torch.zeros((a.cnn_batch, 128, 128, net.cout_p), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    for _ in range(2):
        net.lib.qgn_cnn_forward(net.net, x.data_ptr(), y.data_ptr(), a.cnn_batch, None)
    net.check()
    print(json.dumps({"cnn_batch": a.cnn_batch, "ok": True}))


def run_ensemble(a):
    from . import QGNEnsemble
    from .inputs import ensemble_members
    ws = ensemble_members(a.ensemble)
    gs = [QGNModule(w.params, w.H, w.S, w.U, scheme="bsrk3") for w in ws]
    for g, w in zip(gs, ws):
        g.initialize(w.qp, 0.0, w.dt0)
    ens = QGNEnsemble(gs, precision="mixed")
    ens.advance(a.steps)
    print(json.dumps({"ensemble": a.ensemble, "steps": a.steps, "tuning": ens.tuning()}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="strat1024x8")
    ap.add_argument("--nx", type=int, default=None)
    ap.add_argument("--nz", type=int, default=None)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--precision", default="fp64")
    ap.add_argument("--closure", action="store_true")
    ap.add_argument("--cnn-batch", type=int, default=0)
    ap.add_argument("--cnn-train", type=int, default=0)
    ap.add_argument("--ensemble", type=int, default=0)
    a = ap.parse_args()
    if a.cnn_batch:
        run_cnn(a)
    elif a.ensemble:
        run_ensemble(a)
    else:
        run_model(a)


if __name__ == "__main__":
    main()
