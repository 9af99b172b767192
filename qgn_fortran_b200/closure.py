"""Host side of the learned subgrid closure (csrc/cnn.cu, csrc/closure.cu).

``ClosureNet`` wraps the tensor-core network (periodic 3x3 convolutions, GELU, BF16 with FP32
accumulation) and its Adam training; ``make_dataset`` coarse-grains a high-resolution run into
training samples on the GPU; ``attach`` puts a trained network into a coarse ARK43_QGLeith
model's right-hand side with the energy-budget fallback to QG-Leith.  Device tensors are
torch allocations (plumbing only); every computation runs in ``libqgn_b200.so``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import QGNError


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class ClosureNet:
    """Network with ``2 nz`` inputs (q, psi per layer) and ``nz`` outputs on an H x W grid."""

    def __init__(self, nz: int, H: int, W: int, layers: int = 6, width: int = 64, max_batch: int = 32,
                 seed: int = 0, cin: int | None = None, cout: int | None = None):
        self.lib = _lib.load()
        self.cin = 2 * nz if cin is None else cin
        self.cout = nz if cout is None else cout
        self.H, self.W, self.nlayers, self.width, self.max_batch = H, W, layers, width, max_batch
        net = C.c_void_p()
        rc = self.lib.qgn_cnn_create(self.cin, width, self.cout, layers, H, W, max_batch, seed, C.byref(net))
        if rc != 0:
            raise QGNError(rc, f"qgn_cnn_create(cin={self.cin}, cout={self.cout}, H={H}, W={W})")
        self.net = net
        ci, co = C.c_int(), C.c_int()
        self.lib.qgn_cnn_padded_channels(net, C.byref(ci), C.byref(co))
        self.cin_p, self.cout_p = ci.value, co.value
        self.shapes = []
        for l in range(layers):
            cip = self.cin_p if l == 0 else width
            cop = self.cout_p if l == layers - 1 else width
            self.shapes.append((cop, cip))

    def _check(self, rc, what):
        if rc != 0:
            msg = self.lib.qgn_cnn_last_error(self.net)
            raise QGNError(rc, f"{what}: {msg.decode() if msg else ''}")

    # -- weights ----------------------------------------------------------------------------
    def _unflatten(self, flat):
        out, off = [], 0
        for cop, cip in self.shapes:
            nw = 9 * cop * cip
            out.append((flat[off:off + nw].reshape(9, cop, cip).copy(), flat[off + nw:off + nw + cop].copy()))
            off += nw + cop
        return out

    def get_weights(self):
        flat = np.empty(self.lib.qgn_cnn_num_params(self.net), dtype=np.float32)
        self._check(self.lib.qgn_cnn_get_weights(self.net, _fp(flat)), "qgn_cnn_get_weights")
        return self._unflatten(flat)

    def set_weights(self, layers):
        flat = np.concatenate([np.concatenate([np.asarray(w, np.float32).ravel(), np.asarray(b, np.float32).ravel()])
                               for w, b in layers])
        self._check(self.lib.qgn_cnn_set_weights(self.net, _fp(flat)), "qgn_cnn_set_weights")

    # -- compute ------------------------------------------------------------------------------
    def forward(self, x, y, batch: int, stream: int | None = None):
        """x: device BF16 [batch,H,W,cin_p] (torch tensor), y: device FP32 [batch,H,W,cout_p]."""
        import torch
        torch.cuda.synchronize()
        self._check(self.lib.qgn_cnn_forward(self.net, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), batch,
                                             C.c_void_p(stream) if stream else None), "qgn_cnn_forward")

    def gradients(self, x, y, batch: int):
        import torch
        torch.cuda.synchronize()
        flat = np.empty(self.lib.qgn_cnn_num_params(self.net), dtype=np.float32)
        loss = C.c_double()
        self._check(self.lib.qgn_cnn_gradients(self.net, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), batch,
                                               _fp(flat), C.byref(loss)), "qgn_cnn_gradients")
        return loss.value, self._unflatten(flat)

    def train_step(self, x_all, y_all, idx, batch: int, lr: float, want_loss: bool = True):
        """One Adam step on samples idx (device int32 tensor) of the dataset tensors."""
        loss = C.c_double()
        self._check(self.lib.qgn_cnn_train_step(self.net, C.c_void_p(x_all.data_ptr()), C.c_void_p(y_all.data_ptr()),
                                                C.c_void_p(idx.data_ptr()), batch, float(lr),
                                                C.byref(loss) if want_loss else None), "qgn_cnn_train_step")
        return loss.value if want_loss else None

    def set_engine(self, engine: str):
        """'tcgen05' (TMEM accumulators, default; a small-batch inference runs all layers in one
        launch), 'mma.sync' (warp-level MMA) or 'tcgen05-layers' (one tcgen05 launch per layer)."""
        self._check(self.lib.qgn_cnn_set_engine(self.net, {"tcgen05": 0, "mma.sync": 1, "tcgen05-layers": 2}[engine]),
                    "qgn_cnn_set_engine")

    def check(self):
        self._check(self.lib.qgn_cnn_check(self.net), "qgn_cnn_check")

    def debug_set_counter(self, tile: int, value: int):
        """Failure injection for tests: set one tile's layer counter of the fused inference."""
        self._check(self.lib.qgn_cnn_debug_set_counter(self.net, tile, value), "qgn_cnn_debug_set_counter")

    def stream(self):
        sp = C.c_void_p()
        self._check(self.lib.qgn_cnn_stream(self.net, C.byref(sp)), "qgn_cnn_stream")
        return sp.value

    def close(self):
        if getattr(self, "net", None):
            self.lib.qgn_cnn_destroy(self.net)
            self.net = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def coarse_grain(fine, coarse):
    """coarse (QGNModule) <- sharp spectral cutoff of fine's resident state."""
    rc = fine.lib.qgn_coarse_grain(fine.ctx, coarse.ctx)
    if rc != 0:
        raise QGNError(rc, "qgn_coarse_grain")


def snapshot(fine, coarse, in_scale, out_scale, x, y, cin_p, cout_p):
    """One training sample of fine's resident state into device tensors x (BF16), y (FP32)."""
    isc = np.ascontiguousarray(in_scale, dtype=np.float32)
    osc = np.ascontiguousarray(out_scale, dtype=np.float32)
    rc = fine.lib.qgn_closure_snapshot(fine.ctx, coarse.ctx, _fp(isc), _fp(osc), C.c_void_p(x.data_ptr()),
                                       C.c_void_p(y.data_ptr()), cin_p, cout_p)
    if rc != 0:
        raise QGNError(rc, "qgn_closure_snapshot")


def make_dataset(fine, coarse, n: int, every: int, cin_p: int, cout_p: int, in_scale=None, out_scale=None):
    """Advance ``fine`` and take ``n`` samples ``every`` steps apart.  With no scales given, they
    are estimated from the first samples (inverse standard deviation per channel).  Returns
    (x [n,H,W,cin_p] bf16, y [n,H,W,cout_p] fp32, in_scale, out_scale) on the GPU."""
    import torch

    nz, H, W = coarse.nz, coarse.ny, coarse.nx
    dev = torch.device("cuda")
    if in_scale is None or out_scale is None:
        ones_i, ones_o = np.ones(2 * nz, np.float32), np.ones(nz, np.float32)
        xs = torch.zeros((4, H, W, cin_p), dtype=torch.bfloat16, device=dev)
        ys = torch.zeros((4, H, W, cout_p), dtype=torch.float32, device=dev)
        torch.cuda.synchronize()
        for i in range(4):
            snapshot(fine, coarse, ones_i, ones_o, xs[i], ys[i], cin_p, cout_p)
            fine.advance_resident(every)
        xv = xs.float().cpu().numpy()
        yv = ys.cpu().numpy()
        in_scale = 1.0 / np.maximum(xv[..., :2 * nz].std(axis=(0, 1, 2)), 1e-30)
        out_scale = 1.0 / np.maximum(yv[..., :nz].std(axis=(0, 1, 2)), 1e-30)
    x = torch.zeros((n, H, W, cin_p), dtype=torch.bfloat16, device=dev)
    y = torch.zeros((n, H, W, cout_p), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()      # the model's streams do not order after torch's
    for i in range(n):
        snapshot(fine, coarse, in_scale, out_scale, x[i], y[i], cin_p, cout_p)
        fine.advance_resident(every)
    return x, y, np.asarray(in_scale, np.float32), np.asarray(out_scale, np.float32)


def train(net: ClosureNet, x, y, iters: int, batch: int, lr: float, seed: int = 0, log_every: int = 0):
    """Adam on random batches of the dataset; returns the loss history (every log_every steps)."""
    import torch

    n = x.shape[0]
    g = torch.Generator(device="cpu").manual_seed(seed)
    idx_all = torch.randint(0, n, (max(iters, 1), batch), generator=g, dtype=torch.int32).to("cuda")
    torch.cuda.synchronize()      # the network's stream does not order after torch's
    hist = []
    for it in range(iters):
        want = log_every > 0 and (it % log_every == 0 or it == iters - 1)
        loss = net.train_step(x, y, idx_all[it], batch, lr, want_loss=want)
        if want:
            hist.append((it, loss))
    return hist


def attach(coarse, net: ClosureNet | None, in_scale=None, out_scale=None, A8_background: float = 0.0,
           energy_limit: float = 1.0):
    """Attach (or with net=None detach) the closure of a coarse ARK43_QGLeith QGNModule."""
    if net is None:
        rc = coarse.lib.qgn_closure_attach(coarse.ctx, None, None, None, 0.0, 0.0)
    else:
        isc = np.ascontiguousarray(in_scale, dtype=np.float32)
        osc = np.ascontiguousarray(out_scale, dtype=np.float32)
        rc = coarse.lib.qgn_closure_attach(coarse.ctx, net.net, _fp(isc), _fp(osc), float(A8_background),
                                           float(energy_limit))
    if rc != 0:
        raise QGNError(rc, "qgn_closure_attach")


def stats(coarse):
    ev, fb = C.c_longlong(), C.c_longlong()
    last = np.zeros(3)
    rc = coarse.lib.qgn_closure_stats(coarse.ctx, C.byref(ev), C.byref(fb), last.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise QGNError(rc, "qgn_closure_stats")
    return {"evaluations": ev.value, "fallbacks": fb.value, "dE": last[0], "dZ": last[1], "E": last[2]}
