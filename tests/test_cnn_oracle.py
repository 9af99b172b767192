"""Pins the closure network's CPU oracle (oracle/cnn_oracle.py): bf16 rounding, the periodic
convolution against a direct loop, and backpropagation against finite differences."""
import numpy as np

from oracle.cnn_oracle import CNNOracle, adam_step, bf16, conv, conv_transpose, weight_grad


def test_bf16_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -9, 1.0 + 2.0 ** -7, -2.5, 3.1415927], dtype=np.float32)
    r = bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                      # tie -> even (mantissa 0)
    assert r[2] == 1.0 + 2.0 ** -7          # above the tie rounds up
    assert r[3] == 1.0 + 2.0 ** -7
    assert r[4] == -2.5
    assert r[5] == np.float32(3.140625)


def test_conv_matches_direct_loop():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((2, 5, 6, 3))
    w = rng.standard_normal((9, 4, 3))
    b = rng.standard_normal(4)
    out = conv(x, w, b)
    ref = np.zeros_like(out)
    for bb in range(2):
        for h in range(5):
            for ww in range(6):
                acc = b.copy()
                for tap in range(9):
                    dy, dx = tap // 3 - 1, tap % 3 - 1
                    acc += w[tap] @ x[bb, (h + dy) % 5, (ww + dx) % 6]
                ref[bb, h, ww] = acc
    assert np.allclose(out, ref)
    # adjoints: <conv(x), g> = <x, conv_T(g)> and = <w, weight_grad(x, g)>
    g = rng.standard_normal(out.shape)
    lhs = np.sum(conv(x, w) * g)
    assert np.isclose(lhs, np.sum(x * conv_transpose(g, w)))
    assert np.isclose(lhs, np.sum(w * weight_grad(x, g)))


def test_backprop_matches_finite_differences():
    rng = np.random.default_rng(1)
    shapes = [(8, 4), (8, 8), (2, 8)]
    layers = [(0.4 * rng.standard_normal((9, co, ci)), 0.1 * rng.standard_normal(co)) for co, ci in shapes]
    net = CNNOracle(layers, cout_real=2)
    net.layers = [(w.astype(np.float64), b.astype(np.float64)) for w, b in layers]
    x = rng.standard_normal((2, 4, 5, 4))
    t = rng.standard_normal((2, 4, 5, 2))
    loss, grads = net.loss_and_grads(x, t, emulate=False)
    eps = 1e-6
    for l, (w, b) in enumerate(net.layers):
        for _ in range(4):
            idx = tuple(rng.integers(0, s) for s in w.shape)
            w[idx] += eps
            lp, _ = net.loss_and_grads(x, t, emulate=False)
            w[idx] -= 2 * eps
            lm, _ = net.loss_and_grads(x, t, emulate=False)
            w[idx] += eps
            assert np.isclose((lp - lm) / (2 * eps), grads[l][0][idx], rtol=1e-5, atol=1e-9)
        j = rng.integers(0, b.shape[0])
        b[j] += eps
        lp, _ = net.loss_and_grads(x, t, emulate=False)
        b[j] -= 2 * eps
        lm, _ = net.loss_and_grads(x, t, emulate=False)
        b[j] += eps
        assert np.isclose((lp - lm) / (2 * eps), grads[l][1][j], rtol=1e-5, atol=1e-9)


def test_adam_first_step_is_signed_lr():
    w = np.ones(5, np.float32)
    g = np.array([1.0, -2.0, 0.5, 0.0, 3.0], np.float32)
    w1, m, v = adam_step(w, np.zeros(5), np.zeros(5), g, 1, lr=0.01)
    # bias-corrected first step moves every weight with a nonzero gradient by lr against its sign
    assert np.allclose(w1[[0, 1, 2, 4]], 1.0 - 0.01 * np.sign(g[[0, 1, 2, 4]]), atol=1e-6)
    assert w1[3] == 1.0
