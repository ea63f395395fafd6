"""The CPU restatement of the warm-start network: its backward pass against
finite differences of its own forward pass (FP64), and its parameter layout
against the device handle's."""
import numpy as np
import pytest

import unet_ref as U


def _inputs(rng, B=1, H=16, W=16):
    wta = rng.uniform(0.5, 5.0, (B, H, W))
    cost = rng.uniform(0.0, 1.2, (B, H, W))
    ref = rng.uniform(0.0, 255.0, (B, H, W))
    ut = wta + rng.normal(0.0, 0.2, (B, H, W))
    vt = rng.normal(0.0, 0.01, (B, 2, H, W))
    return wta, cost, ref, ut, vt


def test_layout_matches_layer_table():
    offs, head, n = U.layout()
    assert len(offs) == 14
    assert n == sum(9 * ci * co + co for ci, co in U.LAYERS) + 51
    # ~0.5M parameters (4 levels, 16/32/64/128 channels)
    assert 450_000 < n < 520_000


def test_round_bf16_ties_to_even():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5, 0.0], np.float32)
    r = U.round_bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                      # tie, rounds to the even significand
    assert r[2] == 1.0 + 2.0 ** -6          # tie, rounds up to even
    assert r[3] == -2.5 and r[4] == 0.0


def test_conv_backward_matches_finite_differences():
    rng = np.random.default_rng(5)
    x = rng.normal(size=(2, 5, 7, 16))
    w = rng.normal(size=(8, 16, 9)) * 0.2
    dz = rng.normal(size=(2, 5, 7, 8))
    dx, dw, db = U.conv3x3_backward(x, w, dz)
    f = lambda xx, ww: float(np.sum(dz * U.conv3x3(xx, ww, np.zeros(8))))
    h = 1e-6
    for idx in [(0, 0, 0, 0), (1, 4, 6, 15), (0, 2, 3, 7)]:
        xp, xm = x.copy(), x.copy()
        xp[idx] += h
        xm[idx] -= h
        assert abs((f(xp, w) - f(xm, w)) / (2 * h) - dx[idx]) < 1e-6 * max(1.0, abs(dx[idx]))
    for idx in [(0, 0, 0), (7, 15, 8), (3, 5, 4)]:
        wp, wm = w.copy(), w.copy()
        wp[idx] += h
        wm[idx] -= h
        assert abs((f(x, wp) - f(x, wm)) / (2 * h) - dw[idx]) < 1e-6 * max(1.0, abs(dw[idx]))
    assert np.allclose(db, dz.sum((0, 1, 2)))


def test_network_gradient_matches_finite_differences():
    rng = np.random.default_rng(11)
    p = U.init_params(3).astype(np.float64)
    offs, head, n = U.layout()
    for ci, co, wo, bo in offs:
        p[bo:bo + co] = rng.uniform(0.0, 0.05, co)    # keep most ReLUs open
    norm = (0.25, -1.0, 2.0, 1.0, 0.01, 1.0, 1.0)
    wta, cost, ref, ut, vt = _inputs(rng)
    net = U.Net(p, norm, bf16=False)
    net.forward(wta, cost, ref)
    loss, g = net.backward(ut, vt)

    def L(q):
        m = U.Net(q, norm, bf16=False)
        m.forward(wta, cost, ref)
        return m.loss(ut, vt)

    assert abs(L(p) - loss) < 1e-12
    h = 1e-6
    checked = 0
    for ci, co, wo, bo in offs + [(16, 3, head[0], head[1])]:
        nw = 48 if wo == head[0] else 9 * ci * co
        for k in list(rng.integers(wo, wo + nw, 3)) + [bo]:
            if ci == 16 and wo == offs[0][2] and (k - wo) // 9 % ci >= 3:
                continue                     # padded input channels: zero input, zero gradient
            q1, q2 = p.copy(), p.copy()
            q1[k] += h
            q2[k] -= h
            fd = (L(q1) - L(q2)) / (2 * h)
            assert abs(fd - g[k]) <= 1e-5 * max(abs(fd), 1e-3), (k, fd, g[k])
            checked += 1
    assert checked >= 40
