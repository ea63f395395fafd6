"""CPU restatement of the TGV2 warm-start network (test infrastructure only).

The network has no counterpart in the reference; this module restates, in
numpy, what the device kernels of plane-sweep-cuda_b200/csrc/unet.cu compute,
so that their forward values and gradients can be checked:

* conv3x3: zero-padded 3x3 convolution, NHWC activations, weights
  W[cout][cin][3][3] (tap t = 3*ky + kx), bias, optional ReLU;
* pool: 2x2 average; upcat: nearest 2x upsampling concatenated with a skip
  tensor (upsampled channels first);
* head: 1x1 convolution 16 -> 3, u = wta + u_scale*o0, v = v_scale*(o1, o2);
* loss = mean_p [w_u (u - u*)^2 + w_v |v - v*|^2].

With ``bf16=True`` every tensor the device stores in bfloat16 is rounded to
bfloat16 at the same place (activations, input features, activation
gradients), the rest is FP64; the remaining differences from the device are
its FP32 accumulation order.  With ``bf16=False`` everything is FP64, which is
what the finite-difference check of the gradients uses.
"""
from __future__ import annotations

import numpy as np

LAYERS = ((16, 16), (16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (64, 128), (128, 128),
          (192, 64), (64, 64), (96, 32), (32, 32), (48, 16), (16, 16))
(E0A, E0B, E1A, E1B, E2A, E2B, E3A, E3B, D2A, D2B, D1A, D1B, D0A, D0B) = range(14)


def round_bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    a = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((a + 0x7FFF + ((a >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def layout():
    """Offsets of each layer's W and bias in the flat parameter array, then the head."""
    offs, off = [], 0
    for ci, co in LAYERS:
        w = off
        off += 9 * ci * co
        offs.append((ci, co, w, off))
        off += co
    head = (off, off + 48)
    return offs, head, off + 51


def _patches(x):
    """(B, H, W, C) -> (B, H, W, 9, C) zero-padded 3x3 neighbourhoods."""
    B, H, W, C = x.shape
    xp = np.zeros((B, H + 2, W + 2, C), x.dtype)
    xp[:, 1:-1, 1:-1] = x
    return np.stack([xp[:, ky:ky + H, kx:kx + W] for ky in range(3) for kx in range(3)], axis=3)


def conv3x3(x, w, b=None, relu=False):
    """x (B, H, W, cin), w (cout, cin, 9) -> (B, H, W, cout), FP64."""
    co, ci = w.shape[:2]
    P = _patches(np.asarray(x, np.float64))
    Wr = np.asarray(w, np.float64).reshape(co, ci, 9).transpose(2, 1, 0).reshape(9 * ci, co)
    y = P.reshape(-1, 9 * ci) @ Wr
    if b is not None:
        y = y + np.asarray(b, np.float64)
    if relu:
        y = np.maximum(y, 0.0)
    return y.reshape(x.shape[:3] + (co,))


def conv3x3_backward(x, w, dz):
    """Gradients of sum(dz * conv3x3(x, w)) w.r.t. x, w (cout, cin, 9) and the bias."""
    co, ci = w.shape[:2]
    B, H, W, _ = x.shape
    Wr = np.asarray(w, np.float64).reshape(co, ci, 9).transpose(2, 1, 0).reshape(9 * ci, co)
    dzf = np.asarray(dz, np.float64).reshape(-1, co)
    dP = (dzf @ Wr.T).reshape(B, H, W, 9, ci)
    dxp = np.zeros((B, H + 2, W + 2, ci))
    for t in range(9):
        ky, kx = divmod(t, 3)
        dxp[:, ky:ky + H, kx:kx + W] += dP[:, :, :, t]
    P = _patches(np.asarray(x, np.float64)).reshape(-1, 9 * ci)
    dWr = P.T @ dzf
    dw = dWr.reshape(9, ci, co).transpose(2, 1, 0)
    return dxp[:, 1:-1, 1:-1], dw, dzf.sum(0)


def pool(x, fp32=False):
    """2x2 average; fp32=True repeats the device's FP32 sum order."""
    x = np.asarray(x, np.float32 if fp32 else np.float64)
    s = x[:, 0::2, 0::2] + x[:, 0::2, 1::2]
    s = s + x[:, 1::2, 0::2]
    s = s + x[:, 1::2, 1::2]
    return (s * x.dtype.type(0.25)).astype(np.float64)


def upcat(prev, skip):
    up = np.repeat(np.repeat(prev, 2, axis=1), 2, axis=2)
    return np.concatenate([up, skip], axis=3)


def features(wta, cost, ref255, norm):
    ds, dsh, clip = (np.float32(v) for v in norm[:3])
    d = np.nan_to_num(np.asarray(wta, np.float32), nan=0.0)
    c = np.asarray(cost, np.float32) if cost is not None else np.zeros_like(d)
    c = np.where(np.isnan(c), clip, c)
    f0 = d * ds + dsh
    f1 = np.float32(1) - np.minimum(np.maximum(c, np.float32(0)), clip)
    f2 = np.asarray(ref255, np.float32) * np.float32(1.0 / 255.0) - np.float32(0.5)
    x = np.zeros(d.shape + (16,), np.float64)
    x[..., 0], x[..., 1], x[..., 2] = f0, f1, f2
    return x


class Net:
    """Forward and backward of the warm-start U-Net on the CPU."""

    def __init__(self, params, norm, bf16=True):
        self.p = np.asarray(params, np.float64)
        self.norm = tuple(float(v) for v in norm)
        self.bf16 = bf16
        self.offs, self.head, self.n = layout()
        assert self.p.size == self.n

    def _r(self, x):
        return round_bf16(x) if self.bf16 else x

    def _w(self, l):
        ci, co, w, b = self.offs[l]
        W = self.p[w:w + 9 * ci * co].reshape(co, ci, 9)
        if self.bf16:
            W = round_bf16(W)
        return W, self.p[b:b + co]

    def _conv(self, l, x):
        W, b = self._w(l)
        return self._r(conv3x3(x, W, b, relu=True))

    def forward(self, wta, cost, ref255):
        """wta, cost, ref255: (B, H, W).  Returns u (B, H, W), v (B, 2, H, W)."""
        a = {}
        a["x0"] = self._r(features(wta, cost, ref255, self.norm))
        a["e0a"] = self._conv(E0A, a["x0"])
        a["e0"] = self._conv(E0B, a["e0a"])
        a["p0"] = self._r(pool(a["e0"], self.bf16))
        a["e1a"] = self._conv(E1A, a["p0"])
        a["e1"] = self._conv(E1B, a["e1a"])
        a["p1"] = self._r(pool(a["e1"], self.bf16))
        a["e2a"] = self._conv(E2A, a["p1"])
        a["e2"] = self._conv(E2B, a["e2a"])
        a["p2"] = self._r(pool(a["e2"], self.bf16))
        a["e3a"] = self._conv(E3A, a["p2"])
        a["e3"] = self._conv(E3B, a["e3a"])
        a["c2"] = upcat(a["e3"], a["e2"])
        a["d2a"] = self._conv(D2A, a["c2"])
        a["d2"] = self._conv(D2B, a["d2a"])
        a["c1"] = upcat(a["d2"], a["e1"])
        a["d1a"] = self._conv(D1A, a["c1"])
        a["d1"] = self._conv(D1B, a["d1a"])
        a["c0"] = upcat(a["d1"], a["e0"])
        a["d0a"] = self._conv(D0A, a["c0"])
        a["d0"] = self._conv(D0B, a["d0a"])
        hw, hb = self.head
        Wh = self.p[hw:hw + 48].reshape(3, 16)
        bh = self.p[hb:hb + 3]
        o = a["d0"] @ Wh.T + bh
        _, _, _, us, vs = self.norm[:5]
        wta64 = np.nan_to_num(np.asarray(wta, np.float64), nan=0.0)
        self.a = a
        self.wta = wta64
        u = wta64 + us * o[..., 0]
        v = np.stack([vs * o[..., 1], vs * o[..., 2]], axis=1)
        self.u, self.v = u, v
        return u, v

    def loss(self, ut, vt):
        wu, wv = self.norm[5:7]
        eu = self.u - ut
        ev = self.v - vt
        return float(np.mean(wu * eu ** 2 + wv * (ev[:, 0] ** 2 + ev[:, 1] ** 2)))

    def backward(self, ut, vt):
        """Loss of the last forward and its gradient (flat, the parameter layout)."""
        a = self.a
        g = np.zeros(self.n)
        _, _, _, us, vs, wu, wv = self.norm
        npix = self.u.size
        eu = self.u - ut
        ev = self.v - vt
        go = np.stack([2 * wu * eu * us, 2 * wv * ev[:, 0] * vs, 2 * wv * ev[:, 1] * vs], axis=-1) / npix
        hw, hb = self.head
        Wh = self.p[hw:hw + 48].reshape(3, 16)
        g[hw:hw + 48] = np.einsum("bhwk,bhwc->kc", go, a["d0"]).reshape(-1)
        g[hb:hb + 3] = go.sum((0, 1, 2))
        gd0 = self._r((go @ Wh) * (a["d0"] > 0))

        def cb(l, x, dz, mask):
            W, _ = self._w(l)
            dx, dw, db = conv3x3_backward(x, W, dz)
            ci, co, wo, bo = self.offs[l]
            g[wo:wo + 9 * ci * co] += dw.reshape(-1)
            g[bo:bo + co] += db
            if mask:
                dx = dx * (x > 0)
            return self._r(dx)

        def upback(dc, cp):
            d = dc[..., :cp]
            s = d[:, 0::2, 0::2] + d[:, 0::2, 1::2] + d[:, 1::2, 0::2] + d[:, 1::2, 1::2]
            return self._r(s)

        def poolback(dp, dc, coff, e):
            up = np.repeat(np.repeat(dp, 2, axis=1), 2, axis=2) * 0.25
            return self._r((up + dc[..., coff:]) * (e > 0))

        self.ga = ga = {"d0": gd0}
        gd0a = ga["d0a"] = cb(D0B, a["d0a"], gd0, True)
        gc0 = ga["c0"] = cb(D0A, a["c0"], gd0a, True)
        gd1 = ga["d1"] = upback(gc0, 32)
        gd1a = ga["d1a"] = cb(D1B, a["d1a"], gd1, True)
        gc1 = ga["c1"] = cb(D1A, a["c1"], gd1a, True)
        gd2 = ga["d2"] = upback(gc1, 64)
        gd2a = ga["d2a"] = cb(D2B, a["d2a"], gd2, True)
        gc2 = ga["c2"] = cb(D2A, a["c2"], gd2a, True)
        ge3 = ga["e3"] = upback(gc2, 128)
        ge3a = ga["e3a"] = cb(E3B, a["e3a"], ge3, True)
        gp2 = ga["p2"] = cb(E3A, a["p2"], ge3a, False)
        ge2 = ga["e2"] = poolback(gp2, gc2, 128, a["e2"])
        ge2a = ga["e2a"] = cb(E2B, a["e2a"], ge2, True)
        gp1 = ga["p1"] = cb(E2A, a["p1"], ge2a, False)
        ge1 = ga["e1"] = poolback(gp1, gc1, 64, a["e1"])
        ge1a = ga["e1a"] = cb(E1B, a["e1a"], ge1, True)
        gp0 = ga["p0"] = cb(E1A, a["p0"], ge1a, False)
        ge0 = ga["e0"] = poolback(gp0, gc0, 32, a["e0"])
        ge0a = ga["e0a"] = cb(E0B, a["e0a"], ge0, True)
        cb(E0A, a["x0"], ge0a, False)
        return self.loss(ut, vt), g


def init_params(seed=0):
    """The device handle's He-normal initialisation (mvs_b200.Unet.init_params)."""
    import math
    rng = np.random.default_rng(seed)
    offs, head, n = layout()
    p = np.zeros(n, np.float32)
    for l, (ci, co, wo, bo) in enumerate(offs):
        fan = 9 * (3 if l == 0 else ci)
        w = rng.standard_normal((co, ci, 9)) * math.sqrt(2.0 / fan)
        if l == 0:
            w[:, 3:, :] = 0.0
        p[wo:wo + co * ci * 9] = w.reshape(-1)
    p[head[0]:head[0] + 48] = rng.standard_normal(48) * 0.01
    return p
