"""Warm-start network kernels on the GPU against the CPU restatement
(oracle/unet_ref.py, itself checked against finite differences).

The CPU side rounds to bfloat16 wherever the device stores bfloat16, so the
remaining differences are FP32 accumulation order on the device: a stored
bfloat16 value may land one unit in the last place (2^-7 relative) away from
the rounded FP64 value when the exact sum sits near a rounding boundary."""
import numpy as np
import pytest

import unet_ref as U

pytestmark = pytest.mark.gpu

BF16_ULP = 2.0 ** -7


def _bf16_close(got, ref, scale, exact_frac=0.99):
    """Every value within one bfloat16 ulp of the rounded FP64 value, or within
    2^-17 of `scale` (the sum of the magnitudes of its products: the FP32
    accumulation bound where the products cancel), most values identical."""
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    err = np.abs(got - ref)
    tol = np.maximum(BF16_ULP * np.abs(ref), 2.0 ** -17 * scale)
    bad = err > tol
    assert not bad.any(), f"{bad.sum()} values off by more than 1 ulp; max err {err.max()}"
    assert (err == 0).mean() >= exact_frac, f"only {(err == 0).mean():.4f} identical"


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-30))


CONV_CASES = [(16, 16), (16, 32), (48, 16), (96, 32), (64, 64), (32, 48), (192, 64), (64, 128), (128, 96), (128, 192)]


@pytest.mark.parametrize("cin,cout", CONV_CASES)
def test_conv3x3_forward_and_backward(cuda, cin, cout):
    import torch
    import mvs_b200 as M
    rng = np.random.default_rng(cin * 1000 + cout)
    B, H, W = 2, 20, 12                      # partial 8x16 tiles in both directions
    x = torch.from_numpy(np.maximum(rng.normal(size=(B, H, W, cin)), -0.2).astype(np.float32)).to(cuda)
    x = x.to(torch.bfloat16).contiguous()
    w = torch.from_numpy((rng.normal(size=(cout, cin, 3, 3)) * np.sqrt(2.0 / (9 * cin))).astype(np.float32)).to(cuda)
    b = torch.from_numpy(rng.normal(size=cout).astype(np.float32) * 0.1).to(cuda)
    out = torch.empty((B, H, W, cout), dtype=torch.bfloat16, device=cuda)
    wpack = torch.empty(2 * 9 * cin * cout, dtype=torch.bfloat16, device=cuda)
    err = torch.zeros(1, dtype=torch.int32, device=cuda)
    M.conv3x3_forward(x, w, b, True, out, wpack, err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    xn = x.float().cpu().numpy().astype(np.float64)
    wn = U.round_bf16(w.cpu().numpy()).reshape(cout, cin, 9)
    ref = U.round_bf16(U.conv3x3(xn, wn, b.cpu().numpy(), relu=True))
    _bf16_close(out.float().cpu().numpy(), ref, U.conv3x3(np.abs(xn), np.abs(wn)))

    dz = torch.from_numpy(rng.normal(size=(B, H, W, cout)).astype(np.float32)).to(cuda).to(torch.bfloat16)
    dx = torch.empty((B, H, W, cin), dtype=torch.bfloat16, device=cuda)
    dw = torch.zeros((cout, cin, 3, 3), dtype=torch.float32, device=cuda)
    db = torch.zeros(cout, dtype=torch.float32, device=cuda)
    M.conv3x3_backward(x, w, dz.contiguous(), True, dx, dw, db, wpack, err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    dzn = dz.float().cpu().numpy().astype(np.float64)
    rdx, rdw, rdb = U.conv3x3_backward(xn, wn, dzn)
    _bf16_close(dx.float().cpu().numpy(), U.round_bf16(rdx * (xn > 0)),
                U.conv3x3_backward(xn, np.abs(wn), np.abs(dzn))[0])
    assert _rel(dw.cpu().numpy().reshape(cout, cin, 9), rdw) < 1e-5
    assert _rel(db.cpu().numpy(), rdb) < 1e-5
    # the CUDA-core formulation of the weight gradient agrees too
    dw2 = torch.zeros_like(dw)
    M.conv3x3_backward(x, w, dz.contiguous(), True, None, dw2, None, wpack, err, tensor_cores=False)
    torch.cuda.synchronize()
    assert _rel(dw2.cpu().numpy().reshape(cout, cin, 9), rdw) < 1e-5


def _net_inputs(rng, B, H, W):
    """Random inputs; targets offset coherently from the input depth so that the
    gradients are sums without heavy cancellation."""
    wta = rng.uniform(0.5, 6.0, (B, H, W)).astype(np.float32)
    cost = rng.uniform(0.0, 1.5, (B, H, W)).astype(np.float32)
    ref = rng.uniform(0.0, 255.0, (B, H, W)).astype(np.float32)
    ut = (wta + 0.5 + rng.normal(0.0, 0.05, (B, H, W))).astype(np.float32)
    vt = (0.01 + rng.normal(0.0, 0.002, (B, 2, H, W))).astype(np.float32)
    return wta, cost, ref, ut, vt


def test_network_forward_and_gradients_match_oracle(cuda):
    """Whole network, forward and backward, against the CPU restatement with
    bfloat16 storage.  Activations within a rounding of zero can land on the
    other side of a ReLU on the device (FP32 vs FP64 sums), which switches that
    pixel's gradient path; the per-layer bar (3% relative, cosine > 0.999) is
    the size of that effect between the CPU's own bfloat16 and FP64 passes on
    these inputs, a layout or indexing error gives O(1)."""
    import torch
    import mvs_b200 as M
    B, H, W = 2, 32, 48
    rng = np.random.default_rng(21)
    net = M.Unet(B, H, W)
    p = net.init_params(seed=4)
    p = p.copy()
    for l in range(14):
        ci, co, wo, bo = net.layer_info(l)
        p[bo:bo + co] = rng.uniform(0.0, 0.05, co)
    net.set_params(p)
    wta, cost, ref, ut, vt = _net_inputs(rng, B, H, W)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda)
    d_wta, d_cost, d_ref, d_ut, d_vt = T(wta), T(cost), T(ref), T(ut), T(vt)
    u = torch.empty((B, H, W), device=cuda)
    v = torch.empty((B, 2, H, W), device=cuda)
    net.forward(d_wta, d_cost, d_ref, u, v)
    loss = net.backward(d_ut, d_vt)
    net.check()
    _, g = net.get_params(grads=True)

    o = U.Net(p, M.UNET_DEFAULT_NORM, bf16=True)
    ru, rv = o.forward(wta, cost, ref)
    rloss, rg = o.backward(ut, vt)
    us, vs = M.UNET_DEFAULT_NORM[3:5]
    # predictions: the head is FP32 on the device; the activations it reads may
    # differ by a bfloat16 ulp here and there
    assert np.max(np.abs(u.cpu().numpy() - ru)) < 1e-2 * us
    assert np.max(np.abs(v.cpu().numpy() - rv)) < 1e-2 * vs
    assert abs(loss - rloss) <= 1e-3 * rloss
    offs, head, n = U.layout()
    for l, (ci, co, wo, bo) in enumerate(offs):
        gw = g[wo:wo + 9 * ci * co]
        if l == 0:   # the 13 padded input channels carry zeros: only the 3 features
            gw = gw.reshape(co, ci, 9)[:, :3]
            rgw = rg[wo:wo + 9 * ci * co].reshape(co, ci, 9)[:, :3]
        else:
            rgw = rg[wo:wo + 9 * ci * co]
        cos = float(np.dot(gw.ravel(), rgw.ravel()) / (np.linalg.norm(gw) * np.linalg.norm(rgw)))
        assert _rel(gw, rgw) < 3e-2 and cos > 0.999, (l, _rel(gw, rgw), cos)
        assert _rel(g[bo:bo + co], rg[bo:bo + co]) < 3e-2, l
    assert _rel(g[head[0]:head[0] + 51], rg[head[0]:head[0] + 51]) < 1e-3


def test_training_reduces_loss(cuda):
    """Adam on the device fits a smooth correction of the input depth."""
    import torch
    import mvs_b200 as M
    B, H, W = 4, 64, 64
    rng = np.random.default_rng(8)
    net = M.Unet(B, H, W)
    net.init_params(seed=1)
    yy, xx = np.mgrid[0:H, 0:W] / 64.0
    ref = (127.5 + 100 * np.sin(7 * xx) * np.cos(5 * yy))[None].repeat(B, 0).astype(np.float32)
    wta = (2.0 + xx + 0.5 * yy + rng.normal(0, 0.05, (B, H, W))).astype(np.float32)
    cost = rng.uniform(0.0, 0.5, (B, H, W)).astype(np.float32)
    # the target sits 0.3 m behind a smooth plane through the noisy input
    ut = (2.3 + xx + 0.5 * yy)[None].repeat(B, 0).astype(np.float32)
    vt = np.zeros((B, 2, H, W), np.float32)
    vt[:, 0] = 1.0 / 64.0
    vt[:, 1] = 0.5 / 64.0
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda)
    args = [T(wta), T(cost), T(ref), T(ut), T(vt)]
    first = net.train_step(*args, lr=1e-3)
    for _ in range(200):
        last = net.train_step(*args, lr=1e-3)
    net.check()
    assert np.isfinite(last)
    assert last < 0.05 * first, (first, last)
