"""The on-chip persistent TGV2 iteration (one cooperative launch per
linearisation, state in shared memory, grid barriers) against the fused
launch-per-iteration kernel: the same arithmetic per pixel, so after a fixed
number of iterations u, v, p, q and every r agree bit for bit, on images with
partial tiles and at the full 640x480x8 size.  With an energy tolerance the
persistent kernel sums the energy in another order (per-CTA partials), so the
stopping iteration may move by one check.

The launch-per-iteration form stops on the device: the energy check sets a
flag, later launches return at once and the host polls the flag.  A run it
stops must equal a run of that many iterations without a tolerance."""
import numpy as np
import pytest

import mvs_b200 as M
from mvs_b200 import hostmath as hm, scenes

pytestmark = pytest.mark.gpu

# the persistent kernel, requested explicitly, runs where the image fits one
# tile per SM: 640x480 (140 tiles of 64x35), 600x420 (partial tiles on both
# edges) and 320x240 (fewer tiles than SMs)
CASES = [(640, 480, 8), (600, 420, 3), (640, 480, 1), (320, 240, 4)]


def _setup(cuda, w, h, V, seed=3):
    import torch
    rnd = scenes.GpuRenderer(cuda)
    K = scenes.intrinsics(0.75 * w, 0.75 * w, (w - 1) / 2.0, (h - 1) / 2.0)
    df = rnd.frame(seed, w, h, K, V, baseline=(0.03, 0.08))
    Kf = np.float32(df.ref_cam.K_1based)
    rel = [hm.relative_f32(df.ref_cam.R, df.ref_cam.t, c.R, c.t) for c in df.src_cams]
    rng = np.random.default_rng(seed)
    start = torch.from_numpy((df.depth_gt.cpu().numpy() * (1 + 0.03 * rng.standard_normal((h, w)))).astype(np.float32))
    ws = torch.empty(M.tgv2_workspace_bytes(w, h, V) // 8 + 1, dtype=torch.int64, device=cuda)
    return dict(ref=df.ref, srcs=df.srcs.contiguous(), K=Kf.reshape(9), iK=hm.inv3_f32(Kf).reshape(9),
                Rs=np.stack([r[0].reshape(9) for r in rel]), ts=np.stack([r[1] for r in rel]),
                start=start.to(cuda), ws=ws, w=w, h=h, V=V)


def _run(cuda, s, prm):
    import torch
    u = s["start"].clone()
    v = torch.zeros((2, s["h"], s["w"]), device=cuda)
    pq = torch.zeros((5, s["h"], s["w"]), device=cuda)
    r = torch.zeros((s["V"], s["h"], s["w"]), device=cuda)
    it, e = M.tgv2_run_warm(s["ref"], s["srcs"], s["K"], s["iK"], s["Rs"], s["ts"], prm, s["start"], u, v, pq=pq, r=r,
                            workspace=s["ws"])
    torch.cuda.synchronize()
    return it, e, u.cpu().numpy(), v.cpu().numpy(), pq.cpu().numpy(), r.cpu().numpy()


@pytest.mark.parametrize("w,h,V", CASES)
def test_persistent_equals_launch_per_iteration(cuda, w, h, V):
    s = _setup(cuda, w, h, V)
    a = _run(cuda, s, M.tgv2_params(niters=57, warps=2, iteration_kernel=M.TGV2_ITER_PERSISTENT))
    b = _run(cuda, s, M.tgv2_params(niters=57, warps=2, iteration_kernel=M.TGV2_ITER_LAUNCH))
    assert a[0] == b[0] == 114
    assert a[1] == b[1]
    for x, y in zip(a[2:], b[2:]):
        np.testing.assert_array_equal(x, y)


def test_persistent_tolerance_stop(cuda):
    s = _setup(cuda, 640, 480, 8, seed=5)
    prm = dict(niters=500, warps=1, tol=1e-4, check_every=10, max_iters=500)
    a = _run(cuda, s, M.tgv2_params(**prm, iteration_kernel=M.TGV2_ITER_PERSISTENT))
    b = _run(cuda, s, M.tgv2_params(**prm, iteration_kernel=M.TGV2_ITER_LAUNCH))
    assert abs(a[0] - b[0]) <= 10
    if a[0] == b[0]:
        np.testing.assert_array_equal(a[2], b[2])
    assert abs(a[1] - b[1]) <= 1e-6 * abs(b[1]) + abs(a[1] - b[1]) * (a[0] != b[0])


@pytest.mark.parametrize("w,h,V,niters,warps,tol", [(640, 480, 8, 400, 1, 3e-3), (320, 240, 4, 150, 4, 3e-3)])
def test_device_side_stop_equals_a_fixed_count(cuda, w, h, V, niters, warps, tol):
    """Launches after the tolerance is met change nothing: u, v, p, q, r and the
    energy equal those of a run of the returned iteration count.  (With 150
    iterations per linearisation the small case stops in a later
    linearisation, where the previous energy starts anew.)"""
    s = _setup(cuda, w, h, V, seed=7)
    a = _run(cuda, s, M.tgv2_params(niters=niters, warps=warps, tol=tol, check_every=10,
                                    iteration_kernel=M.TGV2_ITER_LAUNCH))
    it = a[0]
    assert 0 < it < niters * warps and it % 10 == 0
    full, last = divmod(it, niters)
    if last == 0:   # stopped at the end of a linearisation: that many full ones
        b = _run(cuda, s, M.tgv2_params(niters=niters, warps=full, iteration_kernel=M.TGV2_ITER_LAUNCH))
    else:
        # the first `full` linearisations ran completely; the last one stopped after `last`
        b = _run(cuda, s, M.tgv2_params(niters=niters, warps=full + 1, max_iters=it,
                                        iteration_kernel=M.TGV2_ITER_LAUNCH))
    assert b[0] == it
    assert a[1] == b[1]
    for x, y in zip(a[2:], b[2:]):
        np.testing.assert_array_equal(x, y)
