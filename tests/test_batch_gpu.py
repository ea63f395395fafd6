"""Batched uneven frames (one graph launch, persistent work-list kernel)
against the single-frame sweep of each frame: the same aggregated-mode
arithmetic per (pixel, plane) and an order-free 64-bit minimum across plane
chunks, so depth, label and cost agree bit for bit, for any chunking and item
order, and again on a second launch of the same graph (its counters and
winner words re-arm themselves)."""
import numpy as np
import pytest

import mvs_b200 as M
from mvs_b200 import scenes

pytestmark = pytest.mark.gpu

SMALL = [  # (scene, w, h, views, planes, window)
    ("room", 96, 64, 3, 24, 5),
    ("room", 128, 96, 4, 40, 9),
    ("street", 200, 60, 2, 32, 7),
    ("room", 64, 48, 2, 16, 11),
    ("room", 96, 64, 3, 20, 3),
]


def _frames(cuda):
    import torch
    rnd = scenes.GpuRenderer(cuda)
    frames = []
    for k, (sc, w, h, V, P, win) in enumerate(SMALL):
        f = 0.75 * w if sc == "room" else 0.58 * w
        K = scenes.intrinsics(f, f, (w - 1) / 2.0, (h - 1) / 2.0)
        zn, zf = (0.5, 5.0) if sc == "room" else (2.0, 60.0)
        df = rnd.frame(100 + k, w, h, K, V, baseline=(0.05, 0.1) if sc == "room" else (0.2, 0.5), scene=sc)
        rel = [M.relative_pose(df.ref_cam.R, df.ref_cam.t, c.R, c.t) for c in df.src_cams]
        frames.append(dict(ref=df.ref, srcs=df.srcs.contiguous(), rel=rel, K1=df.ref_cam.K_1based,
                           depths=torch.from_numpy(scenes.inverse_depth_planes(zn, zf, P)).to(cuda), window=win,
                           zfar=zf, depth=torch.empty((h, w), device=cuda),
                           labels=torch.empty((h, w), dtype=torch.int32, device=cuda),
                           best=torch.empty((h, w), device=cuda)))
    return frames


def _single(cuda, f):
    import torch
    h, w = f["ref"].shape
    V, P = f["srcs"].shape[0], f["depths"].numel()
    desc = M.sweep_desc(w, h, V, P, f["window"], M.MOMENTS_COMPENSATED, M.SWEEP_AGGREGATED, 1e-4, 0.5, f["zfar"])
    H = torch.empty(V * P * 9, device=cuda)
    M.sweep_homographies(desc, f["K1"], f["rel"], f["depths"], H)
    d = torch.empty((h, w), device=cuda)
    lab = torch.empty((h, w), dtype=torch.int32, device=cuda)
    best = torch.empty((h, w), device=cuda)
    ws = torch.empty(M.sweep_workspace_bytes(desc) // 8 + 1, dtype=torch.int64, device=cuda)
    M.sweep(desc, f["ref"], f["srcs"], H, f["depths"], d, lab, best, None, ws)
    torch.cuda.synchronize()
    return d.cpu().numpy(), lab.cpu().numpy(), best.cpu().numpy()


@pytest.mark.parametrize("tuning", [(8, 2, M.BATCH_ORDER_INTERLEAVED), (0, 1, M.BATCH_ORDER_FRAME),
                                    (16, 3, M.BATCH_ORDER_LARGEST_FIRST)])
def test_batch_matches_single_frame_sweeps(cuda, tuning):
    import torch
    frames = _frames(cuda)
    ref = [_single(cuda, f) for f in frames]
    b = M.Batch(frames, M.MOMENTS_COMPENSATED, tuning=tuning)
    assert b.tuning == tuning
    for rep in range(2):
        for f in frames:
            f["depth"].fill_(-1)
            f["labels"].fill_(-7)
        b.run()
        torch.cuda.synchronize()
        for f, (d, lab, best) in zip(frames, ref):
            np.testing.assert_array_equal(f["labels"].cpu().numpy(), lab)
            np.testing.assert_array_equal(f["depth"].cpu().numpy(), d)
            np.testing.assert_array_equal(f["best"].cpu().numpy(), best)
        lat = b.latencies_ms()
        assert np.all(lat > 0) and np.all(np.isfinite(lat))
    b.close()


def test_batch_autotuner_picks_a_candidate(cuda):
    import torch
    frames = _frames(cuda)
    b = M.Batch(frames, M.MOMENTS_COMPENSATED)
    ppc, ctas, order = b.tuning
    assert ppc in (16, 32, 64, 0) and ctas in (1, 2, 3) and order in (0, 1, 2)
    b.run()
    torch.cuda.synchronize()
    d, lab, best = _single(cuda, frames[1])
    np.testing.assert_array_equal(frames[1]["labels"].cpu().numpy(), lab)
    # the choice is cached per batch shape: a second batch of the same shape skips the search
    b2 = M.Batch(frames, M.MOMENTS_COMPENSATED)
    assert b2.tuning == b.tuning
