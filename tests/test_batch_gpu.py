"""Batched uneven frames (one graph launch, persistent work-list kernel)
against the single-frame sweep of each frame: the same aggregated-mode
arithmetic per (pixel, plane) and an order-free 64-bit minimum across plane
chunks, so depth, label and cost agree bit for bit, for any chunking and item
order, and again on a second launch of the same graph (its counters and
winner words re-arm themselves)."""
import numpy as np
import pytest

import pyoracle as po
import mvs_b200 as M
from mvs_b200 import scenes
from test_sweep_gpu import bf16_round

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


@pytest.mark.parametrize("tuning", [(8, 2, M.BATCH_ORDER_INTERLEAVED, 0), (0, 1, M.BATCH_ORDER_FRAME, 0),
                                    (16, 3, M.BATCH_ORDER_LARGEST_FIRST, 0)])
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
    ppc, ctas, order, step = b.tuning
    assert ppc in (16, 32, 64, 0) and ctas in (1, 2, 3) and order in (0, 1, 2) and step in (0, 1)
    b.run()
    torch.cuda.synchronize()
    if step == 0:   # the widest tile is the single-frame kernel's
        d, lab, best = _single(cuda, frames[1])
        np.testing.assert_array_equal(frames[1]["labels"].cpu().numpy(), lab)
    # the choice is cached per batch shape: a second batch of the same shape skips the search
    b2 = M.Batch(frames, M.MOMENTS_COMPENSATED)
    assert b2.tuning == b.tuning


def _fp64_wta(f):
    """FP64 oracle: argmin over planes of BF16(max(0, 1 - mean NCC over views))."""
    ref = f["ref"].cpu().numpy()
    srcs = list(f["srcs"].cpu().numpy())
    planes = f["depths"].cpu().numpy()
    h, w = ref.shape
    Rref, tref = np.eye(3), np.zeros(3)   # relative poses: the reference camera at the origin
    H64 = po.homographies(f["K1"], Rref, tref, [(np.asarray(R), np.asarray(t)) for R, t in f["rel"]], planes,
                          precision="f64")
    c64 = np.maximum(1.0 - po.sweep_ncc_band(ref, srcs, H64, f["window"], 0, h) / len(srcs), 0.0)
    return np.argmin(bf16_round(c64.astype(np.float32)), axis=0)


def test_batch_narrow_tiles_vs_fp64_oracle(cuda):
    """tile_step 1 (56- or 48-column tiles): its own per-tile shift of the
    compensated sums, so the labels are checked against the FP64 oracle, with
    the bar of the single-frame aggregated sweep's small frames."""
    import torch
    frames = _frames(cuda)
    b = M.Batch(frames, M.MOMENTS_COMPENSATED, tuning=(16, 2, M.BATCH_ORDER_FRAME, 1))
    assert b.tuning[3] == 1
    b.run()
    torch.cuda.synchronize()
    for f in frames:
        lab = f["labels"].cpu().numpy()
        o = _fp64_wta(f)
        same = float(np.mean(lab == o))
        near = float(np.mean(np.abs(lab.astype(np.int64) - o) <= 1))
        assert same >= 0.99 and near >= 0.999, (f["ref"].shape, same, near)
    b.close()


def _big_frames(cuda):
    """A 1242x375 street frame (KITTI intrinsics, 4 views, 128 planes, 7x7) and a
    640x480 box-room frame with the bench's 8 views, 256 planes and 9x9."""
    import torch
    rnd = scenes.GpuRenderer(cuda)
    out = []
    for kind, seed, w, h, K, V, P, win, zn, zf, base in [
            ("street", 77, 1242, 375, scenes.intrinsics(721.5, 721.5, 609.6, 172.9), 4, 128, 7, 2.0, 60.0,
             (0.2, 0.5)),
            ("room", 78, 640, 480, scenes.intrinsics(481.2, 481.2, 319.5, 239.5), 8, 256, 9, 0.4, 8.0,
             (0.02, 0.10))]:
        df = rnd.frame(seed, w, h, K, V, baseline=base, scene=kind)
        rel = [M.relative_pose(df.ref_cam.R, df.ref_cam.t, c.R, c.t) for c in df.src_cams]
        out.append(dict(ref=df.ref, srcs=df.srcs.contiguous(), rel=rel, K1=df.ref_cam.K_1based,
                        depths=torch.from_numpy(scenes.inverse_depth_planes(zn, zf, P)).to(cuda), window=win,
                        zfar=zf, depth=torch.empty((h, w), device=cuda),
                        labels=torch.empty((h, w), dtype=torch.int32, device=cuda),
                        best=torch.empty((h, w), device=cuda)))
    return out


def test_batch_full_size_frames_match_single_frame(cuda):
    """Real sizes in one batch: a 1242x375 street frame and a 640x480, 8-view,
    256-plane frame, bit for bit against the single-frame sweep of each."""
    import torch
    frames = _big_frames(cuda)
    ref = [_single(cuda, f) for f in frames]
    b = M.Batch(frames, M.MOMENTS_COMPENSATED, tuning=(32, 3, M.BATCH_ORDER_LARGEST_FIRST, 0))
    b.run()
    torch.cuda.synchronize()
    for f, (d, lab, best) in zip(frames, ref):
        np.testing.assert_array_equal(f["labels"].cpu().numpy(), lab)
        np.testing.assert_array_equal(f["depth"].cpu().numpy(), d)
        np.testing.assert_array_equal(f["best"].cpu().numpy(), best)
    b.close()
