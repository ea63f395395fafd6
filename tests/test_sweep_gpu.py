"""Plane sweep on the GPU against the reference and the oracle.

Parity bars (stated per output):
* reference arithmetic (MVS_MOMENTS_REFERENCE) fed the reference's float
  homographies: per-view best NCC, labels and the averaged depthmap are
  bit-identical to the reference's own kernels run on the CPU;
* FP64 homographies built on the device: per-view labels identical on
  >= 99.9% of pixels and within one plane elsewhere;
* compensated moments: labels against the FP64 oracle, same bar.
"""
import numpy as np
import pytest

import pyoracle as po
import mvs_b200 as M
from mvs_b200 import hostmath as hm, scenes

pytestmark = pytest.mark.gpu

SWEEP_GOLDEN = ["sweep_inverse_w5", "sweep_refloop_w7", "sweep_inverse_w3_negthr"]


def float_H(K, Rref, tref, poses, planes):
    invK = hm.inv3_f32(K)
    out = []
    for Rs, ts in poses:
        Rrel, trel = hm.relative_f32(Rref, tref, Rs, ts)
        out.append([hm.homography_f32(np.float32(K), invK, Rrel, trel, d).reshape(9) for d in planes])
    return np.asarray(out, np.float32)


def run_sweep(cuda, ref, srcs, planes, win, K=None, Rref=None, tref=None, poses=None, H=None,
              moments=M.MOMENTS_REFERENCE, mode=M.SWEEP_PER_VIEW, nccthresh=0.5, zfar=5.0, cost=False):
    import torch
    h, w = ref.shape
    V, P = len(srcs), len(planes)
    desc = M.sweep_desc(w, h, V, P, win, moments, mode, 1e-4, nccthresh, zfar)
    d_ref = torch.from_numpy(np.ascontiguousarray(ref, np.float32)).to(cuda)
    d_srcs = torch.from_numpy(np.ascontiguousarray(np.stack(srcs), np.float32)).to(cuda)
    d_depths = torch.from_numpy(np.ascontiguousarray(planes, np.float32)).to(cuda)
    if H is None:
        rel = [M.relative_pose(Rref, tref, Rs, ts) for Rs, ts in poses]
        d_H = torch.empty(V * P * 9, dtype=torch.float32, device=cuda)
        M.sweep_homographies(desc, K, rel, d_depths, d_H)
    else:
        d_H = torch.from_numpy(np.ascontiguousarray(H, np.float32)).to(cuda)
    nl = V if mode == M.SWEEP_PER_VIEW else 1
    depth = torch.empty((h, w), dtype=torch.float32, device=cuda)
    labels = torch.empty((nl, h, w), dtype=torch.int32, device=cuda)
    best = torch.empty((nl, h, w), dtype=torch.float32, device=cuda)
    d_cost = torch.empty((P, h, w), dtype=torch.int16, device=cuda) if cost else None
    ws = torch.empty(M.sweep_workspace_bytes(desc) // 8 + 1, dtype=torch.int64, device=cuda)
    M.sweep(desc, d_ref, d_srcs, d_H, d_depths, depth, labels, best, d_cost, ws)
    torch.cuda.synchronize()
    out = dict(depth=depth.cpu().numpy(), label=labels.cpu().numpy(), best=best.cpu().numpy(), H=d_H.cpu().numpy())
    if cost:
        out["cost"] = d_cost.cpu().numpy().view(np.uint16)
    return out


def label_agreement(a, b):
    same = float(np.mean(a == b))
    near = float(np.mean(np.abs(a.astype(np.int64) - b.astype(np.int64)) <= 1))
    return same, near


@pytest.mark.parametrize("name", SWEEP_GOLDEN)
def test_reference_arithmetic_bit_exact_vs_reference(cuda, golden, name):
    g = golden(name)
    poses = [(g["Rsrc"][i], g["tsrc"][i]) for i in range(len(g["Rsrc"]))]
    H = float_H(g["K"], g["Rref"], g["tref"], poses, g["planes"])
    r = run_sweep(cuda, g["ref"], list(g["srcs"]), g["planes"], int(g["win"]), H=H, nccthresh=float(g["nccthresh"]),
                  zfar=float(g["zfar"]))
    np.testing.assert_array_equal(r["best"], g["best"])
    np.testing.assert_array_equal(r["label"], g["label"])
    np.testing.assert_array_equal(r["depth"], g["depth"])


def assert_label_parity(lab, best, ref_lab, ref_best, same_min=0.999, tie_tol=1e-3, weak=0.5):
    """Labels identical on >= same_min of the pixels; elsewhere within one plane, except
    where the match is a tie (the two best NCCs agree to tie_tol) or too weak to enter the
    depthmap (both best NCCs <= the NCC threshold, `weak`)."""
    d = np.abs(lab.astype(np.int64) - ref_lab.astype(np.int64))
    same = float(np.mean(d == 0))
    far = d > 1
    assert same >= same_min, (same, float(np.mean(far)))
    tie = np.abs(best - ref_best) < tie_tol
    unused = np.maximum(best, ref_best) <= weak
    assert np.all((tie | unused)[far]), (float(np.mean(far)), best[far & ~(tie | unused)][:8],
                                         ref_best[far & ~(tie | unused)][:8])
    return same


@pytest.mark.parametrize("name", SWEEP_GOLDEN)
def test_fp64_homographies_label_parity(cuda, golden, name):
    g = golden(name)
    poses = [(g["Rsrc"][i], g["tsrc"][i]) for i in range(len(g["Rsrc"]))]
    r = run_sweep(cuda, g["ref"], list(g["srcs"]), g["planes"], int(g["win"]), K=g["K"].astype(np.float64),
                  Rref=g["Rref"], tref=g["tref"], poses=poses, nccthresh=float(g["nccthresh"]), zfar=float(g["zfar"]))
    assert_label_parity(r["label"], r["best"], g["label"], g["best"], same_min=0.995)
    # the device homographies agree with the reference's float ones to float precision
    Hf = float_H(g["K"], g["Rref"], g["tref"], poses, g["planes"]).reshape(-1, 9)
    np.testing.assert_allclose(r["H"].reshape(-1, 9), Hf, rtol=2e-5, atol=2e-5)


def test_c1_fp64_homographies_with_reference_moments(cuda):
    """FP64 device homographies with the reference's naive moments, against the reference's
    arithmetic.  The naive E[x^2]-E[x]^2 magnifies the ~1e-7 relative difference of the
    homographies into NCC changes of ~1e-5, which reorders near-tied planes: labels agree on
    >= 99% of pixels and every other pixel is within one plane or a tie.  Bit-exact parity
    with the reference uses the reference's float homographies (tests above)."""
    fr, planes, win = scenes.config_small(seed=1)
    poses = [(c.R, c.t) for c in fr.src_cams]
    K1 = fr.ref_cam.K_1based
    H = po.homographies(K1, fr.ref_cam.R, fr.ref_cam.t, poses, planes, precision="f32")
    o = po.sweep(fr.ref, fr.srcs, H, planes, win, zfar=5.0, precision="f32")
    r = run_sweep(cuda, fr.ref, fr.srcs, planes, win, K=K1, Rref=fr.ref_cam.R, tref=fr.ref_cam.t, poses=poses,
                  zfar=5.0)
    assert_label_parity(r["label"], r["best"], o["label"], o["best"], same_min=0.99)


def test_c1_size_reference_arithmetic_bit_exact(cuda):
    """320x240, 4 views, 64 inverse-depth planes, 7x7: the GPU equals the f32 oracle bit for bit."""
    fr, planes, win = scenes.config_small(seed=1)
    poses = [(c.R, c.t) for c in fr.src_cams]
    K1 = fr.ref_cam.K_1based
    H = po.homographies(K1, fr.ref_cam.R, fr.ref_cam.t, poses, planes, precision="f32")
    o = po.sweep(fr.ref, fr.srcs, H, planes, win, zfar=5.0, precision="f32")
    r = run_sweep(cuda, fr.ref, fr.srcs, planes, win, H=H, zfar=5.0)
    np.testing.assert_array_equal(r["best"], o["best"])
    np.testing.assert_array_equal(r["label"], o["label"])
    np.testing.assert_array_equal(r["depth"], o["depth"])


def test_c1_compensated_vs_fp64_oracle(cuda):
    """Compensated moments + FP64 homographies against the FP64 oracle: >= 99.8% identical
    labels, all others within one plane or ties, winning NCC within 1e-4; and closer to the
    FP64 oracle than the reference's own float arithmetic is."""
    fr, planes, win = scenes.config_small(seed=1)
    poses = [(c.R, c.t) for c in fr.src_cams]
    K1 = fr.ref_cam.K_1based
    H64 = po.homographies(K1, fr.ref_cam.R, fr.ref_cam.t, poses, planes, precision="f64")
    o = po.sweep(fr.ref, fr.srcs, H64, planes, win, zfar=5.0, precision="f64")
    r = run_sweep(cuda, fr.ref, fr.srcs, planes, win, K=K1, Rref=fr.ref_cam.R, tref=fr.ref_cam.t, poses=poses,
                  moments=M.MOMENTS_COMPENSATED, zfar=5.0)
    same = assert_label_parity(r["label"], r["best"], o["label"], o["best"], same_min=0.998)
    # winning NCC where both agree on the plane: 99.9% within 1e-4, all within 1e-3 (sliding
    # FP32 window sums carry a few rounding steps more than direct sums)
    m = r["label"] == o["label"]
    err = np.abs(r["best"][m] - o["best"][m])
    assert np.quantile(err, 0.999) < 1e-4 and err.max() < 1e-3, (np.quantile(err, 0.999), err.max())
    H32 = po.homographies(K1, fr.ref_cam.R, fr.ref_cam.t, poses, planes, precision="f32")
    ref_arith = po.sweep(fr.ref, fr.srcs, H32, planes, win, zfar=5.0, precision="f32")
    assert same >= float(np.mean(ref_arith["label"] == o["label"]))


def bf16_round(x):
    x = np.ascontiguousarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (u.astype(np.uint32) << 16).view(np.float32)


@pytest.mark.parametrize("win,width,height", [(7, 96, 64), (3, 70, 45), (5, 131, 40), (11, 120, 70), (15, 77, 52)])
def test_aggregated_bf16_wta_vs_fp64_oracle(cuda, win, width, height):
    """Every tile layout of the aggregated kernel: 64-wide tiles with 8-output
    runs (3x3 to 9x9, regions of 66 to 72 columns) and 56-wide tiles with
    7-output runs (11x11 and up); frame sizes that do not divide the tiles."""
    fr, planes, win = scenes.config_tiny(seed=5, width=width, height=height, n_src=3, n_planes=24, win=win)
    poses = [(c.R, c.t) for c in fr.src_cams]
    K1 = fr.ref_cam.K_1based
    H64 = po.homographies(K1, fr.ref_cam.R, fr.ref_cam.t, poses, planes, precision="f64")
    L = po.oracle_lib()
    h, w = fr.ref.shape
    ncc = np.zeros((len(poses), len(planes), h, w))
    for v in range(len(poses)):
        for p in range(len(planes)):
            buf = np.zeros((h, w))
            L.orc_sweep_ncc_f64(w, h, po._fp(po._f32(fr.ref)), po._fp(po._f32(fr.srcs[v])),
                                po._dp(np.ascontiguousarray(H64[v, p])), win, 1e-4, po._dp(buf))
            ncc[v, p] = buf
    cost = bf16_round(np.maximum(1.0 - ncc.mean(0), 0).astype(np.float32))
    lab = np.argmin(cost, axis=0)
    r = run_sweep(cuda, fr.ref, fr.srcs, planes, win, K=K1, Rref=fr.ref_cam.R, tref=fr.ref_cam.t, poses=poses,
                  moments=M.MOMENTS_COMPENSATED, mode=M.SWEEP_AGGREGATED, zfar=5.0, cost=True)
    same, near = label_agreement(r["label"][0], lab)
    assert same >= 0.99 and near >= 0.999, (same, near)
    # the stored cost volume and a separate WTA pass over it give the same labels
    gpu_cost = (r["cost"].astype(np.uint32) << 16).view(np.float32)
    assert np.max(np.abs(gpu_cost - cost)) <= 0.02
    np.testing.assert_array_equal(np.argmin(gpu_cost, axis=0), r["label"][0])


def test_wta_volume_kernel(cuda):
    import torch
    rng = np.random.default_rng(0)
    P, h, w = 37, 24, 40
    cost = bf16_round(rng.random((P, h, w), dtype=np.float32) * 2)
    cost[5, 3, 7] = cost[:, 3, 7].min()          # a tie: the earlier plane wins
    bits = (cost.view(np.uint32) >> 16).astype(np.uint16)
    depths = np.linspace(1, 2, P).astype(np.float32)
    d_cost = torch.from_numpy(bits.view(np.int16)).to(cuda)
    d_depths = torch.from_numpy(depths).to(cuda)
    depth = torch.empty((h, w), device=cuda)
    labels = torch.empty((h, w), dtype=torch.int32, device=cuda)
    best = torch.empty((h, w), device=cuda)
    M.sweep_wta_volume(d_cost, d_depths, h * w, P, 9.0, depth, labels, best)
    torch.cuda.synchronize()
    lab = np.argmin(cost, axis=0)
    np.testing.assert_array_equal(labels.cpu().numpy(), lab)
    np.testing.assert_array_equal(depth.cpu().numpy(), depths[lab])


@pytest.mark.parametrize("win", [3, 9, 15])
def test_window_sizes_and_ragged_tiles(cuda, win):
    """Odd sizes that do not divide the tile; image only slightly larger than the window."""
    fr, planes, _ = scenes.config_tiny(seed=7, width=win + 5, height=win + 2, n_src=2, n_planes=9, win=win)
    poses = [(c.R, c.t) for c in fr.src_cams]
    H = po.homographies(fr.ref_cam.K_1based, fr.ref_cam.R, fr.ref_cam.t, poses, planes, precision="f32")
    o = po.sweep(fr.ref, fr.srcs, H, planes, win, zfar=5.0, precision="f32")
    r = run_sweep(cuda, fr.ref, fr.srcs, planes, win, H=H, zfar=5.0)
    np.testing.assert_array_equal(r["best"], o["best"])
    np.testing.assert_array_equal(r["label"], o["label"])
    np.testing.assert_array_equal(r["depth"], o["depth"])


def test_flat_source_gives_no_match_and_zfar(cuda):
    """A constant source: NCC is 0 except where the warp leaves the image (zero fill) and the
    window straddles the border; the GPU matches the oracle there bit for bit, and pixels
    where no view passes the NCC threshold get zfar."""
    fr, planes, win = scenes.config_tiny(seed=8, width=48, height=40, n_src=2, n_planes=6, win=5)
    srcs = [np.full_like(fr.srcs[0], 77.0), np.full_like(fr.srcs[1], 12.5)]
    poses = [(c.R, c.t) for c in fr.src_cams]
    H = po.homographies(fr.ref_cam.K_1based, fr.ref_cam.R, fr.ref_cam.t, poses, planes, precision="f32")
    o = po.sweep(fr.ref, srcs, H, planes, win, zfar=3.25, precision="f32")
    r = run_sweep(cuda, fr.ref, srcs, planes, win, H=H, zfar=3.25)
    np.testing.assert_array_equal(r["label"], o["label"])
    np.testing.assert_array_equal(r["depth"], o["depth"])
    assert np.mean(r["label"] == -1) > 0.5
    none = np.all(r["best"] <= 0.5, axis=0)
    assert np.all(r["depth"][none] == np.float32(3.25))


def test_many_plane_chunks_match_single_chunk(cuda):
    """A small image with many planes is split into plane chunks merged by 64-bit max; same result."""
    fr, _, win = scenes.config_tiny(seed=9, width=40, height=32, n_src=1, n_planes=8, win=5)
    planes = scenes.inverse_depth_planes(0.5, 5.0, 300)
    poses = [(c.R, c.t) for c in fr.src_cams]
    H = po.homographies(fr.ref_cam.K_1based, fr.ref_cam.R, fr.ref_cam.t, poses, planes, precision="f32")
    o = po.sweep(fr.ref, fr.srcs, H, planes, win, zfar=5.0, precision="f32")
    r = run_sweep(cuda, fr.ref, fr.srcs, planes, win, H=H, zfar=5.0)
    np.testing.assert_array_equal(r["label"], o["label"])
    np.testing.assert_array_equal(r["best"], o["best"])


def test_full_size_properties(cuda):
    """640x480, 8 views, 256 planes, 9x9 (compensated): labels in range, deterministic, depth
    consistent with the per-view labels, and close to the ray-cast ground truth."""
    fr, planes, win = scenes.config_full(seed=2)
    poses = [(c.R, c.t) for c in fr.src_cams]
    args = dict(K=fr.ref_cam.K_1based, Rref=fr.ref_cam.R, tref=fr.ref_cam.t, poses=poses,
                moments=M.MOMENTS_COMPENSATED, zfar=8.0)
    r1 = run_sweep(cuda, fr.ref, fr.srcs, planes, win, **args)
    r2 = run_sweep(cuda, fr.ref, fr.srcs, planes, win, **args)
    np.testing.assert_array_equal(r1["label"], r2["label"])
    np.testing.assert_array_equal(r1["depth"], r2["depth"])
    lab = r1["label"]
    assert lab.min() >= -1 and lab.max() < len(planes)
    # the averaged depth is the reference combine of the per-view labels
    vd = np.where(lab >= 0, planes[np.clip(lab, 0, None)], 0).astype(np.float32)
    ok = r1["best"] > 0.5
    cnt = ok.sum(0).astype(np.float32)
    s = np.zeros(fr.ref.shape, np.float32)
    for v in range(len(poses)):
        s = (s + np.where(ok[v], vd[v], 0)).astype(np.float32)
    want = np.where(cnt > 0, s / np.where(cnt > 0, cnt, 1), 8.0).astype(np.float32)
    np.testing.assert_allclose(r1["depth"], want, rtol=1e-6)
    rel = np.abs(r1["depth"] - fr.depth_gt) / fr.depth_gt
    assert np.median(rel[cnt > 0]) < 0.03


@pytest.mark.parametrize("moments,win", [(M.MOMENTS_COMPENSATED, 9), (M.MOMENTS_COMPENSATED, 15),
                                         (M.MOMENTS_REFERENCE, 5)])
def test_tma_staged_form_equals_gather_form(cuda, moments, win, monkeypatch):
    """The aggregated sweep with TMA-staged source regions (MVS_SWEEP_STAGING=tma)
    against the gather form: cost volume, labels, depth and best cost bit for
    bit, at 640x480 with 8 views and 96 planes, and on a frame whose rows are
    not whole 16-byte groups (the gather form then runs)."""
    fr, planes, _ = scenes.config_full(seed=2)
    planes = planes[::4].copy() if win == 9 else planes[::8].copy()
    poses = [(c.R, c.t) for c in fr.src_cams]
    args = dict(K=fr.ref_cam.K_1based, Rref=fr.ref_cam.R, tref=fr.ref_cam.t, poses=poses, moments=moments,
                mode=M.SWEEP_AGGREGATED, zfar=8.0, cost=True)
    monkeypatch.delenv("MVS_SWEEP_STAGING", raising=False)
    want = run_sweep(cuda, fr.ref, fr.srcs, planes, win, **args)
    monkeypatch.setenv("MVS_SWEEP_STAGING", "tma")
    got = run_sweep(cuda, fr.ref, fr.srcs, planes, win, **args)
    for k in ("cost", "label", "depth", "best"):
        np.testing.assert_array_equal(got[k], want[k])
    # 638 columns: rows of 2552 bytes, not whole 16-byte groups
    ref, srcs = fr.ref[:, :638].copy(), [s[:, :638].copy() for s in fr.srcs]
    got = run_sweep(cuda, ref, srcs, planes[:16], win, **args)
    monkeypatch.delenv("MVS_SWEEP_STAGING")
    want = run_sweep(cuda, ref, srcs, planes[:16], win, **args)
    np.testing.assert_array_equal(got["label"], want["label"])
