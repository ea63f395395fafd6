"""Headless reconstruction (mvs_b200.pipeline: sweep -> TV-L1 denoise ->
histogram fusion -> surface points -> PLY) on a few views of one seeded box
room.  The GPU chain equals the same chain over the CPU oracle in the
reference's float arithmetic (same voxels, same centres), and the extracted
band of voxels (-1 < u < 0, what the reference's viewer shows: after one TV-L1
step per frame it reaches well behind the surfaces) starts at the rendered
surfaces."""
import math

import numpy as np
import pytest

import pyoracle as po
from mvs_b200 import pipeline, scenes

pytestmark = pytest.mark.gpu


def _frames(seed=21, n=4, w=160, h=120):
    rng = np.random.default_rng(seed)
    sc = scenes.box_room(seed)
    f = 0.75 * w
    K = scenes.intrinsics(f, f, (w - 1) / 2.0, (h - 1) / 2.0)
    frames, cams = [], []
    for i in range(n):
        a = 0.5 * i / max(n - 1, 1)
        center = np.array([0.6 * math.sin(a), -0.2, -1.8 + 0.2 * math.cos(a)])
        R0, t0 = scenes.look_at(center, np.array([0.2 * math.sin(a), 0.3, 2.0]))
        ref_cam = scenes.Camera(K, R0, t0, w, h)
        src = []
        for k in range(3):
            ang = 2 * math.pi * k / 3
            c = center + R0.T @ np.array([0.06 * math.cos(ang), 0.06 * math.sin(ang), 0.0])
            Rs = scenes.rot_xyz(*np.radians(rng.uniform(-1, 1, 3))) @ R0
            src.append(scenes.Camera(K, Rs, -Rs @ c, w, h))
        inten, depth = sc.render(ref_cam)
        imgs = [(sc.render(c)[0] * 255).astype(np.float32) for c in src]
        frames.append(dict(ref=(inten * 255).astype(np.float32), srcs=np.stack(imgs), K=ref_cam.K_1based,
                           R=R0, t=t0, src_R=[c.R for c in src], src_t=[c.t for c in src]))
        cams.append((ref_cam, depth))
    return frames, cams


def oracle_reconstruct(frames, a, b, ss, fs, dn=pipeline.DenoiseSettings()):
    """The same chain over the CPU oracle in the reference's float arithmetic:
    sweep (float homographies), TV-L1 denoise, one histogram + U + P step per
    frame, voxels with lo < u < hi at their centres (x fastest)."""
    vol = po.Volume(fs.bins, fs.dims, a, b, precision="f32")
    for fr in frames:
        poses = list(zip(fr["src_R"], fr["src_t"]))
        H = po.homographies(fr["K"], fr["R"], fr["t"], poses, ss.plane_depths, precision="f32")
        d = po.sweep(fr["ref"], list(fr["srcs"]), H, ss.plane_depths, ss.window, stdthresh=ss.std_threshold,
                     nccthresh=ss.ncc_threshold, zfar=ss.zfar, precision="f32")["depth"]
        d = po.tvl1_denoise(fr["ref"], d, ss.znear, ss.zfar, niters=dn.niters, lam=dn.lam, tau=dn.tau,
                            sigma=dn.sigma, theta=dn.theta, beta=dn.beta, gamma=dn.gamma, precision="f32")
        vol.histogram(d, fr["K"], fr["R"], fr["t"], fs.threshold)
        vol.update_u(fs.tau, fs.lam)
        vol.update_p(fs.sigma)
    vw, vh, vd = fs.dims
    idx = np.nonzero((vol.u > -1) & (vol.u < 0))[0]
    x, y, z = idx % vw, (idx // vw) % vh, idx // (vw * vh)
    a32, b32 = np.float32(a), np.float32(b)
    s32 = b32 - a32
    return np.stack([a32[k] + s32[k] * ((c + .5) / n).astype(np.float32)
                     for k, (c, n) in enumerate(((x, vw), (y, vh), (z, vd)))], 1)


def test_reconstruction_follows_the_oracle_and_the_surfaces(cuda, tmp_path):
    frames, cams = _frames()
    a, b = np.array([-2.0, -1.5, -2.5]), np.array([2.0, 1.5, 2.5])
    fs = pipeline.FusionSettings(dims=(64, 48, 80), bins=8, threshold=0.1)
    ss = pipeline.SweepSettings(znear=0.5, zfar=6.0, n_planes=48, window=5,
                                plane_depths=scenes.inverse_depth_planes(0.5, 6.0, 48))
    ply = tmp_path / "fused.ply"
    pts, col, vol = pipeline.reconstruct(frames, a, b, sweep=ss, fusion=fs, ply_path=ply)
    vol.close()
    assert len(pts) > 500 and col.shape == pts.shape
    assert ply.read_bytes().startswith(b"ply\n")
    world = pts.copy()
    world[:, 0] = -world[:, 0]                      # the viewer's x flip undone
    # the whole chain in the reference's arithmetic: the same voxels, the same centres
    np.testing.assert_array_equal(world, oracle_reconstruct(frames, a, b, ss, fs))

    # geometry: the extracted band (-1 < u < 0, as the reference shows it) starts
    # at the rendered surfaces of the first frame and lies behind them
    voxel = float(np.max((b - a) / np.array(fs.dims)))
    ref_cam, depth = cams[0]
    pc = world @ ref_cam.R.T + ref_cam.t
    pc = pc[pc[:, 2] > 0.1]
    uv = pc @ ref_cam.K.T
    u, v = uv[:, 0] / uv[:, 2], uv[:, 1] / uv[:, 2]
    ins = (u >= 0) & (v >= 0) & (u <= ref_cam.width - 1) & (v <= ref_cam.height - 1)
    ui, vi = np.round(u[ins]).astype(int), np.round(v[ins]).astype(int)
    z = pc[ins, 2]
    sd = z - depth[vi, ui]
    assert ins.sum() > 200
    assert (sd < -2 * voxel).mean() < 0.15          # few points in the free space in front
    key = vi * ref_cam.width + ui                  # nearest point along each pixel's ray
    order = np.lexsort((z, key))
    first = order[np.r_[True, key[order][1:] != key[order][:-1]]]
    assert np.median(np.abs(sd[first])) < 3 * voxel, np.median(np.abs(sd[first]))
