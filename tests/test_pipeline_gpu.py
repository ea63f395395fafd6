"""Headless reconstruction (mvs_b200.pipeline: sweep -> TV-L1 denoise ->
histogram fusion -> surface points -> PLY) on a few views of one seeded box
room: the fused surface points must lie on the rendered surfaces."""
import math

import numpy as np
import pytest

import mvs_b200 as M
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


def test_reconstruction_lies_on_the_surfaces(cuda, tmp_path):
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
    voxel = float(np.max((b - a) / np.array(fs.dims)))
    ref_cam, depth = cams[0]
    pc = world @ ref_cam.R.T + ref_cam.t
    front = pc[:, 2] > 0.1
    uv = (pc[front] @ ref_cam.K.T)
    u, v = uv[:, 0] / uv[:, 2], uv[:, 1] / uv[:, 2]
    ins = (u >= 0) & (v >= 0) & (u <= ref_cam.width - 1) & (v <= ref_cam.height - 1)
    zi = depth[np.round(v[ins]).astype(int), np.round(u[ins]).astype(int)]
    dz = np.abs(pc[front][ins, 2] - zi)
    assert ins.sum() > 200
    # surface voxels sit within a couple of voxels of the rendered depth
    assert np.median(dz) < 2 * voxel, (np.median(dz), voxel)
