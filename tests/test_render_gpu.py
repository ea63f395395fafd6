"""The device ray caster (mvs_render_scene) against the CPU caster of
mvs_b200.scenes on the same scene and cameras (FP64 both; the device may pick
the other lattice cell where a coordinate sits exactly on a cell border, and
its 3x3 products round in another order)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scene", ["room", "street"])
def test_render_matches_cpu(cuda, scene):
    from mvs_b200 import scenes
    w, h = (96, 72) if scene == "room" else (160, 48)
    K = scenes.intrinsics(0.75 * w, 0.75 * w, (w - 1) / 2.0, (h - 1) / 2.0)
    sc, ref_cam, cams = scenes.frame_geometry(7, w, h, K, 3, baseline=(0.05, 0.3), scene=scene)
    g = scenes.GpuRenderer(cuda)
    gray, depth = g.render(sc, [ref_cam] + cams)
    for k, cam in enumerate([ref_cam] + cams):
        inten, d = sc.render(cam)
        cd = d.astype(np.float32)
        ci = (inten * 255.0).astype(np.float32)
        gd = depth[k].cpu().numpy()
        gi = gray[k].cpu().numpy()
        assert np.max(np.abs(gd - cd) / cd) < 1e-6
        close = np.abs(gi - ci) <= 1e-3
        assert close.mean() >= 0.999, close.mean()


def test_device_frame_matches_make_frame(cuda):
    from mvs_b200 import scenes
    K = scenes.intrinsics(48.0, 48.0, 31.5, 23.5)
    fr = scenes.make_frame(3, 64, 48, K, 2, baseline=(0.05, 0.08))
    df = scenes.GpuRenderer(cuda).frame(3, 64, 48, K, 2, baseline=(0.05, 0.08))
    assert np.allclose(df.ref.cpu().numpy(), fr.ref, atol=1e-3)
    assert np.allclose(df.srcs.cpu().numpy(), np.stack(fr.srcs), atol=1e-3)
    assert np.allclose(df.depth_gt.cpu().numpy(), fr.depth_gt, rtol=1e-6)
    for a, b in zip(df.src_cams, fr.src_cams):
        assert np.array_equal(a.R, b.R) and np.array_equal(a.t, b.t)
