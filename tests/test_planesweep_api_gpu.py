"""The PlaneSweep drop-in (mvs_ps_* C handle, host buffers) end to end on the GPU.

Driven exactly as the reference's GUI drives PlaneSweep (pclviewer.cpp:329-439):
set images, poses and K, then RunAlgorithm / CudaDenoise / TGV and read the
host depthmaps back.  With the reference arithmetic and float homographies the
depthmaps are bit-identical to the reference's own kernels.
"""
import numpy as np
import pytest

import pyoracle as po
import mvs_b200 as M
from mvs_b200 import scenes

pytestmark = pytest.mark.gpu


def make_ps(g, planes_from_list):
    ps = M.PlaneSweep()
    ps.set_reference(g["ref"], g["Rref"], g["tref"])
    ps.set_sources(list(g["srcs"]), list(g["Rsrc"]), list(g["tsrc"]))
    ps.setK(g["K"])
    ps.setZ(float(g["znear"]), float(g["zfar"]))
    ps.setWindowSize(int(g["win"]))
    ps.setNumberofImages(len(g["srcs"]))
    ps.setNCCthreshold(float(g["nccthresh"]))
    ps.setSTDthreshold(float(g["stdthresh"]))
    if planes_from_list:
        ps.setPlaneDepths(g["planes"])
    else:
        ps.setNumberofPlanes(24)
    ps.setSweepOptions(M.MOMENTS_REFERENCE, M.SWEEP_PER_VIEW, fp64_homographies=False)
    return ps


@pytest.mark.parametrize("name,from_list", [("sweep_inverse_w5", True), ("sweep_refloop_w7", False)])
def test_run_algorithm_bit_exact(cuda, golden, name, from_list):
    g = golden(name)
    ps = make_ps(g, from_list)
    ps.RunAlgorithm()
    assert ps.getPlaneCount() == len(g["planes"])
    np.testing.assert_array_equal(ps.getDepthmap(), g["depth"])
    np.testing.assert_array_equal(ps.getViewLabels(), g["label"])
    np.testing.assert_array_equal(ps.getViewBest(), g["best"])
    # ConvertDepthtoUChar (planesweep.cpp:279-290)
    d = g["depth"]
    zn, zf = np.float32(g["znear"]), np.float32(g["zfar"])
    want8 = np.where(d == d, (np.float32(255) * np.clip((d - zn) / (zf - zn), 0, 1)).astype(np.uint8), 255)
    np.testing.assert_array_equal(ps.getDepthmap8u(), want8.astype(np.uint8))
    # a caller's buffer is filled in place; one of another shape or type is refused
    buf = np.full(g["depth"].shape, -1.0, np.float32)
    assert ps.getDepthmap(out=buf) is buf
    np.testing.assert_array_equal(buf, g["depth"])
    buf8 = np.zeros(g["depth"].shape, np.uint8)
    np.testing.assert_array_equal(ps.getDepthmap8u(out=buf8), want8.astype(np.uint8))
    with pytest.raises(ValueError):
        ps.getDepthmap(out=np.empty(g["depth"].shape, np.float64))
    with pytest.raises(ValueError):
        ps.getDepthmap(out=np.empty((3, 3), np.float32))


def test_denoise_tgv_and_points_follow_the_reference(cuda, golden):
    g = golden("sweep_refloop_w7")
    ps = make_ps(g, False)
    ps.RunAlgorithm()
    ps.CudaDenoise(niters=25)
    den = ps.getDepthmapDenoised()
    want, _ = po.ref_tvl1_denoise(g["ref"], g["depth"], float(g["znear"]), float(g["zfar"]), niters=25) \
        if po.ref_lib() else (po.tvl1_denoise(g["ref"], g["depth"], float(g["znear"]), float(g["zfar"]), niters=25,
                                              precision="f32"), 0)
    np.testing.assert_array_equal(den, want)
    assert ps.getDepthmapDenoisedPtr() != 0
    X, Y, Z = ps.get3Dcoordinates()
    assert np.isfinite(X).all() and np.isfinite(Z).all()
    ps.TGV(niters=5, warps=2)
    u = ps.getDepthmapTGV()
    uo, _, _ = po.tgv2(g["ref"], list(g["srcs"]), g["K"], g["Rref"], g["tref"],
                       [(g["Rsrc"][i], g["tsrc"][i]) for i in range(len(g["Rsrc"]))], niters=5, warps=2,
                       precision="f32")
    np.testing.assert_array_equal(u, uo)


def test_errors_are_reported_not_raised_on_device(cuda):
    ps = M.PlaneSweep()
    with pytest.raises(M.MvsError):
        ps.RunAlgorithm()            # no images yet
    with pytest.raises(M.MvsError):
        ps.setWindowSize(4)          # even window


def test_images_set_again_between_runs(cuda, golden):
    """The image setters upload while they stage and RunAlgorithm skips those
    uploads: new sources, a repeated run and a new frame size on one handle give
    the depthmaps of fresh handles (never a stale device image)."""
    g = golden("sweep_inverse_w5")
    ps = make_ps(g, True)
    ps.RunAlgorithm()
    np.testing.assert_array_equal(ps.getDepthmap(), g["depth"])
    ps.RunAlgorithm()   # nothing set again: the same images
    np.testing.assert_array_equal(ps.getDepthmap(), g["depth"])
    # other sources (the list reversed), then the originals again
    g2 = dict(g)
    g2["srcs"], g2["Rsrc"], g2["tsrc"] = g["srcs"][::-1], g["Rsrc"][::-1], g["tsrc"][::-1]
    ps.set_sources(list(g2["srcs"]), list(g2["Rsrc"]), list(g2["tsrc"]))
    ps.RunAlgorithm()
    fresh = make_ps(g2, True)
    fresh.RunAlgorithm()
    np.testing.assert_array_equal(ps.getDepthmap(), fresh.getDepthmap())
    ps.set_sources(list(g["srcs"]), list(g["Rsrc"]), list(g["tsrc"]))
    ps.RunAlgorithm()
    np.testing.assert_array_equal(ps.getDepthmap(), g["depth"])
    # a smaller frame (the top-left crop) on the same handle
    h, w = g["ref"].shape
    g3 = dict(g)
    g3["ref"] = np.ascontiguousarray(g["ref"][: h - 8, : w - 16])
    g3["srcs"] = np.ascontiguousarray(np.asarray(g["srcs"])[:, : h - 8, : w - 16])
    ps.set_reference(g3["ref"], g3["Rref"], g3["tref"])
    ps.set_sources(list(g3["srcs"]), list(g3["Rsrc"]), list(g3["tsrc"]))
    ps.RunAlgorithm()
    fresh3 = make_ps(g3, True)
    fresh3.RunAlgorithm()
    assert ps.getDepthmap().shape == (h - 8, w - 16)
    np.testing.assert_array_equal(ps.getDepthmap(), fresh3.getDepthmap())
    # the reference set again alone, after the sources
    ps.set_reference(g3["ref"], g3["Rref"], g3["tref"])
    ps.RunAlgorithm()
    np.testing.assert_array_equal(ps.getDepthmap(), fresh3.getDepthmap())
    for p in (ps, fresh, fresh3):
        p.close()


def test_page_locked_images_are_uploaded_from_the_callers_memory(cuda, golden):
    """Images in page-locked memory are uploaded from the caller's buffer while the handle
    copies them: the depthmaps equal the reference's, and the caller may overwrite its buffers
    as soon as the setter returns (the run still sees the images it was given)."""
    import torch
    g = golden("sweep_inverse_w5")

    def pinned(a):
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).pin_memory()
        return t, t.numpy()

    t_ref, h_ref = pinned(g["ref"])
    t_srcs, h_srcs = pinned(np.asarray(g["srcs"]))
    ps = make_ps(g, True)
    ps.set_reference(h_ref, g["Rref"], g["tref"])
    ps.set_sources(h_srcs, np.asarray(g["Rsrc"]), np.asarray(g["tsrc"]))
    h_ref[...] = 0.0
    h_srcs[...] = 0.0
    ps.RunAlgorithm()
    np.testing.assert_array_equal(ps.getDepthmap(), g["depth"])
    # other sources through the same pinned buffer, against a fresh handle fed pageable arrays
    g2 = dict(g)
    g2["srcs"], g2["Rsrc"], g2["tsrc"] = g["srcs"][::-1], g["Rsrc"][::-1], g["tsrc"][::-1]
    h_srcs[...] = np.asarray(g2["srcs"])
    ps.set_sources(h_srcs, np.asarray(g2["Rsrc"]), np.asarray(g2["tsrc"]))
    h_srcs[...] = 0.0
    ps.RunAlgorithm()
    fresh = make_ps(g2, True)
    fresh.RunAlgorithm()
    np.testing.assert_array_equal(ps.getDepthmap(), fresh.getDepthmap())
    for p in (ps, fresh):
        p.close()


def test_getters_refuse_a_map_of_another_frame_size(cuda, golden):
    """After the reference is set again at another size, the last run's maps no
    longer fit the getters' width*height contract: they are refused, not copied."""
    g = golden("sweep_inverse_w5")
    ps = make_ps(g, True)
    ps.RunAlgorithm()
    h, w = g["ref"].shape
    ps.set_reference(np.ascontiguousarray(g["ref"][: h // 2, : w // 2]), g["Rref"], g["tref"])
    for get in (ps.getDepthmap, ps.getDepthmap8u, ps.getViewLabels, ps.getViewBest):
        with pytest.raises(M.MvsError):
            get()
    ps.set_reference(g["ref"], g["Rref"], g["tref"])   # the run's size again
    np.testing.assert_array_equal(ps.getDepthmap(), g["depth"])
    ps.close()


def _rel_like_the_handle(Rref, tref, Rsrc, tsrc):
    """RunAlgorithm's FP64 relative pose from the float poses: Rsrc * Rref^-1
    with the adjugate / determinant inverse, in the same operation order."""
    m = [float(x) for x in np.asarray(Rref, np.float32).reshape(9)]
    rs = [float(x) for x in np.asarray(Rsrc, np.float32).reshape(9)]
    tr = [float(x) for x in np.asarray(tref, np.float32).reshape(3)]
    ts = [float(x) for x in np.asarray(tsrc, np.float32).reshape(3)]
    det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) + m[2] * (m[3] * m[7] - m[4] * m[6])
    inv = [(m[4] * m[8] - m[5] * m[7]) / det, (m[2] * m[7] - m[1] * m[8]) / det, (m[1] * m[5] - m[2] * m[4]) / det,
           (m[5] * m[6] - m[3] * m[8]) / det, (m[0] * m[8] - m[2] * m[6]) / det, (m[2] * m[3] - m[0] * m[5]) / det,
           (m[3] * m[7] - m[4] * m[6]) / det, (m[1] * m[6] - m[0] * m[7]) / det, (m[0] * m[4] - m[1] * m[3]) / det]
    Ro = [rs[3 * r] * inv[c] + rs[3 * r + 1] * inv[3 + c] + rs[3 * r + 2] * inv[6 + c] for r in range(3) for c in range(3)]
    to = [ts[r] - (Ro[3 * r] * tr[0] + Ro[3 * r + 1] * tr[1] + Ro[3 * r + 2] * tr[2]) for r in range(3)]
    return np.array(Ro).reshape(3, 3), np.array(to)


def test_full_size_frame_through_the_handle_equals_device_entry_point(cuda):
    """640x480, 8 views (11 MB of images: staged by several threads and uploaded
    MB by MB as they are copied): the handle's depthmap is bit-identical to
    mvs_sweep's on device copies of the same images and homographies."""
    import torch
    fr, planes, win = scenes.config_full(seed=6)
    planes = planes[::4].copy()          # 64 planes: the upload path does not depend on them
    V = len(fr.srcs)
    K1 = np.float32(fr.ref_cam.K_1based)
    ps = M.PlaneSweep()
    ps.setK(K1)
    ps.setPlaneDepths(planes)
    ps.setWindowSize(win)
    ps.setNumberofImages(V)
    ps.setZ(0.4, 8.0)
    ps.setSweepOptions(M.MOMENTS_COMPENSATED, M.SWEEP_AGGREGATED, True)
    Rs = np.stack([c.R for c in fr.src_cams]).astype(np.float32)
    ts = np.stack([c.t for c in fr.src_cams]).astype(np.float32)
    ps.set_reference(fr.ref, fr.ref_cam.R, fr.ref_cam.t)
    ps.set_sources(np.stack(fr.srcs), Rs, ts)
    ps.RunAlgorithm()
    got = ps.getDepthmap()
    ps.close()
    h, w = fr.ref.shape
    desc = M.sweep_desc(w, h, V, len(planes), win, M.MOMENTS_COMPENSATED, M.SWEEP_AGGREGATED, 1e-4, 0.5, 8.0)
    d_ref = torch.from_numpy(np.ascontiguousarray(fr.ref, np.float32)).to(cuda)
    d_srcs = torch.from_numpy(np.ascontiguousarray(np.stack(fr.srcs), np.float32)).to(cuda)
    d_depths = torch.from_numpy(np.ascontiguousarray(planes, np.float32)).to(cuda)
    H = torch.empty((V, len(planes), 9), dtype=torch.float32, device=cuda)
    rel = [_rel_like_the_handle(fr.ref_cam.R, fr.ref_cam.t, Rs[v], ts[v]) for v in range(V)]
    M.sweep_homographies(desc, np.float64(K1), rel, d_depths, H)
    depth = torch.empty((h, w), dtype=torch.float32, device=cuda)
    ws = torch.empty(M.sweep_workspace_bytes(desc), dtype=torch.uint8, device=cuda)
    M.sweep(desc, d_ref, d_srcs, H, d_depths, depth, workspace=ws)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(got, depth.cpu().numpy())
