"""The 320x240 configuration (4 views, 64 inverse-depth planes, 7x7 window) end to
end through the PlaneSweep handle, as the reference's GUI drives it: RunAlgorithm,
then TGV2 in the two splits of "100 iterations" (the reference's own 15 x 30 run
from u = 1, planesweep.cpp:381-536 with its defaults; and 100 iterations in one
linearisation started from the sweep depthmap).  Everything runs in the
reference's float arithmetic, so each result equals the f32 oracle bit for bit
(the oracle itself equals the reference's kernels on these inputs,
tests/test_oracle.py)."""
import numpy as np
import pytest

import pyoracle as po
import mvs_b200 as M
from mvs_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1():
    fr, planes, win = scenes.config_small(seed=1)
    assert fr.ref.shape == (240, 320) and len(fr.srcs) == 4 and len(planes) == 64 and win == 7
    poses = [(c.R, c.t) for c in fr.src_cams]
    K1 = fr.ref_cam.K_1based
    H = po.homographies(K1, fr.ref_cam.R, fr.ref_cam.t, poses, planes, precision="f32")
    o = po.sweep(fr.ref, fr.srcs, H, planes, win, zfar=5.0, precision="f32")
    return fr, planes, win, poses, K1, o


def handle(c1):
    fr, planes, win, poses, K1, _ = c1
    ps = M.PlaneSweep()
    ps.set_reference(fr.ref, fr.ref_cam.R, fr.ref_cam.t)
    ps.set_sources(list(fr.srcs), [p[0] for p in poses], [p[1] for p in poses])
    ps.setK(np.float32(K1))
    ps.setZ(0.5, 5.0)
    ps.setWindowSize(win)
    ps.setNumberofImages(len(fr.srcs))
    ps.setPlaneDepths(planes)
    ps.setSweepOptions(M.MOMENTS_REFERENCE, M.SWEEP_PER_VIEW, fp64_homographies=False)
    return ps


def test_c1_sweep_then_tgv2_100_iterations_from_the_sweep(cuda, c1):
    fr, planes, win, poses, K1, o = c1
    ps = handle(c1)
    ps.RunAlgorithm()
    depth = ps.getDepthmap()
    np.testing.assert_array_equal(depth, o["depth"])
    it, _ = ps.TGVext(M.tgv2_params(niters=100, warps=1), start=1)
    assert it == 100
    want, n, _ = po.tgv2(fr.ref, fr.srcs, K1, fr.ref_cam.R, fr.ref_cam.t, poses, niters=100, warps=1,
                         u_init=depth, precision="f32")
    np.testing.assert_array_equal(ps.getDepthmapTGV(), want)
    ps.close()


def test_c1_reference_default_tgv_from_one(cuda, c1):
    """PlaneSweep::TGV with its defaults (30 iterations x 15 linearisations, u = 1)."""
    fr, planes, win, poses, K1, _ = c1
    ps = handle(c1)
    ps.TGV()
    want, n, _ = po.tgv2(fr.ref, fr.srcs, K1, fr.ref_cam.R, fr.ref_cam.t, poses, niters=30, warps=15,
                         precision="f32")
    assert n == 450
    np.testing.assert_array_equal(ps.getDepthmapTGV(), want)
    ps.close()
