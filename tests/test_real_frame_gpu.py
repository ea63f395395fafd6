"""The reference's own sample frames through the PlaneSweep handle, as its GUI
drives them (pclviewer.cpp:329-439): reference image and four sources, the
calibration's K and poses, the float plane loop over [0.1, 1] m, a 5x5
window; then CudaDenoise and TGV2 from the sweep depthmap.  The frames are the
grey images downsampled 4x and rounded to 8 bits (both engines see the same
values); every output equals the reference's own kernels bit for bit."""
import numpy as np
import pytest

import mvs_b200 as M

pytestmark = pytest.mark.gpu


def test_real_frame_through_the_handle(cuda, golden):
    g = golden("real_frame")
    ims = g["images"].astype(np.float32)
    ps = M.PlaneSweep()
    ps.set_reference(ims[0], g["Rref"], g["tref"])
    ps.set_sources(list(ims[1:]), list(g["Rsrc"]), list(g["tsrc"]))
    ps.setK(g["K"])
    ps.setZ(float(g["znear"]), float(g["zfar"]))
    ps.setNumberofPlanes(int(g["n_planes"]))
    ps.setWindowSize(int(g["win"]))
    ps.setNumberofImages(len(ims) - 1)
    ps.setSweepOptions(M.MOMENTS_REFERENCE, M.SWEEP_PER_VIEW, fp64_homographies=False)
    ps.RunAlgorithm()
    assert ps.getPlaneCount() == len(g["planes"])
    np.testing.assert_array_equal(ps.getDepthmap(), g["depth"])
    np.testing.assert_array_equal(ps.getViewLabels().reshape(g["label"].shape), g["label"])
    ps.CudaDenoise(niters=50)
    np.testing.assert_array_equal(ps.getDepthmapDenoised(), g["denoised"])
    it, _ = ps.TGVext(M.tgv2_params(niters=40, warps=2), start=1)
    assert it == 80
    np.testing.assert_array_equal(ps.getDepthmapTGV(), g["tgv"])
    ps.close()
