"""Host float math that feeds the kernels equals the reference's Matrix3D arithmetic."""
import numpy as np

import pyoracle as po
from mvs_b200 import hostmath as hm, scenes


def test_homographies_equal_reference_construction():
    fr, planes, _ = scenes.config_tiny(seed=17, n_src=3, n_planes=11)
    K1 = fr.ref_cam.K_1based
    p = [(c.R, c.t) for c in fr.src_cams]
    Ho = po.homographies(K1, fr.ref_cam.R, fr.ref_cam.t, p, planes, precision="f32")
    invK = hm.inv3_f32(K1)
    for v, (Rs, ts) in enumerate(p):
        Rrel, trel = hm.relative_f32(fr.ref_cam.R, fr.ref_cam.t, Rs, ts)
        for k, d in enumerate(planes):
            np.testing.assert_array_equal(hm.homography_f32(np.float32(K1), invK, Rrel, trel, d).reshape(9), Ho[v, k])
    L = po.ref_lib()
    if L is not None:
        H = np.zeros(9, np.float32)
        Rs, ts = p[1]
        L.ref_homography(po._fp(np.float32(K1).reshape(9).copy()), po._fp(np.float32(fr.ref_cam.R).reshape(9).copy()),
                         po._fp(np.float32(fr.ref_cam.t).copy()), po._fp(np.float32(Rs).reshape(9).copy()),
                         po._fp(np.float32(ts).copy()), 0, planes[4], po._fp(H))
        np.testing.assert_array_equal(H, Ho[1, 4])


def test_alternative_relative_method():
    rng = np.random.default_rng(2)
    R1 = scenes.rot_xyz(*rng.uniform(-1, 1, 3))
    R2 = scenes.rot_xyz(*rng.uniform(-1, 1, 3))
    t1, t2 = rng.normal(size=3), rng.normal(size=3)
    a = hm.relative_f32(R1, t1, R2, t2, alternative=True)
    b = po.relative(R1, t1, R2, t2, alternative=True, precision="f32")
    np.testing.assert_array_equal(a[0].reshape(9), b[0])
    np.testing.assert_array_equal(a[1], b[1])
