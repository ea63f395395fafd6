"""TGV2 towards a sparse depthmap (PlaneSweep::TGVdenoiseFromSparse) on the GPU.

The fused iteration performs the reference's arithmetic statement for
statement (planesweep.cpp:596-674, TGV2_kernels.cu:54-85,340-445), so with
beta = 0 (tensor entries exactly 1 / 0 / 1 or unit gradients) the result is
bit-identical to the reference's own kernels run on the CPU (golden fixtures)
and to the C restatement at every size.  With beta != 0 the tensor goes
through CUDA's expf / powf where the reference ran the host libm: a few ulps
in T, which moves the result by < 1e-6 relative over these iteration counts
(one-ulp perturbations of T on 30% of the pixels: 6e-7), so that case is held
to 1e-5 relative.
"""
import numpy as np
import pytest

import pyoracle as po
import mvs_b200 as M

pytestmark = pytest.mark.gpu

PARAM_NAMES = ("alpha0", "alpha1", "tau", "sigma", "theta", "beta", "gamma")


def run_sparse(cuda, ref, depthmap, sparse, zfar, niters, **kw):
    import torch
    h, w = depthmap.shape
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(cuda)
    d_ref, d_dep, d_sp = t(ref), t(depthmap), t(sparse)
    out = torch.empty((h, w), dtype=torch.float32, device=cuda)
    ws = torch.empty(M.tgv2_sparse_workspace_bytes(w, h) // 8 + 1, dtype=torch.int64, device=cuda)
    M.tgv2_sparse(d_ref, d_dep, d_sp, zfar, out, ws, niters, **kw)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def sparse_case(seed, w, h, frac=0.15):
    rng = np.random.default_rng(seed)
    ref = (rng.random((h, w)) * 255).astype(np.float32)
    depth = (1 + 3 * rng.random((h, w))).astype(np.float32)
    sparse = np.where(rng.random((h, w)) < frac, depth * (1 + 0.01 * rng.standard_normal((h, w))), 0)
    return ref, depth, sparse.astype(np.float32)


def test_sparse_bit_exact_vs_reference(cuda, golden):
    g = golden("tgv_sparse")
    kw = dict(zip(PARAM_NAMES, (float(x) for x in g["params"])))
    out = run_sparse(cuda, g["ref"], g["depthmap"], g["sparse"], float(g["zfar"]), int(g["niters"]), **kw)
    np.testing.assert_array_equal(out, g["out"])


def test_sparse_tensor_vs_reference(cuda, golden):
    g = golden("tgv_sparse_tensor")
    kw = dict(zip(PARAM_NAMES, (float(x) for x in g["params"])))
    out = run_sparse(cuda, g["ref"], g["depthmap"], g["sparse"], float(g["zfar"]), int(g["niters"]), **kw)
    rel = np.abs(out - g["out"]) / np.abs(g["out"])
    assert rel.max() <= 1e-5, rel.max()


@pytest.mark.parametrize("w,h,niters", [(1, 17, 9), (17, 1, 9), (2, 2, 5), (33, 7, 12), (97, 61, 30)])
def test_sparse_ragged_sizes_bit_exact_vs_oracle(cuda, w, h, niters):
    ref, depth, sparse = sparse_case(w * 131 + h, w, h)
    out = run_sparse(cuda, ref, depth, sparse, 6.0, niters)
    want = po.tgv_sparse(ref, depth, sparse, 6.0, niters, precision="f32")
    np.testing.assert_array_equal(out, want)


def test_sparse_zero_iterations_is_the_scaled_start(cuda):
    ref, depth, sparse = sparse_case(3, 40, 30)
    out = run_sparse(cuda, ref, depth, sparse, 7.0, 0)
    want = po.tgv_sparse(ref, depth, sparse, 7.0, 0, precision="f32")
    np.testing.assert_array_equal(out, want)


def test_sparse_full_frame_bit_exact_vs_oracle(cuda):
    """640 x 480 (the bench frame size), 100 iterations, alpha / tau / sigma off
    their defaults; theta must not change anything."""
    ref, depth, sparse = sparse_case(640, 640, 480, frac=0.05)
    kw = dict(alpha0=1.7, alpha1=1.1, tau=0.03, sigma=1.5)
    out = run_sparse(cuda, ref, depth, sparse, 8.0, 100, theta=1.0, **kw)
    out2 = run_sparse(cuda, ref, depth, sparse, 8.0, 100, theta=0.25, **kw)
    want = po.tgv_sparse(ref, depth, sparse, 8.0, 100, precision="f32", **kw)
    np.testing.assert_array_equal(out, want)
    np.testing.assert_array_equal(out2, out)


def test_planesweep_handle_tgv_denoise_from_sparse(cuda, golden):
    """RunAlgorithm, then TGVdenoiseFromSparse through the host-buffer handle:
    the sweep depthmap is the start, the result lands in the TGV getters."""
    g = golden("sweep_inverse_w5")
    ps = M.PlaneSweep()
    ps.set_reference(g["ref"], g["Rref"], g["tref"])
    ps.set_sources(list(g["srcs"]), list(g["Rsrc"]), list(g["tsrc"]))
    ps.setK(g["K"])
    ps.setZ(float(g["znear"]), float(g["zfar"]))
    ps.setWindowSize(int(g["win"]))
    ps.setNumberofImages(len(g["srcs"]))
    ps.setPlaneDepths(g["planes"])
    ps.setSweepOptions(M.MOMENTS_REFERENCE, M.SWEEP_PER_VIEW, fp64_homographies=False)
    with pytest.raises(M.MvsError):
        ps.TGVdenoiseFromSparse(np.zeros_like(g["ref"]), 10)   # no depthmap yet
    ps.RunAlgorithm()
    dm = ps.getDepthmap()
    rng = np.random.default_rng(5)
    sparse = np.where(rng.random(dm.shape) < 0.2, g["depth_gt"], 0).astype(np.float32)
    ps.TGVdenoiseFromSparse(sparse, 40, alpha0=2.0, alpha1=1.5, tau=0.02, sigma=1.0)
    got = ps.getDepthmapTGV()
    want = po.tgv_sparse(g["ref"], dm, sparse, float(g["zfar"]), 40, precision="f32")
    np.testing.assert_array_equal(got, want)
    with pytest.raises(ValueError):
        ps.TGVdenoiseFromSparse(sparse[:-1], 10)


def test_sparse_vs_the_reference_gpu_build(cuda):
    """Against the reference's own kernels compiled for this GPU (its nvcc build
    contracts multiply-adds, so agreement is to rounding, not bits), with two
    theta values: the over-relaxation the reference computes is not read, in
    its GPU build as in its CPU build."""
    if po.ref_gpu_lib() is None:
        pytest.skip("oracle/_ref/libmvs_ref_gpu.so not built")
    ref, depth, sparse = sparse_case(11, 97, 61, frac=0.2)
    out = run_sparse(cuda, ref, depth, sparse, 6.0, 40)
    for theta in (1.0, 0.3):
        ru, ms = po.ref_gpu_tgv_sparse(ref, depth, sparse, 6.0, 40, theta=theta)
        assert ms >= 0
        rel = np.abs(out - ru) / np.abs(ru)
        assert rel.max() <= 1e-5, (theta, rel.max())
