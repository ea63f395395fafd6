"""The CPU oracle pinned to the reference (CPU only).

* against the committed golden fixtures (outputs of the reference's own
  kernels compiled for the CPU by tests/golden/make_golden.py): the f32 oracle
  is bit-exact, the f64 oracle within stated tolerances;
* against the reference-on-CPU library live, on fresh seeded inputs, when it
  was built here (oracle/_ref/libmvs_ref.so).
"""
import numpy as np
import pytest

import pyoracle as po
from mvs_b200 import scenes

SWEEPS = ["sweep_inverse_w5", "sweep_refloop_w7", "sweep_inverse_w3_negthr"]


def poses(g):
    return [(g["Rsrc"][i], g["tsrc"][i]) for i in range(len(g["Rsrc"]))]


@pytest.mark.parametrize("name", SWEEPS)
def test_sweep_f32_bit_exact_vs_golden(golden, name):
    g = golden(name)
    H = po.homographies(g["K"], g["Rref"], g["tref"], poses(g), g["planes"], precision="f32")
    o = po.sweep(g["ref"], list(g["srcs"]), H, g["planes"], int(g["win"]), nccthresh=float(g["nccthresh"]),
                 zfar=float(g["zfar"]), precision="f32")
    np.testing.assert_array_equal(o["best"], g["best"])
    np.testing.assert_array_equal(o["vdepth"], g["vdepth"])
    np.testing.assert_array_equal(o["label"], g["label"])
    np.testing.assert_array_equal(o["depth"], g["depth"])


@pytest.mark.parametrize("name", SWEEPS)
def test_sweep_f64_labels_vs_golden(golden, name):
    g = golden(name)
    H = po.homographies(g["K"], g["Rref"], g["tref"], poses(g), g["planes"], precision="f64")
    o = po.sweep(g["ref"], list(g["srcs"]), H, g["planes"], int(g["win"]), nccthresh=float(g["nccthresh"]),
                 zfar=float(g["zfar"]), precision="f64")
    # FP64 moments differ from the reference's naive float moments only where the NCC curve
    # is flat: the labels agree almost everywhere, and where they differ by more than one
    # plane the two maxima are equal to float resolution (a tie broken differently).
    d = np.abs(o["label"] - g["label"])
    assert np.mean(d == 0) >= 0.995
    far = d > 1
    assert np.mean(far) <= 1e-3
    assert np.all(np.abs(o["best"][far] - g["best"][far]) < 1e-4)


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_sweep_ncc_band_equals_full_frame_rows(precision):
    """The row-band cost used for full-size checks equals the same rows of the
    full-frame per-view NCC summed over views, bit for bit: a band at the top
    (mirrored rows above the frame), one inside and one at the bottom."""
    fr, planes, win = scenes.config_tiny(seed=11, width=37, height=29, n_src=3, n_planes=5, win=7)
    pz = [(c.R, c.t) for c in fr.src_cams]
    H = po.homographies(fr.ref_cam.K_1based, fr.ref_cam.R, fr.ref_cam.t, pz, planes, precision=precision)
    L = po.oracle_lib()
    dt = np.float32 if precision == "f32" else np.float64
    P = po._fp if precision == "f32" else po._dp
    h, w = fr.ref.shape
    full = np.zeros((len(planes), h, w), dt)
    for p in range(len(planes)):
        for v in range(len(pz)):
            buf = np.zeros((h, w), dt)
            getattr(L, f"orc_sweep_ncc_{precision}")(w, h, po._fp(po._f32(fr.ref)), po._fp(po._f32(fr.srcs[v])),
                                                     P(np.ascontiguousarray(H[v, p], dt)), win, 1e-4, P(buf))
            full[p] = (full[p] + buf).astype(dt)
    for y0, y1 in [(0, 6), (9, 20), (25, 29)]:
        band = po.sweep_ncc_band(fr.ref, fr.srcs, H, win, y0, y1, precision=precision)
        np.testing.assert_array_equal(band, full[:, y0:y1])


def test_reference_plane_loop(golden):
    g = golden("sweep_refloop_w7")
    np.testing.assert_array_equal(po.plane_list(float(g["znear"]), float(g["zfar"]), 24), g["planes"])
    np.testing.assert_array_equal(scenes.reference_plane_list(float(g["znear"]), float(g["zfar"]), 24), g["planes"])
    # the reference's float loop can drop the last plane (planesweep.cpp:200)
    assert len(po.plane_list(0.1, 1.0, 200)) == 199


@pytest.mark.parametrize("name", ["tgv_from_one", "tgv_from_depth", "tgv_aniso"])
def test_tgv2_f32_bit_exact_vs_golden(golden, name):
    """tgv_aniso: beta = 1.5, gamma = 0.8, the anisotropic tensor on."""
    g = golden(name)
    u0 = None if str(g["start"]) == "one" else g["depth_gt"]
    bg = dict(beta=float(g["beta"]), gamma=float(g["gamma"])) if "beta" in g else {}
    u, n, _ = po.tgv2(g["ref"], list(g["srcs"]), g["K"], g["Rref"], g["tref"], poses(g), niters=int(g["niters"]),
                      warps=int(g["warps"]), u_init=u0, precision="f32", **bg)
    np.testing.assert_array_equal(u, g["u"])
    u64, _, _ = po.tgv2(g["ref"], list(g["srcs"]), g["K"], g["Rref"], g["tref"], poses(g),
                        niters=int(g["niters"]), warps=int(g["warps"]), u_init=u0, precision="f64", **bg)
    assert np.max(np.abs(u64 - g["u"]) / np.abs(u64)) < 1e-4


def test_tvl1_f32_bit_exact_vs_golden(golden):
    g = golden("tvl1_denoise")
    o = po.tvl1_denoise(g["ref"], g["depth_in"], float(g["znear"]), float(g["zfar"]), niters=int(g["niters"]),
                        precision="f32")
    np.testing.assert_array_equal(o, g["out"])


SPARSE_PARAMS = ("alpha0", "alpha1", "tau", "sigma", "theta", "beta", "gamma")


@pytest.mark.parametrize("name", ["tgv_sparse", "tgv_sparse_tensor"])
def test_tgv_sparse_f32_bit_exact_vs_golden(golden, name):
    """PlaneSweep::TGVdenoiseFromSparse: the f32 restatement equals the
    reference's kernels bit for bit (with the reference's v / vbar aliasing);
    the f64 form stays within 1e-5 relative of them."""
    g = golden(name)
    kw = dict(zip(SPARSE_PARAMS, (float(x) for x in g["params"])))
    args = (g["ref"], g["depthmap"], g["sparse"], float(g["zfar"]), int(g["niters"]))
    np.testing.assert_array_equal(po.tgv_sparse(*args, precision="f32", **kw), g["out"])
    o64 = po.tgv_sparse(*args, precision="f64", **kw)
    assert np.max(np.abs(o64 - g["out"]) / np.abs(g["out"])) < 1e-5
    # theta reaches only the over-relaxed u, which nothing reads
    kw["theta"] = 0.1
    np.testing.assert_array_equal(po.tgv_sparse(*args, precision="f32", **kw), g["out"])


@pytest.mark.parametrize("name", ["fusion_b7_decoupled", "fusion_b8_interleaved", "fusion_b2_decoupled",
                                  "fusion_b10_decoupled"])
def test_fusion_f32_bit_exact_vs_golden(golden, name):
    g = golden(name)
    v = po.Volume(int(g["bins"]), tuple(g["dims"]), g["vol_min"], g["vol_max"], precision="f32")
    thr, tau, lam, sigma = float(g["thr"]), float(g["tau"]), float(g["lam"]), float(g["sigma"])
    if bool(g["interleaved"]):
        for m in range(len(g["depths"])):
            v.histogram(g["depths"][m], g["K"][m], g["R"][m], g["t"][m], thr)
            v.update_u(tau, lam)
            v.update_p(sigma)
    else:
        for m in range(len(g["depths"])):
            v.histogram(g["depths"][m], g["K"][m], g["R"][m], g["t"][m], thr)
        for _ in range(int(g["iters"])):
            v.update_u(tau, lam)
            v.update_p(sigma)
    np.testing.assert_array_equal(v.hist, g["hist"])
    np.testing.assert_array_equal(v.u, g["u"])
    np.testing.assert_array_equal(v.v, g["v"])
    np.testing.assert_array_equal(v.p, g["p"])


def test_bin_centers():
    np.testing.assert_array_equal(po.bin_centers(7), np.float32([-1, -1, -0.5, 0, 0.5, 1, 1]))
    np.testing.assert_array_equal(po.bin_centers(3), np.float32([-1, 0, 1]))
    np.testing.assert_array_equal(po.bin_centers(2), np.float32([-1, 1]))


def prox_closed_form(bins, h, u, tl):
    """The closed-form median the CUDA U kernel uses (numpy float32 restatement)."""
    c = po.bin_centers(bins)
    h = np.asarray(h, np.int64)
    total = h.sum()
    pre = np.cumsum(h)
    B = np.array([max(np.float32(np.float32(u) + np.float32(tl) * np.float32(total - 2 * pre[j - 1])), np.float32(-1))
                  for j in range(1, bins + 1)], np.float32)[::-1]
    lo, hi = np.float32(np.inf), np.float32(-np.inf)
    for i in range(bins + 1):
        a_lo = c[i - 1] if i > 0 else -np.inf
        b_lo = B[bins - 1 - i] if bins - 1 - i >= 0 else -np.inf
        lo = min(lo, max(a_lo, b_lo))
        a_hi = c[i] if i < bins else np.inf
        b_hi = B[bins - i] if bins - i < bins else np.inf
        hi = max(hi, min(a_hi, b_hi))
    return np.float32(min(max(max(np.float32(u), np.float32(-1)), lo), hi))


@pytest.mark.parametrize("bins", [2, 3, 5, 7, 8, 10])
def test_prox_closed_form_equals_insertion_sort(bins):
    rng = np.random.default_rng(bins)
    L = po.oracle_lib()
    tau, lam = np.float32(0.1), np.float32(0.5)
    tl = np.float32(tau * lam)
    for _ in range(400):
        h = rng.integers(0, 30, bins).astype(np.uint16)
        if rng.random() < 0.2:
            h[:] = 0
        u = np.float32(rng.uniform(-4, 4))
        want = L.orc_prox_hist_f32(bins, h.ctypes.data_as(po._U16), float(u), float(tau), float(lam))
        assert prox_closed_form(bins, h, u, tl) == np.float32(want)


needs_ref = pytest.mark.skipif(po.ref_lib() is None, reason="reference-on-CPU library not built here")


@needs_ref
@pytest.mark.parametrize("bins", [3, 7, 10])
def test_fp64_fusion_u_median_equals_sorted_selection(bins):
    """The FP64 oracle's U step (merge selection) against a plain sort: the
    median (rank N) of the bin centres, u and u + tau lambda W_j, each raised
    to the lowest centre as the reference's insertion leaves it."""
    rng = np.random.default_rng(bins)
    dims = (9, 7, 5)
    n = 9 * 7 * 5
    o = po.Volume(bins, dims, [0, 0, 0], [1, 1, 1], precision="f64")
    o.hist[:] = rng.integers(0, 9, o.hist.shape)
    o.hist[:, :10] = 0
    u0 = rng.uniform(-2.5, 2.5, n)
    o.u[:] = u0
    tau, lam = 0.1, 0.5
    o.update_u(tau, lam)   # p = 0: the divergence term vanishes
    c = po.bin_centers(bins).astype(np.float64)
    h = o.hist.astype(np.int64)
    for i in range(n):
        W = [-h[:j, i].sum() + h[j:, i].sum() for j in range(1, bins + 1)]
        vals = np.concatenate([c, [u0[i]], u0[i] + tau * lam * np.asarray(W, np.float64)])
        vals = np.maximum(vals, c[0])
        assert o.u[i] == np.sort(vals)[bins], i


def test_live_sweep_vs_reference():
    fr, planes, win = scenes.config_tiny(seed=101, width=72, height=50, n_src=3, n_planes=20, win=9)
    p = [(c.R, c.t) for c in fr.src_cams]
    r = po.ref_sweep(fr.ref, fr.srcs, fr.ref_cam.K_1based, fr.ref_cam.R, fr.ref_cam.t, p, planes, win, zfar=5.0)
    H = po.homographies(fr.ref_cam.K_1based, fr.ref_cam.R, fr.ref_cam.t, p, planes, precision="f32")
    o = po.sweep(fr.ref, fr.srcs, H, planes, win, zfar=5.0, precision="f32")
    np.testing.assert_array_equal(o["depth"], r["depth"])
    np.testing.assert_array_equal(o["best"], r["best"])


@needs_ref
def test_live_fusion_and_tgv_vs_reference():
    fi = scenes.fusion_sequence(102, 2, 40, 30)
    rv = po.RefVolume(6, (14, 12, 10), fi.vol_min, fi.vol_max)
    ov = po.Volume(6, (14, 12, 10), fi.vol_min, fi.vol_max, precision="f32")
    for d, c in zip(fi.depths, fi.cams):
        rv.histogram(d, c.K, c.R, c.t, 0.07)
        ov.histogram(d, c.K, c.R, c.t, 0.07)
    for _ in range(5):
        rv.update_u(0.1, 0.5), rv.update_p(1.0)
        ov.update_u(0.1, 0.5), ov.update_p(1.0)
    got = rv.get()
    np.testing.assert_array_equal(got["hist"], ov.hist)
    np.testing.assert_array_equal(got["u"], ov.u)
    fr, _, _ = scenes.config_tiny(seed=103, width=40, height=32, n_src=2)
    p = [(c.R, c.t) for c in fr.src_cams]
    ur, _ = po.ref_tgv(fr.ref, fr.srcs, fr.ref_cam.K_1based, fr.ref_cam.R, fr.ref_cam.t, p, niters=7, warps=2,
                       beta=1.5, gamma=0.8)
    uo, _, _ = po.tgv2(fr.ref, fr.srcs, fr.ref_cam.K_1based, fr.ref_cam.R, fr.ref_cam.t, p, niters=7, warps=2,
                       beta=1.5, gamma=0.8, precision="f32")
    np.testing.assert_array_equal(ur, uo)
    rng = np.random.default_rng(104)
    sp = np.where(rng.random(fr.depth_gt.shape) < 0.3, fr.depth_gt, 0).astype(np.float32)
    d0 = (fr.depth_gt * 1.05).astype(np.float32)
    sr = po.ref_tgv_sparse(fr.ref, d0, sp, 6.0, 11, beta=1.5, gamma=0.8, theta=0.7)
    so = po.tgv_sparse(fr.ref, d0, sp, 6.0, 11, beta=1.5, gamma=0.8, precision="f32")
    np.testing.assert_array_equal(sr, so)


def test_real_frame_f32_bit_exact_vs_golden(golden):
    """The reference's own sample frames (grey, downsampled): the f32 oracle
    equals the reference's kernels on the sweep (its float plane loop), the
    TV-L1 denoise of that depthmap and TGV2 from it."""
    g = golden("real_frame")
    ref, srcs = g["images"][0].astype(np.float32), [im.astype(np.float32) for im in g["images"][1:]]
    poses = [(g["Rsrc"][i], g["tsrc"][i]) for i in range(len(srcs))]
    H = po.homographies(g["K"], g["Rref"], g["tref"], poses, g["planes"], precision="f32")
    o = po.sweep(ref, srcs, H, g["planes"], int(g["win"]), zfar=float(g["zfar"]), precision="f32")
    np.testing.assert_array_equal(o["depth"], g["depth"])
    np.testing.assert_array_equal(o["label"], g["label"])
    den = po.tvl1_denoise(ref, g["depth"], float(g["znear"]), float(g["zfar"]), niters=50, precision="f32")
    np.testing.assert_array_equal(den, g["denoised"])
    u, _, _ = po.tgv2(ref, srcs, g["K"], g["Rref"], g["tref"], poses, niters=40, warps=2, u_init=g["depth"],
                      precision="f32")
    np.testing.assert_array_equal(u, g["tgv"])
