"""Generate the golden fixtures in tests/golden/*.npz from the reference itself.

The reference's own kernels (kernels.cu, TGV2_kernels.cu, fusion.cu) are
compiled for the CPU by ``make -C oracle ref`` (oracle/Makefile, shim in
oracle/ref_shim.h, driver oracle/ref_driver.cpp) and run here on seeded
synthetic inputs.  Each fixture stores its inputs and the reference's outputs,
so the tests need neither the reference tree nor the scene generator to agree
across machines.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "plane-sweep-cuda_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

import pyoracle as po  # noqa: E402
from mvs_b200 import scenes  # noqa: E402

# The reference's src/ folder (its sample frames); MVS_REFERENCE_SRC overrides the default.
REFERENCE_SRC = pathlib.Path(os.environ.get("MVS_REFERENCE_SRC", "/root/reference/src"))


def frame_arrays(fr):
    return dict(ref=fr.ref, srcs=np.stack(fr.srcs), K=fr.ref_cam.K_1based.astype(np.float32),
                Rref=fr.ref_cam.R.astype(np.float32), tref=fr.ref_cam.t.astype(np.float32),
                Rsrc=np.stack([c.R for c in fr.src_cams]).astype(np.float32),
                tsrc=np.stack([c.t for c in fr.src_cams]).astype(np.float32),
                depth_gt=fr.depth_gt)


def poses(a):
    return [(a["Rsrc"][i], a["tsrc"][i]) for i in range(len(a["Rsrc"]))]


def sweep_case(name, seed, w, h, n_src, n_planes, win, planes_kind, znear=0.5, zfar=5.0, nccthresh=0.5):
    fr, planes, _ = scenes.config_tiny(seed=seed, width=w, height=h, n_src=n_src, n_planes=n_planes, win=win)
    a = frame_arrays(fr)
    if planes_kind == "inverse":
        pl = planes
        r = po.ref_sweep(a["ref"], list(a["srcs"]), a["K"], a["Rref"], a["tref"], poses(a), pl, win, znear=znear,
                         zfar=zfar, nccthresh=nccthresh)
    else:  # the reference's own float loop over [znear, zfar]
        pl = po.plane_list(znear, zfar, n_planes)
        r = po.ref_sweep(a["ref"], list(a["srcs"]), a["K"], a["Rref"], a["tref"], poses(a), None, win, znear=znear,
                         zfar=zfar, nplanes=n_planes, nccthresh=nccthresh)
    np.savez_compressed(HERE / f"{name}.npz", **a, planes=pl, win=win, znear=znear, zfar=zfar, nccthresh=nccthresh,
                        stdthresh=1e-4, depth=r["depth"], best=r["best"], vdepth=r["vdepth"],
                        label=po.labels_from_depth(r["vdepth"], pl))


def tgv_case(name, seed, w, h, n_src, niters, warps, start, beta=0.0, gamma=1.0):
    """PlaneSweep::TGV; beta != 0 turns the anisotropic diffusion tensor on
    (TGV2_kernels.cu:257-298), which then weights the P and U steps."""
    fr, _, _ = scenes.config_tiny(seed=seed, width=w, height=h, n_src=n_src)
    a = frame_arrays(fr)
    u_init = None if start == "one" else a["depth_gt"]
    u, _ = po.ref_tgv(a["ref"], list(a["srcs"]), a["K"], a["Rref"], a["tref"], poses(a), niters=niters, warps=warps,
                      u_init=u_init, beta=beta, gamma=gamma)
    np.savez_compressed(HERE / f"{name}.npz", **a, niters=niters, warps=warps, start=start, beta=beta, gamma=gamma,
                        u=u)


def tvl1_case(name, seed, w, h, niters):
    fr, _, _ = scenes.config_tiny(seed=seed, width=w, height=h, n_src=1)
    rng = np.random.default_rng(seed)
    d0 = (fr.depth_gt * (1 + 0.02 * rng.standard_normal(fr.depth_gt.shape))).astype(np.float32)
    znear, zfar = 0.5, 5.0
    out, _ = po.ref_tvl1_denoise(fr.ref, d0, znear, zfar, niters=niters)
    np.savez_compressed(HERE / f"{name}.npz", ref=fr.ref, depth_in=d0, znear=znear, zfar=zfar, niters=niters, out=out)


def tgv_sparse_case(name, seed, w, h, niters, frac, **kw):
    """PlaneSweep::TGVdenoiseFromSparse: start at a noisy depthmap, pull
    towards a sparse set of (noisy) samples, the rest of the pixels 0."""
    fr, _, _ = scenes.config_tiny(seed=seed, width=w, height=h, n_src=1)
    rng = np.random.default_rng(seed)
    gt = fr.depth_gt
    d0 = (gt * (1 + 0.03 * rng.standard_normal(gt.shape))).astype(np.float32)
    sparse = np.where(rng.random(gt.shape) < frac, gt * (1 + 0.005 * rng.standard_normal(gt.shape)), 0)
    sparse = sparse.astype(np.float32)
    zfar = 5.0
    out = po.ref_tgv_sparse(fr.ref, d0, sparse, zfar, niters, **kw)
    np.savez_compressed(HERE / f"{name}.npz", ref=fr.ref, depthmap=d0, sparse=sparse, zfar=zfar, niters=niters,
                        params=np.array([kw.get(k, d) for k, d in SPARSE_DEFAULTS]), out=out)


# (name, default) of PlaneSweep::TGVdenoiseFromSparse's numeric arguments, in order
SPARSE_DEFAULTS = (("alpha0", 2.0), ("alpha1", 1.5), ("tau", 0.02), ("sigma", 1.0), ("theta", 1.0), ("beta", 0.0),
                   ("gamma", 1.0))


def fusion_case(name, seed, dims, bins, n_maps, w, h, iters, interleaved):
    fi = scenes.fusion_sequence(seed, n_maps, w, h)
    vol = po.RefVolume(bins, dims, fi.vol_min, fi.vol_max)
    thr, tau, lam, sigma = 0.05, 0.1, 0.5, 1.0
    Ks = np.stack([c.K for c in fi.cams]).astype(np.float32)
    Rs = np.stack([c.R for c in fi.cams]).astype(np.float32)
    ts = np.stack([c.t for c in fi.cams]).astype(np.float32)
    depths = np.stack(fi.depths)
    if interleaved:   # FusionUpdateIteration per map (pclviewer.cpp:1040)
        for m in range(n_maps):
            vol.histogram(depths[m], Ks[m], Rs[m], ts[m], thr)
            vol.update_u(tau, lam)
            vol.update_p(sigma)
    else:             # all votes first, then `iters` primal-dual steps
        for m in range(n_maps):
            vol.histogram(depths[m], Ks[m], Rs[m], ts[m], thr)
        hist_only = vol.get()["hist"]
        for _ in range(iters):
            vol.update_u(tau, lam)
            vol.update_p(sigma)
    g = vol.get()
    np.savez_compressed(HERE / f"{name}.npz", depths=depths, K=Ks, R=Rs, t=ts, vol_min=fi.vol_min.astype(np.float32),
                        vol_max=fi.vol_max.astype(np.float32), dims=np.array(dims), bins=bins, thr=thr, tau=tau,
                        lam=lam, sigma=sigma, iters=iters, interleaved=interleaved, u=g["u"], v=g["v"], p=g["p"],
                        hist=g["hist"])


def main(only=None):
    """Regenerate every fixture, or only those whose names are listed."""
    if po.ref_lib() is None:
        raise SystemExit("oracle/_ref/libmvs_ref.so is not built (make -C oracle ref)")
    if only:
        for n in only:
            CASES[n]()
        return
    sweep_case("sweep_inverse_w5", seed=11, w=64, h=48, n_src=2, n_planes=16, win=5, planes_kind="inverse")
    sweep_case("sweep_refloop_w7", seed=12, w=56, h=40, n_src=3, n_planes=24, win=7, planes_kind="refloop")
    sweep_case("sweep_inverse_w3_negthr", seed=13, w=40, h=36, n_src=2, n_planes=12, win=3, planes_kind="inverse",
               nccthresh=-0.25)
    tgv_case("tgv_from_one", seed=21, w=48, h=40, n_src=2, niters=10, warps=3, start="one")
    tgv_case("tgv_from_depth", seed=22, w=48, h=40, n_src=3, niters=25, warps=2, start="depth")
    tgv_case("tgv_aniso", seed=23, w=56, h=44, n_src=3, niters=20, warps=2, start="depth", beta=1.5, gamma=0.8)
    tvl1_case("tvl1_denoise", seed=31, w=48, h=40, niters=40)
    fusion_case("fusion_b7_decoupled", seed=41, dims=(20, 16, 12), bins=7, n_maps=3, w=48, h=40, iters=12,
                interleaved=False)
    fusion_case("fusion_b8_interleaved", seed=42, dims=(18, 14, 10), bins=8, n_maps=4, w=48, h=40, iters=0,
                interleaved=True)
    fusion_case("fusion_b2_decoupled", seed=43, dims=(12, 10, 8), bins=2, n_maps=2, w=40, h=32, iters=6,
                interleaved=False)
    fusion_case("fusion_b10_decoupled", seed=44, dims=(12, 10, 8), bins=10, n_maps=3, w=40, h=32, iters=6,
                interleaved=False)
    for c in CASES.values():
        c()
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)


def real_frame_case(name, n_src=4, factor=4, n_planes=64, win=5, znear=0.1, zfar=1.0):
    """The reference's own sample frames (src/PlaneSweep/im0..9.png with
    Calibration.txt), grey as the GUI converts them (pclviewer.cpp:870-885,
    weights defines.h:19-21), box-downsampled by `factor` and rounded to 8 bits
    so the fixture stays small; K from the calibration line, scaled to the
    smaller image; the poses as the GUI passes them (pclviewer.cpp:346-405).
    Outputs of the reference's own kernels: the sweep with its float plane
    loop, the TV-L1 denoise of that depthmap, and TGV2 from it."""
    from PIL import Image
    src_dir = REFERENCE_SRC / "PlaneSweep"
    lines = (src_dir / "Calibration.txt").read_text().splitlines()
    fx, fy, cx, cy, sk = (float(x) for x in lines[0].split())
    W0, H0 = 640, 480
    K0 = np.array([[fx * W0, (1 - sk) * W0, cx * W0], [0, fy * H0, cy * H0], [0, 0, 1]])
    poses = []
    for k, ln in enumerate(lines):
        if ln.startswith("Transform"):
            m = np.array([[float(x) for x in lines[k + r].split()] for r in (1, 2, 3)])
            poses.append((m[:, :3].astype(np.float32), m[:, 3].astype(np.float32)))
    imgs = []
    for i in range(n_src + 1):
        rgb = np.asarray(Image.open(src_dir / f"im{i}.png").convert("RGB"), np.float64)
        gray = (0.2989 * rgb[..., 0] + 0.1140 * rgb[..., 2] + 0.5870 * rgb[..., 1]).astype(np.float32)
        h, w = gray.shape[0] // factor, gray.shape[1] // factor
        g = gray[:h * factor, :w * factor].reshape(h, factor, w, factor).mean(axis=(1, 3))
        imgs.append(np.clip(np.rint(g), 0, 255).astype(np.uint8))
    # 1-based pixel centres: full-resolution X = factor * X' - (factor - 1) / 2
    S = np.array([[1 / factor, 0, (factor - 1) / (2 * factor)], [0, 1 / factor, (factor - 1) / (2 * factor)], [0, 0, 1]])
    K = (S @ K0).astype(np.float32)
    ref, srcs = imgs[0].astype(np.float32), [im.astype(np.float32) for im in imgs[1:]]
    Rref, tref = poses[0]
    src_poses = poses[1:n_src + 1]
    r = po.ref_sweep(ref, srcs, K, Rref, tref, src_poses, None, win, znear=znear, zfar=zfar, nplanes=n_planes)
    planes = po.plane_list(znear, zfar, n_planes)
    den, _ = po.ref_tvl1_denoise(ref, r["depth"], znear, zfar, niters=50)
    tgv, _ = po.ref_tgv(ref, srcs, K, Rref, tref, src_poses, niters=40, warps=2, u_init=r["depth"])
    np.savez_compressed(HERE / f"{name}.npz", images=np.stack(imgs), K=K, Rref=Rref, tref=tref,
                        Rsrc=np.stack([p[0] for p in src_poses]), tsrc=np.stack([p[1] for p in src_poses]),
                        planes=planes, win=win, znear=znear, zfar=zfar, n_planes=n_planes,
                        depth=r["depth"], label=po.labels_from_depth(r["vdepth"], planes).astype(np.int16),
                        denoised=den, tgv=tgv)


CASES = {
    "tgv_aniso": lambda: tgv_case("tgv_aniso", seed=23, w=56, h=44, n_src=3, niters=20, warps=2, start="depth",
                                  beta=1.5, gamma=0.8),
    "tgv_sparse": lambda: tgv_sparse_case("tgv_sparse", seed=51, w=48, h=40, niters=60, frac=0.1),
    "real_frame": lambda: real_frame_case("real_frame"),
    "tgv_sparse_tensor": lambda: tgv_sparse_case("tgv_sparse_tensor", seed=52, w=37, h=29, niters=45, frac=0.25,
                                                 alpha0=1.3, alpha1=0.9, tau=0.05, sigma=2.0, theta=0.5, beta=2.5,
                                                 gamma=0.7),
}


if __name__ == "__main__":
    main(sys.argv[1:])
