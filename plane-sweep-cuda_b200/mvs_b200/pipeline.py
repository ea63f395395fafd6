"""Headless reconstruction: frames -> plane sweep -> TV-L1 denoise -> TV-L1
histogram fusion -> surface points (PLY).

The sequence of PCLViewer::on_reconstruct_button_clicked
(pclviewer.cpp:972-1083) without the GUI: per frame the PlaneSweep handle
runs RunAlgorithm and CudaDenoise, and FusionUpdateIteration fuses the
denoised device depthmap (getDepthmapDenoisedPtr) into the volume with the
world -> reference pose (RelativeMatrices of the identity and the reference
pose) and the sweep's K; afterwards the voxels with -1 < u < 0 become the
point cloud, x negated and coloured by the viewer's depth colour map of their
x position (pclviewer.cpp:1058-1074), written as PLY instead of shown by PCL.
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class SweepSettings:
    znear: float = 0.4
    zfar: float = 8.0
    n_planes: int = 64
    window: int = 5
    std_threshold: float = 1e-4
    ncc_threshold: float = 0.5
    plane_depths: np.ndarray | None = None   # None: the reference's uniform plane loop


@dataclasses.dataclass
class DenoiseSettings:
    """PlaneSweep::CudaDenoise parameters (the GUI's defaults)."""
    niters: int = 100
    lam: float = 0.3
    tau: float = 0.02
    sigma: float = 6.0
    theta: float = 1.0
    beta: float = 0.0
    gamma: float = 1.0


@dataclasses.dataclass
class FusionSettings:
    dims: tuple = (128, 128, 128)
    bins: int = 8
    threshold: float = 0.05
    tau: float = 0.1
    lam: float = 0.5
    sigma: float = 1.0


def reconstruct(frames, corner_a, corner_b, sweep=SweepSettings(), denoise=DenoiseSettings(),
                fusion=FusionSettings(), ply_path=None, binary=False):
    """Fuse `frames` into a volume over the box corner_a..corner_b.

    Each frame: dict(ref=(H, W) 0..255, srcs=(V, H, W), K=1-based 3x3, R, t
    (world -> camera of the reference), src_R, src_t (lists, world -> camera)).
    Returns (points (N, 3) float32 with x negated as the viewer shows them,
    colours (N, 3) uint8, the FusionVolume)."""
    import mvs_b200 as M
    ps = M.PlaneSweep()
    vol = M.FusionVolume(fusion.dims, fusion.bins, corner_a, corner_b)
    try:
        for fr in frames:
            ref = np.ascontiguousarray(fr["ref"], np.float32)
            H, W = ref.shape
            K = np.asarray(fr["K"], np.float32)
            ps.setK(K)
            ps.setZ(sweep.znear, sweep.zfar)
            ps.setNumberofPlanes(sweep.n_planes)
            if sweep.plane_depths is not None:
                ps.setPlaneDepths(np.asarray(sweep.plane_depths, np.float32))
            ps.setWindowSize(sweep.window)
            ps.setSTDthreshold(sweep.std_threshold)
            ps.setNCCthreshold(sweep.ncc_threshold)
            ps.set_reference(ref, fr["R"], fr["t"])
            srcs = np.ascontiguousarray(fr["srcs"], np.float32)
            ps.setNumberofImages(len(srcs))
            ps.set_sources(srcs, np.stack(fr["src_R"]), np.stack(fr["src_t"]))
            ps.RunAlgorithm()
            ps.CudaDenoise(denoise.niters, denoise.lam, denoise.tau, denoise.sigma, denoise.theta, denoise.beta,
                           denoise.gamma)
            # RelativeMatrices(R, T, I, 0, HostRef.R, HostRef.t): world -> reference camera
            R = np.asarray(fr["R"], np.float32)
            t = np.asarray(fr["t"], np.float32)
            vol.iteration(ps.getDepthmapDenoisedPtr(), K, R, t, fusion.threshold, fusion.tau, fusion.lam,
                          fusion.sigma, shape=(H, W))
        pts = vol.extract(-1.0, 0.0)
        a = np.asarray(corner_a, np.float32)
        size = np.asarray(corner_b, np.float32) - a
        gray = (np.float32(255) * (pts[:, 0] - a[0]) / size[0]).astype(np.uint8)
        colours = M.depth_color(gray)
        out = pts.copy()
        out[:, 0] = -out[:, 0]
        if ply_path is not None:
            M.write_ply(ply_path, out, colours, binary=binary)
        return out, colours, vol
    finally:
        ps.close()
