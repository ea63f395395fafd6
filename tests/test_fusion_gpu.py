"""TV-L1 histogram fusion on the GPU against the reference (golden fixtures) and the oracle.

Histograms are integer counts: bit-exact.  u, v, p follow the reference's
float arithmetic statement for statement: bit-exact against the reference's
own kernels; against the FP64 oracle the bar is 1e-4 relative on u.
"""
import numpy as np
import pytest

import pyoracle as po
import mvs_b200 as M
from mvs_b200 import scenes

pytestmark = pytest.mark.gpu

CASES = ["fusion_b7_decoupled", "fusion_b8_interleaved", "fusion_b2_decoupled", "fusion_b10_decoupled"]


def run_fusion(cuda, g):
    import torch
    dims = tuple(int(x) for x in g["dims"])
    vol = M.FusionVolume(dims, int(g["bins"]), g["vol_min"], g["vol_max"])
    depths = torch.from_numpy(np.ascontiguousarray(g["depths"], np.float32)).to(cuda)
    thr, tau, lam, sigma = float(g["thr"]), float(g["tau"]), float(g["lam"]), float(g["sigma"])
    if bool(g["interleaved"]):
        for m in range(depths.shape[0]):
            vol.iteration(depths[m], g["K"][m], g["R"][m], g["t"][m], thr, tau, lam, sigma)
    else:
        vol.histogram(depths, g["K"], g["R"], g["t"], thr)
        vol.tvl1(int(g["iters"]), tau, lam, sigma)
    torch.cuda.synchronize()
    out = vol.download()
    vol.close()
    return out


@pytest.mark.parametrize("name", CASES)
def test_fusion_bit_exact_vs_reference(cuda, golden, name):
    g = golden(name)
    r = run_fusion(cuda, g)
    assert g["hist"].sum() > 0
    np.testing.assert_array_equal(r["hist"], g["hist"])
    np.testing.assert_array_equal(r["u"], g["u"])
    np.testing.assert_array_equal(r["v"], g["v"])
    np.testing.assert_array_equal(r["p"], g["p"])


def test_fusion_vs_fp64_oracle(cuda):
    """64^3 volume, 6 depthmaps, 7 bins, 30 iterations: histograms exact, u within 1e-4 of FP64."""
    import torch
    fi = scenes.fusion_sequence(9, 6, 96, 72)
    dims, bins = (64, 64, 64), 7
    Ks = np.stack([c.K for c in fi.cams]).astype(np.float32)
    Rs = np.stack([c.R for c in fi.cams]).astype(np.float32)
    ts = np.stack([c.t for c in fi.cams]).astype(np.float32)
    vol = M.FusionVolume(dims, bins, fi.vol_min, fi.vol_max)
    vol.histogram(torch.from_numpy(np.stack(fi.depths)).to(cuda), Ks, Rs, ts, 0.05)
    vol.tvl1(30, 0.1, 0.5, 1.0)
    torch.cuda.synchronize()
    r = vol.download()
    o = po.Volume(bins, dims, fi.vol_min, fi.vol_max, precision="f64")
    for m in range(len(fi.depths)):
        o.histogram(fi.depths[m], Ks[m], Rs[m], ts[m], 0.05)
    np.testing.assert_array_equal(r["hist"], o.hist)
    for _ in range(30):
        o.update_u(0.1, 0.5)
        o.update_p(1.0)
    err = np.abs(r["u"] - o.u) / np.maximum(np.abs(o.u), 1e-3)
    assert np.quantile(err, 0.999) <= 1e-4 and err.max() <= 1e-3, (np.quantile(err, 0.999), err.max())


def prox_want(hist, u0, bins, tau, lam):
    L = po.oracle_lib()
    return np.array([L.orc_prox_hist_f32(bins, np.ascontiguousarray(hist[:, i]).ctypes.data_as(po._U16),
                                         float(np.float32(np.float64(u0[i]))), np.float32(tau), np.float32(lam))
                     for i in range(hist.shape[1])], np.float32)


@pytest.mark.parametrize("bins,top", [(7, 12), (7, 4000), (10, 12), (10, 4000)])
def test_prox_median_matches_insertion_sort(cuda, bins, top):
    """The closed-form median of the U kernel against sortedHist's insertion (structs.h:241-262):
    random histograms and start values, u read back after one U step with p = 0.  Counts up to
    12 (and 200 in a few voxels), and up to 4000: the volume counts in 16 bits."""
    import torch
    rng = np.random.default_rng(3)
    dims = (16, 8, 8)
    n = dims[0] * dims[1] * dims[2]
    vol = M.FusionVolume(dims, bins, [0, 0, 0], [1, 1, 1])
    hist = rng.integers(0, top, size=(bins, n)).astype(np.uint16)
    hist[:, :50] = 0
    hist[0, 50:60] = 200
    u0 = rng.uniform(-3, 3, n).astype(np.float32)
    vol.upload(u=u0, v=np.zeros(n, np.float32), p=np.zeros((3, n), np.float32), hist=hist)
    tau, lam = 0.1, 0.5
    vol.update_u(tau, lam)
    torch.cuda.synchronize()
    r = vol.download()
    np.testing.assert_array_equal(r["u"], prox_want(hist, u0, bins, tau, lam))


class _DeviceArray:
    """A device pointer of the library as an array that torch can wrap without a copy."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (ptr, False),
                                         "strides": None, "version": 3}


def test_counts_written_through_device_pointer(cuda):
    """Counts written by the caller through mvs_fusion_device_state's pointer reach the next U
    step (counts below 40, then one count of 300), and after a reset and a histogram pass the U
    step reads that pass's counts."""
    import torch
    rng = np.random.default_rng(5)
    dims, bins = (16, 8, 8), 7
    n = dims[0] * dims[1] * dims[2]
    vol = M.FusionVolume(dims, bins, [0, 0, 0], [1, 1, 1])
    u0 = rng.uniform(-3, 3, n).astype(np.float32)
    zeros = dict(v=np.zeros(n, np.float32), p=np.zeros((3, n), np.float32))
    tau, lam = 0.1, 0.5
    st = vol.device_state()
    hs = st["hist_stride"]
    for top in (40, 300):
        hist = rng.integers(0, 40, size=(bins, n)).astype(np.uint16)
        hist[2, 77] = top
        dev = np.zeros((n, hs), np.uint16)
        dev[:, :bins] = hist.T
        vol.upload(u=u0, **zeros)
        st = vol.device_state()
        view = torch.as_tensor(_DeviceArray(st["hist"], (n, hs), "<i2"), device=cuda)
        view.copy_(torch.from_numpy(dev.view(np.int16)).to(cuda))
        torch.cuda.synchronize()
        vol.update_u(tau, lam)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(vol.download()["u"], prox_want(hist, u0, bins, tau, lam))
    vol.reset()
    fi = scenes.fusion_sequence(9, 2, 96, 72)
    vol.set_volume(fi.vol_min, fi.vol_max)
    Ks = np.stack([c.K for c in fi.cams]).astype(np.float32)
    Rs = np.stack([c.R for c in fi.cams]).astype(np.float32)
    ts = np.stack([c.t for c in fi.cams]).astype(np.float32)
    vol.histogram(torch.from_numpy(np.stack(fi.depths)).to(cuda), Ks, Rs, ts, 0.05)
    vol.upload(u=u0, **zeros)
    vol.update_u(tau, lam)
    torch.cuda.synchronize()
    r = vol.download()
    assert r["hist"].sum() > 0
    np.testing.assert_array_equal(r["u"], prox_want(r["hist"], u0, bins, tau, lam))


def test_extract_surface_points(cuda):
    dims = (10, 8, 6)
    n = 10 * 8 * 6
    vol = M.FusionVolume(dims, 7, [-1, -1, -1], [1, 1, 2])
    u = np.linspace(-1.5, 1.5, n).astype(np.float32)
    vol.upload(u=u)
    pts = vol.extract(-1.0, 0.0)
    idx = np.nonzero((u > -1) & (u < 0))[0]
    x, y, z = idx % 10, (idx // 10) % 8, idx // 80
    a = np.float32([-1, -1, -1])
    s = np.float32([2, 2, 3])
    want = np.stack([a[0] + s[0] * ((x + .5) / 10).astype(np.float32),
                     a[1] + s[1] * ((y + .5) / 8).astype(np.float32),
                     a[2] + s[2] * ((z + .5) / 6).astype(np.float32)], 1).astype(np.float32)
    np.testing.assert_array_equal(pts, want)
