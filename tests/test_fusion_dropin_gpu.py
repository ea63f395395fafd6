"""The C++ fusion drop-in (include/mvs_b200.hpp) compiled and run as a C++ caller.

tests/cpp/fusion_dropin.cpp is built with g++ against the header and
libmvs_b200.so and drives fusionData<8> the way the reference's GUI does
(pclviewer.cpp:972-1083): FusionUpdateIteration<8> per depthmap (fusion.cu.h:
91-99), copyTo into AoS fusionvoxel<8> rows at a padded pitch (fusion.h:
933-947).  The first snapshot equals the reference's own kernels run on the
same inputs (golden fusion_b8_interleaved) bit for bit; the second, after one
more U and P step taken once the shallow copies (fusion.h:176-182) were
destroyed, equals the same steps through the C ABI.
"""
import pathlib
import shutil
import subprocess

import numpy as np
import pytest

import mvs_b200 as M

pytestmark = pytest.mark.gpu

ROOT = pathlib.Path(__file__).resolve().parent.parent
SRC = ROOT / "tests" / "cpp" / "fusion_dropin.cpp"
LIB = ROOT / "plane-sweep-cuda_b200" / "mvs_b200" / "libmvs_b200.so"
CUDA = pathlib.Path("/usr/local/cuda")

VOXEL = np.dtype([("u", "<f4"), ("v", "<f4"), ("p", "<f4", 3), ("h", "u1", 8)])   # fusionvoxel<8>: 28 bytes


def _build(tmp):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.fail("g++ is needed to build the C++ drop-in test")
    exe = tmp / "fusion_dropin"
    cmd = [gxx, "-std=c++17", "-O1", "-I", str(ROOT / "include"), "-I", str(CUDA / "include"), str(SRC), "-o",
           str(exe), str(LIB), "-L", str(CUDA / "lib64"), "-lcudart", f"-Wl,-rpath,{LIB.parent}",
           f"-Wl,-rpath,{CUDA / 'lib64'}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _unpack(raw, rows, w, pitch):
    out = np.empty(rows * w, VOXEL)
    for r in range(rows):
        out[r * w:(r + 1) * w] = np.frombuffer(raw, VOXEL, count=w, offset=r * pitch)
    return out


def test_cpp_fusion_dropin_matches_reference_and_c_abi(cuda, golden, tmp_path):
    import torch
    g = golden("fusion_b8_interleaved")
    assert int(g["bins"]) == 8 and bool(g["interleaved"])
    w, h, d = (int(x) for x in g["dims"])
    nm, mh, mw = g["depths"].shape
    thr, tau, lam, sigma = float(g["thr"]), float(g["tau"]), float(g["lam"]), float(g["sigma"])
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        np.asarray([w, h, d, nm, mw, mh], np.int32).tofile(f)
        np.concatenate([g["vol_min"], g["vol_max"]]).astype(np.float32).tofile(f)
        np.asarray([thr], np.float32).tofile(f)
        np.asarray([tau, lam, sigma], np.float64).tofile(f)
        for k in ("depths", "K", "R", "t"):
            np.ascontiguousarray(g[k], np.float32).tofile(f)
    exe = _build(tmp_path)
    out = tmp_path / "out.bin"
    r = subprocess.run([str(exe), str(inp), str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    raw = out.read_bytes()
    pitch = int(np.frombuffer(raw, np.int32, count=1)[0])
    assert pitch == w * VOXEL.itemsize + 36 and VOXEL.itemsize == 28
    rows = h * d
    body = raw[4:]
    assert len(body) == 2 * rows * pitch
    first, second = _unpack(body[:rows * pitch], rows, w, pitch), _unpack(body[rows * pitch:], rows, w, pitch)
    # snapshot 1: the reference's own FusionUpdateIteration<8> on the same inputs
    np.testing.assert_array_equal(first["u"], g["u"])
    np.testing.assert_array_equal(first["v"], g["v"])
    np.testing.assert_array_equal(first["p"], g["p"].T)
    np.testing.assert_array_equal(first["h"], g["hist"].T.astype(np.uint8))
    # snapshot 2: the same run plus one U and P step through the C ABI
    vol = M.FusionVolume((w, h, d), 8, g["vol_min"], g["vol_max"])
    maps = torch.from_numpy(np.ascontiguousarray(g["depths"])).to(cuda)
    for m in range(nm):
        vol.iteration(maps[m], g["K"][m], g["R"][m], g["t"][m], thr, tau, lam, sigma)
    vol.update_u(tau, lam)
    vol.update_p(sigma)
    torch.cuda.synchronize()
    c = vol.download()
    vol.close()
    np.testing.assert_array_equal(second["u"], c["u"])
    np.testing.assert_array_equal(second["v"], c["v"])
    np.testing.assert_array_equal(second["p"], c["p"].T)
    np.testing.assert_array_equal(second["h"], c["hist"].T.astype(np.uint8))
