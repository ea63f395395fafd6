"""Data formats either side of the path: the ICL-NUIM camera reader against a
float32 restatement of Reader::getcamK / computeRT (reader.cpp:181-225), the
PLY writer (read back) and the viewer's depth colour map (pclviewer.cpp:1084-1115)."""
import math

import numpy as np
import pytest

import mvs_b200 as M

ICL = """cam_pos      = [0.790932, 1.300000, 1.462270]';
cam_dir      = [-0.599, 0.104, -0.7935]';
cam_up       = [0.0, 1.0, 0.05]';
cam_lookat   = [0, 0, 1]';
cam_sky      = [0, 1, 0]';
cam_right    = [1.3333, 0.0, -0.02]';
cam_fpoint   = [0, 0, 10]';
cam_angle    = 90;
"""


def _f32(*v):
    return [np.float32(x) for x in v]


def _len(v):
    return np.sqrt(np.float32(np.float32(v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]))


def _cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def _icl_restated(pos, d, up, right, w, h):
    focal = float(_len(d))
    aspect = float(_len(right))
    angle = 2 * math.atan(aspect / 2 / focal)
    aspect = aspect / float(_len(up))
    psx = 2 * focal * math.tan(0.5 * angle) / w
    psy = 2 * focal * math.tan(0.5 * angle) / aspect / h
    psx, psy = psx / focal, psy / focal
    K = np.array([[1.0 / psx, 0, (w + 1) * 0.5], [0, -1.0 / psy, (h + 1) * 0.5], [0, 0, 1]], np.float32)
    L = _len(d)
    z = [d[0] / L, d[1] / L, d[2] / L]
    c = _cross(up, z)
    inv = np.float32(1) / np.sqrt(np.float32(np.float32(c[0] * c[0] + c[1] * c[1]) + c[2] * c[2]))
    x = [c[0] * inv, c[1] * inv, c[2] * inv]
    y = _cross(z, x)
    R = np.array([x, y, z], np.float32).T
    return K, R, np.array(pos, np.float32)


def test_icl_camera_matches_restatement(tmp_path):
    f = tmp_path / "scene_00_0000.txt"
    f.write_text(ICL)
    K, R, t = M.read_icl_camera(f)
    rK, rR, rt = _icl_restated(_f32(0.790932, 1.3, 1.46227), _f32(-0.599, 0.104, -0.7935), _f32(0.0, 1.0, 0.05),
                               _f32(1.3333, 0.0, -0.02), 640, 480)
    np.testing.assert_array_equal(K, rK)
    np.testing.assert_array_equal(R, rR)
    np.testing.assert_array_equal(t, rt)
    assert K[1, 1] < 0 and K[0, 2] == 320.5 and K[1, 2] == 240.5
    # an orthonormal camera -> world rotation (up tilted, so not exactly)
    assert np.allclose(R.T @ R, np.eye(3), atol=1e-5)


def test_icl_camera_errors(tmp_path):
    with pytest.raises(M.MvsError):
        M.read_icl_camera(tmp_path / "missing.txt")
    f = tmp_path / "partial.txt"
    f.write_text("cam_pos = [1, 2, 3]';\ncam_dir = [0, 0, 1]';\n")
    with pytest.raises(M.MvsError):
        M.read_icl_camera(f)


@pytest.mark.parametrize("binary", [False, True])
def test_ply_roundtrip(tmp_path, binary):
    rng = np.random.default_rng(0)
    xyz = rng.normal(size=(57, 3)).astype(np.float32)
    rgb = rng.integers(0, 256, (57, 3)).astype(np.uint8)
    p = tmp_path / "c.ply"
    M.write_ply(p, xyz, rgb, binary=binary)
    data = p.read_bytes()
    head, body = data.split(b"end_header\n", 1)
    assert b"element vertex 57" in head
    if binary:
        rec = np.frombuffer(body, dtype=np.dtype([("p", "<f4", 3), ("c", "u1", 3)]))
        np.testing.assert_array_equal(rec["p"], xyz)
        np.testing.assert_array_equal(rec["c"], rgb)
    else:
        rows = [ln.split() for ln in body.decode().strip().splitlines()]
        np.testing.assert_array_equal(np.array([[float(v) for v in r[:3]] for r in rows], np.float32), xyz)
        np.testing.assert_array_equal(np.array([[int(v) for v in r[3:]] for r in rows], np.uint8), rgb)


def test_depth_color_bands():
    c = M.depth_color(np.array([0, 31, 32, 95, 96, 159, 160, 223, 224, 255], np.uint8))
    np.testing.assert_array_equal(c, [[0, 0, 128], [0, 0, 252], [0, 0, 255], [0, 252, 255], [0, 255, 255],
                                      [252, 255, 3], [255, 255, 0], [255, 3, 0], [255, 0, 0], [131, 0, 0]])
