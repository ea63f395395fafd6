"""Seeded synthetic multiview scenes (CPU ray caster).

These stand in for the ICL-NUIM living-room and KITTI sequences that the
reference reads from disk (reader.cpp:147-231, kitti_reader.cpp), which are not
available here.  Everything is generated from a seed, so every test and bench
run sees the same pixels.

Conventions follow the reference:

* poses are world->camera, ``X_cam = R @ X_world + t`` (the
  ``alternativemethod == false`` branch of PlaneSweep::RelativeMatrices,
  planesweep.cpp:541-543);
* ``Camera.K`` is the usual 0-based pinhole matrix (pixel centre (0,0) is the
  first pixel).  The plane sweep and TGV2 kernels of the reference treat pixel
  (l, k) as (l+1, k+1) and subtract 1 after projection (kernels.cu:39-40,
  TGV2_kernels.cu:157-177), so they want ``K_1based`` (principal point + 1);
  fusion projects with 0-based pixels (fusion.cu:20-24) and wants ``K``;
* grayscale images are float32 in [0, 255] for the sweep (the GUI feeds the
  sweep 0..255 grey, pclviewer.cpp:870-885); TGV2 divides them by 255 itself
  (planesweep.cpp:419,436).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Camera:
    K: np.ndarray          # 3x3 float64, 0-based pixel convention
    R: np.ndarray          # 3x3 float64, world -> camera
    t: np.ndarray          # 3   float64
    width: int
    height: int

    @property
    def K_1based(self) -> np.ndarray:
        K = self.K.copy()
        K[0, 2] += 1.0
        K[1, 2] += 1.0
        return K

    @property
    def center(self) -> np.ndarray:
        return -self.R.T @ self.t


@dataclasses.dataclass
class Frame:
    """One reference view plus its source views."""
    ref: np.ndarray            # (H, W) float32, 0..255
    srcs: list                 # list of (H, W) float32, 0..255
    ref_cam: Camera
    src_cams: list             # list of Camera
    depth_gt: np.ndarray       # (H, W) float32, camera-z depth of the reference view


# ---------------------------------------------------------------------------
# 3-D value noise
# ---------------------------------------------------------------------------

class ValueNoise3D:
    """Seeded 4-octave value noise in [0, 1] on a periodic integer lattice."""

    def __init__(self, seed: int, octaves: int = 4, base_freq: float = 3.0,
                 lattice: int = 64):
        rng = np.random.default_rng(seed)
        self.table = rng.random(lattice ** 3, dtype=np.float64).reshape(
            lattice, lattice, lattice)
        self.lattice = lattice
        self.octaves = octaves
        self.base_freq = base_freq
        self.offsets = rng.random((octaves, 3)) * lattice

    def _octave(self, p: np.ndarray, o: int) -> np.ndarray:
        n = self.lattice
        q = p + self.offsets[o]
        i0 = np.floor(q).astype(np.int64)
        f = q - i0
        f = f * f * (3.0 - 2.0 * f)            # smoothstep
        i0 %= n
        i1 = (i0 + 1) % n
        T = self.table
        x0, y0, z0 = i0[..., 0], i0[..., 1], i0[..., 2]
        x1, y1, z1 = i1[..., 0], i1[..., 1], i1[..., 2]
        fx, fy, fz = f[..., 0], f[..., 1], f[..., 2]
        c000 = T[x0, y0, z0]; c100 = T[x1, y0, z0]
        c010 = T[x0, y1, z0]; c110 = T[x1, y1, z0]
        c001 = T[x0, y0, z1]; c101 = T[x1, y0, z1]
        c011 = T[x0, y1, z1]; c111 = T[x1, y1, z1]
        c00 = c000 + fx * (c100 - c000)
        c10 = c010 + fx * (c110 - c010)
        c01 = c001 + fx * (c101 - c001)
        c11 = c011 + fx * (c111 - c011)
        c0 = c00 + fy * (c10 - c00)
        c1 = c01 + fy * (c11 - c01)
        return c0 + fz * (c1 - c0)

    def __call__(self, p: np.ndarray) -> np.ndarray:
        acc = np.zeros(p.shape[:-1], dtype=np.float64)
        amp, freq, norm = 1.0, self.base_freq, 0.0
        for o in range(self.octaves):
            acc += amp * self._octave(p * freq, o)
            norm += amp
            amp *= 0.5
            freq *= 2.0
        return acc / norm


# ---------------------------------------------------------------------------
# geometry
# ---------------------------------------------------------------------------

def rot_xyz(ax: float, ay: float, az: float) -> np.ndarray:
    cx, sx = math.cos(ax), math.sin(ax)
    cy, sy = math.cos(ay), math.sin(ay)
    cz, sz = math.cos(az), math.sin(az)
    Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return Rz @ Ry @ Rx


def look_at(center: np.ndarray, target: np.ndarray,
            up=(0.0, -1.0, 0.0)) -> tuple[np.ndarray, np.ndarray]:
    """World->camera (R, t) for a camera at ``center`` looking at ``target``.

    Camera axes: x right, y down, z forward (the pinhole convention used by
    the reference's K matrices)."""
    z = np.asarray(target, float) - np.asarray(center, float)
    z /= np.linalg.norm(z)
    x = np.cross(z, -np.asarray(up, float))
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    R = np.stack([x, y, z])
    t = -R @ np.asarray(center, float)
    return R, t


class BoxScene:
    """Axis-aligned boxes: one 'room' seen from inside plus solid boxes.

    World frame: x right, y down (floor at +y), z forward."""

    def __init__(self, room_min, room_max, boxes, noise: ValueNoise3D,
                 inside_room: bool = True):
        self.room_min = np.asarray(room_min, float)
        self.room_max = np.asarray(room_max, float)
        self.boxes = [(np.asarray(a, float), np.asarray(b, float)) for a, b in boxes]
        self.noise = noise
        self.inside_room = inside_room

    def cast(self, origin: np.ndarray, dirs: np.ndarray) -> np.ndarray:
        """Ray parameter of the first hit for rays ``origin + s * dirs``."""
        inv = 1.0 / np.where(np.abs(dirs) < 1e-12, 1e-12, dirs)
        best = np.full(dirs.shape[:-1], np.inf)
        if self.inside_room:
            t1 = (self.room_min - origin) * inv
            t2 = (self.room_max - origin) * inv
            tfar = np.min(np.maximum(t1, t2), axis=-1)
            best = np.where(tfar > 1e-6, tfar, best)
        for a, b in self.boxes:
            t1 = (a - origin) * inv
            t2 = (b - origin) * inv
            tnear = np.max(np.minimum(t1, t2), axis=-1)
            tfar = np.min(np.maximum(t1, t2), axis=-1)
            hit = (tnear <= tfar) & (tnear > 1e-6)
            best = np.where(hit & (tnear < best), tnear, best)
        return best

    def render(self, cam: Camera, depth_only: bool = False) -> tuple[np.ndarray, np.ndarray]:
        """(intensity in [0,1], camera-z depth), both (H, W) float64.  With
        ``depth_only`` the texture lookup is skipped and intensity is None."""
        H, W = cam.height, cam.width
        xs, ys = np.meshgrid(np.arange(W, dtype=float), np.arange(H, dtype=float))
        pix = np.stack([xs, ys, np.ones_like(xs)], -1)
        rays_cam = pix @ np.linalg.inv(cam.K).T          # z component == 1
        dirs = rays_cam @ cam.R                          # R^T * ray
        origin = cam.center
        s = self.cast(origin, dirs)
        miss = ~np.isfinite(s)
        s = np.where(miss, 50.0, s)
        if depth_only:
            return None, s
        pts = origin + dirs * s[..., None]
        inten = self.noise(pts)
        inten = np.where(miss, 0.5, inten)
        return inten, s                                  # s is camera z depth


def box_room(seed: int) -> BoxScene:
    """4 x 3 x 5 m room (walls, floor, ceiling) with a few boxes on the floor."""
    rng = np.random.default_rng(seed + 7919)
    boxes = []
    for _ in range(4):
        sx, sy, sz = rng.uniform(0.3, 0.9, 3)
        cx = rng.uniform(-1.4, 1.4)
        cz = rng.uniform(-0.5, 2.0)
        boxes.append(((cx - sx / 2, 1.5 - sy, cz - sz / 2),
                      (cx + sx / 2, 1.5, cz + sz / 2)))
    return BoxScene((-2.0, -1.5, -2.5), (2.0, 1.5, 2.5), boxes,
                    ValueNoise3D(seed, base_freq=4.0))


def street(seed: int) -> BoxScene:
    """Ground plane (a very wide flat box) plus random boxes, for KITTI-like frames."""
    rng = np.random.default_rng(seed + 104729)
    boxes = [((-60.0, 1.65, -10.0), (60.0, 2.65, 120.0))]   # road/ground slab
    for _ in range(14):
        sx, sy, sz = rng.uniform(1.5, 4.5), rng.uniform(1.2, 3.0), rng.uniform(2.0, 6.0)
        side = rng.choice([-1.0, 1.0])
        cx = side * rng.uniform(3.0, 9.0)
        cz = rng.uniform(6.0, 60.0)
        boxes.append(((cx - sx / 2, 1.65 - sy, cz - sz / 2),
                      (cx + sx / 2, 1.65, cz + sz / 2)))
    boxes.append(((-40.0, -12.0, 80.0), (40.0, 1.65, 82.0)))  # far facade
    return BoxScene((0, 0, 0), (0, 0, 0), boxes,
                    ValueNoise3D(seed, base_freq=0.8), inside_room=False)


def intrinsics(fx: float, fy: float, cx: float, cy: float) -> np.ndarray:
    return np.array([[fx, 0.0, cx], [0.0, fy, cy], [0.0, 0.0, 1.0]])


def frame_geometry(seed: int, width: int, height: int, K: np.ndarray,
                   n_src: int, baseline=(0.05, 0.05), rot_deg: float = 2.0,
                   scene: str = "room") -> tuple[BoxScene, Camera, list]:
    """Scene, reference camera and source cameras of ``make_frame``.

    Source centres sit on an arc (a circle in the reference camera's x-y
    plane) with radius drawn from ``baseline`` (metres); each source camera
    gets an independent seeded rotation of up to ``rot_deg`` degrees per axis.
    """
    rng = np.random.default_rng(seed)
    if scene == "room":
        sc = box_room(seed)
        center = np.array([rng.uniform(-0.3, 0.3), rng.uniform(-0.2, 0.2), -2.0])
        target = center + np.array([rng.uniform(-0.3, 0.3), rng.uniform(-0.1, 0.2), 3.0])
    else:
        sc = street(seed)
        center = np.array([0.0, 0.0, 0.0])
        target = np.array([rng.uniform(-0.5, 0.5), 0.3, 20.0])
    R0, t0 = look_at(center, target)
    ref_cam = Camera(K.astype(float), R0, t0, width, height)
    cams = []
    for i in range(n_src):
        ang = 2.0 * math.pi * (i + rng.uniform(-0.2, 0.2)) / max(n_src, 1)
        r = rng.uniform(baseline[0], baseline[1])
        off_cam = np.array([r * math.cos(ang), r * math.sin(ang), 0.0])
        c = center + R0.T @ off_cam
        d = np.radians(rng.uniform(-rot_deg, rot_deg, 3))
        Rs = rot_xyz(*d) @ R0
        ts = -Rs @ c
        cams.append(Camera(K.astype(float), Rs, ts, width, height))
    return sc, ref_cam, cams


def make_frame(seed: int, width: int, height: int, K: np.ndarray,
               n_src: int, baseline=(0.05, 0.05), rot_deg: float = 2.0,
               scene: str = "room") -> Frame:
    """Reference view + ``n_src`` source views around it (see frame_geometry)."""
    sc, ref_cam, cams = frame_geometry(seed, width, height, K, n_src, baseline, rot_deg, scene)
    inten, depth = sc.render(ref_cam)
    srcs = [(sc.render(cam)[0] * 255.0).astype(np.float32) for cam in cams]
    return Frame((inten * 255.0).astype(np.float32), srcs, ref_cam, cams,
                 depth.astype(np.float32))


@dataclasses.dataclass
class DeviceFrame:
    """A frame rendered on the GPU: ``ref`` (H, W), ``srcs`` (V, H, W) in
    0..255 and ``depth_gt`` (H, W) are float32 CUDA tensors."""
    ref: object
    srcs: object
    ref_cam: Camera
    src_cams: list
    depth_gt: object


class GpuRenderer:
    """Renders BoxScene views with the library's ray caster (mvs_render_scene).

    The same scene and cameras give the CPU caster's pixels up to rounding
    order (FP64 throughout)."""

    def __init__(self, device="cuda"):
        self.device = device

    def _desc(self, sc: BoxScene):
        import torch
        from . import BoxSceneDesc
        table = torch.from_numpy(np.ascontiguousarray(sc.noise.table, dtype=np.float64)).to(self.device)
        boxes = np.ascontiguousarray([np.concatenate([a, b]) for a, b in sc.boxes], dtype=np.float64).reshape(-1)
        d = BoxSceneDesc()
        d.inside_room = int(sc.inside_room)
        d.n_boxes = len(sc.boxes)
        for k in range(3):
            d.room_min[k] = float(sc.room_min[k])
            d.room_max[k] = float(sc.room_max[k])
        import ctypes
        d.h_boxes = boxes.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        d.d_noise = table.data_ptr()
        d.lattice = sc.noise.lattice
        d.octaves = sc.noise.octaves
        d.base_freq = float(sc.noise.base_freq)
        for o in range(sc.noise.octaves):
            for k in range(3):
                d.offsets[o][k] = float(sc.noise.offsets[o][k])
        return d, (table, boxes)

    def render(self, sc: BoxScene, cams, with_image=True):
        """(gray255 (N, H, W) or None, depth (N, H, W)) for a list of cameras."""
        import torch
        from . import render_scene
        desc, keep = self._desc(sc)
        H, W = cams[0].height, cams[0].width
        depth = torch.empty((len(cams), H, W), dtype=torch.float32, device=self.device)
        gray = torch.empty_like(depth) if with_image else None
        for k, cam in enumerate(cams):
            render_scene(desc, np.linalg.inv(cam.K), cam.R, cam.center, W, H,
                         None if gray is None else gray[k], depth[k])
        torch.cuda.current_stream().synchronize()   # keeps the host table and boxes alive until done
        del keep
        return gray, depth

    def frame(self, seed: int, width: int, height: int, K: np.ndarray, n_src: int,
              baseline=(0.05, 0.05), rot_deg: float = 2.0, scene: str = "room") -> DeviceFrame:
        sc, ref_cam, cams = frame_geometry(seed, width, height, K, n_src, baseline, rot_deg, scene)
        gray, depth = self.render(sc, [ref_cam] + cams)
        return DeviceFrame(gray[0], gray[1:].contiguous(), ref_cam, cams, depth[0])


def inverse_depth_planes(znear: float, zfar: float, n: int) -> np.ndarray:
    """``n`` fronto-parallel plane depths uniform in inverse depth, near to far."""
    inv = np.linspace(1.0 / znear, 1.0 / zfar, n)
    return (1.0 / inv).astype(np.float32)


def reference_plane_list(znear: float, zfar: float, n: int) -> np.ndarray:
    """The depth list PlaneSweepThread walks (planesweep.cpp:169,200).

    ``dstep = (zfar - znear) / (n - 1)`` and ``for (float d = znear; d <= zfar;
    d += dstep)``, all in float32, so the count can be n or n-1 depending on
    rounding, exactly as in the reference."""
    zn, zf = np.float32(znear), np.float32(zfar)
    dstep = np.float32((zf - zn) / np.float32(n - 1))
    out = []
    d = zn
    while d <= zf:
        out.append(d)
        d = np.float32(d + dstep)
    return np.array(out, dtype=np.float32)


# ---------------------------------------------------------------------------
# configurations
# ---------------------------------------------------------------------------

def config_small(seed: int = 1) -> tuple[Frame, np.ndarray, int]:
    """320x240, 4 views on a 5 cm arc, 64 inverse-depth planes over [0.5, 5] m, 7x7."""
    K = intrinsics(240.0, 240.0, 160.0, 120.0)
    fr = make_frame(seed, 320, 240, K, 4, baseline=(0.05, 0.05))
    return fr, inverse_depth_planes(0.5, 5.0, 64), 7


def config_full(seed: int = 2) -> tuple[Frame, np.ndarray, int]:
    """640x480, 8 views with 2-10 cm baselines, 256 inverse-depth planes over [0.4, 8] m, 9x9."""
    K = intrinsics(481.2, 481.2, 319.5, 239.5)
    fr = make_frame(seed, 640, 480, K, 8, baseline=(0.02, 0.10))
    return fr, inverse_depth_planes(0.4, 8.0, 256), 9


def config_tiny(seed: int = 3, width: int = 64, height: int = 48, n_src: int = 2,
                n_planes: int = 16, win: int = 5):
    """Small case the scalar oracles finish in well under a second."""
    f = 0.75 * width
    K = intrinsics(f, f, (width - 1) / 2.0, (height - 1) / 2.0)
    fr = make_frame(seed, width, height, K, n_src, baseline=(0.05, 0.08))
    return fr, inverse_depth_planes(0.5, 5.0, n_planes), win


def config_street(seed: int, width: int = 1242, height: int = 375, n_src: int = 4):
    K = intrinsics(721.5, 721.5, 609.6, 172.9)
    return make_frame(seed, width, height, K, n_src, baseline=(0.05, 0.5),
                      rot_deg=1.0, scene="street")


# ---------------------------------------------------------------------------
# fusion inputs
# ---------------------------------------------------------------------------

@dataclasses.dataclass
class FusionInput:
    depths: list               # list of (H, W) float32 depthmaps (camera z)
    cams: list                 # list of Camera (0-based K, world->camera)
    vol_min: np.ndarray        # volume corner a
    vol_max: np.ndarray        # volume corner b


def fusion_sequence(seed: int, n_maps: int, width: int, height: int,
                    noise_frac: float = 0.01, outlier_frac: float = 0.02,
                    cube: float = 5.0, fx: float | None = None) -> FusionInput:
    """Depthmaps of the box room along a smooth seeded trajectory.

    Gaussian depth noise with sigma = ``noise_frac`` * depth and
    ``outlier_frac`` of the pixels replaced by uniform random depths."""
    rng = np.random.default_rng(seed)
    sc = box_room(seed)
    f = 0.75 * width if fx is None else fx
    K = intrinsics(f, f, (width - 1) / 2.0, (height - 1) / 2.0)
    depths, cams = [], []
    phase = rng.uniform(0, 2 * math.pi)
    for i in range(n_maps):
        a = phase + 0.9 * i / max(n_maps - 1, 1)
        center = np.array([0.8 * math.sin(a), -0.3 + 0.1 * math.sin(2 * a),
                           -1.6 + 0.4 * math.cos(a)])
        target = np.array([0.3 * math.sin(a + 1.0), 0.3, 2.0])
        R, t = look_at(center, target)
        cam = Camera(K, R, t, width, height)
        _, d = sc.render(cam, depth_only=True)
        d = d * (1.0 + noise_frac * rng.standard_normal(d.shape))
        out = rng.random(d.shape) < outlier_frac
        d = np.where(out, rng.uniform(0.3, 6.0, d.shape), d)
        depths.append(d.astype(np.float32))
        cams.append(cam)
    half = cube / 2.0
    return FusionInput(depths, cams, np.array([-half, -1.5, -2.5]),
                       np.array([half, -1.5 + cube, 2.5]))


# ---------------------------------------------------------------------------
# batched uneven frames
# ---------------------------------------------------------------------------

@dataclasses.dataclass
class BatchFrameSpec:
    kind: str          # "room320", "room640", "street"
    seed: int
    width: int
    height: int
    K: np.ndarray      # 0-based
    n_src: int
    n_planes: int
    window: int
    znear: float
    zfar: float
    baseline: tuple
    rot_deg: float
    scene: str


def batch_workload(seed: int = 4, n: int = 48) -> list:
    """Mixed frames: 320x240 and 640x480 box rooms and 1242x375 street frames
    (KITTI-like intrinsics fx = 721.5, cx = 609.6, cy = 172.9), 64-256
    inverse-depth planes, 4-8 source views and 5x5 to 11x11 windows, drawn
    from `seed`."""
    rng = np.random.default_rng(seed)
    kinds = ("room320", "room640", "street")
    out = []
    for i in range(n):
        kind = kinds[i % 3] if i < 3 else kinds[int(rng.integers(0, 3))]
        P = int(rng.choice([64, 96, 128, 160, 192, 224, 256]))
        V = int(rng.integers(4, 9))
        win = int(rng.choice([5, 7, 9, 11]))
        s = seed * 1000 + i
        if kind == "room320":
            spec = BatchFrameSpec(kind, s, 320, 240, intrinsics(240.0, 240.0, 160.0, 120.0), V, P, win, 0.5, 5.0,
                                  (0.05, 0.05), 2.0, "room")
        elif kind == "room640":
            spec = BatchFrameSpec(kind, s, 640, 480, intrinsics(481.2, 481.2, 319.5, 239.5), V, P, win, 0.4, 8.0,
                                  (0.02, 0.10), 2.0, "room")
        else:
            spec = BatchFrameSpec(kind, s, 1242, 375, intrinsics(721.5, 721.5, 609.6, 172.9), V, P, win, 2.0, 80.0,
                                  (0.05, 0.5), 1.0, "street")
        out.append(spec)
    return out
