"""Python binding of libmvs_b200 (ctypes over the C ABI of include/mvs_b200.h).

The compute path is the CUDA library only: the first call into it opens
``libmvs_b200.so`` and raises ``ImportError`` if it is missing or cannot be
loaded -- there is no CPU fallback.  The pure-host modules of the package
(``scenes``, ``dist``, ``hostmath``) can be imported without opening it.  Device memory for the device-pointer entry
points is handled with torch tensors (plumbing only; no torch math runs on the
product path).

Main entry points
    sweep(...)               fused plane sweep over device tensors
    sweep_homographies(...)  FP64 per-plane homographies on the device
    tgv2_run(...)            TGV2 refinement over device tensors
    tvl1_denoise(...)        TV-L1 depth denoise over device tensors
    FusionVolume             TV-L1 histogram fusion volume (mvs_fusion handle)
    PlaneSweep               the reference's PlaneSweep API over host arrays
                             (mvs_ps_* handle: host buffers in, host out)
"""
from __future__ import annotations

import ctypes as C
import math
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "libmvs_b200.so"

MVS_OK = 0
MVS_ERR_ARG, MVS_ERR_NOMEM, MVS_ERR_CUDA, MVS_ERR_TIMEOUT, MVS_ERR_STATE, MVS_ERR_NOTBUILT = -1, -2, -3, -4, -5, -6
MOMENTS_REFERENCE, MOMENTS_COMPENSATED = 0, 1
SWEEP_PER_VIEW, SWEEP_AGGREGATED = 0, 1


class MvsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libmvs_b200 error {code}: {msg}")
        self.code = code


class _Library:
    """libmvs_b200.so, opened on the first call into it.

    Signatures declared with ``_sig`` are bound when the library opens.  A
    missing or unloadable library raises ``ImportError`` at that first call:
    there is no fallback."""

    def __init__(self):
        self._cdll = None
        self._sigs = []

    def declare(self, name, res, args):
        self._sigs.append((name, res, list(args)))
        if self._cdll is not None:
            self._bind(self._cdll, name, res, args)

    @staticmethod
    def _bind(cdll, name, res, args):
        f = getattr(cdll, name)
        f.restype = res
        f.argtypes = list(args)

    def load(self):
        if self._cdll is None:
            if not LIB_PATH.exists():
                raise ImportError(f"{LIB_PATH} is missing: build it with `python plane-sweep-cuda_b200/build.py`")
            try:
                cdll = C.CDLL(str(LIB_PATH))
            except OSError as e:  # pragma: no cover - depends on the box
                raise ImportError(f"cannot load {LIB_PATH}: {e}") from e
            for name, res, args in self._sigs:
                self._bind(cdll, name, res, args)
            self._cdll = cdll
        return self._cdll

    def __getattr__(self, name):
        return getattr(self.load(), name)


_L = _Library()

_F = C.POINTER(C.c_float)
_D = C.POINTER(C.c_double)
_I32 = C.POINTER(C.c_int32)
_U8 = C.POINTER(C.c_uint8)
_U16 = C.POINTER(C.c_uint16)
_VP = C.c_void_p


class SweepDesc(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("n_views", C.c_int32), ("n_planes", C.c_int32),
                ("window", C.c_int32), ("moments", C.c_int32), ("mode", C.c_int32),
                ("std_threshold", C.c_float), ("ncc_threshold", C.c_float), ("zfar", C.c_float)]


class TGV2Params(C.Structure):
    _fields_ = [("niters", C.c_int32), ("warps", C.c_int32), ("lam", C.c_double), ("alpha0", C.c_double),
                ("alpha1", C.c_double), ("tau", C.c_double), ("sigma", C.c_double), ("beta", C.c_double),
                ("gamma", C.c_double), ("tol", C.c_double), ("check_every", C.c_int32), ("max_iters", C.c_int32),
                ("iteration_kernel", C.c_int32), ("stop_window", C.c_int32)]


class TVL1Params(C.Structure):
    _fields_ = [("niters", C.c_int32), ("lam", C.c_double), ("tau", C.c_double), ("sigma", C.c_double),
                ("theta", C.c_double), ("beta", C.c_double), ("gamma", C.c_double)]


class BoxSceneDesc(C.Structure):
    _fields_ = [("inside_room", C.c_int32), ("n_boxes", C.c_int32), ("room_min", C.c_double * 3),
                ("room_max", C.c_double * 3), ("h_boxes", C.POINTER(C.c_double)), ("d_noise", C.c_void_p),
                ("lattice", C.c_int32), ("octaves", C.c_int32), ("base_freq", C.c_double),
                ("offsets", (C.c_double * 3) * 8)]


class BatchFrameDesc(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("n_views", C.c_int32), ("n_planes", C.c_int32),
                ("window", C.c_int32), ("std_threshold", C.c_float), ("zfar", C.c_float), ("d_ref", C.c_void_p),
                ("d_srcs", C.c_void_p), ("d_depths", C.c_void_p), ("h_K9", C.POINTER(C.c_double)),
                ("h_Rrel", C.POINTER(C.c_double)), ("h_trel", C.POINTER(C.c_double)), ("d_depth", C.c_void_p),
                ("d_labels", C.c_void_p), ("d_best", C.c_void_p)]


class BatchTuning(C.Structure):
    _fields_ = [("planes_per_chunk", C.c_int32), ("ctas_per_sm", C.c_int32), ("order", C.c_int32),
                ("tile_step", C.c_int32)]


def _sig(name, res, *args):
    _L.declare(name, res, args)


_sig("mvs_last_error", C.c_char_p)
_sig("mvs_version", C.c_int)
_sig("mvs_set_device", C.c_int, C.c_int)
_sig("mvs_host_alloc", C.c_void_p, C.c_size_t)
_sig("mvs_host_free", None, C.c_void_p)
_sig("mvs_sweep_workspace_bytes", C.c_size_t, C.POINTER(SweepDesc))
_sig("mvs_sweep_homographies", C.c_int, C.POINTER(SweepDesc), _D, _D, _D, _VP, _VP, _VP)
_sig("mvs_sweep", C.c_int, C.POINTER(SweepDesc), _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, C.c_size_t, _VP)
_sig("mvs_sweep_noalloc", C.c_int, C.POINTER(SweepDesc), _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP)
_sig("mvs_sweep_noalloc_scratch_bytes", C.c_size_t)
_sig("mvs_sweep_wta_volume", C.c_int, _VP, _VP, C.c_int32, C.c_int32, C.c_float, _VP, _VP, _VP, _VP)
_sig("mvs_tgv2_workspace_bytes", C.c_size_t, C.c_int32, C.c_int32, C.c_int32)
_sig("mvs_tgv2_run", C.c_int, C.c_int32, C.c_int32, C.c_int32, _VP, _VP, _F, _F, _F, _F, C.POINTER(TGV2Params),
     C.c_int32, C.c_float, _VP, _I32, _D, _VP, C.c_size_t, _VP)
_sig("mvs_tgv2_run_warm", C.c_int, C.c_int32, C.c_int32, C.c_int32, _VP, _VP, _F, _F, _F, _F, C.POINTER(TGV2Params),
     _VP, _VP, _VP, C.c_double, C.c_double, _VP, _VP, _I32, _D, _VP, C.c_size_t, _VP)
_sig("mvs_render_scene", C.c_int, C.POINTER(BoxSceneDesc), _D, _D, _D, C.c_int32, C.c_int32, _VP, _VP, _VP)
_sig("mvs_unet_create", C.c_int, C.POINTER(_VP), C.c_int32, C.c_int32, C.c_int32, _F)
_sig("mvs_unet_destroy", C.c_int, _VP)
_sig("mvs_unet_param_count", C.c_int64, _VP)
_sig("mvs_unet_layer_info", C.c_int, _VP, C.c_int32, _I32, _I32, C.POINTER(C.c_int64), C.POINTER(C.c_int64))
_sig("mvs_unet_set_params", C.c_int, _VP, _F)
_sig("mvs_unet_get_params", C.c_int, _VP, _F, _F)
_sig("mvs_unet_forward", C.c_int, _VP, _VP, _VP, _VP, _VP, _VP, _VP)
_sig("mvs_unet_backward", C.c_int, _VP, _VP, _VP, _D, _VP)
_sig("mvs_unet_adam_step", C.c_int, _VP, C.c_float, C.c_float, C.c_float, C.c_float, _VP)
_sig("mvs_unet_train_step", C.c_int, _VP, _VP, _VP, _VP, _VP, _VP, C.c_float, _D, _VP)
_sig("mvs_unet_check", C.c_int, _VP, _VP)
_sig("mvs_conv3x3_forward", C.c_int, _VP, C.c_int32, _VP, _VP, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
     C.c_int32, _VP, _VP, _VP, _VP)
_sig("mvs_conv3x3_backward", C.c_int, _VP, C.c_int32, _VP, _VP, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
     C.c_int32, _VP, _VP, _VP, _VP, _VP, C.c_int32, _VP)
_sig("mvs_batch_create", C.c_int, C.POINTER(_VP), C.POINTER(BatchFrameDesc), C.c_int32, C.c_int32,
     C.POINTER(BatchTuning))
_sig("mvs_batch_destroy", C.c_int, _VP)
_sig("mvs_batch_get_tuning", C.c_int, _VP, C.POINTER(BatchTuning))
_sig("mvs_batch_set_poses", C.c_int, _VP, _D, _D, _VP)
_sig("mvs_batch_run", C.c_int, _VP, _VP)
_sig("mvs_batch_frame_latency_ms", C.c_int, _VP, _F, _VP)
_sig("mvs_batch_work_items", C.c_int64, _VP)
_sig("mvs_read_icl_camera", C.c_int, C.c_char_p, C.c_int32, C.c_int32, _F, _F, _F)
_sig("mvs_write_ply", C.c_int, C.c_char_p, _F, C.POINTER(C.c_uint8), C.c_int64, C.c_int32)
_sig("mvs_depth_color", None, C.POINTER(C.c_uint8), C.c_int64, C.POINTER(C.c_uint8))
_sig("mvs_tgv2_sparse_workspace_bytes", C.c_size_t, C.c_int32, C.c_int32)
_sig("mvs_tgv2_sparse", C.c_int, C.c_int32, C.c_int32, _VP, _VP, _VP, C.c_float, C.c_int32, *([C.c_double] * 7), _VP,
     _VP, C.c_size_t, _VP)
_sig("mvs_tvl1_workspace_bytes", C.c_size_t, C.c_int32, C.c_int32)
_sig("mvs_tvl1_denoise", C.c_int, C.c_int32, C.c_int32, _VP, _VP, C.c_float, C.c_float, C.POINTER(TVL1Params),
     _VP, C.c_size_t, _VP)
_sig("mvs_compute3d", C.c_int, C.c_int32, C.c_int32, _VP, _F, _F, _F, _VP, _VP, _VP, _VP)
_sig("mvs_fusion_create", C.c_int, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _F, _F, C.POINTER(_VP))
_sig("mvs_fusion_destroy", C.c_int, _VP)
_sig("mvs_fusion_set_volume", C.c_int, _VP, _F, _F)
_sig("mvs_fusion_reset", C.c_int, _VP, _VP)
_sig("mvs_fusion_histogram", C.c_int, _VP, _VP, C.c_int32, C.c_int32, C.c_int32, _F, _F, _F, C.c_float, _VP)
_sig("mvs_fusion_tvl1", C.c_int, _VP, C.c_int32, C.c_double, C.c_double, C.c_double, _VP)
_sig("mvs_fusion_update_u", C.c_int, _VP, C.c_double, C.c_double, _VP)
_sig("mvs_fusion_update_p", C.c_int, _VP, C.c_double, _VP)
_sig("mvs_fusion_iteration", C.c_int, _VP, _VP, C.c_int32, C.c_int32, _F, _F, _F, C.c_float, C.c_double,
     C.c_double, C.c_double, _VP)
_sig("mvs_fusion_download", C.c_int, _VP, _F, _F, _F, _U16)
_sig("mvs_fusion_upload", C.c_int, _VP, _F, _F, _F, _U16)
_sig("mvs_fusion_device_state", C.c_int, _VP, C.POINTER(_VP), C.POINTER(_VP), C.POINTER(_VP), C.POINTER(_VP), _I32)
_sig("mvs_fusion_extract", C.c_int, _VP, C.c_float, C.c_float, _F, C.c_int64, C.POINTER(C.c_int64))
_sig("mvs_ps_create", C.c_int, C.POINTER(_VP))
_sig("mvs_ps_destroy", C.c_int, _VP)
_sig("mvs_ps_set_reference", C.c_int, _VP, _F, C.c_int32, C.c_int32, _F, _F)
_sig("mvs_ps_set_sources", C.c_int, _VP, _F, C.c_int32, _F, _F)
_sig("mvs_ps_set_K", C.c_int, _VP, _F)
_sig("mvs_ps_set_z", C.c_int, _VP, C.c_float, C.c_float)
_sig("mvs_ps_set_number_of_planes", C.c_int, _VP, C.c_int32)
_sig("mvs_ps_set_number_of_images", C.c_int, _VP, C.c_int32)
_sig("mvs_ps_set_window_size", C.c_int, _VP, C.c_int32)
_sig("mvs_ps_set_std_threshold", C.c_int, _VP, C.c_float)
_sig("mvs_ps_set_ncc_threshold", C.c_int, _VP, C.c_float)
_sig("mvs_ps_set_alternative_relative_matrix_method", C.c_int, _VP, C.c_int32)
_sig("mvs_ps_set_plane_depths", C.c_int, _VP, _F, C.c_int32)
_sig("mvs_ps_set_sweep_options", C.c_int, _VP, C.c_int32, C.c_int32, C.c_int32)
_sig("mvs_ps_run_algorithm", C.c_int, _VP)
_sig("mvs_ps_cuda_denoise", C.c_int, _VP, C.c_int32, *([C.c_double] * 6))
_sig("mvs_ps_tgv", C.c_int, _VP, C.c_int32, C.c_int32, *([C.c_double] * 7))
_sig("mvs_ps_tgv_denoise_from_sparse", C.c_int, _VP, _F, C.c_int32, *([C.c_double] * 7))
_sig("mvs_ps_tgv_ext", C.c_int, _VP, C.POINTER(TGV2Params), C.c_int32, _F, _I32, _D)
_sig("mvs_ps_get_size", C.c_int, _VP, _I32, _I32)
for _n in ("depthmap", "depthmap_denoised", "depthmap_tgv"):
    _sig(f"mvs_ps_get_{_n}", C.c_int, _VP, _F)
for _n in ("depthmap8u", "depthmap8u_denoised", "depthmap8u_tgv"):
    _sig(f"mvs_ps_get_{_n}", C.c_int, _VP, _U8)
_sig("mvs_ps_get_depthmap_denoised_ptr", C.c_int, _VP, C.POINTER(_VP))
_sig("mvs_ps_get_view_labels", C.c_int, _VP, _I32)
_sig("mvs_ps_get_view_best", C.c_int, _VP, _F)
_sig("mvs_ps_get_3d_coordinates", C.c_int, _VP, _F, _F, _F)
_sig("mvs_ps_get_plane_count", C.c_int, _VP, _I32)
_sig("mvs_ps_get_last_kernel_ms", C.c_int, _VP, _F)


def lib():
    """The opened ctypes library (opens it on the first call)."""
    return _L.load()


def check(rc):
    if rc != MVS_OK:
        raise MvsError(rc, _L.mvs_last_error().decode(errors="replace"))
    return rc


def _fp(a):
    return None if a is None else a.ctypes.data_as(_F)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(t):
    """Device pointer of a CUDA tensor (None -> NULL)."""
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("expected a contiguous CUDA tensor")
    return C.c_void_p(t.data_ptr())


def _stream(stream):
    if stream is None:
        import torch
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return C.c_void_p(int(stream))


# ---------------------------------------------------------------------------
# plane sweep (device tensors)
# ---------------------------------------------------------------------------

def sweep_desc(width, height, n_views, n_planes, window, moments=MOMENTS_REFERENCE, mode=SWEEP_PER_VIEW,
               std_threshold=1e-4, ncc_threshold=0.5, zfar=1.0):
    return SweepDesc(width, height, n_views, n_planes, window, moments, mode, std_threshold, ncc_threshold, zfar)


def relative_pose(Rref, tref, Rsrc, tsrc, alternative=False):
    """PlaneSweep::RelativeMatrices in float64 (reference -> source)."""
    Rref, tref, Rsrc, tsrc = (np.asarray(x, np.float64) for x in (Rref, tref, Rsrc, tsrc))
    if not alternative:
        Rrel = Rsrc @ np.linalg.inv(Rref)
        return Rrel, tsrc - Rrel @ tref
    return Rsrc.T @ Rref, Rsrc.T @ (tref - tsrc)


def sweep_homographies(desc, K_1based, rel_poses, depths, H_out, stream=None):
    """FP64 homographies on the device. rel_poses: list of (Rrel, trel)."""
    K = np.ascontiguousarray(np.asarray(K_1based, np.float64).reshape(9))
    R = np.ascontiguousarray(np.stack([np.asarray(p[0], np.float64).reshape(9) for p in rel_poses]))
    t = np.ascontiguousarray(np.stack([np.asarray(p[1], np.float64).reshape(3) for p in rel_poses]))
    check(_L.mvs_sweep_homographies(C.byref(desc), K.ctypes.data_as(_D), R.ctypes.data_as(_D),
                                    t.ctypes.data_as(_D), _ptr(depths), _ptr(H_out), _stream(stream)))


def sweep_workspace_bytes(desc):
    return int(_L.mvs_sweep_workspace_bytes(C.byref(desc)))


def sweep(desc, ref, srcs, H, depths, depth_out, labels=None, best=None, cost=None, workspace=None, stream=None):
    ws_bytes = 0 if workspace is None else workspace.numel() * workspace.element_size()
    check(_L.mvs_sweep(C.byref(desc), _ptr(ref), _ptr(srcs), _ptr(H), _ptr(depths), _ptr(depth_out), _ptr(labels),
                       _ptr(best), _ptr(cost), _ptr(workspace), ws_bytes, _stream(stream)))


def sweep_wta_volume(cost, depths, n_pixels, n_planes, zfar, depth_out, labels=None, best=None, stream=None):
    check(_L.mvs_sweep_wta_volume(_ptr(cost), _ptr(depths), n_pixels, n_planes, zfar, _ptr(depth_out),
                                  _ptr(labels), _ptr(best), _stream(stream)))


# ---------------------------------------------------------------------------
# TGV2 / TV-L1 (device tensors)
# ---------------------------------------------------------------------------

TGV2_ITER_AUTO, TGV2_ITER_LAUNCH, TGV2_ITER_PERSISTENT = 0, 1, 2


TGV2_STOP_WINDOW_DEFAULT = 5


def tgv2_params(niters=30, warps=15, lam=0.5, alpha0=2.0, alpha1=1.5, tau=0.02, sigma=1.0, beta=0.0, gamma=1.0,
                tol=0.0, check_every=10, max_iters=0, iteration_kernel=TGV2_ITER_AUTO,
                stop_window=TGV2_STOP_WINDOW_DEFAULT):
    """mvs_tgv2_params.  With tol > 0 the run stops at the first energy check
    j >= stop_window where |E_j - E_{j-W}| <= tol * W * |E_{j-W}| (W =
    stop_window; checks every check_every iterations of a linearisation)."""
    return TGV2Params(niters, warps, lam, alpha0, alpha1, tau, sigma, beta, gamma, tol, check_every, max_iters,
                      iteration_kernel, stop_window)


def float_cams(K_1based, rel_poses):
    """The reference's float K, K^-1 (cofactor form) and float relative poses."""
    from . import hostmath
    K = np.asarray(K_1based, np.float32).reshape(3, 3)
    invK = hostmath.inv3_f32(K)
    Rs = np.stack([np.asarray(p[0], np.float32).reshape(9) for p in rel_poses])
    ts = np.stack([np.asarray(p[1], np.float32).reshape(3) for p in rel_poses])
    return K.reshape(9).copy(), invK.reshape(9).copy(), Rs, ts


def tgv2_run(ref255, srcs255, K9, invK9, Rrel, trel, params, u, u_from_input=False, u_init=1.0, workspace=None,
             stream=None):
    h, w = ref255.shape[-2:]
    V = srcs255.shape[0]
    it = C.c_int32(0)
    e = C.c_double(0)
    ws_bytes = 0 if workspace is None else workspace.numel() * workspace.element_size()
    K9, invK9, Rrel, trel = (_f32(x) for x in (K9, invK9, Rrel, trel))
    check(_L.mvs_tgv2_run(w, h, V, _ptr(ref255), _ptr(srcs255), _fp(K9), _fp(invK9), _fp(Rrel), _fp(trel),
                          C.byref(params), int(u_from_input), u_init, _ptr(u), C.byref(it), C.byref(e),
                          _ptr(workspace), ws_bytes, _stream(stream)))
    return it.value, e.value


def tgv2_run_warm(ref255, srcs255, K9, invK9, Rrel, trel, params, u_lin, u, v=None, dual_sigma=0.0,
                  dual_sigma_r=0.0, pq=None, r=None, workspace=None, stream=None):
    """TGV2 linearised at ``u_lin`` with the primal started at ``u`` (in/out)
    and ``v`` ((2, H, W), in/out, or None for 0); optional dual state ``pq``
    ((5, H, W)) and ``r`` ((V, H, W)), in/out.  Returns (iterations, final
    energy)."""
    h, w = ref255.shape[-2:]
    V = srcs255.shape[0]
    it = C.c_int32(0)
    e = C.c_double(0)
    ws_bytes = 0 if workspace is None else workspace.numel() * workspace.element_size()
    K9, invK9, Rrel, trel = (_f32(x) for x in (K9, invK9, Rrel, trel))
    check(_L.mvs_tgv2_run_warm(w, h, V, _ptr(ref255), _ptr(srcs255), _fp(K9), _fp(invK9), _fp(Rrel), _fp(trel),
                               C.byref(params), _ptr(u_lin), _ptr(u), _ptr(v), float(dual_sigma),
                               float(dual_sigma_r), _ptr(pq), _ptr(r), C.byref(it),
                               C.byref(e), _ptr(workspace), ws_bytes, _stream(stream)))
    return it.value, e.value


def render_scene(scene_desc, invK, R, center, width, height, gray255, depth, stream=None):
    """Ray cast one view of a box scene on the device (see scenes.GpuRenderer)."""
    invK, R, center = (np.ascontiguousarray(a, dtype=np.float64) for a in (invK, R, center))
    check(_L.mvs_render_scene(C.byref(scene_desc), invK.ctypes.data_as(_D), R.ctypes.data_as(_D),
                              center.ctypes.data_as(_D), width, height, _ptr(gray255), _ptr(depth),
                              _stream(stream)))


def tgv2_workspace_bytes(w, h, V):
    return int(_L.mvs_tgv2_workspace_bytes(w, h, V))


def tgv2_sparse_workspace_bytes(w, h):
    return int(_L.mvs_tgv2_sparse_workspace_bytes(w, h))


def tgv2_sparse(ref255, depthmap, sparse, zfar, out, workspace, niters, alpha0=2.0, alpha1=1.5, tau=0.02, sigma=1.0,
                theta=1.0, beta=0.0, gamma=1.0, stream=None):
    """TGV2 from ``depthmap`` towards ``sparse`` (0 = no sample), all device
    float32 H x W; ``out`` receives the result (PlaneSweep::TGVdenoiseFromSparse,
    planesweep.cpp:596-674)."""
    h, w = depthmap.shape[-2:]
    check(_L.mvs_tgv2_sparse(w, h, _ptr(ref255), _ptr(depthmap), _ptr(sparse), zfar, niters, alpha0, alpha1, tau,
                             sigma, theta, beta, gamma, _ptr(out), _ptr(workspace),
                             workspace.numel() * workspace.element_size(), _stream(stream)))


def tvl1_params(niters=100, lam=0.3, tau=0.02, sigma=6.0, theta=1.0, beta=0.0, gamma=1.0):
    return TVL1Params(niters, lam, tau, sigma, theta, beta, gamma)


def tvl1_workspace_bytes(w, h):
    return int(_L.mvs_tvl1_workspace_bytes(w, h))


def tvl1_denoise(ref255, depth, znear, zfar, params, workspace, stream=None):
    h, w = depth.shape[-2:]
    check(_L.mvs_tvl1_denoise(w, h, _ptr(ref255), _ptr(depth), znear, zfar, C.byref(params), _ptr(workspace),
                              workspace.numel() * workspace.element_size(), _stream(stream)))


def compute3d(depth, invK9, Rr9, t3, X, Y, Z, stream=None):
    h, w = depth.shape[-2:]
    invK9, Rr9, t3 = (_f32(x) for x in (invK9, Rr9, t3))
    check(_L.mvs_compute3d(w, h, _ptr(depth), _fp(invK9), _fp(Rr9), _fp(t3), _ptr(X), _ptr(Y), _ptr(Z),
                           _stream(stream)))


# ---------------------------------------------------------------------------
# data formats
# ---------------------------------------------------------------------------

def read_icl_camera(path, width=640, height=480):
    """(K (1-based, float32 3x3), R (camera->world, 3x3), t (3)) of an ICL-NUIM camera file."""
    K = np.zeros(9, np.float32)
    R = np.zeros(9, np.float32)
    t = np.zeros(3, np.float32)
    check(_L.mvs_read_icl_camera(str(path).encode(), width, height, _fp(K), _fp(R), _fp(t)))
    return K.reshape(3, 3), R.reshape(3, 3), t


def write_ply(path, xyz, rgb=None, binary=False):
    xyz = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
    c = None
    if rgb is not None:
        rgb = np.ascontiguousarray(rgb, np.uint8).reshape(-1, 3)
        assert len(rgb) == len(xyz)
        c = rgb.ctypes.data_as(C.POINTER(C.c_uint8))
    check(_L.mvs_write_ply(str(path).encode(), _fp(xyz), c, len(xyz), int(binary)))


def depth_color(gray):
    g = np.ascontiguousarray(gray, np.uint8).reshape(-1)
    out = np.empty((g.size, 3), np.uint8)
    _L.mvs_depth_color(g.ctypes.data_as(C.POINTER(C.c_uint8)), g.size, out.ctypes.data_as(C.POINTER(C.c_uint8)))
    return out


# ---------------------------------------------------------------------------
# batched frames
# ---------------------------------------------------------------------------

BATCH_ORDER_FRAME, BATCH_ORDER_LARGEST_FIRST, BATCH_ORDER_INTERLEAVED = 0, 1, 2


class Batch:
    """Handle on mvs_batch: many frames swept (aggregated mode) in one graph launch.

    ``frames``: dicts with ``ref`` (H, W), ``srcs`` (V, H, W), ``depths`` (P)
    CUDA float32 tensors, ``K1`` (3x3, 1-based), ``rel`` (list of (R, t) per
    view), ``window``, ``zfar``, optional ``std_threshold`` and the output
    tensors ``depth`` (H, W) and optional ``labels`` (int32) / ``best``.
    ``tuning``: None (autotune) or (planes_per_chunk, ctas_per_sm, order[, tile_step])."""

    def __init__(self, frames, moments=MOMENTS_COMPENSATED, tuning=None):
        descs = (BatchFrameDesc * len(frames))()
        keep = []
        for d, f in zip(descs, frames):
            H, W = f["ref"].shape
            V = f["srcs"].shape[0]
            K = np.ascontiguousarray(f["K1"], np.float64).reshape(9)
            R = np.ascontiguousarray(np.stack([np.asarray(r, np.float64).reshape(9) for r, _ in f["rel"]]))
            t = np.ascontiguousarray(np.stack([np.asarray(tt, np.float64).reshape(3) for _, tt in f["rel"]]))
            keep += [K, R, t]
            d.width, d.height, d.n_views, d.n_planes, d.window = W, H, V, f["depths"].numel(), f["window"]
            d.std_threshold = f.get("std_threshold", 1e-4)
            d.zfar = f["zfar"]
            d.d_ref, d.d_srcs, d.d_depths = (x.data_ptr() for x in (f["ref"], f["srcs"], f["depths"]))
            d.h_K9, d.h_Rrel, d.h_trel = (a.ctypes.data_as(_D) for a in (K, R, t))
            d.d_depth = f["depth"].data_ptr()
            d.d_labels = f["labels"].data_ptr() if f.get("labels") is not None else None
            d.d_best = f["best"].data_ptr() if f.get("best") is not None else None
        tn = None
        if tuning is not None:
            tn = BatchTuning(*tuning)
        h = _VP()
        check(_L.mvs_batch_create(C.byref(h), descs, len(frames), moments, None if tn is None else C.byref(tn)))
        self._h = h
        self.n = len(frames)

    def close(self):
        if getattr(self, "_h", None) and _L._cdll is not None:
            _L.mvs_batch_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()

    @property
    def tuning(self):
        t = BatchTuning()
        check(_L.mvs_batch_get_tuning(self._h, C.byref(t)))
        return (t.planes_per_chunk, t.ctas_per_sm, t.order, t.tile_step)

    @property
    def work_items(self):
        return int(_L.mvs_batch_work_items(self._h))

    def run(self, stream=None):
        check(_L.mvs_batch_run(self._h, _stream(stream)))

    def latencies_ms(self, stream=None):
        out = np.empty(self.n, np.float32)
        check(_L.mvs_batch_frame_latency_ms(self._h, out.ctypes.data_as(_F), _stream(stream)))
        return out


# ---------------------------------------------------------------------------
# TGV2 warm-start network
# ---------------------------------------------------------------------------

UNET_LAYERS = ((16, 16), (16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (64, 128), (128, 128),
               (192, 64), (64, 64), (96, 32), (32, 32), (48, 16), (16, 16))
UNET_DEFAULT_NORM = (0.25, -1.0, 2.0, 1.0, 0.01, 1.0, 1.0)


class Unet:
    """Handle on mvs_unet: forward, backward, Adam, parameters (FP32 host arrays)."""

    def __init__(self, batch, height, width, norm=UNET_DEFAULT_NORM):
        self.batch, self.height, self.width = batch, height, width
        self.norm = tuple(float(x) for x in norm)
        nm = np.asarray(self.norm, np.float32)
        h = _VP()
        check(_L.mvs_unet_create(C.byref(h), batch, height, width, nm.ctypes.data_as(_F)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and _L._cdll is not None:
            _L.mvs_unet_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()

    @property
    def n_params(self):
        return int(_L.mvs_unet_param_count(self._h))

    def layer_info(self, layer):
        ci, co = C.c_int32(), C.c_int32()
        wo, bo = C.c_int64(), C.c_int64()
        check(_L.mvs_unet_layer_info(self._h, layer, C.byref(ci), C.byref(co), C.byref(wo), C.byref(bo)))
        return ci.value, co.value, wo.value, bo.value

    def init_params(self, seed=0):
        """He-normal 3x3 weights (input channels beyond the 3 features of the
        first layer at zero), zero biases, a small random head."""
        rng = np.random.default_rng(seed)
        p = np.zeros(self.n_params, np.float32)
        for l in range(len(UNET_LAYERS)):
            ci, co, wo, bo = self.layer_info(l)
            fan = 9 * (3 if l == 0 else ci)
            w = rng.standard_normal((co, ci, 9)) * math.sqrt(2.0 / fan)
            if l == 0:
                w[:, 3:, :] = 0.0
            p[wo:wo + co * ci * 9] = w.reshape(-1)
        ci, co, wo, bo = self.layer_info(len(UNET_LAYERS))
        p[wo:wo + 48] = rng.standard_normal(48) * 0.01
        self.set_params(p)
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.n_params
        check(_L.mvs_unet_set_params(self._h, p.ctypes.data_as(_F)))

    def get_params(self, grads=False):
        p = np.empty(self.n_params, np.float32)
        g = np.empty(self.n_params, np.float32) if grads else None
        check(_L.mvs_unet_get_params(self._h, p.ctypes.data_as(_F), None if g is None else g.ctypes.data_as(_F)))
        return (p, g) if grads else p

    def forward(self, wta, cost, ref255, u_out=None, v_out=None, stream=None):
        check(_L.mvs_unet_forward(self._h, _ptr(wta), _ptr(cost), _ptr(ref255), _ptr(u_out), _ptr(v_out),
                                  _stream(stream)))

    def backward(self, u_target, v_target, stream=None):
        loss = C.c_double(0)
        check(_L.mvs_unet_backward(self._h, _ptr(u_target), _ptr(v_target), C.byref(loss), _stream(stream)))
        return loss.value

    def adam_step(self, lr, beta1=0.9, beta2=0.999, eps=1e-8, stream=None):
        check(_L.mvs_unet_adam_step(self._h, lr, beta1, beta2, eps, _stream(stream)))

    def train_step(self, wta, cost, ref255, u_target, v_target, lr, stream=None):
        loss = C.c_double(0)
        check(_L.mvs_unet_train_step(self._h, _ptr(wta), _ptr(cost), _ptr(ref255), _ptr(u_target), _ptr(v_target),
                                     lr, C.byref(loss), _stream(stream)))
        return loss.value

    def check(self, stream=None):
        check(_L.mvs_unet_check(self._h, _stream(stream)))


def conv3x3_forward(x, w, bias, relu, out, wpack, err, stream=None):
    """x (B, H, W, cin) bf16, w (cout, cin, 3, 3) float32 CUDA tensors."""
    B, H, W, cin = x.shape
    cout = w.shape[0]
    check(_L.mvs_conv3x3_forward(_ptr(x), cin, _ptr(w), _ptr(bias), cout, B, H, W, int(relu), _ptr(out), _ptr(wpack),
                                 _ptr(err), _stream(stream)))


def conv3x3_backward(x, w, dz, mask_x, dx, dw, db, wpack, err, tensor_cores=True, stream=None):
    B, H, W, cin = x.shape
    cout = w.shape[0]
    check(_L.mvs_conv3x3_backward(_ptr(x), cin, _ptr(w), _ptr(dz), cout, B, H, W, int(mask_x), _ptr(dx), _ptr(dw),
                                  _ptr(db), _ptr(wpack), _ptr(err), int(tensor_cores), _stream(stream)))


# ---------------------------------------------------------------------------
# fusion
# ---------------------------------------------------------------------------

class FusionVolume:
    """TV-L1 histogram fusion volume: dims = (width, height, depth) voxels."""

    def __init__(self, dims, bins, corner_a, corner_b):
        self.dims = tuple(int(d) for d in dims)
        self.bins = int(bins)
        self.n = self.dims[0] * self.dims[1] * self.dims[2]
        h = _VP()
        check(_L.mvs_fusion_create(*self.dims, self.bins, _fp(_f32(corner_a)), _fp(_f32(corner_b)), C.byref(h)))
        self.h = h

    def close(self):
        # _L is None once the interpreter is tearing the module down
        if getattr(self, "h", None) and self.h.value and _L is not None:
            _L.mvs_fusion_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()

    def reset(self, stream=None):
        check(_L.mvs_fusion_reset(self.h, _stream(stream)))

    def set_volume(self, a, b):
        check(_L.mvs_fusion_set_volume(self.h, _fp(_f32(a)), _fp(_f32(b))))

    def histogram(self, depths, Ks, Rs, ts, threshold, stream=None):
        """depths: CUDA tensor (M, H, W); Ks/Rs: (M,3,3); ts: (M,3) (world->camera, 0-based K)."""
        M, h, w = depths.shape
        K = _f32(np.asarray(Ks).reshape(M, 9))
        R = _f32(np.asarray(Rs).reshape(M, 9))
        t = _f32(np.asarray(ts).reshape(M, 3))
        check(_L.mvs_fusion_histogram(self.h, _ptr(depths), M, w, h, _fp(K), _fp(R), _fp(t), threshold,
                                      _stream(stream)))

    def tvl1(self, iters, tau, lam, sigma, stream=None):
        check(_L.mvs_fusion_tvl1(self.h, iters, tau, lam, sigma, _stream(stream)))

    def update_u(self, tau, lam, stream=None):
        check(_L.mvs_fusion_update_u(self.h, tau, lam, _stream(stream)))

    def update_p(self, sigma, stream=None):
        check(_L.mvs_fusion_update_p(self.h, sigma, _stream(stream)))

    def iteration(self, depth, K, R, t, threshold, tau, lam, sigma, stream=None, shape=None):
        """One FusionUpdateIteration: ``depth`` a CUDA tensor (H, W), or a raw
        device pointer (int, e.g. PlaneSweep.getDepthmapDenoisedPtr()) with
        ``shape`` = (H, W)."""
        if isinstance(depth, int):
            h, w = shape
            dp = C.c_void_p(depth)
        else:
            h, w = depth.shape[-2:]
            dp = _ptr(depth)
        check(_L.mvs_fusion_iteration(self.h, dp, w, h, _fp(_f32(K)), _fp(_f32(R)), _fp(_f32(t)), threshold,
                                      tau, lam, sigma, _stream(stream)))

    def download(self):
        u, v = np.zeros(self.n, np.float32), np.zeros(self.n, np.float32)
        p = np.zeros((3, self.n), np.float32)
        hist = np.zeros((self.bins, self.n), np.uint16)
        check(_L.mvs_fusion_download(self.h, _fp(u), _fp(v), _fp(p), hist.ctypes.data_as(_U16)))
        return dict(u=u, v=v, p=p, hist=hist)

    def upload(self, u=None, v=None, p=None, hist=None):
        hp = None if hist is None else np.ascontiguousarray(hist, np.uint16).ctypes.data_as(_U16)
        check(_L.mvs_fusion_upload(self.h, _fp(None if u is None else _f32(u)), _fp(None if v is None else _f32(v)),
                                   _fp(None if p is None else _f32(p)), hp))

    def device_state(self):
        u, v, p, hist = _VP(), _VP(), _VP(), _VP()
        hs = C.c_int32(0)
        check(_L.mvs_fusion_device_state(self.h, C.byref(u), C.byref(v), C.byref(p), C.byref(hist), C.byref(hs)))
        return dict(u=u.value, v=v.value, p=p.value, hist=hist.value, hist_stride=hs.value)

    def extract(self, lo=-1.0, hi=0.0, capacity=None):
        cnt = C.c_int64(0)
        check(_L.mvs_fusion_extract(self.h, lo, hi, None, 0, C.byref(cnt)))
        n = cnt.value if capacity is None else min(cnt.value, capacity)
        out = np.zeros((n, 3), np.float32)
        if n:
            check(_L.mvs_fusion_extract(self.h, lo, hi, _fp(out), n, C.byref(cnt)))
        return out


# ---------------------------------------------------------------------------
# PlaneSweep (host buffers, the reference's class API)
# ---------------------------------------------------------------------------

class PlaneSweep:
    """The reference's PlaneSweep (planesweep.h:27-510) over the mvs_ps_* C handle.

    Images are host float32 arrays (0..255 grey); poses world->camera."""

    def __init__(self):
        h = _VP()
        check(_L.mvs_ps_create(C.byref(h)))
        self.h = h
        self.shape = None
        self.n_views = 0

    def close(self):
        # _L is None once the interpreter is tearing the module down
        if getattr(self, "h", None) and self.h.value and _L is not None:
            _L.mvs_ps_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()

    def set_reference(self, img, R, t):
        img = _f32(img)
        self.shape = img.shape
        check(_L.mvs_ps_set_reference(self.h, _fp(img), img.shape[1], img.shape[0], _fp(_f32(R)), _fp(_f32(t))))

    def set_sources(self, imgs, Rs, ts):
        imgs = _f32(np.stack(imgs)) if isinstance(imgs, (list, tuple)) else _f32(imgs)
        self.n_views = imgs.shape[0]
        Rs = _f32(Rs if isinstance(Rs, np.ndarray) else np.stack(Rs))
        ts = _f32(ts if isinstance(ts, np.ndarray) else np.stack(ts))
        check(_L.mvs_ps_set_sources(self.h, _fp(imgs), imgs.shape[0], _fp(Rs), _fp(ts)))

    def setK(self, K):
        check(_L.mvs_ps_set_K(self.h, _fp(_f32(K))))

    def setZ(self, n, f):
        check(_L.mvs_ps_set_z(self.h, n, f))

    def setNumberofPlanes(self, n):
        check(_L.mvs_ps_set_number_of_planes(self.h, n))

    def setNumberofImages(self, n):
        check(_L.mvs_ps_set_number_of_images(self.h, n))

    def setWindowSize(self, n):
        check(_L.mvs_ps_set_window_size(self.h, n))

    def setSTDthreshold(self, t):
        check(_L.mvs_ps_set_std_threshold(self.h, t))

    def setNCCthreshold(self, t):
        check(_L.mvs_ps_set_ncc_threshold(self.h, t))

    def setAlternativeRelativeMatrixMethod(self, alt):
        check(_L.mvs_ps_set_alternative_relative_matrix_method(self.h, int(bool(alt))))

    def setPlaneDepths(self, depths):
        d = None if depths is None else _f32(depths)
        check(_L.mvs_ps_set_plane_depths(self.h, _fp(d), 0 if d is None else len(d)))

    def setSweepOptions(self, moments=MOMENTS_REFERENCE, mode=SWEEP_PER_VIEW, fp64_homographies=True):
        check(_L.mvs_ps_set_sweep_options(self.h, moments, mode, int(bool(fp64_homographies))))

    def RunAlgorithm(self):
        check(_L.mvs_ps_run_algorithm(self.h))

    def CudaDenoise(self, niters=100, lam=0.3, tau=0.02, sigma=6.0, theta=1.0, beta=0.0, gamma=1.0):
        check(_L.mvs_ps_cuda_denoise(self.h, niters, lam, tau, sigma, theta, beta, gamma))

    def TGV(self, niters=30, warps=15, lam=0.5, alpha0=2.0, alpha1=1.5, tau=0.02, sigma=1.0, beta=0.0, gamma=1.0):
        check(_L.mvs_ps_tgv(self.h, niters, warps, lam, alpha0, alpha1, tau, sigma, beta, gamma))

    def TGVdenoiseFromSparse(self, depth, niters, alpha0=2.0, alpha1=1.5, tau=0.02, sigma=1.0, theta=1.0, beta=0.0,
                             gamma=1.0):
        sp = _f32(depth)
        if sp.shape != self.shape:
            raise ValueError(f"sparse depthmap shape {sp.shape} != {self.shape}")
        check(_L.mvs_ps_tgv_denoise_from_sparse(self.h, _fp(sp), niters, alpha0, alpha1, tau, sigma, theta, beta,
                                                gamma))

    def TGVext(self, params, start=1, u_init=None):
        it = C.c_int32(0)
        e = C.c_double(0)
        ui = None if u_init is None else _f32(u_init)
        check(_L.mvs_ps_tgv_ext(self.h, C.byref(params), start, _fp(ui), C.byref(it), C.byref(e)))
        return it.value, e.value

    def _img(self, name, dtype=np.float32, out=None):
        # every element is written: the library refuses a map of another size.
        # `out`: a C-contiguous array of the frame's shape and type to fill (a
        # caller that keeps one avoids a fresh allocation per frame)
        if out is None:
            out = np.empty(self.shape, dtype)
        elif out.dtype != dtype or out.shape != tuple(self.shape) or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous {np.dtype(dtype).name} array of shape {tuple(self.shape)}")
        ptr = out.ctypes.data_as(_F if dtype == np.float32 else _U8)
        check(getattr(_L, f"mvs_ps_get_{name}")(self.h, ptr))
        return out

    def getDepthmap(self, out=None):
        return self._img("depthmap", out=out)

    def getDepthmap8u(self, out=None):
        return self._img("depthmap8u", np.uint8, out)

    def getDepthmapDenoised(self, out=None):
        return self._img("depthmap_denoised", out=out)

    def getDepthmap8uDenoised(self, out=None):
        return self._img("depthmap8u_denoised", np.uint8, out)

    def getDepthmapTGV(self, out=None):
        return self._img("depthmap_tgv", out=out)

    def getDepthmap8uTGV(self, out=None):
        return self._img("depthmap8u_tgv", np.uint8, out)

    def getDepthmapDenoisedPtr(self):
        p = _VP()
        check(_L.mvs_ps_get_depthmap_denoised_ptr(self.h, C.byref(p)))
        return p.value

    def getViewLabels(self):
        out = np.zeros((self.n_views,) + tuple(self.shape), np.int32)
        check(_L.mvs_ps_get_view_labels(self.h, out.ctypes.data_as(_I32)))
        return out

    def getViewBest(self):
        out = np.zeros((self.n_views,) + tuple(self.shape), np.float32)
        check(_L.mvs_ps_get_view_best(self.h, _fp(out)))
        return out

    def get3Dcoordinates(self):
        X, Y, Z = (np.zeros(self.shape, np.float32) for _ in range(3))
        check(_L.mvs_ps_get_3d_coordinates(self.h, _fp(X), _fp(Y), _fp(Z)))
        return X, Y, Z

    def getPlaneCount(self):
        n = C.c_int32(0)
        check(_L.mvs_ps_get_plane_count(self.h, C.byref(n)))
        return n.value

    def getLastKernelMs(self):
        ms = C.c_float(0)
        check(_L.mvs_ps_get_last_kernel_ms(self.h, C.byref(ms)))
        return ms.value
