"""ctypes bindings for the CPU oracle and the reference-on-CPU library.

TEST INFRASTRUCTURE ONLY: imported by tests/, the fixture generator,
``__graft_entry__.smoke()`` and the CPU-baseline legs of bench.py, always as
the checker.  The product path never imports this module.

Two libraries, both built by ``make -C oracle``:

* ``_ref/libmvs_oracle.so`` -- the C restatement (mvs_oracle.c), f32 and f64;
* ``_ref/libmvs_ref.so``    -- the reference's own kernels compiled for the
  CPU (only when the reference tree was present at build time).
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
_F = C.POINTER(C.c_float)
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int32)
_U16 = C.POINTER(C.c_uint16)


def _fp(a):
    return None if a is None else a.ctypes.data_as(_F)


def _dp(a):
    return None if a is None else a.ctypes.data_as(_D)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


_oracle = None
_ref = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        path = HERE / "_ref" / "libmvs_oracle.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} missing: run `make -C oracle oracle`")
        _oracle = C.CDLL(str(path))
        _declare_oracle(_oracle)
    return _oracle


def ref_lib():
    """The reference compiled for the CPU, or None if it was not built."""
    global _ref
    if _ref is None:
        path = HERE / "_ref" / "libmvs_ref.so"
        if not path.exists():
            return None
        _ref = C.CDLL(str(path))
        _declare_ref(_ref)
    return _ref


def _declare_oracle(L):
    for S, T in (("f32", C.c_float), ("f64", C.c_double)):
        P = C.POINTER(T)
        getattr(L, f"orc_inv3_{S}").argtypes = [P, P]
        getattr(L, f"orc_relative_{S}").argtypes = [P, P, P, P, C.c_int, P, P]
        getattr(L, f"orc_homography_{S}").argtypes = [P, P, P, P, T, P]
        getattr(L, f"orc_sweep_view_{S}").argtypes = [C.c_int, C.c_int, _F, _F, P, _F, C.c_int, C.c_int,
                                                      C.c_double, P, P, _I]
        getattr(L, f"orc_sweep_ncc_{S}").argtypes = [C.c_int, C.c_int, _F, _F, P, C.c_int, C.c_double, P]
        getattr(L, f"orc_sweep_ncc_band_{S}").argtypes = [C.c_int, C.c_int, C.c_int, _F, _F, P, C.c_int, C.c_int,
                                                          C.c_double, C.c_int, C.c_int, P]
        getattr(L, f"orc_sweep_combine_{S}").argtypes = [C.c_int, C.c_int, C.c_int, P, P, C.c_double,
                                                         C.c_double, P]
        getattr(L, f"orc_tensor_{S}").argtypes = [C.c_int, C.c_int, P, C.c_double, C.c_double, P, P, P, P]
        getattr(L, f"orc_tgv2_linearize_{S}").argtypes = [C.c_int, C.c_int, P, P, P, P, P, P, P, P, P]
        getattr(L, f"orc_tgv2_iteration_{S}").argtypes = ([C.c_int] * 3 + [P] * 21 + [C.c_double] * 5)
        getattr(L, f"orc_tgv2_energy_{S}").argtypes = [C.c_int] * 3 + [P] * 10 + [C.c_double] * 3
        getattr(L, f"orc_tgv2_energy_{S}").restype = C.c_double
        getattr(L, f"orc_tgv_sparse_iteration_{S}").argtypes = [C.c_int] * 2 + [P] * 15 + [C.c_double] * 4
        getattr(L, f"orc_tvl1_denoise_{S}").argtypes = ([C.c_int, C.c_int, P, P, C.c_double, C.c_double, C.c_int]
                                                        + [C.c_double] * 6 + [P])
        getattr(L, f"orc_fusion_histogram_{S}").argtypes = [C.c_int] * 4 + [_F, _F, _U16, _F, C.c_int, C.c_int,
                                                                            P, P, P, C.c_double]
        getattr(L, f"orc_fusion_u_{S}").argtypes = [C.c_int] * 4 + [_U16, P, P, P, C.c_double, C.c_double]
        getattr(L, f"orc_fusion_p_{S}").argtypes = [C.c_int] * 3 + [P, P, C.c_double]
        getattr(L, f"orc_compute3d_{S}").argtypes = [C.c_int, C.c_int, P, P, P, P, P, P, P]
    L.orc_bin_centers.argtypes = [C.c_int, _F]
    L.orc_prox_hist_f32.argtypes = [C.c_int, _U16, C.c_float, C.c_float, C.c_float]
    L.orc_prox_hist_f32.restype = C.c_float
    L.orc_plane_list.argtypes = [C.c_float, C.c_float, C.c_int, _F, C.c_int]
    L.orc_plane_list.restype = C.c_int


def _declare_ref(L):
    L.ref_tgv_sparse.restype = C.c_double
    L.ref_tgv_sparse.argtypes = [C.c_int, C.c_int, _F, _F, _F, C.c_float, C.c_int] + [C.c_double] * 7 + [_F]
    L.ref_sweep.argtypes = [C.c_int, C.c_int, _F, _F, C.c_int, _F, _F, _F, _F, _F, C.c_int, _F, C.c_int,
                            C.c_float, C.c_float, C.c_int, C.c_float, C.c_float, _F, _F, _F]
    L.ref_sweep.restype = C.c_double
    L.ref_plane_list.argtypes = [C.c_float, C.c_float, C.c_int, _F, C.c_int]
    L.ref_plane_list.restype = C.c_int
    L.ref_homography.argtypes = [_F, _F, _F, _F, _F, C.c_int, C.c_float, _F]
    L.ref_tgv.argtypes = ([C.c_int, C.c_int, _F, _F, C.c_int, _F, _F, _F, _F, _F, C.c_int, C.c_int, C.c_int]
                          + [C.c_double] * 7 + [_F, _F])
    L.ref_tgv.restype = C.c_double
    L.ref_tvl1_denoise.argtypes = ([C.c_int, C.c_int, _F, _F, C.c_float, C.c_float, C.c_int]
                                   + [C.c_double] * 6 + [_F])
    L.ref_tvl1_denoise.restype = C.c_double
    L.ref_compute3d.argtypes = [C.c_int, C.c_int, _F, _F, _F, _F, C.c_int, _F, _F, _F]
    L.ref_fusion_create.argtypes = [C.c_int] * 4 + [_F, _F]
    L.ref_fusion_create.restype = C.c_void_p
    L.ref_fusion_destroy.argtypes = [C.c_void_p]
    L.ref_fusion_histogram.argtypes = [C.c_void_p, _F, C.c_int, C.c_int, _F, _F, _F, C.c_float]
    L.ref_fusion_histogram.restype = C.c_double
    L.ref_fusion_u.argtypes = [C.c_void_p, C.c_double, C.c_double]
    L.ref_fusion_u.restype = C.c_double
    L.ref_fusion_p.argtypes = [C.c_void_p, C.c_double]
    L.ref_fusion_p.restype = C.c_double
    L.ref_fusion_get.argtypes = [C.c_void_p, _F, _F, _F, _U16]
    L.ref_fusion_set.argtypes = [C.c_void_p, _F, _F, _F, _U16]
    L.ref_fusion_bin_centers.argtypes = [C.c_int, _F]


# ---------------------------------------------------------------------------
# cameras
# ---------------------------------------------------------------------------

def _mat(dt, m):
    return np.ascontiguousarray(np.asarray(m).reshape(-1), dtype=dt)


def relative(Rref, tref, Rsrc, tsrc, alternative=False, precision="f64"):
    dt = np.float32 if precision == "f32" else np.float64
    L = oracle_lib()
    P = _fp if precision == "f32" else _dp
    Rrel, trel = np.zeros(9, dt), np.zeros(3, dt)
    args = [_mat(dt, Rref), _mat(dt, tref), _mat(dt, Rsrc), _mat(dt, tsrc)]
    getattr(L, f"orc_relative_{precision}")(*[P(a) for a in args], int(alternative), P(Rrel), P(trel))
    return Rrel, trel


def homographies(K_1based, Rref, tref, src_poses, depths, alternative=False, precision="f64"):
    """(nsrc, nplanes, 9) homographies built as PlaneSweepThread builds them."""
    dt = np.float32 if precision == "f32" else np.float64
    L = oracle_lib()
    P = _fp if precision == "f32" else _dp
    K = _mat(dt, K_1based)
    invK = np.zeros(9, dt)
    getattr(L, f"orc_inv3_{precision}")(P(K), P(invK))
    out = np.zeros((len(src_poses), len(depths), 9), dt)
    fn = getattr(L, f"orc_homography_{precision}")
    for v, (Rs, ts) in enumerate(src_poses):
        Rrel, trel = relative(Rref, tref, Rs, ts, alternative, precision)
        for p, d in enumerate(depths):
            H = np.zeros(9, dt)
            fn(P(K), P(invK), P(Rrel), P(trel), dt(d), P(H))
            out[v, p] = H
    return out


# ---------------------------------------------------------------------------
# plane sweep
# ---------------------------------------------------------------------------

def sweep(ref, srcs, H, depths, winsize, stdthresh=1e-4, nccthresh=0.5, zfar=1.0, precision="f64"):
    """Per-view argmax plus the cross-view average, as RunAlgorithm computes it.

    Returns dict(depth, best (V,H,W), vdepth (V,H,W), label (V,H,W) int32)."""
    L = oracle_lib()
    dt = np.float32 if precision == "f32" else np.float64
    P = _fp if precision == "f32" else _dp
    h, w = ref.shape
    V = len(srcs)
    ref = _f32(ref)
    depths = _f32(depths)
    best = np.zeros((V, h, w), dt)
    vdepth = np.zeros((V, h, w), dt)
    label = np.zeros((V, h, w), np.int32)
    fn = getattr(L, f"orc_sweep_view_{precision}")
    for v in range(V):
        Hv = np.ascontiguousarray(H[v], dtype=dt)
        fn(w, h, _fp(ref), _fp(_f32(srcs[v])), P(Hv), _fp(depths), len(depths), winsize, stdthresh,
           P(best[v]), P(vdepth[v]), label[v].ctypes.data_as(_I))
    out = np.zeros((h, w), dt)
    getattr(L, f"orc_sweep_combine_{precision}")(w, h, V, P(best), P(vdepth), nccthresh, zfar, P(out))
    return dict(depth=out, best=best, vdepth=vdepth, label=label)


def sweep_ncc_band(ref, srcs, H, winsize, y0, y1, stdthresh=1e-4, precision="f64"):
    """Sum over the source views of every plane's NCC on output rows [y0, y1):
    (nplanes, y1 - y0, W), as orc_sweep_ncc computes each view on the full
    frame.  H is (nviews, nplanes, 9)."""
    L = oracle_lib()
    dt = np.float32 if precision == "f32" else np.float64
    P = _fp if precision == "f32" else _dp
    h, w = ref.shape
    V, NP = H.shape[0], H.shape[1]
    out = np.zeros((NP, y1 - y0, w), dt)
    getattr(L, f"orc_sweep_ncc_band_{precision}")(w, h, V, _fp(_f32(ref)), _fp(_f32(np.stack(srcs))),
                                                  P(np.ascontiguousarray(H, dt)), NP, winsize, stdthresh, y0, y1,
                                                  P(out))
    return out


def ref_sweep(ref, srcs, K_1based, Rref, tref, src_poses, planes, winsize, znear=0.1, zfar=1.0,
              nplanes=None, stdthresh=1e-4, nccthresh=0.5, alternative=False):
    """The reference's own sweep on the CPU.  ``planes`` None -> its float loop."""
    L = ref_lib()
    if L is None:
        raise FileNotFoundError("oracle/_ref/libmvs_ref.so not built")
    h, w = ref.shape
    V = len(srcs)
    S = _f32(np.stack(srcs))
    Rs = _f32(np.stack([p[0] for p in src_poses]))
    ts = _f32(np.stack([p[1] for p in src_poses]))
    out = np.zeros((h, w), np.float32)
    best = np.zeros((V, h, w), np.float32)
    vdepth = np.zeros((V, h, w), np.float32)
    pl = None if planes is None else _f32(planes)
    n = len(planes) if planes is not None else int(nplanes)
    secs = L.ref_sweep(w, h, _fp(_f32(ref)), _fp(S), V, _fp(_f32(K_1based)), _fp(_f32(Rref)), _fp(_f32(tref)),
                       _fp(Rs), _fp(ts), int(alternative), _fp(pl), n, znear, zfar, winsize, stdthresh, nccthresh,
                       _fp(out), _fp(best), _fp(vdepth))
    return dict(depth=out, best=best, vdepth=vdepth, seconds=secs)


_ref_gpu = None


def ref_gpu_lib():
    """The reference's own CUDA kernels compiled for the B200, or None if not built."""
    global _ref_gpu
    if _ref_gpu is None:
        path = HERE / "_ref" / "libmvs_ref_gpu.so"
        if not path.exists():
            return None
        L = C.CDLL(str(path))
        P = _F
        L.ref_gpu_sweep.restype = C.c_double
        L.ref_gpu_sweep.argtypes = [C.c_int, C.c_int, P, P, C.c_int, P, P, P, P, P, C.c_int, P, C.c_int,
                                    C.c_float, C.c_float, C.c_int, C.c_float, C.c_float, P]
        L.ref_gpu_tgv.restype = C.c_double
        L.ref_gpu_tgv.argtypes = ([C.c_int, C.c_int, P, P, C.c_int, P, P, P, P, P, C.c_int, C.c_int, C.c_int] +
                                  [C.c_double] * 7 + [P, P])
        L.ref_gpu_tgv_sparse.restype = C.c_double
        L.ref_gpu_tgv_sparse.argtypes = [C.c_int, C.c_int, P, P, P, C.c_float, C.c_int] + [C.c_double] * 7 + [P]
        _ref_gpu = L
    return _ref_gpu


def ref_gpu_tgv_sparse(ref, depthmap, sparse, zfar, niters, alpha0=2.0, alpha1=1.5, tau=0.02, sigma=1.0, theta=1.0,
                       beta=0.0, gamma=1.0):
    """PlaneSweep::TGVdenoiseFromSparse's call sequence with the reference's
    own kernels on the GPU; returns (u, device ms)."""
    L = ref_gpu_lib()
    if L is None:
        raise FileNotFoundError("oracle/_ref/libmvs_ref_gpu.so not built")
    h, w = ref.shape
    out = np.zeros((h, w), np.float32)
    ms = L.ref_gpu_tgv_sparse(w, h, _fp(_f32(ref)), _fp(_f32(depthmap)), _fp(_f32(sparse)), float(zfar), niters,
                              alpha0, alpha1, tau, sigma, theta, beta, gamma, _fp(out))
    return out, ms


def ref_gpu_sweep(ref, srcs, K_1based, Rref, tref, src_poses, planes, winsize, zfar, stdthresh=1e-4,
                  nccthresh=0.5, alternative=False):
    """The reference's RunAlgorithm call sequence with its own kernels on the
    GPU; returns (depth, device ms of the compute)."""
    L = ref_gpu_lib()
    if L is None:
        raise FileNotFoundError("oracle/_ref/libmvs_ref_gpu.so not built")
    h, w = ref.shape
    V = len(srcs)
    S = _f32(np.stack(srcs))
    Rs = _f32(np.stack([p[0] for p in src_poses]))
    ts = _f32(np.stack([p[1] for p in src_poses]))
    out = np.zeros((h, w), np.float32)
    pl = _f32(planes)
    ms = L.ref_gpu_sweep(w, h, _fp(_f32(ref)), _fp(S), V, _fp(_f32(K_1based)), _fp(_f32(Rref)), _fp(_f32(tref)),
                         _fp(Rs), _fp(ts), int(alternative), _fp(pl), len(pl), float(pl[0]), float(zfar), winsize,
                         stdthresh, nccthresh, _fp(out))
    return out, ms


def ref_gpu_tgv(ref, srcs, K_1based, Rref, tref, src_poses, niters, warps, u_init=None, lam=0.5, alpha0=2.0,
                alpha1=1.5, tau=0.02, sigma=1.0, beta=0.0, gamma=1.0, alternative=False):
    """The reference's PlaneSweep::TGV call sequence with its own kernels on the
    GPU; returns (u, device ms of the iterations)."""
    L = ref_gpu_lib()
    if L is None:
        raise FileNotFoundError("oracle/_ref/libmvs_ref_gpu.so not built")
    h, w = ref.shape
    V = len(srcs)
    S = _f32(np.stack(srcs))
    Rs = _f32(np.stack([p[0] for p in src_poses]))
    ts = _f32(np.stack([p[1] for p in src_poses]))
    out = np.zeros((h, w), np.float32)
    ui = None if u_init is None else _f32(u_init)
    ms = L.ref_gpu_tgv(w, h, _fp(_f32(ref)), _fp(S), V, _fp(_f32(K_1based)), _fp(_f32(Rref)), _fp(_f32(tref)),
                       _fp(Rs), _fp(ts), int(alternative), niters, warps, lam, alpha0, alpha1, tau, sigma, beta,
                       gamma, _fp(ui), _fp(out))
    return out, ms


def ref_tgv_sparse(ref, depthmap, sparse, zfar, niters, alpha0=2.0, alpha1=1.5, tau=0.02, sigma=1.0, theta=1.0,
                   beta=0.0, gamma=1.0):
    """The reference's PlaneSweep::TGVdenoiseFromSparse on the CPU (its own kernels)."""
    L = ref_lib()
    if L is None:
        raise FileNotFoundError("oracle/_ref/libmvs_ref.so not built")
    h, w = ref.shape
    out = np.zeros((h, w), np.float32)
    L.ref_tgv_sparse(w, h, _fp(_f32(ref)), _fp(_f32(depthmap)), _fp(_f32(sparse)), float(zfar), niters, alpha0, alpha1,
                     tau, sigma, theta, beta, gamma, _fp(out))
    return out


def labels_from_depth(vdepth, planes):
    """Per-view plane index from the reference's stored depth (0 -> -1)."""
    planes = np.asarray(planes, np.float32)
    lab = np.full(vdepth.shape, -1, np.int32)
    for p, d in enumerate(planes):
        lab[(vdepth == d) & (lab < 0)] = p
    return lab


def plane_list(znear, zfar, n):
    L = oracle_lib()
    out = np.zeros(n + 4, np.float32)
    k = L.orc_plane_list(znear, zfar, n, _fp(out), len(out))
    return out[:k].copy()


# ---------------------------------------------------------------------------
# TGV2
# ---------------------------------------------------------------------------

def tensor(img01, beta=0.0, gamma=1.0, precision="f64"):
    L = oracle_lib()
    dt = np.float32 if precision == "f32" else np.float64
    P = _fp if precision == "f32" else _dp
    h, w = img01.shape
    img = np.ascontiguousarray(img01, dt)
    T = [np.zeros((h, w), dt) for _ in range(4)]
    getattr(L, f"orc_tensor_{precision}")(w, h, P(img), beta, gamma, *[P(t) for t in T])
    return T


class TGV2State:
    """Primal/dual state of the TGV2 iteration (names as in planesweep.cpp:404-411)."""

    FIELDS = ("u", "u1x", "u1y", "ubar", "u1xbar", "u1ybar", "Px", "Py", "Qx", "Qy", "Qz", "Qw", "prodsum")

    def __init__(self, h, w, V, dt):
        for f in self.FIELDS:
            setattr(self, f, np.zeros((h, w), dt))
        self.r = np.zeros((V, h, w), dt)
        self.u0 = np.zeros((h, w), dt)


def tgv2_setup(ref255, srcs255, K_1based, Rref, tref, src_poses, alternative=False, precision="f64"):
    dt = np.float32 if precision == "f32" else np.float64
    L = oracle_lib()
    P = _fp if precision == "f32" else _dp
    scale = np.float32(1.0 / 255.0) if precision == "f32" else 1.0 / 255.0
    ref01 = np.ascontiguousarray(np.asarray(ref255, dt) * scale, dt)
    src01 = [np.ascontiguousarray(np.asarray(s, dt) * scale, dt) for s in srcs255]
    K = _mat(dt, K_1based)
    invK = np.zeros(9, dt)
    getattr(L, f"orc_inv3_{precision}")(P(K), P(invK))
    rel = [relative(Rref, tref, Rs, ts, alternative, precision) for Rs, ts in src_poses]
    return dict(ref01=ref01, src01=src01, K=K, invK=invK, rel=rel, dt=dt, P=P)


def tgv2_linearize(setup, u0, precision="f64"):
    L = oracle_lib()
    P, dt = setup["P"], setup["dt"]
    h, w = u0.shape
    V = len(setup["src01"])
    It = np.zeros((V, h, w), dt)
    Iu = np.zeros((V, h, w), dt)
    u0 = np.ascontiguousarray(u0, dt)
    for v in range(V):
        Rrel, trel = setup["rel"][v]
        getattr(L, f"orc_tgv2_linearize_{precision}")(w, h, P(setup["src01"][v]), P(setup["ref01"]), P(u0),
                                                      P(setup["K"]), P(setup["invK"]), P(Rrel), P(trel),
                                                      P(It[v]), P(Iu[v]))
    return It, Iu


def tgv2(ref255, srcs255, K_1based, Rref, tref, src_poses, niters=30, warps=15, lam=0.5, alpha0=2.0,
         alpha1=1.5, tau=0.02, sigma=1.0, beta=0.0, gamma=1.0, u_init=None, alternative=False,
         precision="f64", tol=0.0, check_every=10, max_iters=None, stop_window=5):
    """PlaneSweep::TGV (planesweep.cpp:381-536) driven from Python over the C
    kernels.  With ``tol > 0`` the energy E_j is evaluated every
    ``check_every`` iterations of a linearisation and the run stops at the
    first check j >= W with |E_j - E_{j-W}| <= tol * W * |E_{j-W}|, W =
    ``stop_window`` (the stopping rule of mvs_tgv2_params); ``max_iters``
    caps the total count.

    Returns (u, iterations, energies)."""
    L = oracle_lib()
    st = tgv2_setup(ref255, srcs255, K_1based, Rref, tref, src_poses, alternative, precision)
    P, dt = st["P"], st["dt"]
    h, w = st["ref01"].shape
    V = len(srcs255)
    T = tensor(st["ref01"], beta, gamma, precision)
    S = TGV2State(h, w, V, dt)
    S.u[:] = 1.0 if u_init is None else u_init
    total, energies, done = 0, [], False
    cap = warps * niters if max_iters is None else max_iters
    it_fn = getattr(L, f"orc_tgv2_iteration_{precision}")
    en_fn = getattr(L, f"orc_tgv2_energy_{precision}")
    for _ in range(warps):
        if done:
            break
        S.u0[:] = S.u
        S.ubar[:] = S.u
        for f in ("Px", "Py", "Qx", "Qy", "Qz", "Qw", "u1x", "u1y", "u1xbar", "u1ybar"):
            getattr(S, f)[:] = 0
        S.r[:] = 0
        It, Iu = tgv2_linearize(st, S.u0, precision)
        hist = []
        for k in range(niters):
            it_fn(w, h, V, *[P(t) for t in T], P(It), P(Iu), P(S.u0), P(S.u), P(S.u1x), P(S.u1y), P(S.ubar),
                  P(S.u1xbar), P(S.u1ybar), P(S.Px), P(S.Py), P(S.Qx), P(S.Qy), P(S.Qz), P(S.Qw), P(S.r),
                  P(S.prodsum), lam, alpha0, alpha1, tau, sigma)
            total += 1
            if tol > 0 and (k + 1) % check_every == 0:
                E = en_fn(w, h, V, *[P(t) for t in T], P(It), P(Iu), P(S.u0), P(S.u), P(S.u1x), P(S.u1y),
                          lam, alpha0, alpha1)
                energies.append(E)
                hist.append(E)
                if len(hist) > stop_window and abs(hist[-1 - stop_window] - E) <= tol * stop_window * abs(
                        hist[-1 - stop_window]):
                    done = True
                    break
            if total >= cap:
                done = True
                break
    return S.u.copy(), total, energies


def tgv2_warm(ref255, srcs255, K_1based, Rref, tref, src_poses, u_lin, u_start, v_start, dual_sigma, dual_sigma_r,
              max_iters=500, lam=0.5, alpha0=2.0, alpha1=1.5, tau=0.008, sigma=2.5, beta=0.0, gamma=1.0,
              tol=1e-4, check_every=10, stop_window=5, alternative=False):
    """A warm-started TGV2 run as mvs_tgv2_run_warm makes it, in FP64 (one
    linearisation): the data term linearised at ``u_lin``, the primal started
    at ``u_start`` and ``v_start`` (2, H, W), the duals one dual step of size
    ``dual_sigma`` (p, q) and ``dual_sigma_r`` (r) from zero with the
    iteration's own operators and projections (P of TGV2_kernels.cu:340-365,
    Q of :54-85, R of :87-105), then the iterations of PlaneSweep::TGV with the
    given steps and the same stopping rule as ``tgv2``.

    Returns (u, iterations, energies)."""
    L = oracle_lib()
    precision = "f64"
    st = tgv2_setup(ref255, srcs255, K_1based, Rref, tref, src_poses, alternative, precision)
    P, dt = st["P"], st["dt"]
    h, w = st["ref01"].shape
    V = len(srcs255)
    T = tensor(st["ref01"], beta, gamma, precision)
    S = TGV2State(h, w, V, dt)
    S.u0[:] = u_lin
    S.u[:] = u_start
    S.ubar[:] = S.u
    S.u1x[:] = v_start[0]
    S.u1y[:] = v_start[1]
    S.u1xbar[:] = S.u1x
    S.u1ybar[:] = S.u1y
    It, Iu = tgv2_linearize(st, S.u0, precision)
    xn = np.minimum(np.arange(w) + 1, w - 1)
    yn = np.minimum(np.arange(h) + 1, h - 1)
    u, vx, vy = (np.asarray(a, np.float64) for a in (S.u, S.u1x, S.u1y))
    T11, T12, T21, T22 = (np.asarray(t, np.float64) for t in T)
    if dual_sigma > 0:
        xg, yg = u[:, xn] - u - vx, u[yn, :] - u - vy
        sc = alpha1 * dual_sigma
        dx, dy = sc * (T11 * xg + T12 * yg), sc * (T21 * xg + T22 * yg)
        d = np.maximum(1.0, np.sqrt(dx * dx + dy * dy))
        S.Px[:], S.Py[:] = dx / d, dy / d
        sc = alpha0 * dual_sigma
        dx, dy = sc * (vx[:, xn] - vx), sc * (vy[yn, :] - vy)
        dz = sc * ((vx[yn, :] - vx) + (vy[:, xn] - vy)) / 2.0
        d = np.maximum(1.0, np.sqrt(dx * dx + dy * dy + 2 * dz * dz))
        S.Qx[:], S.Qy[:], S.Qz[:], S.Qw[:] = dx / d, dy / d, dz / d, dz / d
    if dual_sigma_r > 0:
        q = dual_sigma_r * lam * (np.asarray(It, np.float64) + (u - np.asarray(S.u0, np.float64)) * Iu)
        S.r[:] = q / np.maximum(1.0, np.abs(q))
    it_fn = getattr(L, f"orc_tgv2_iteration_{precision}")
    en_fn = getattr(L, f"orc_tgv2_energy_{precision}")
    total, energies, hist = 0, [], []
    for k in range(max_iters):
        it_fn(w, h, V, *[P(t) for t in T], P(It), P(Iu), P(S.u0), P(S.u), P(S.u1x), P(S.u1y), P(S.ubar),
              P(S.u1xbar), P(S.u1ybar), P(S.Px), P(S.Py), P(S.Qx), P(S.Qy), P(S.Qz), P(S.Qw), P(S.r),
              P(S.prodsum), lam, alpha0, alpha1, tau, sigma)
        total += 1
        if tol > 0 and (k + 1) % check_every == 0:
            E = en_fn(w, h, V, *[P(t) for t in T], P(It), P(Iu), P(S.u0), P(S.u), P(S.u1x), P(S.u1y), lam,
                      alpha0, alpha1)
            energies.append(E)
            hist.append(E)
            if len(hist) > stop_window and abs(hist[-1 - stop_window] - E) <= tol * stop_window * abs(
                    hist[-1 - stop_window]):
                break
    return S.u.copy(), total, energies


def tgv_sparse(ref255, depthmap, sparse, zfar, niters, alpha0=2.0, alpha1=1.5, tau=0.02, sigma=1.0, theta=1.0,
               beta=0.0, gamma=1.0, precision="f64", T=None):
    """PlaneSweep::TGVdenoiseFromSparse (planesweep.cpp:596-674) over the C
    restatement: weights = (sparse > 0), Ds = sparse * (1/zfar), u = depthmap *
    (1/zfar), the anisotropic tensor of ref/255, ``niters`` iterations, u * zfar.
    ``theta`` only reaches the over-relaxed u, which nothing reads.  ``T``
    (T11, T12, T21, T22) replaces the tensor when given."""
    L = oracle_lib()
    dt = np.float32 if precision == "f32" else np.float64
    P = _fp if precision == "f32" else _dp
    h, w = depthmap.shape
    one = dt(1)
    inv_zfar = dt(np.float32(1) / np.float32(zfar)) if precision == "f32" else 1.0 / zfar
    sp = np.asarray(sparse, dt)
    wgt = np.ascontiguousarray(np.where(sp > 0, one, dt(0)), dt)
    Ds = np.ascontiguousarray(sp * inv_zfar, dt)
    u = np.ascontiguousarray(np.asarray(depthmap, dt) * inv_zfar, dt)
    scale = np.float32(1) / np.float32(255) if precision == "f32" else 1.0 / 255.0
    if T is None:
        T = tensor(np.ascontiguousarray(np.asarray(ref255, dt) * dt(scale), dt), beta, gamma, precision)
    T = [np.ascontiguousarray(t, dt) for t in T]
    st = [np.zeros((h, w), dt) for _ in range(8)]   # vx, vy, Px, Py, Qx, Qy, Qz, Qw
    fn = getattr(L, f"orc_tgv_sparse_iteration_{precision}")
    for _ in range(niters):
        fn(w, h, *[P(t) for t in T], P(wgt), P(Ds), P(u), *[P(a) for a in st], alpha0, alpha1, tau, sigma)
    return (u * dt(zfar)).astype(dt)


def ref_tgv(ref255, srcs255, K_1based, Rref, tref, src_poses, niters=30, warps=15, lam=0.5, alpha0=2.0,
            alpha1=1.5, tau=0.02, sigma=1.0, beta=0.0, gamma=1.0, u_init=None, alternative=False):
    L = ref_lib()
    h, w = ref255.shape
    V = len(srcs255)
    out = np.zeros((h, w), np.float32)
    Rs = _f32(np.stack([p[0] for p in src_poses]))
    ts = _f32(np.stack([p[1] for p in src_poses]))
    ui = None if u_init is None else _f32(u_init)
    secs = L.ref_tgv(w, h, _fp(_f32(ref255)), _fp(_f32(np.stack(srcs255))), V, _fp(_f32(K_1based)),
                     _fp(_f32(Rref)), _fp(_f32(tref)), _fp(Rs), _fp(ts), int(alternative), niters, warps, lam,
                     alpha0, alpha1, tau, sigma, beta, gamma, _fp(ui), _fp(out))
    return out, secs


# ---------------------------------------------------------------------------
# TV-L1 depth denoise
# ---------------------------------------------------------------------------

def tvl1_denoise(ref255, depth, znear, zfar, niters=100, lam=0.3, tau=0.02, sigma=6.0, theta=1.0, beta=0.0,
                 gamma=1.0, precision="f64"):
    L = oracle_lib()
    dt = np.float32 if precision == "f32" else np.float64
    P = _fp if precision == "f32" else _dp
    h, w = depth.shape
    out = np.zeros((h, w), dt)
    getattr(L, f"orc_tvl1_denoise_{precision}")(w, h, P(np.ascontiguousarray(ref255, dt)),
                                                P(np.ascontiguousarray(depth, dt)), znear, zfar, niters, lam,
                                                tau, sigma, theta, beta, gamma, P(out))
    return out


def ref_tvl1_denoise(ref255, depth, znear, zfar, niters=100, lam=0.3, tau=0.02, sigma=6.0, theta=1.0,
                     beta=0.0, gamma=1.0):
    L = ref_lib()
    h, w = depth.shape
    out = np.zeros((h, w), np.float32)
    secs = L.ref_tvl1_denoise(w, h, _fp(_f32(ref255)), _fp(_f32(depth)), znear, zfar, niters, lam, tau, sigma,
                              theta, beta, gamma, _fp(out))
    return out, secs


# ---------------------------------------------------------------------------
# fusion
# ---------------------------------------------------------------------------

def bin_centers(bins):
    out = np.zeros(bins, np.float32)
    oracle_lib().orc_bin_centers(bins, _fp(out))
    return out


class Volume:
    """SoA fusion volume: u, v (n), p (3, n), hist (bins, n) uint16; x fastest."""

    def __init__(self, bins, dims, a, b, precision="f64"):
        self.bins = bins
        self.dims = tuple(int(d) for d in dims)            # (vw, vh, vd)
        self.a = _f32(a)
        self.b = _f32(b)
        self.precision = precision
        dt = np.float32 if precision == "f32" else np.float64
        n = self.dims[0] * self.dims[1] * self.dims[2]
        self.u = np.zeros(n, dt)
        self.v = np.zeros(n, dt)
        self.p = np.zeros((3, n), dt)
        self.hist = np.zeros((bins, n), np.uint16)

    def histogram(self, depth, K, R, t, thr):
        L = oracle_lib()
        pr = self.precision
        dt = np.float32 if pr == "f32" else np.float64
        P = _fp if pr == "f32" else _dp
        h, w = depth.shape
        vw, vh, vd = self.dims
        getattr(L, f"orc_fusion_histogram_{pr}")(self.bins, vw, vh, vd, _fp(self.a), _fp(self.b),
                                                 self.hist.ctypes.data_as(_U16), _fp(_f32(depth)), w, h,
                                                 P(_mat(dt, K)), P(_mat(dt, R)), P(_mat(dt, t)), thr)

    def update_u(self, tau, lam):
        L = oracle_lib()
        pr = self.precision
        P = _fp if pr == "f32" else _dp
        vw, vh, vd = self.dims
        getattr(L, f"orc_fusion_u_{pr}")(self.bins, vw, vh, vd, self.hist.ctypes.data_as(_U16), P(self.u),
                                         P(self.v), P(self.p), tau, lam)

    def update_p(self, sigma):
        L = oracle_lib()
        pr = self.precision
        P = _fp if pr == "f32" else _dp
        vw, vh, vd = self.dims
        getattr(L, f"orc_fusion_p_{pr}")(vw, vh, vd, P(self.v), P(self.p), sigma)


class RefVolume:
    """fusionData<bins> driven through the reference's own kernels on the CPU."""

    def __init__(self, bins, dims, a, b):
        self.L = ref_lib()
        self.bins = bins
        self.dims = tuple(int(d) for d in dims)
        self.h = self.L.ref_fusion_create(bins, *self.dims, _fp(_f32(a)), _fp(_f32(b)))

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_fusion_destroy(self.h)
            self.h = None

    def histogram(self, depth, K, R, t, thr):
        h, w = depth.shape
        return self.L.ref_fusion_histogram(self.h, _fp(_f32(depth)), w, h, _fp(_f32(K)), _fp(_f32(R)),
                                           _fp(_f32(t)), thr)

    def update_u(self, tau, lam):
        return self.L.ref_fusion_u(self.h, tau, lam)

    def update_p(self, sigma):
        return self.L.ref_fusion_p(self.h, sigma)

    def get(self):
        n = self.dims[0] * self.dims[1] * self.dims[2]
        u, v, p = np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros((3, n), np.float32)
        hist = np.zeros((self.bins, n), np.uint16)
        self.L.ref_fusion_get(self.h, _fp(u), _fp(v), _fp(p), hist.ctypes.data_as(_U16))
        return dict(u=u, v=v, p=p, hist=hist)

    def set(self, u=None, v=None, p=None, hist=None):
        self.L.ref_fusion_set(self.h, _fp(None if u is None else _f32(u)), _fp(None if v is None else _f32(v)),
                              _fp(None if p is None else _f32(p)),
                              None if hist is None else np.ascontiguousarray(hist, np.uint16).ctypes.data_as(_U16))
