"""Float32 host math that feeds the kernels, in the reference's operation order.

The reference builds K^-1, the relative poses and (on its CPU path) the
per-plane homographies with its float Matrix3D type (structs.h:410-764,
helper_structs.h:159-291): rows dotted with columns as a.x*b.x + a.y*b.y +
a.z*b.z, the cofactor inverse divided by the determinant.  These helpers do the
same in numpy float32 scalars, so the device receives the same floats the
reference's kernels receive.  (The C++ classes in include/mvs_b200.hpp do the
same for C++ callers.)
"""
from __future__ import annotations

import numpy as np

f = np.float32


def _dot(a0, a1, a2, b0, b1, b2):
    return f(f(f(a0 * b0) + f(a1 * b1)) + f(a2 * b2))


def matmul_f32(A, B):
    A = np.asarray(A, f).reshape(3, 3)
    B = np.asarray(B, f).reshape(3, 3)
    C = np.zeros((3, 3), f)
    for r in range(3):
        for c in range(3):
            C[r, c] = _dot(A[r, 0], A[r, 1], A[r, 2], B[0, c], B[1, c], B[2, c])
    return C


def matvec_f32(A, v):
    A = np.asarray(A, f).reshape(3, 3)
    v = np.asarray(v, f).reshape(3)
    return np.array([_dot(A[r, 0], A[r, 1], A[r, 2], v[0], v[1], v[2]) for r in range(3)], f)


def inv3_f32(M):
    """Matrix3D::inv (structs.h:584-593)."""
    m = np.asarray(M, f).reshape(3, 3)
    d = f(f(f(m[0, 0] * f(f(m[1, 1] * m[2, 2]) - f(m[1, 2] * m[2, 1])))
            - f(m[0, 1] * f(f(m[1, 0] * m[2, 2]) - f(m[1, 2] * m[2, 0]))))
          + f(m[0, 2] * f(f(m[1, 0] * m[2, 1]) - f(m[1, 1] * m[2, 0]))))

    def c(a, b, x, y):
        return f(f(f(a * b) - f(x * y)) / d)

    return np.array([
        [c(m[1, 1], m[2, 2], m[1, 2], m[2, 1]), c(m[0, 2], m[2, 1], m[0, 1], m[2, 2]), c(m[0, 1], m[1, 2], m[0, 2], m[1, 1])],
        [c(m[1, 2], m[2, 0], m[1, 0], m[2, 2]), c(m[0, 0], m[2, 2], m[0, 2], m[2, 0]), c(m[0, 2], m[1, 0], m[0, 0], m[1, 2])],
        [c(m[1, 0], m[2, 1], m[1, 1], m[2, 0]), c(m[0, 1], m[2, 0], m[0, 0], m[2, 1]), c(m[0, 0], m[1, 1], m[0, 1], m[1, 0])],
    ], f)


def relative_f32(Rref, tref, Rsrc, tsrc, alternative=False):
    """PlaneSweep::RelativeMatrices (planesweep.cpp:538-549) in float."""
    Rref = np.asarray(Rref, f).reshape(3, 3)
    Rsrc = np.asarray(Rsrc, f).reshape(3, 3)
    tref = np.asarray(tref, f).reshape(3)
    tsrc = np.asarray(tsrc, f).reshape(3)
    if not alternative:
        Rrel = matmul_f32(Rsrc, inv3_f32(Rref))
        trel = (tsrc - matvec_f32(Rrel, tref)).astype(f)
    else:
        St = Rsrc.T.copy()
        Rrel = matmul_f32(St, Rref)
        trel = matvec_f32(St, (tref - tsrc).astype(f))
    return Rrel, trel


def homography_f32(K, invK, Rrel, trel, d):
    """H = K (Rrel + t e3^T / d) K^-1, H /= H22, as PlaneSweepThread (planesweep.cpp:196-203)."""
    M = np.zeros((3, 3), f)
    M[:, 2] = np.asarray(trel, f).reshape(3)
    M = (np.asarray(Rrel, f).reshape(3, 3) + (M / f(d)).astype(f)).astype(f)
    H = matmul_f32(matmul_f32(K, M), invK)
    return (H / H[2, 2]).astype(f)
