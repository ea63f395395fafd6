/* Generic body of the CPU oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * Included twice by mvs_oracle.c: once with R = float (the reference's own
 * arithmetic: float storage, the double intermediates it uses, the same
 * operation order, compiled without FMA contraction) and once with R = double
 * (the FP64 oracle).  Each routine cites the reference code it restates.
 *
 * Macros expected from the includer: R, FN(name), SQRTR, FABSR, FLOORR,
 * ROUNDR, EXPR, POWR, FMAXR, FMINR.
 */

/* ---- 3x3 helpers: Matrix3D (structs.h:410-764, helper_structs.h:159-291) ---- */

static R FN(dot3)(const R *a, const R *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

static void FN(matmul)(const R *A, const R *B, R *C)
{
    /* operator*(Matrix3D, Matrix3D): rows of A dotted with columns of B */
    R out[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            R col[3] = {B[j], B[3 + j], B[6 + j]};
            out[3 * i + j] = FN(dot3)(A + 3 * i, col);
        }
    memcpy(C, out, sizeof(out));
}

static void FN(matvec)(const R *A, const R *v, R *out)
{
    R o[3] = {FN(dot3)(A, v), FN(dot3)(A + 3, v), FN(dot3)(A + 6, v)};
    memcpy(out, o, sizeof(o));
}

static void FN(transpose)(const R *A, R *T)
{
    R o[9] = {A[0], A[3], A[6], A[1], A[4], A[7], A[2], A[5], A[8]};
    memcpy(T, o, sizeof(o));
}

/* Matrix3D::det / Matrix3D::inv, structs.h:571-593 (cofactors / det) */
void FN(orc_inv3)(const R *m, R *out)
{
    const R *r0 = m, *r1 = m + 3, *r2 = m + 6;
    R d = r0[0] * (r1[1] * r2[2] - r1[2] * r2[1]) - r0[1] * (r1[0] * r2[2] - r1[2] * r2[0]) +
          r0[2] * (r1[0] * r2[1] - r1[1] * r2[0]);
    R o[9] = {(r1[1] * r2[2] - r1[2] * r2[1]) / d, (r0[2] * r2[1] - r0[1] * r2[2]) / d,
              (r0[1] * r1[2] - r0[2] * r1[1]) / d, (r1[2] * r2[0] - r1[0] * r2[2]) / d,
              (r0[0] * r2[2] - r0[2] * r2[0]) / d, (r0[2] * r1[0] - r0[0] * r1[2]) / d,
              (r1[0] * r2[1] - r1[1] * r2[0]) / d, (r0[1] * r2[0] - r0[0] * r2[1]) / d,
              (r0[0] * r1[1] - r0[1] * r1[0]) / d};
    memcpy(out, o, sizeof(o));
}

/* PlaneSweep::RelativeMatrices, planesweep.cpp:538-549 */
void FN(orc_relative)(const R *Rref, const R *tref, const R *Rsrc, const R *tsrc, int alternative,
                      R *Rrel, R *trel)
{
    if (!alternative) {
        R inv[9], Rt[3];
        FN(orc_inv3)(Rref, inv);
        FN(matmul)(Rsrc, inv, Rrel);
        FN(matvec)(Rrel, tref, Rt);
        for (int i = 0; i < 3; ++i) trel[i] = tsrc[i] - Rt[i];
    } else {
        R St[9], dt[3];
        FN(transpose)(Rsrc, St);
        FN(matmul)(St, Rref, Rrel);
        for (int i = 0; i < 3; ++i) dt[i] = tref[i] - tsrc[i];
        FN(matvec)(St, dt, trel);
    }
}

/* H = K (Rrel + t e3^T / d) K^-1, H /= H(2,2)  (planesweep.cpp:196-203) */
void FN(orc_homography)(const R *K, const R *invK, const R *Rrel, const R *trel, R d, R *H)
{
    R M[9], T[9];
    for (int i = 0; i < 9; ++i) M[i] = 0;
    /* tr.row(2) = trel; tr = tr.trans(): column 2 holds trel */
    M[2] = trel[0];
    M[5] = trel[1];
    M[8] = trel[2];
    for (int i = 0; i < 9; ++i) M[i] = Rrel[i] + M[i] / d;
    FN(matmul)(K, M, T);
    FN(matmul)(T, invK, T);
    R s = T[8];
    for (int i = 0; i < 9; ++i) H[i] = T[i] / s;
}

/* ---- plane sweep: kernels.cu:4-235, planesweep.cpp:74-259 ---- */

static int FN(mirror)(int k, int n)
{
    /* windowed_mean_*_kernel boundary, kernels.cu:203-204 / 228-229 */
    if (k < 0) k = -k;
    if (k > n - 1) k = 2 * (n - 1) - k;
    return k;
}

/* windowed_mean_column_kernel then windowed_mean_row_kernel (kernels.cu:187-235) */
static void FN(box_mean)(int w, int h, const R *in, int win, int squared, R *tmp, R *out)
{
    const int n = win / 2;
    ORC_PAR
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            R m = 0;
            for (int i = -n; i <= n; ++i) {
                R v = in[FN(mirror)(y + i, h) * w + x];
                m += squared ? v * v : v;
            }
            tmp[y * w + x] = m / (R)win;
        }
    ORC_PAR
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            R m = 0;
            for (int i = -n; i <= n; ++i) m += tmp[y * w + FN(mirror)(x + i, w)];
            out[y * w + x] = m / (R)win;
        }
}

/* calculate_STD_kernel, kernels.cu:103-120 */
static void FN(std_from)(int n, const R *mean, const R *msq, R *std)
{
    for (int i = 0; i < n; ++i) {
        R var = msq[i] - mean[i] * mean[i];
        std[i] = var > 0 ? SQRTR(var) : 0;
    }
}

/* transform_indexes_kernel + bilinear_interpolation_kernel_GPU (kernels.cu:4-44) */
static void FN(warp)(int w, int h, const R *src, const R *H, R *out)
{
    ORC_PAR
    for (int k = 0; k < h; ++k)
        for (int l = 0; l < w; ++l) {
            R p[3] = {(R)(l + 1), (R)(k + 1), (R)1}, q[3];
            FN(matvec)(H, p, q);
            R xs = q[0] / q[2] - 1, ys = q[1] / q[2] - 1;
            R fx = FLOORR(xs), fy = FLOORR(ys);
            /* out-of-range or non-finite coordinates read as outside (0) */
            if (!(fx >= 0 && fy >= 0 && fx + 1 <= (R)(w - 1) && fy + 1 <= (R)(h - 1))) {
                out[k * w + l] = 0;
                continue;
            }
            int ix = (int)fx, iy = (int)fy;
            R a = xs - (R)ix, b = ys - (R)iy;
            R t1 = a * src[iy * w + ix + 1] + (1 - a) * src[iy * w + ix];
            R t2 = a * src[(iy + 1) * w + ix + 1] + (1 - a) * src[(iy + 1) * w + ix];
            out[k * w + l] = b * t2 + (1 - b) * t1;
        }
}

typedef struct {
    R *refv, *refmean, *refstd, *warped, *tmp, *wmean, *wsq, *wstd, *prod, *pmean;
} FN(sweep_ws);

static void FN(ws_alloc)(FN(sweep_ws) *s, size_t n)
{
    R **f[] = {&s->refv, &s->refmean, &s->refstd, &s->warped, &s->tmp, &s->wmean, &s->wsq, &s->wstd,
               &s->prod, &s->pmean};
    for (size_t i = 0; i < sizeof(f) / sizeof(f[0]); ++i) *f[i] = (R *)calloc(n, sizeof(R));
}

static void FN(ws_free)(FN(sweep_ws) *s)
{
    R *f[] = {s->refv, s->refmean, s->refstd, s->warped, s->tmp, s->wmean, s->wsq, s->wstd, s->prod, s->pmean};
    for (size_t i = 0; i < sizeof(f) / sizeof(f[0]); ++i) free(f[i]);
}

static void FN(ref_moments)(int w, int h, const float *ref, int win, FN(sweep_ws) *s)
{
    const size_t n = (size_t)w * h;
    for (size_t i = 0; i < n; ++i) s->refv[i] = (R)ref[i];
    FN(box_mean)(w, h, s->refv, win, 0, s->tmp, s->refmean);
    FN(box_mean)(w, h, s->refv, win, 1, s->tmp, s->wsq);
    FN(std_from)((int)n, s->refmean, s->wsq, s->refstd);
}

/* One plane: NCC image as PlaneSweepThread computes it (planesweep.cpp:205-243,
 * calcNCC_kernel kernels.cu:46-64).  srcR is the source as R. */
static void FN(plane_ncc)(int w, int h, const R *srcR, const R *H, int win, R st, FN(sweep_ws) *s, R *ncc)
{
    const size_t n = (size_t)w * h;
    FN(warp)(w, h, srcR, H, s->warped);
    FN(box_mean)(w, h, s->warped, win, 0, s->tmp, s->wmean);
    FN(box_mean)(w, h, s->warped, win, 1, s->tmp, s->wsq);
    FN(std_from)((int)n, s->wmean, s->wsq, s->wstd);
    for (size_t i = 0; i < n; ++i) s->prod[i] = s->refv[i] * s->warped[i];
    FN(box_mean)(w, h, s->prod, win, 0, s->tmp, s->pmean);
    ORC_PAR
    for (size_t i = 0; i < n; ++i) {
        if (s->refstd[i] < st || s->wstd[i] < st) ncc[i] = 0;
        else ncc[i] = (s->pmean[i] - s->refmean[i] * s->wmean[i]) / (s->refstd[i] * s->wstd[i]);
    }
}

void FN(orc_sweep_ncc)(int w, int h, const float *ref, const float *src, const R *H9, int winsize,
                       double stdthresh, R *ncc)
{
    const size_t n = (size_t)w * h;
    FN(sweep_ws) s;
    FN(ws_alloc)(&s, n);
    R *srcR = (R *)malloc(n * sizeof(R));
    for (size_t i = 0; i < n; ++i) srcR[i] = (R)src[i];
    FN(ref_moments)(w, h, ref, winsize, &s);
    FN(plane_ncc)(w, h, srcR, H9, winsize, (R)stdthresh, &s, ncc);
    free(srcR);
    FN(ws_free)(&s);
}

/* PlaneSweepThread's plane loop with update_arrays_kernel (kernels.cu:66-82):
 * best starts at 0 and only a strictly larger NCC replaces it, so ties keep
 * the earlier plane and NCC <= 0 never wins (label -1, depth 0). */
void FN(orc_sweep_view)(int w, int h, const float *ref, const float *src, const R *H, const float *depths,
                        int nplanes, int winsize, double stdthresh, R *best, R *depth, int32_t *label)
{
    const size_t n = (size_t)w * h;
    FN(sweep_ws) s;
    FN(ws_alloc)(&s, n);
    R *srcR = (R *)malloc(n * sizeof(R)), *ncc = (R *)malloc(n * sizeof(R));
    for (size_t i = 0; i < n; ++i) {
        srcR[i] = (R)src[i];
        best[i] = 0;
        depth[i] = 0;
        if (label) label[i] = -1;
    }
    FN(ref_moments)(w, h, ref, winsize, &s);
    for (int p = 0; p < nplanes; ++p) {
        FN(plane_ncc)(w, h, srcR, H + 9 * p, winsize, (R)stdthresh, &s, ncc);
        ORC_PAR
        for (size_t i = 0; i < n; ++i)
            if (ncc[i] > best[i]) {
                best[i] = ncc[i];
                depth[i] = (R)depths[p];
                if (label) label[i] = p;
            }
    }
    free(srcR);
    free(ncc);
    FN(ws_free)(&s);
}

/* sum_depthmap_NCC_kernel + element_rdivide_kernel + set_QNAN_value_kernel
 * (kernels.cu:84-101,145-157,331-340; planesweep.cpp:126-131) */
void FN(orc_sweep_combine)(int w, int h, int nview, const R *best, const R *depth, double nccthresh,
                           double zfar, R *out)
{
    const size_t n = (size_t)w * h;
    for (size_t i = 0; i < n; ++i) {
        R sum = 0, cnt = 0;
        for (int v = 0; v < nview; ++v)
            if (best[v * n + i] > (R)nccthresh) {
                sum += depth[v * n + i];
                cnt++;
            }
        R r = cnt != 0 ? sum / cnt : (R)NAN;
        out[i] = r != r ? (R)zfar : r;
    }
}

/* ---- aggregated matching cost over a band of rows ----
 * For output rows [y0, y1) of a w x h frame: the sum over the nview source
 * views of the NCC of every plane, computed exactly as orc_sweep_ncc (the
 * warp, the mirrored box means and calcNCC of kernels.cu:4-64,103-120,187-235)
 * but only on the rows the band needs: the warped source on rows
 * [max(0, y0 - r), min(h, y1 + r)), r = winsize / 2, which holds every row the
 * mirrored column windows of the band read.  Pixels are independent, so the
 * band equals the same rows of the full-frame computation.  Planes run in
 * parallel.  H is [nview][nplanes][9]; out is [nplanes][y1 - y0][w]. */
static void FN(box_mean_band)(int w, int h, const R *in, int lo, int win, int y0, int y1, R *tmp, R *out)
{
    const int n = win / 2;
    for (int y = y0; y < y1; ++y)
        for (int x = 0; x < w; ++x) {
            R m = 0;
            for (int i = -n; i <= n; ++i) m += in[(size_t)(FN(mirror)(y + i, h) - lo) * w + x];
            tmp[(size_t)(y - y0) * w + x] = m / (R)win;
        }
    for (int y = y0; y < y1; ++y)
        for (int x = 0; x < w; ++x) {
            R m = 0;
            for (int i = -n; i <= n; ++i) m += tmp[(size_t)(y - y0) * w + FN(mirror)(x + i, w)];
            out[(size_t)(y - y0) * w + x] = m / (R)win;
        }
}

static void FN(warp_rows)(int w, int h, const float *src, const R *H, int lo, int hi, R *out)
{
    for (int k = lo; k < hi; ++k)
        for (int l = 0; l < w; ++l) {
            R p[3] = {(R)(l + 1), (R)(k + 1), (R)1}, q[3];
            FN(matvec)(H, p, q);
            R xs = q[0] / q[2] - 1, ys = q[1] / q[2] - 1;
            R fx = FLOORR(xs), fy = FLOORR(ys);
            R v = 0;
            if (fx >= 0 && fy >= 0 && fx + 1 <= (R)(w - 1) && fy + 1 <= (R)(h - 1)) {
                int ix = (int)fx, iy = (int)fy;
                R a = xs - (R)ix, b = ys - (R)iy;
                R t1 = a * (R)src[iy * w + ix + 1] + (1 - a) * (R)src[iy * w + ix];
                R t2 = a * (R)src[(iy + 1) * w + ix + 1] + (1 - a) * (R)src[(iy + 1) * w + ix];
                v = b * t2 + (1 - b) * t1;
            }
            out[(size_t)(k - lo) * w + l] = v;
        }
}

void FN(orc_sweep_ncc_band)(int w, int h, int nview, const float *ref, const float *srcs, const R *H, int nplanes,
                            int winsize, double stdthresh, int y0, int y1, R *out)
{
    const int r = winsize / 2, lo = y0 - r > 0 ? y0 - r : 0, hi = y1 + r < h ? y1 + r : h;
    const size_t nb = (size_t)(y1 - y0) * w, nr = (size_t)(hi - lo) * w;
    const R st = (R)stdthresh;
    R *refv = (R *)malloc(nr * sizeof(R)), *rm = (R *)malloc(nb * sizeof(R)), *rs = (R *)malloc(nb * sizeof(R)),
      *t0 = (R *)malloc(nb * sizeof(R)), *sq = (R *)malloc(nr * sizeof(R));
    for (size_t i = 0; i < nr; ++i) {
        refv[i] = (R)ref[(size_t)lo * w + i];
        sq[i] = refv[i] * refv[i];
    }
    FN(box_mean_band)(w, h, refv, lo, winsize, y0, y1, t0, rm);
    FN(box_mean_band)(w, h, sq, lo, winsize, y0, y1, t0, rs);
    FN(std_from)((int)nb, rm, rs, rs);
    free(t0);
    free(sq);
#pragma omp parallel for schedule(dynamic)
    for (int p = 0; p < nplanes; ++p) {
        R *wp = (R *)malloc(nr * sizeof(R)), *w2 = (R *)malloc(nr * sizeof(R)), *pr = (R *)malloc(nr * sizeof(R)),
          *tmp = (R *)malloc(nb * sizeof(R)), *wm = (R *)malloc(nb * sizeof(R)), *wq = (R *)malloc(nb * sizeof(R)),
          *pm = (R *)malloc(nb * sizeof(R));
        R *o = out + (size_t)p * nb;
        for (size_t i = 0; i < nb; ++i) o[i] = 0;
        for (int v = 0; v < nview; ++v) {
            FN(warp_rows)(w, h, srcs + (size_t)v * w * h, H + ((size_t)v * nplanes + p) * 9, lo, hi, wp);
            for (size_t i = 0; i < nr; ++i) {
                w2[i] = wp[i] * wp[i];
                pr[i] = refv[i] * wp[i];
            }
            FN(box_mean_band)(w, h, wp, lo, winsize, y0, y1, tmp, wm);
            FN(box_mean_band)(w, h, w2, lo, winsize, y0, y1, tmp, wq);
            FN(box_mean_band)(w, h, pr, lo, winsize, y0, y1, tmp, pm);
            FN(std_from)((int)nb, wm, wq, wq);
            for (size_t i = 0; i < nb; ++i)
                if (!(rs[i] < st || wq[i] < st)) o[i] += (pm[i] - rm[i] * wm[i]) / (rs[i] * wq[i]);
        }
        free(wp); free(w2); free(pr); free(tmp); free(wm); free(wq); free(pm);
    }
    free(refv); free(rm); free(rs);
}

/* ---- TGV2: TGV2_kernels.cu, planesweep.cpp:381-536 ---- */

/* Anisotropic_diffusion_tensor_kernel, TGV2_kernels.cu:257-298 */
void FN(orc_tensor)(int w, int h, const R *img, double beta, double gamma, R *T11, R *T12, R *T21, R *T22)
{
    const R bt = (R)beta, gm = (R)gamma;
    ORC_PAR
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            int i = y * w + x, xn = x + 1 < w - 1 ? x + 1 : w - 1, yn = y + 1 < h - 1 ? y + 1 : h - 1;
            R gx = img[y * w + xn] - img[i];
            R gy = img[yn * w + x] - img[i];
            R d = SQRTR(gx * gx + gy * gy);
            if (d > 0) {
                gx = gx / d;
                gy = gy / d;
                R k = EXPR(-bt * POWR(d, gm));
                T11[i] = k * gx * gx + gy * gy;
                T12[i] = (k - 1) * gx * gy;
                T21[i] = (k - 1) * gx * gy;
                T22[i] = k * gy * gy + gx * gx;
            } else {
                T11[i] = 1;
                T12[i] = 0;
                T21[i] = 0;
                T22[i] = 1;
            }
        }
}

/* Per-view linearisation at u0 (planesweep.cpp:460-483):
 * TGV2_transform_coordinates_kernel (TGV2_kernels.cu:141-179),
 * TGV2_calculate_coordinate_derivatives_kernel (:194-219),
 * TGV2_calculate_derivativeF_kernel (:221-236), bilinear_interpolation,
 * TGV2_calculate_Iu_kernel (:238-255) and subtract_kernel (:181-192). */
void FN(orc_tgv2_linearize)(int w, int h, const R *src01, const R *ref01, const R *u0, const R *K,
                            const R *invK, const R *Rrel, const R *trel, R *It, R *Iu)
{
    const size_t n = (size_t)w * h;
    R *xs = (R *)malloc(n * sizeof(R)), *ys = (R *)malloc(n * sizeof(R)), *X = (R *)malloc(n * sizeof(R)),
      *Y = (R *)malloc(n * sizeof(R)), *Z = (R *)malloc(n * sizeof(R)), *dfx = (R *)malloc(n * sizeof(R)),
      *dfy = (R *)malloc(n * sizeof(R)), *Iw = (R *)malloc(n * sizeof(R));
    const R fx = K[0], fy = K[4];
    R RinvK[9];
    FN(matmul)(Rrel, invK, RinvK);
    ORC_PAR
    for (int k = 0; k < h; ++k)
        for (int l = 0; l < w; ++l) {
            const int i = k * w + l;
            R a[3] = {(R)(l + 1), (R)(k + 1), (R)1}, ka[3], x1[3], x2[3], kx[3], dX[3];
            FN(matvec)(invK, a, ka);
            for (int c = 0; c < 3; ++c) x1[c] = u0[i] * ka[c];
            FN(matvec)(Rrel, x1, x2);
            for (int c = 0; c < 3; ++c) x2[c] = x2[c] + trel[c];
            X[i] = x2[0];
            Y[i] = x2[1];
            Z[i] = x2[2];
            FN(matvec)(K, x2, kx);
            xs[i] = kx[0] / kx[2] - 1;
            ys[i] = kx[1] / kx[2] - 1;
            FN(matvec)(RinvK, a, dX);
            dfx[i] = fx * (dX[0] * Z[i] - X[i] * dX[2]) / (Z[i] * Z[i]);
            dfy[i] = fy * (dX[1] * Z[i] - Y[i] * dX[2]) / (Z[i] * Z[i]);
        }
    /* bilinear_interpolation at the transformed coordinates (kernels.cu:4-29) */
    ORC_PAR
    for (int k = 0; k < h; ++k)
        for (int l = 0; l < w; ++l) {
            const int i = k * w + l;
            R fxx = FLOORR(xs[i]), fyy = FLOORR(ys[i]);
            if (!(fxx >= 0 && fyy >= 0 && fxx + 1 <= (R)(w - 1) && fyy + 1 <= (R)(h - 1))) {
                Iw[i] = 0;
                continue;
            }
            int ix = (int)fxx, iy = (int)fyy;
            R aa = xs[i] - (R)ix, bb = ys[i] - (R)iy;
            R t1 = aa * src01[iy * w + ix + 1] + (1 - aa) * src01[iy * w + ix];
            R t2 = aa * src01[(iy + 1) * w + ix + 1] + (1 - aa) * src01[(iy + 1) * w + ix];
            Iw[i] = bb * t2 + (1 - bb) * t1;
        }
    ORC_PAR
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            int i = y * w + x, xn = x + 1 < w - 1 ? x + 1 : w - 1, yn = y + 1 < h - 1 ? y + 1 : h - 1;
            double gx = Iw[y * w + xn] - Iw[i];
            double gy = Iw[yn * w + x] - Iw[i];
            Iu[i] = (R)(gx * dfx[i] + gy * dfy[i]);
            It[i] = Iw[i] - ref01[i];
        }
    free(xs); free(ys); free(X); free(Y); free(Z); free(dfx); free(dfy); free(Iw);
}

/* One primal-dual iteration (planesweep.cpp:485-509):
 * TGV2_updateP_tensor_weighed_kernel (TGV2_kernels.cu:340-365),
 * TGV2_updateQ_kernel (:54-85), prodsum = 0, TGV2_updateR_kernel per view
 * (:87-105) and TGV2_updateU_tensor_weighed_kernel (:300-338).  Each step is
 * a separate full-image pass, as in the reference. */
void FN(orc_tgv2_iteration)(int w, int h, int nview, const R *T11, const R *T12, const R *T21, const R *T22,
                            const R *It, const R *Iu, const R *u0, R *u, R *u1x, R *u1y, R *ubar, R *u1xbar,
                            R *u1ybar, R *Px, R *Py, R *Qx, R *Qy, R *Qz, R *Qw, R *r, R *prodsum,
                            double lambda_, double alpha0_, double alpha1_, double tau_, double sigma_)
{
    const size_t n = (size_t)w * h;
    const R lambda = (R)lambda_, alpha0 = (R)alpha0_, alpha1 = (R)alpha1_, tau = (R)tau_, sigma = (R)sigma_;
    ORC_PAR
    for (int yy = 0; yy < h; ++yy)
        for (int xx = 0; xx < w; ++xx) {
            int i = yy * w + xx, xn = xx + 1 < w - 1 ? xx + 1 : w - 1, yn = yy + 1 < h - 1 ? yy + 1 : h - 1;
            double x = ubar[yy * w + xn] - ubar[i] - u1xbar[i];
            double y = ubar[yn * w + xx] - ubar[i] - u1ybar[i];
            double dx = Px[i] + alpha1 * sigma * (T11[i] * x + T12[i] * y);
            double dy = Py[i] + alpha1 * sigma * (T21[i] * x + T22[i] * y);
            double d = FMAXR(1, sqrt(dx * dx + dy * dy));
            Px[i] = (R)(dx / d);
            Py[i] = (R)(dy / d);
        }
    ORC_PAR
    for (int yy = 0; yy < h; ++yy)
        for (int xx = 0; xx < w; ++xx) {
            int i = yy * w + xx, xn = xx + 1 < w - 1 ? xx + 1 : w - 1, yn = yy + 1 < h - 1 ? yy + 1 : h - 1;
            R dx_u1x = u1xbar[yy * w + xn] - u1xbar[i];
            R dy_u1x = u1xbar[yn * w + xx] - u1xbar[i];
            R dx_u1y = u1ybar[yy * w + xn] - u1ybar[i];
            R dy_u1y = u1ybar[yn * w + xx] - u1ybar[i];
            double dx = Qx[i] + alpha0 * sigma * dx_u1x;
            double dy = Qy[i] + alpha0 * sigma * dy_u1y;
            double dz = Qz[i] + alpha0 * sigma * (dy_u1x + dx_u1y) / (R)2;
            double dw = Qw[i] + alpha0 * sigma * (dy_u1x + dx_u1y) / (R)2;
            double d = FMAXR(1, sqrt(dx * dx + dy * dy + dz * dz + dw * dw));
            Qx[i] = (R)(dx / d);
            Qy[i] = (R)(dy / d);
            Qz[i] = (R)(dz / d);
            Qw[i] = (R)(dw / d);
        }
    for (size_t i = 0; i < n; ++i) prodsum[i] = 0;
    for (int v = 0; v < nview; ++v) {
        R *rv = r + (size_t)v * n;
        const R *itv = It + (size_t)v * n, *iuv = Iu + (size_t)v * n;
        ORC_PAR
        for (size_t i = 0; i < n; ++i) {
            rv[i] = rv[i] + sigma * lambda * (itv[i] + (u[i] - u0[i]) * iuv[i]);
            rv[i] = rv[i] / FMAXR(1, FABSR(rv[i]));
            prodsum[i] += rv[i] * iuv[i];
        }
    }
    ORC_PAR
    for (int yy = 0; yy < h; ++yy)
        for (int xx = 0; xx < w; ++xx) {
            int i = yy * w + xx, xp = xx - 1 > 0 ? xx - 1 : 0, yp = yy - 1 > 0 ? yy - 1 : 0;
            R uprev = u[i], u1xprev = u1x[i], u1yprev = u1y[i];
            R c_px = Px[i], c_py = Py[i], xp_px = Px[yy * w + xp], yp_px = Px[yp * w + xx],
              xp_py = Py[yy * w + xp], yp_py = Py[yp * w + xx];
            u[i] = u[i] - tau * (-alpha1 * (T11[i] * (c_px - xp_px) + T12[i] * (c_py - xp_py) +
                                            T21[i] * (c_px - yp_px) + T22[i] * (c_py - yp_py)) +
                                 lambda * prodsum[i]);
            u1x[i] = u1x[i] - tau * (-alpha1 * (T11[i] * c_px + T12[i] * c_py) -
                                     alpha0 * (Qx[i] - Qx[yy * w + xp] + Qz[i] - Qz[yp * w + xx]));
            u1y[i] = u1y[i] - tau * (-alpha1 * (T21[i] * c_px + T22[i] * c_py) -
                                     alpha0 * (Qz[i] - Qz[yy * w + xp] + Qy[i] - Qy[yp * w + xx]));
            ubar[i] = 2 * u[i] - uprev;
            u1xbar[i] = 2 * u1x[i] - u1xprev;
            u1ybar[i] = 2 * u1y[i] - u1yprev;
        }
}

/* TGV2 energy that the iterations above minimise (no reference symbol: the
 * reference runs a fixed iteration count).  Same discrete operators as the
 * dual steps: forward differences with the clamped index x+1 -> min(x+1,W-1),
 *   E = a1 * sum |T (grad u - v)|_2 + a0 * sum |eps(v)|  (eps = (dx vx, dy vy,
 *       (dy vx + dx vy)/2, (dy vx + dx vy)/2), both off-diagonals counted as
 *       in TGV2_updateQ_kernel) + lambda * sum_i sum |It_i + (u - u0) Iu_i|.
 * Accumulated in double. */
double FN(orc_tgv2_energy)(int w, int h, int nview, const R *T11, const R *T12, const R *T21, const R *T22,
                           const R *It, const R *Iu, const R *u0, const R *u, const R *u1x, const R *u1y,
                           double lambda, double alpha0, double alpha1)
{
    const size_t n = (size_t)w * h;
    /* per-row partial sums, added in row order: the same result for any
     * number of threads */
    double *rows = (double *)calloc((size_t)3 * h, sizeof(double));
    ORC_PAR
    for (int yy = 0; yy < h; ++yy) {
        double e1 = 0, e0 = 0, ed = 0;
        for (int xx = 0; xx < w; ++xx) {
            int i = yy * w + xx, xn = xx + 1 < w - 1 ? xx + 1 : w - 1, yn = yy + 1 < h - 1 ? yy + 1 : h - 1;
            double gx = (double)u[yy * w + xn] - u[i] - u1x[i];
            double gy = (double)u[yn * w + xx] - u[i] - u1y[i];
            double tx = T11[i] * gx + T12[i] * gy, ty = T21[i] * gx + T22[i] * gy;
            e1 += sqrt(tx * tx + ty * ty);
            double a = (double)u1x[yy * w + xn] - u1x[i], b = (double)u1y[yn * w + xx] - u1y[i];
            double c = 0.5 * (((double)u1x[yn * w + xx] - u1x[i]) + ((double)u1y[yy * w + xn] - u1y[i]));
            e0 += sqrt(a * a + b * b + 2 * c * c);
            for (int v = 0; v < nview; ++v)
                ed += fabs((double)It[v * n + i] + ((double)u[i] - u0[i]) * Iu[v * n + i]);
        }
        rows[3 * yy] = e1;
        rows[3 * yy + 1] = e0;
        rows[3 * yy + 2] = ed;
    }
    double e1 = 0, e0 = 0, ed = 0;
    for (int yy = 0; yy < h; ++yy) {
        e1 += rows[3 * yy];
        e0 += rows[3 * yy + 1];
        ed += rows[3 * yy + 2];
    }
    free(rows);
    return alpha1 * e1 + alpha0 * e0 + lambda * ed;
}

/* ---- TGV2 towards a sparse depthmap: PlaneSweep::TGVdenoiseFromSparse
 * (planesweep.cpp:596-674).  One iteration of its loop (planesweep.cpp:638-649):
 * TGV2_updateP_tensor_weighed_kernel (TGV2_kernels.cu:340-365) on u itself,
 * TGV2_updateQ_kernel (:54-85) and TGV2_updateU_sparseDepthTensor_kernel
 * (:399-430), each a full-image pass.  The reference passes vxbar / vybar as
 * both v and its over-relaxation, so v keeps the plain update (the
 * over-relaxation v + theta (v - v) is v itself); the over-relaxed u it also
 * writes is never read and is left out. ---- */
void FN(orc_tgv_sparse_iteration)(int w, int h, const R *T11, const R *T12, const R *T21, const R *T22,
                                  const R *wgt, const R *Ds, R *u, R *vx, R *vy, R *Px, R *Py, R *Qx, R *Qy,
                                  R *Qz, R *Qw, double alpha0_, double alpha1_, double tau_, double sigma_)
{
    const R alpha0 = (R)alpha0_, alpha1 = (R)alpha1_, tau = (R)tau_, sigma = (R)sigma_;
    ORC_PAR
    for (int yy = 0; yy < h; ++yy)
        for (int xx = 0; xx < w; ++xx) {
            int i = yy * w + xx, xn = xx + 1 < w - 1 ? xx + 1 : w - 1, yn = yy + 1 < h - 1 ? yy + 1 : h - 1;
            double x = u[yy * w + xn] - u[i] - vx[i];
            double y = u[yn * w + xx] - u[i] - vy[i];
            double dx = Px[i] + alpha1 * sigma * (T11[i] * x + T12[i] * y);
            double dy = Py[i] + alpha1 * sigma * (T21[i] * x + T22[i] * y);
            double d = FMAXR(1, sqrt(dx * dx + dy * dy));
            Px[i] = (R)(dx / d);
            Py[i] = (R)(dy / d);
        }
    ORC_PAR
    for (int yy = 0; yy < h; ++yy)
        for (int xx = 0; xx < w; ++xx) {
            int i = yy * w + xx, xn = xx + 1 < w - 1 ? xx + 1 : w - 1, yn = yy + 1 < h - 1 ? yy + 1 : h - 1;
            R dx_u1x = vx[yy * w + xn] - vx[i];
            R dy_u1x = vx[yn * w + xx] - vx[i];
            R dx_u1y = vy[yy * w + xn] - vy[i];
            R dy_u1y = vy[yn * w + xx] - vy[i];
            double dx = Qx[i] + alpha0 * sigma * dx_u1x;
            double dy = Qy[i] + alpha0 * sigma * dy_u1y;
            double dz = Qz[i] + alpha0 * sigma * (dy_u1x + dx_u1y) / (R)2;
            double dw = Qw[i] + alpha0 * sigma * (dy_u1x + dx_u1y) / (R)2;
            double d = FMAXR(1, sqrt(dx * dx + dy * dy + dz * dz + dw * dw));
            Qx[i] = (R)(dx / d);
            Qy[i] = (R)(dy / d);
            Qz[i] = (R)(dz / d);
            Qw[i] = (R)(dw / d);
        }
    ORC_PAR
    for (int yy = 0; yy < h; ++yy)
        for (int xx = 0; xx < w; ++xx) {
            int i = yy * w + xx, xp = xx - 1 > 0 ? xx - 1 : 0, yp = yy - 1 > 0 ? yy - 1 : 0;
            R c_px = Px[i], c_py = Py[i], xp_px = Px[yy * w + xp], yp_px = Px[yp * w + xx],
              xp_py = Py[yy * w + xp], yp_py = Py[yp * w + xx];
            u[i] = (u[i] + tau * (alpha1 * (T11[i] * (c_px - xp_px) + T12[i] * (c_py - xp_py) +
                                            T21[i] * (c_px - yp_px) + T22[i] * (c_py - yp_py)) +
                                  wgt[i] * Ds[i])) /
                   (1 + tau * wgt[i]);
            vx[i] = vx[i] - tau * (-alpha1 * (T11[i] * c_px + T12[i] * c_py) -
                                   alpha0 * (Qx[i] - Qx[yy * w + xp] + Qz[i] - Qz[yp * w + xx]));
            vy[i] = vy[i] - tau * (-alpha1 * (T21[i] * c_px + T22[i] * c_py) -
                                   alpha0 * (Qz[i] - Qz[yy * w + xp] + Qy[i] - Qy[yp * w + xx]));
        }
}

/* ---- TV-L1 depth denoise: PlaneSweep::CudaDenoise (planesweep.cpp:297-379) ---- */

void FN(orc_tvl1_denoise)(int w, int h, const R *ref255, const R *depth, double znear_, double zfar_, int niters,
                          double lambda_, double tau_, double sigma_, double theta_, double beta, double gamma,
                          R *out)
{
    const size_t n = (size_t)w * h;
    const R znear = (R)znear_, zfar = (R)zfar_;
    R *ref = (R *)malloc(n * sizeof(R)), *raw = (R *)malloc(n * sizeof(R)), *Rr = (R *)calloc(n, sizeof(R)),
      *Px = (R *)calloc(n, sizeof(R)), *Py = (R *)calloc(n, sizeof(R)), *T11 = (R *)malloc(n * sizeof(R)),
      *T12 = (R *)malloc(n * sizeof(R)), *T21 = (R *)malloc(n * sizeof(R)), *T22 = (R *)malloc(n * sizeof(R));
    const R inv255 = (R)1 / (R)255;
    for (size_t i = 0; i < n; ++i) ref[i] = ref255[i] * inv255;
    FN(orc_tensor)(w, h, ref, beta, gamma, T11, T12, T21, T22);
    const R xscale = (R)1 / (zfar - znear);
    const R inputscale = (R)(-sigma_ / (double)(zfar - znear));
    for (size_t i = 0; i < n; ++i) {
        out[i] = (depth[i] + -znear) * xscale;
        raw[i] = (depth[i] + -znear) * inputscale;
    }
    const R tau = (R)tau_, theta = (R)theta_, lambda = (R)lambda_, sigma = (R)sigma_;
    for (int it = 0; it < niters; ++it) {
        const R cs = (R)(it == 0 ? 1 + sigma_ : sigma_);
        /* denoising_TVL1_calculateP_tensor_weighed_kernel, kernels.cu:283-307 */
        ORC_PAR
        for (int yy = 0; yy < h; ++yy)
            for (int xx = 0; xx < w; ++xx) {
                int i = yy * w + xx, xn = xx + 1 < w - 1 ? xx + 1 : w - 1, yn = yy + 1 < h - 1 ? yy + 1 : h - 1;
                double x = out[yy * w + xn] - out[i];
                double y = out[yn * w + xx] - out[i];
                double dx = Px[i] + cs * (T11[i] * x + T12[i] * y);
                double dy = Py[i] + cs * (T21[i] * x + T22[i] * y);
                double d = FMAXR(1, sqrt(dx * dx + dy * dy));
                Px[i] = (R)(dx / d);
                Py[i] = (R)(dy / d);
            }
        /* denoising_TVL1_update_kernel, kernels.cu:342-370 */
        ORC_PAR
        for (int yy = 0; yy < h; ++yy)
            for (int xx = 0; xx < w; ++xx) {
                int i = yy * w + xx, yp = yy - 1 < 0 ? 0 : yy - 1;
                double x_new;
                Rr[i] += raw[i];
                Rr[i] += sigma * out[i];
                if (Rr[i] > lambda) Rr[i] = lambda;
                if (Rr[i] < -lambda) Rr[i] = -lambda;
                if (xx == 0) x_new = out[i] + tau * (Py[i] - Py[yp * w + xx]) - tau * Rr[i];
                else x_new = out[i] + tau * (Px[i] - Px[i - 1] + Py[i] - Py[yp * w + xx]) - tau * Rr[i];
                out[i] = (R)(x_new + theta * (x_new - out[i]));
            }
    }
    for (size_t i = 0; i < n; ++i) out[i] = out[i] * (zfar - znear) + znear;
    free(ref); free(raw); free(Rr); free(Px); free(Py); free(T11); free(T12); free(T21); free(T22);
}

/* ---- fusion: fusion.cu:5-70, fusion.h:360-364,773-907, structs.h:212-284 ---- */

/* FusionUpdateHistogram_kernel + fusionData::updateHist.  hist holds `bins`
 * planes of vw*vh*vd counts (x fastest).  Voxels whose projection falls
 * outside [0, w-1] x [0, h-1] do not vote; there is no z > 0 test, as in the
 * reference. */
void FN(orc_fusion_histogram)(int bins, int vw, int vh, int vd, const float *a, const float *b, uint16_t *hist,
                              const float *depth, int w, int h, const R *K, const R *Rm, const R *t, double thr_)
{
    const size_t n = (size_t)vw * vh * vd;
    const R ax = (R)a[0], ay = (R)a[1], az = (R)a[2];
    const R sx = (R)b[0] - ax, sy = (R)b[1] - ay, sz = (R)b[2] - az;
    const R thr = bins == 2 ? 0 : (R)thr_;
    ORC_PAR
    for (int z = 0; z < vd; ++z)
        for (int y = 0; y < vh; ++y)
            for (int x = 0; x < vw; ++x) {
                R c[3] = {ax + sx * (R)((x + .5) / vw), ay + sy * (R)((y + .5) / vh), az + sz * (R)((z + .5) / vd)};
                R cc[3], kc[3];
                FN(matvec)(Rm, c, cc);
                for (int k = 0; k < 3; ++k) cc[k] = cc[k] + t[k];
                FN(matvec)(K, cc, kc);
                R px = kc[0] / kc[2], py = kc[1] / kc[2];
                if (px < 0 || px > (R)(w - 1) || py < 0 || py > (R)(h - 1)) continue;
                R fx = FLOORR(px), fy = FLOORR(py);
                int x0 = (int)FMAXR(fx, 0), y0 = (int)FMAXR(fy, 0);
                int x1 = (int)FMINR((R)(x0 + 1), (R)(w - 1)), y1 = (int)FMINR((R)(y0 + 1), (R)(h - 1));
                R frx = px - fx, fry = py - fy;
                R d00 = depth[x0 + y0 * w], d10 = depth[x1 + y0 * w];
                R d01 = depth[x0 + y1 * w], d11 = depth[x1 + y1 * w];
                /* bilinterp (dev_functions.h:33-38): lerp in y, then in x */
                R l0 = d00 + fry * (d01 - d00), l1 = d10 + fry * (d11 - d10);
                R dep = l0 + frx * (l1 - l0);
                R sd = dep - kc[2];
                size_t vi = (size_t)x + (size_t)vw * (y + (size_t)vh * z);
                int bin;
                if (sd >= thr) bin = bins - 1;
                else if (sd <= -thr) bin = 0;
                else {
                    R q = ROUNDR((sd + thr) / ((R)2 * thr) * (R)(bins - 3) + 1);
                    R m = FMINR(q, (R)(bins - 2));
                    bin = (int)(unsigned char)m;
                }
                hist[(size_t)bin * n + vi]++;
            }
}

/* FusionUpdateU_kernel (fusion.cu:45-57) with divPBwd (fusion.h:793-802) and
 * proxHist (fusion.h:851-858). p holds 3 planes (x, y, z components). */
void FN(orc_fusion_u)(int bins, int vw, int vh, int vd, const uint16_t *hist, R *u, R *v, const R *p,
                      double tau, double lambda)
{
    const size_t n = (size_t)vw * vh * vd, sy = vw, sz = (size_t)vw * vh;
    const R *px = p, *py = p + n, *pz = p + 2 * n;
    float centers[16];
    orc_bin_centers(bins, centers);
    ORC_PAR
    for (int z = 0; z < vd; ++z)
        for (int y = 0; y < vh; ++y)
            for (int x = 0; x < vw; ++x) {
                size_t i = x + sy * y + sz * z;
                R div = px[i] + py[i] + pz[i];
                if (x > 0) div -= px[i - 1];
                if (y > 0) div -= py[i - sy];
                if (z > 0) div -= pz[i - sz];
                const double un = u[i];
                const double uu = un - tau * (-(double)div);
                uint16_t hh[16];
                for (int k = 0; k < bins; ++k) hh[k] = hist[(size_t)k * n + i];
                R unew;
#if ORC_IS_F32
                unew = orc_prox_hist_f32(bins, hh, (float)uu, (float)tau, (float)lambda);
#else
                {
                    /* the same selection in double: values below the smallest
                     * element are raised to it, as the float insertion does.
                     * The median (rank N of the 2N+1 values) is taken by a
                     * merge of the sorted bin centres, the sorted proximal
                     * points u + tau lambda W_j and u itself. */
                    const double lo = centers[0];
                    double pts[16];
                    long W = 0;
                    for (int k = 1; k <= bins; ++k) W += hh[k - 1];
                    for (int j = 1; j <= bins; ++j) {
                        W -= 2 * (long)hh[j - 1];   /* W_j = -sum_{k<=j} h_k + sum_{k>j} h_k */
                        double pj = uu + tau * lambda * (double)W;
                        pj = pj < lo ? lo : pj;
                        int b1 = j - 1;
                        while (b1 > 0 && pts[b1 - 1] > pj) {
                            pts[b1] = pts[b1 - 1];
                            --b1;
                        }
                        pts[b1] = pj;
                    }
                    const double uc = uu < lo ? lo : uu;
                    int ia = 0, ib = 0, took_u = 0;
                    double cur = 0;
                    for (int k = 0; k <= bins; ++k) {
                        const double ca = ia < bins ? (double)centers[ia] : INFINITY;
                        const double cb = ib < bins ? pts[ib] : INFINITY;
                        const double cu = took_u ? INFINITY : uc;
                        if (ca <= cb && ca <= cu) cur = centers[ia++];
                        else if (cb <= cu) cur = pts[ib++];
                        else {
                            cur = cu;
                            took_u = 1;
                        }
                    }
                    unew = cur;
                }
#endif
                u[i] = unew;
                v[i] = (R)((double)(2 * unew) - un);
            }
}

/* FusionUpdateP_kernel (fusion.cu:59-70): p <- proj(p + sigma * gradVFwd),
 * gradVFwd zero at the far faces (fusion.h:773-781). */
void FN(orc_fusion_p)(int vw, int vh, int vd, const R *v, R *p, double sigma_)
{
    const size_t n = (size_t)vw * vh * vd, sy = vw, sz = (size_t)vw * vh;
    R *px = p, *py = p + n, *pz = p + 2 * n;
    const R sigma = (R)sigma_;
    ORC_PAR
    for (int z = 0; z < vd; ++z)
        for (int y = 0; y < vh; ++y)
            for (int x = 0; x < vw; ++x) {
                size_t i = x + sy * y + sz * z;
                R g[3] = {0, 0, 0};
                if (x < vw - 1) g[0] = v[i + 1] - v[i];
                if (y < vh - 1) g[1] = v[i + sy] - v[i];
                if (z < vd - 1) g[2] = v[i + sz] - v[i];
                R q[3] = {px[i] + sigma * g[0], py[i] + sigma * g[1], pz[i] + sigma * g[2]};
                R d = FMAXR(1, SQRTR(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]));
                px[i] = q[0] / d;
                py[i] = q[1] / d;
                pz[i] = q[2] / d;
            }
}

/* compute3D_kernel (kernels.cu:405-429): X = Rr (z K^-1 (x+1, y+1, 1)) + t
 * for z < 5.5, else z = -9. */
void FN(orc_compute3d)(int w, int h, const R *depth, const R *invK, const R *Rr, const R *t, R *X, R *Y, R *Z)
{
    ORC_PAR
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            int i = y * w + x;
            R z = depth[i];
            X[i] = 0;
            Y[i] = 0;
            if (z < (R)5.5) {
                R a[3] = {(R)(x + 1), (R)(y + 1), (R)1}, zk[9], b[3], c[3];
                for (int k = 0; k < 9; ++k) zk[k] = z * invK[k];
                FN(matvec)(zk, a, b);
                FN(matvec)(Rr, b, c);
                X[i] = c[0] + t[0];
                Y[i] = c[1] + t[1];
                Z[i] = c[2] + t[2];
            } else {
                Z[i] = -9;
            }
        }
}
