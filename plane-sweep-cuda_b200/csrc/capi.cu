// C ABI of libmvs_b200: argument checks, workspace carving and launches.
// The kernels live in sweep.cu, tgv2.cu, tvl1.cu and fusion.cu.
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <new>
#include <vector>

#include "common.cuh"

namespace mvs {

static thread_local char g_err[512] = "";

int set_error(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int check_launch(const char *what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(MVS_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return MVS_OK;
}

void clear_error() { g_err[0] = 0; }

// sweep.cu
int sweep_pick_chunks(int win, int w, int h, int V, int P, int mode);
int sweep_launch(const mvs_sweep_desc *d, const float *ref, const float *srcs, const float *H, const float *depths,
                 float *depth, int32_t *labels, float *best, uint16_t *cost, unsigned long long *scratch,
                 int n_chunks, void *stream, float4 *quad = nullptr);
size_t sweep_scratch_bytes(const mvs_sweep_desc *d);
size_t sweep_quad_bytes(const mvs_sweep_desc *d);
int sweep_wta_volume(const uint16_t *cost, const float *depths, int n, int P, float zfar, float *depth,
                     int32_t *labels, float *best, void *stream);
int sweep_homographies(const double *K, const double *invK, const double *Rrel, const double *trel,
                       const float *depths, int V, int P, float *H, void *stream);
// tgv2.cu
size_t tgv2_workspace_bytes(int w, int h, int V);
int tgv2_run(int w, int h, int V, const float *ref255, const float *srcs255, const float *K9, const float *invK9,
             const float *Rrel, const float *trel, const mvs_tgv2_params *prm, int u_from_input, float u_init,
             float *u, int *iters_out, double *energy_out, void *ws, cudaStream_t st,
             const TGV2Warm *warm = nullptr);
size_t tgv2_sparse_workspace_bytes(int w, int h);
int tgv2_sparse_run(int w, int h, const float *ref255, const float *depthmap, const float *sparse, float zfar,
                    int niters, double alpha0, double alpha1, double tau, double sigma, double beta, double gamma,
                    float *out, void *ws, cudaStream_t st);
// tvl1.cu
size_t tvl1_workspace_bytes(int w, int h);
int tvl1_run(int w, int h, const float *ref255, float *depth, float znear, float zfar, const mvs_tvl1_params *prm,
             void *ws, cudaStream_t st);
// fusion.cu
int fusion_hist_stride(int bins);
int fusion_histogram(int vw, int vh, int vd, int bins, const float *a, const float *b, uint16_t *hist,
                     const float *depths, int nmaps, int w, int h, const float *d_cams, float thr, cudaStream_t st);
int fusion_update_u(int vw, int vh, int vd, int bins, const uint16_t *hist, float *u, float *v, const float *p,
                    double tau, double lambda, cudaStream_t st);
int fusion_update_p(int vw, int vh, int vd, const float *v, float *p, double sigma, cudaStream_t st);
long fusion_extract_blocks(long n);
int fusion_extract(int vw, int vh, int vd, const float *a, const float *b, const float *u, float lo, float hi,
                   unsigned long long *d_counts, unsigned long long *h_counts, float *d_xyz, long capacity,
                   long *total, cudaStream_t st);

// ---- misc kernels ------------------------------------------------------------------

// compute3D_kernel (kernels.cu:405-429).
__global__ void compute3d_kernel(const float *__restrict__ depth, int w, int h, float ik0, float ik1, float ik2,
                                 float ik3, float ik4, float ik5, float ik6, float ik7, float ik8, float r0, float r1,
                                 float r2, float r3, float r4, float r5, float r6, float r7, float r8, float t0,
                                 float t1, float t2, float *__restrict__ X, float *__restrict__ Y,
                                 float *__restrict__ Z)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const int i = y * w + x;
    const float z = depth[i];
    if (z < 5.5) {
        // Rrel * (z * invK * (x+1, y+1, 1)) + trel: z scales the matrix first
        const float a = (float)(x + 1), b = (float)(y + 1);
        const float m0 = (z * ik0) * a + (z * ik1) * b + (z * ik2) * 1.f;
        const float m1 = (z * ik3) * a + (z * ik4) * b + (z * ik5) * 1.f;
        const float m2 = (z * ik6) * a + (z * ik7) * b + (z * ik8) * 1.f;
        X[i] = r0 * m0 + r1 * m1 + r2 * m2 + t0;
        Y[i] = r3 * m0 + r4 * m1 + r5 * m2 + t1;
        Z[i] = r6 * m0 + r7 * m1 + r8 * m2 + t2;
    } else {
        Z[i] = -9.f;
    }
}

}  // namespace mvs

using namespace mvs;

// ---- fusion handle ----------------------------------------------------------------

struct mvs_fusion {
    int w, h, d, bins, hs;
    float a[3], b[3];
    size_t n;
    float *u = nullptr, *v = nullptr, *p = nullptr;
    uint16_t *hist = nullptr;
    float *cams = nullptr;          // device, kMaxMaps * 21
    float *h_cams = nullptr;        // pinned staging
    unsigned long long *d_counts = nullptr, *h_counts = nullptr;
    float *d_xyz = nullptr;
    size_t xyz_cap = 0;
};

static constexpr int kMaxMaps = 64;

extern "C" {

const char *mvs_last_error(void) { return g_err; }

int mvs_version(void) { return 1 * 10000 + 0 * 100 + 0; }

// Page-locked allocations are tagged with a header so that a fall-back
// malloc (when page-locking fails) is freed the right way.
struct HostBlock {
    int pinned;
    int pad[3];
};

void *mvs_host_alloc(size_t bytes)
{
    void *p = nullptr;
    if (cudaMallocHost(&p, bytes + sizeof(HostBlock)) == cudaSuccess && p) {
        ((HostBlock *)p)->pinned = 1;
        return (char *)p + sizeof(HostBlock);
    }
    cudaGetLastError();
    p = malloc(bytes + sizeof(HostBlock));
    if (!p) return nullptr;
    ((HostBlock *)p)->pinned = 0;
    return (char *)p + sizeof(HostBlock);
}

void mvs_host_free(void *q)
{
    if (!q) return;
    HostBlock *b = (HostBlock *)((char *)q - sizeof(HostBlock));
    if (b->pinned) cudaFreeHost(b);
    else free(b);
}

int mvs_set_device(int device)
{
    clear_error();
    MVS_TRY_CUDA(cudaSetDevice(device));
    return MVS_OK;
}

// ---- sweep ----------------------------------------------------------------------------

}  // extern "C"

int mvs::check_sweep_desc(const mvs_sweep_desc *d)
{
    if (!d) return set_error(MVS_ERR_ARG, "null sweep descriptor");
    if (d->width <= 0 || d->height <= 0 || d->n_views <= 0 || d->n_planes <= 0)
        return set_error(MVS_ERR_ARG, "empty sweep (w=%d h=%d views=%d planes=%d)", d->width, d->height,
                         d->n_views, d->n_planes);
    if (d->window < 3 || d->window > 15 || !(d->window & 1))
        return set_error(MVS_ERR_ARG, "window %d must be odd, 3..15", d->window);
    if (d->width < d->window || d->height < d->window)
        return set_error(MVS_ERR_ARG, "image %dx%d smaller than the %d-pixel window", d->width, d->height, d->window);
    if (d->moments != MVS_MOMENTS_REFERENCE && d->moments != MVS_MOMENTS_COMPENSATED)
        return set_error(MVS_ERR_ARG, "unknown moments mode %d", d->moments);
    if (d->mode != MVS_SWEEP_PER_VIEW && d->mode != MVS_SWEEP_AGGREGATED)
        return set_error(MVS_ERR_ARG, "unknown sweep mode %d", d->mode);
    if ((long long)d->width * d->height > (1ll << 30)) return set_error(MVS_ERR_ARG, "image too large");
    // the aggregated mode keeps the running best as (bf16 cost << 16 | plane)
    if (d->mode == MVS_SWEEP_AGGREGATED && d->n_planes > 65535)
        return set_error(MVS_ERR_ARG, "aggregated mode: at most 65535 planes (%d)", d->n_planes);
    return MVS_OK;
}

extern "C" {

size_t mvs_sweep_workspace_bytes(const mvs_sweep_desc *d)
{
    if (check_sweep_desc(d)) return 0;
    // winner words, then the sources' 2x2 neighbourhoods
    return (sweep_scratch_bytes(d) + 255) / 256 * 256 + sweep_quad_bytes(d);
}

int mvs_sweep_homographies(const mvs_sweep_desc *d, const double *K, const double *Rrel, const double *trel,
                           const float *depths, float *H, void *stream)
{
    clear_error();
    if (int rc = check_sweep_desc(d)) return rc;
    if (!K || !Rrel || !trel || !depths || !H) return set_error(MVS_ERR_ARG, "null pointer");
    // K^-1 in double (adjugate / determinant)
    const double *m = K;
    const double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                       m[2] * (m[3] * m[7] - m[4] * m[6]);
    if (det == 0.0 || !isfinite(det)) return set_error(MVS_ERR_ARG, "K is singular");
    double inv[9] = {(m[4] * m[8] - m[5] * m[7]) / det, (m[2] * m[7] - m[1] * m[8]) / det,
                     (m[1] * m[5] - m[2] * m[4]) / det, (m[5] * m[6] - m[3] * m[8]) / det,
                     (m[0] * m[8] - m[2] * m[6]) / det, (m[2] * m[3] - m[0] * m[5]) / det,
                     (m[3] * m[7] - m[4] * m[6]) / det, (m[1] * m[6] - m[0] * m[7]) / det,
                     (m[0] * m[4] - m[1] * m[3]) / det};
    return sweep_homographies(K, inv, Rrel, trel, depths, d->n_views, d->n_planes, H, stream);
}

int mvs_sweep(const mvs_sweep_desc *d, const float *ref, const float *srcs, const float *H, const float *depths,
              float *depth, int32_t *labels, float *best, uint16_t *cost, void *ws, size_t ws_bytes, void *stream)
{
    clear_error();
    if (int rc = check_sweep_desc(d)) return rc;
    if (!ref || !srcs || !H || !depths || !depth) return set_error(MVS_ERR_ARG, "null input/output pointer");
    const size_t need = mvs_sweep_workspace_bytes(d);
    if (!ws || ws_bytes < need)
        return set_error(MVS_ERR_ARG, "workspace of %zu bytes needed, %zu given", need, ws ? ws_bytes : (size_t)0);
    if (((uintptr_t)ws) & 7) return set_error(MVS_ERR_ARG, "workspace must be 8-byte aligned");
    if (d->mode == MVS_SWEEP_PER_VIEW && cost) return set_error(MVS_ERR_ARG, "cost volume is an aggregated-mode output");
    const int chunks = sweep_pick_chunks(d->window, d->width, d->height, d->n_views, d->n_planes, d->mode);
    float4 *quad = (float4 *)((char *)ws + (sweep_scratch_bytes(d) + 255) / 256 * 256);
    return sweep_launch(d, ref, srcs, H, depths, depth, labels, best, cost, (unsigned long long *)ws, chunks, stream,
                        quad);
}

int mvs_sweep_wta_volume(const uint16_t *cost, const float *depths, int32_t n_pixels, int32_t n_planes, float zfar,
                         float *depth, int32_t *labels, float *best, void *stream)
{
    clear_error();
    if (!cost || !depths || !depth || n_pixels <= 0 || n_planes <= 0) return set_error(MVS_ERR_ARG, "bad argument");
    if (n_planes > 65535) return set_error(MVS_ERR_ARG, "at most 65535 planes in a cost volume");
    return sweep_wta_volume(cost, depths, n_pixels, n_planes, zfar, depth, labels, best, stream);
}

// ---- TGV2 -----------------------------------------------------------------------------

size_t mvs_tgv2_workspace_bytes(int32_t w, int32_t h, int32_t V)
{
    if (w <= 0 || h <= 0 || V <= 0) return 0;
    return tgv2_workspace_bytes(w, h, V);
}

int mvs_tgv2_run(int32_t w, int32_t h, int32_t V, const float *ref255, const float *srcs255, const float *K9,
                 const float *invK9, const float *Rrel, const float *trel, const mvs_tgv2_params *prm,
                 int32_t u_from_input, float u_init, float *u, int32_t *iters_out, double *energy_out, void *ws,
                 size_t ws_bytes, void *stream)
{
    clear_error();
    if (w < 2 || h < 2 || V <= 0) return set_error(MVS_ERR_ARG, "bad size %dx%d, %d views", w, h, V);
    if (!ref255 || !srcs255 || !K9 || !invK9 || !Rrel || !trel || !prm || !u) return set_error(MVS_ERR_ARG, "null pointer");
    if (prm->niters < 0 || prm->warps < 0) return set_error(MVS_ERR_ARG, "negative iteration count");
    const size_t need = tgv2_workspace_bytes(w, h, V);
    if (!ws || ws_bytes < need) return set_error(MVS_ERR_ARG, "workspace of %zu bytes needed", need);
    int it = 0;
    int rc = tgv2_run(w, h, V, ref255, srcs255, K9, invK9, Rrel, trel, prm, u_from_input, u_init, u, &it, energy_out,
                      ws, (cudaStream_t)stream);
    if (iters_out) *iters_out = it;
    return rc;
}

int mvs_tgv2_run_warm(int32_t w, int32_t h, int32_t V, const float *ref255, const float *srcs255, const float *K9,
                      const float *invK9, const float *Rrel, const float *trel, const mvs_tgv2_params *prm,
                      const float *u_lin, float *u, float *v, double dual_sigma, double dual_sigma_r,
                      float *pq, float *r, int32_t *iters_out,
                      double *energy_out, void *ws, size_t ws_bytes, void *stream)
{
    clear_error();
    if (w < 2 || h < 2 || V <= 0) return set_error(MVS_ERR_ARG, "bad size %dx%d, %d views", w, h, V);
    if (!ref255 || !srcs255 || !K9 || !invK9 || !Rrel || !trel || !prm || !u || !u_lin)
        return set_error(MVS_ERR_ARG, "null pointer");
    if (prm->niters < 0 || prm->warps < 0) return set_error(MVS_ERR_ARG, "negative iteration count");
    if (!(dual_sigma >= 0) || !(dual_sigma_r >= 0)) return set_error(MVS_ERR_ARG, "dual steps must be >= 0");
    const size_t need = tgv2_workspace_bytes(w, h, V);
    if (!ws || ws_bytes < need) return set_error(MVS_ERR_ARG, "workspace of %zu bytes needed", need);
    TGV2Warm warm{u_lin, v, dual_sigma, dual_sigma_r, pq, r};
    int it = 0;
    int rc = tgv2_run(w, h, V, ref255, srcs255, K9, invK9, Rrel, trel, prm, 1, 0.f, u, &it, energy_out, ws,
                      (cudaStream_t)stream, &warm);
    if (iters_out) *iters_out = it;
    return rc;
}

size_t mvs_tgv2_sparse_workspace_bytes(int32_t w, int32_t h)
{
    if (w <= 0 || h <= 0) return 0;
    return tgv2_sparse_workspace_bytes(w, h);
}

int mvs_tgv2_sparse(int32_t w, int32_t h, const float *ref255, const float *depthmap, const float *sparse, float zfar,
                    int32_t niters, double alpha0, double alpha1, double tau, double sigma, double theta, double beta,
                    double gamma, float *out, void *ws, size_t ws_bytes, void *stream)
{
    clear_error();
    (void)theta;   // enters only the over-relaxed u, which the iteration never reads
    if (w < 1 || h < 1) return set_error(MVS_ERR_ARG, "bad size %dx%d", w, h);
    if ((int64_t)w * h > INT32_MAX) return set_error(MVS_ERR_ARG, "image too large");
    if (!ref255 || !depthmap || !sparse || !out) return set_error(MVS_ERR_ARG, "null pointer");
    if (niters < 0) return set_error(MVS_ERR_ARG, "negative iteration count");
    if (!(zfar != 0.f)) return set_error(MVS_ERR_ARG, "zfar == 0");
    const size_t need = tgv2_sparse_workspace_bytes(w, h);
    if (!ws || ws_bytes < need) return set_error(MVS_ERR_ARG, "workspace of %zu bytes needed", need);
    return tgv2_sparse_run(w, h, ref255, depthmap, sparse, zfar, niters, alpha0, alpha1, tau, sigma, beta, gamma, out,
                           ws, (cudaStream_t)stream);
}

// ---- TV-L1 ------------------------------------------------------------------------------

size_t mvs_tvl1_workspace_bytes(int32_t w, int32_t h)
{
    if (w <= 0 || h <= 0) return 0;
    return tvl1_workspace_bytes(w, h);
}

int mvs_tvl1_denoise(int32_t w, int32_t h, const float *ref255, float *depth, float znear, float zfar,
                     const mvs_tvl1_params *prm, void *ws, size_t ws_bytes, void *stream)
{
    clear_error();
    if (w < 2 || h < 2) return set_error(MVS_ERR_ARG, "bad size %dx%d", w, h);
    if (!ref255 || !depth || !prm) return set_error(MVS_ERR_ARG, "null pointer");
    if (!(zfar != znear)) return set_error(MVS_ERR_ARG, "znear == zfar");
    const size_t need = tvl1_workspace_bytes(w, h);
    if (!ws || ws_bytes < need) return set_error(MVS_ERR_ARG, "workspace of %zu bytes needed", need);
    return tvl1_run(w, h, ref255, depth, znear, zfar, prm, ws, (cudaStream_t)stream);
}

// ---- compute3D ----------------------------------------------------------------------------

int mvs_compute3d(int32_t w, int32_t h, const float *depth, const float *ik, const float *R, const float *t, float *X,
                  float *Y, float *Z, void *stream)
{
    clear_error();
    if (w <= 0 || h <= 0 || !depth || !ik || !R || !t || !X || !Y || !Z) return set_error(MVS_ERR_ARG, "bad argument");
    if (Z != depth)
        MVS_TRY_CUDA(cudaMemcpyAsync(Z, depth, sizeof(float) * (size_t)w * h, cudaMemcpyDeviceToDevice,
                                     (cudaStream_t)stream));
    dim3 b(32, 8), g(ceil_div(w, 32), ceil_div(h, 8));
    compute3d_kernel<<<g, b, 0, (cudaStream_t)stream>>>(Z, w, h, ik[0], ik[1], ik[2], ik[3], ik[4], ik[5], ik[6],
                                                         ik[7], ik[8], R[0], R[1], R[2], R[3], R[4], R[5], R[6], R[7],
                                                         R[8], t[0], t[1], t[2], X, Y, Z);
    return check_launch("compute3d_kernel");
}

// ---- fusion ---------------------------------------------------------------------------------

int mvs_fusion_create(int32_t w, int32_t h, int32_t d, int32_t bins, const float *a, const float *b, mvs_fusion **out)
{
    clear_error();
    if (!out) return set_error(MVS_ERR_ARG, "null output");
    *out = nullptr;
    if (w <= 0 || h <= 0 || d <= 0) return set_error(MVS_ERR_ARG, "empty volume");
    if (bins < 2 || bins > 10) return set_error(MVS_ERR_ARG, "bins %d not supported (2..10)", bins);
    if (!a || !b) return set_error(MVS_ERR_ARG, "null volume corner");
    mvs_fusion *f = new (std::nothrow) mvs_fusion;
    if (!f) return set_error(MVS_ERR_NOMEM, "host allocation failed");
    f->w = w;
    f->h = h;
    f->d = d;
    f->bins = bins;
    f->hs = fusion_hist_stride(bins);
    memcpy(f->a, a, sizeof(f->a));
    memcpy(f->b, b, sizeof(f->b));
    f->n = (size_t)w * h * d;
    cudaError_t e = cudaMalloc(&f->u, f->n * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&f->v, f->n * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&f->p, 3 * f->n * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&f->hist, f->n * f->hs * sizeof(uint16_t));
    if (e == cudaSuccess) e = cudaMalloc(&f->cams, kMaxMaps * kMapCamFloats * sizeof(float));
    if (e == cudaSuccess) e = cudaMallocHost(&f->h_cams, kMaxMaps * kMapCamFloats * sizeof(float));
    const long nb = fusion_extract_blocks((long)f->n);
    if (e == cudaSuccess) e = cudaMalloc(&f->d_counts, nb * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMallocHost(&f->h_counts, nb * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        mvs_fusion_destroy(f);
        return set_error(MVS_ERR_NOMEM, "fusion volume allocation: %s", cudaGetErrorString(e));
    }
    int rc = mvs_fusion_reset(f, nullptr);
    if (rc == MVS_OK) rc = cudaDeviceSynchronize() == cudaSuccess ? MVS_OK : set_error(MVS_ERR_CUDA, "reset failed");
    if (rc) {
        mvs_fusion_destroy(f);
        return rc;
    }
    *out = f;
    return MVS_OK;
}

int mvs_fusion_destroy(mvs_fusion *f)
{
    if (!f) return MVS_OK;
    cudaFree(f->u);
    cudaFree(f->v);
    cudaFree(f->p);
    cudaFree(f->hist);
    cudaFree(f->cams);
    cudaFreeHost(f->h_cams);
    cudaFree(f->d_counts);
    cudaFreeHost(f->h_counts);
    cudaFree(f->d_xyz);
    delete f;
    return MVS_OK;
}

int mvs_fusion_set_volume(mvs_fusion *f, const float *a, const float *b)
{
    clear_error();
    if (!f || !a || !b) return set_error(MVS_ERR_ARG, "null argument");
    memcpy(f->a, a, sizeof(f->a));
    memcpy(f->b, b, sizeof(f->b));
    return MVS_OK;
}

int mvs_fusion_reset(mvs_fusion *f, void *stream)
{
    clear_error();
    if (!f) return set_error(MVS_ERR_ARG, "null volume");
    cudaStream_t st = (cudaStream_t)stream;
    MVS_TRY_CUDA(cudaMemsetAsync(f->u, 0, f->n * sizeof(float), st));
    MVS_TRY_CUDA(cudaMemsetAsync(f->v, 0, f->n * sizeof(float), st));
    MVS_TRY_CUDA(cudaMemsetAsync(f->p, 0, 3 * f->n * sizeof(float), st));
    MVS_TRY_CUDA(cudaMemsetAsync(f->hist, 0, f->n * f->hs * sizeof(uint16_t), st));
    return MVS_OK;
}

int mvs_fusion_histogram(mvs_fusion *f, const float *depths, int32_t n_maps, int32_t w, int32_t h, const float *K,
                         const float *R, const float *t, float thr, void *stream)
{
    clear_error();
    if (!f || !depths || !K || !R || !t || n_maps < 0 || w < 2 || h < 2) return set_error(MVS_ERR_ARG, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    for (int m0 = 0; m0 < n_maps; m0 += kMaxMaps) {
        const int nm = std::min(kMaxMaps, n_maps - m0);
        // the staging buffer may still feed a copy of the previous batch
        MVS_TRY_CUDA(cudaStreamSynchronize(st));
        for (int m = 0; m < nm; ++m) {
            float *c = f->h_cams + kMapCamFloats * m;
            memcpy(c, K + 9 * (m0 + m), 9 * sizeof(float));
            memcpy(c + 9, R + 9 * (m0 + m), 9 * sizeof(float));
            memcpy(c + 18, t + 3 * (m0 + m), 3 * sizeof(float));
        }
        MVS_TRY_CUDA(cudaMemcpyAsync(f->cams, f->h_cams, nm * kMapCamFloats * sizeof(float), cudaMemcpyHostToDevice, st));
        int rc = fusion_histogram(f->w, f->h, f->d, f->bins, f->a, f->b, f->hist, depths + (size_t)m0 * w * h, nm, w, h,
                                  f->cams, thr, st);
        if (rc) return rc;
    }
    return MVS_OK;
}

int mvs_fusion_update_u(mvs_fusion *f, double tau, double lambda, void *stream)
{
    clear_error();
    if (!f) return set_error(MVS_ERR_ARG, "null volume");
    return fusion_update_u(f->w, f->h, f->d, f->bins, f->hist, f->u, f->v, f->p, tau, lambda, (cudaStream_t)stream);
}

int mvs_fusion_update_p(mvs_fusion *f, double sigma, void *stream)
{
    clear_error();
    if (!f) return set_error(MVS_ERR_ARG, "null volume");
    return fusion_update_p(f->w, f->h, f->d, f->v, f->p, sigma, (cudaStream_t)stream);
}

int mvs_fusion_tvl1(mvs_fusion *f, int32_t n_iters, double tau, double lambda, double sigma, void *stream)
{
    clear_error();
    if (!f || n_iters < 0) return set_error(MVS_ERR_ARG, "bad argument");
    for (int k = 0; k < n_iters; ++k) {
        int rc = fusion_update_u(f->w, f->h, f->d, f->bins, f->hist, f->u, f->v, f->p, tau, lambda,
                                 (cudaStream_t)stream);
        if (!rc) rc = fusion_update_p(f->w, f->h, f->d, f->v, f->p, sigma, (cudaStream_t)stream);
        if (rc) return rc;
    }
    return MVS_OK;
}

int mvs_fusion_iteration(mvs_fusion *f, const float *depth, int32_t w, int32_t h, const float *K, const float *R,
                         const float *t, float thr, double tau, double lambda, double sigma, void *stream)
{
    int rc = mvs_fusion_histogram(f, depth, 1, w, h, K, R, t, thr, stream);
    if (!rc) rc = mvs_fusion_update_u(f, tau, lambda, stream);
    if (!rc) rc = mvs_fusion_update_p(f, sigma, stream);
    return rc;
}

int mvs_fusion_download(mvs_fusion *f, float *u, float *v, float *p, uint16_t *hist)
{
    clear_error();
    if (!f) return set_error(MVS_ERR_ARG, "null volume");
    MVS_TRY_CUDA(cudaDeviceSynchronize());
    if (u) MVS_TRY_CUDA(cudaMemcpy(u, f->u, f->n * sizeof(float), cudaMemcpyDeviceToHost));
    if (v) MVS_TRY_CUDA(cudaMemcpy(v, f->v, f->n * sizeof(float), cudaMemcpyDeviceToHost));
    if (p) MVS_TRY_CUDA(cudaMemcpy(p, f->p, 3 * f->n * sizeof(float), cudaMemcpyDeviceToHost));
    if (hist) {
        // [n][hs] on the device -> one plane per bin on the host
        std::vector<uint16_t> tmp;
        try {
            tmp.resize(f->n * f->hs);
        } catch (...) {
            return set_error(MVS_ERR_NOMEM, "host allocation failed");
        }
        MVS_TRY_CUDA(cudaMemcpy(tmp.data(), f->hist, tmp.size() * sizeof(uint16_t), cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < f->n; ++i)
            for (int k = 0; k < f->bins; ++k) hist[(size_t)k * f->n + i] = tmp[i * f->hs + k];
    }
    return MVS_OK;
}

int mvs_fusion_upload(mvs_fusion *f, const float *u, const float *v, const float *p, const uint16_t *hist)
{
    clear_error();
    if (!f) return set_error(MVS_ERR_ARG, "null volume");
    MVS_TRY_CUDA(cudaDeviceSynchronize());
    if (u) MVS_TRY_CUDA(cudaMemcpy(f->u, u, f->n * sizeof(float), cudaMemcpyHostToDevice));
    if (v) MVS_TRY_CUDA(cudaMemcpy(f->v, v, f->n * sizeof(float), cudaMemcpyHostToDevice));
    if (p) MVS_TRY_CUDA(cudaMemcpy(f->p, p, 3 * f->n * sizeof(float), cudaMemcpyHostToDevice));
    if (hist) {
        std::vector<uint16_t> tmp;
        try {
            tmp.assign(f->n * f->hs, 0);
        } catch (...) {
            return set_error(MVS_ERR_NOMEM, "host allocation failed");
        }
        for (size_t i = 0; i < f->n; ++i)
            for (int k = 0; k < f->bins; ++k) tmp[i * f->hs + k] = hist[(size_t)k * f->n + i];
        MVS_TRY_CUDA(cudaMemcpy(f->hist, tmp.data(), tmp.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
    }
    return MVS_OK;
}

int mvs_fusion_device_state(mvs_fusion *f, float **u, float **v, float **p, uint16_t **hist, int32_t *hs)
{
    clear_error();
    if (!f) return set_error(MVS_ERR_ARG, "null volume");
    if (u) *u = f->u;
    if (v) *v = f->v;
    if (p) *p = f->p;
    if (hist) *hist = f->hist;
    if (hs) *hs = f->hs;
    return MVS_OK;
}

int mvs_fusion_extract(mvs_fusion *f, float lo, float hi, float *h_xyz, int64_t capacity, int64_t *count)
{
    clear_error();
    if (!f || !count || capacity < 0 || (capacity > 0 && !h_xyz)) return set_error(MVS_ERR_ARG, "bad argument");
    if ((size_t)capacity > f->xyz_cap) {
        cudaFree(f->d_xyz);
        f->d_xyz = nullptr;
        f->xyz_cap = 0;
        MVS_TRY_CUDA(cudaMalloc(&f->d_xyz, 3 * (size_t)capacity * sizeof(float)));
        f->xyz_cap = (size_t)capacity;
    }
    long total = 0;
    int rc = fusion_extract(f->w, f->h, f->d, f->a, f->b, f->u, lo, hi, f->d_counts, f->h_counts,
                            capacity > 0 ? f->d_xyz : nullptr, (long)capacity, &total, nullptr);
    if (rc) return rc;
    *count = total;
    const long m = std::min<long>(total, (long)capacity);
    if (m > 0) MVS_TRY_CUDA(cudaMemcpy(h_xyz, f->d_xyz, 3 * (size_t)m * sizeof(float), cudaMemcpyDeviceToHost));
    return MVS_OK;
}

}  // extern "C"
