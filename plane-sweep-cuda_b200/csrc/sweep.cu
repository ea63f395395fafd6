// Fused plane sweep for sm_100a.
//
// One CTA owns a TW x 32 tile of reference pixels for one source view (or,
// in the aggregated mode, for all views) and walks a chunk of planes.  Per
// plane it
//   A0  warps the source over the tile plus its window halo into shared
//       memory (homography + bilinear, the arithmetic of
//       transform_indexes_kernel / bilinear_interpolation_kernel_GPU,
//       kernels.cu:4-44; mirrored halo as windowed_mean_*, kernels.cu:203-229),
//   A1  forms per-column window sums of w, w^2 and ref*w (72 columns x 3
//       strips of 11 rows, one per thread),
//   B   forms the row sums, the NCC (calcNCC_kernel, kernels.cu:46-64) and
//       keeps the running best per pixel in registers (update_arrays_kernel,
//       kernels.cu:66-82: strictly greater wins, so ties keep the earlier
//       plane and NCC <= 0 never wins).
// This replaces the reference's 12 full-image launches per plane and view
// (planesweep.cpp:205-249) with two barriers per plane and view and no HBM
// traffic except the source gathers (L1/L2 resident) and the results (one
// word per pixel; in the aggregated mode also the BF16 cost per pixel and
// plane, written as 16-byte runs).
//
// Moments:
//   MVS_MOMENTS_REFERENCE   the reference's box means (column pass then row
//                           pass, each sum divided by the window side), its
//                           naive std and NCC formula, in its operation order;
//                           with -fmad=false the results are the reference's
//                           roundings exactly.
//   MVS_MOMENTS_COMPENSATED window sums of values shifted by a per-tile
//                           constant (the mean of the tile's reference region),
//                           kept as sliding sums and combined as n*Sxx - Sx^2
//                           with a fused multiply-add, so the variance does not
//                           cancel catastrophically.  A window whose n*Sxx - Sx^2
//                           is within the rounding bound of the sums
//                           (kappa * Sxx) counts as flat (std 0): constant
//                           windows, such as the zero fill outside the source,
//                           then give NCC 0 exactly as in exact arithmetic.
#include <cuda.h>            // CUtensorMap
#include <cudaTypedefs.h>    // PFN_cuTensorMapEncodeTiled
#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#include "common.cuh"
#include "div_win.cuh"

namespace mvs {
namespace {

constexpr int THREADS = 256;
constexpr int TH = 32;        // output rows per tile
constexpr int RWMAX = 72;     // region columns held in shared memory
constexpr int RHMAX = TH + 15;   // region rows of the largest window (15), plus the row the last A1 strip reads past it
// Row pitch of the column-sum and moment arrays.  Pass B gives the 8 lanes of
// a quarter warp 8 consecutive rows at one column: 76 = 12 (mod 32) floats
// puts their 16-byte words on 8 distinct groups of 4 banks.
constexpr int CSP = 76;
constexpr int STRIP = 11;     // output rows per pass-A1 thread (the last strip has 10)

// TWS narrows the tile by 8 output columns per step (the batched sweep's
// autotuner picks it; every other launch uses the widest tile, TWS = 0).
template <int WIN, int TWS = 0>
struct Geo {
    static constexpr int R = WIN / 2;
    static constexpr int TW = ((RWMAX - 2 * R) / 8 - TWS) * 8;  // output columns: 64 up to 9x9, 56 above
    static constexpr int RUN = TW / 8;                     // outputs per thread in pass B
    static constexpr int RW = TW + 2 * R;                  // region columns used
    static constexpr int RH = TH + 2 * R;                  // region rows
    // passes A0 / A1: three threads per region column (216 of the 256 at
    // 72 columns); A0 thread (c, s) warps rows s, s + 3, ...; A1 thread
    // (c, s) forms the column sums of output rows [11 s, 11 s + 11)
    static constexpr int COLT = 3 * RW;
    static constexpr int A0ROWS = (RH + 2) / 3;
    static constexpr int SROWS = STRIP + 2 * R;            // region rows per pass-A1 strip
    static_assert(RW <= RWMAX && RH <= RHMAX && COLT <= THREADS, "region too large");
    static_assert(3 * STRIP >= TH && 2 * STRIP < TH, "three strips cover the tile");
    static_assert(2 * STRIP + SROWS <= RHMAX, "strip reads stay inside the region arrays");
};

// pass B thread -> (output row, run of RUN columns): the 8 lanes of a
// quarter warp take 8 consecutive rows of one run, so their 16-byte loads
// of a run fall on distinct banks (CSP above); a warp stores 8 rows x 32
// contiguous cost values.
__device__ __forceinline__ int b_row() { return (int)(threadIdx.x & 7) + 8 * (int)(threadIdx.x >> 6); }
__device__ __forceinline__ int b_seg() { return (int)(threadIdx.x >> 3) & 7; }

struct SweepArgs {
    const float *ref;
    const float *srcs;
    const float *H;        // [V][P][9]
    const float *depths;   // [P]
    int w, h, V, P;
    int planes_per_chunk;
    int n_chunks;
    float stdthresh;
    unsigned long long *packed;   // PER_VIEW: [V][n] best (ncc bits << 32 | ~plane)
    unsigned long long *wta;      // AGGREGATED: [n] (cost bits << 32 | plane)
    uint16_t *cost;               // AGGREGATED: [P][n] bf16 or null
    const float4 *quad;           // AGGREGATED: [V][n] 2x2 neighbourhoods of the sources, or null
    int *err;                     // TMA-staged form: set when a staging wait gave up
};

// ---- pass A0: warp the region into shared memory ------------------------------

// Thread (c, s) = (t % RW, t / RW) always owns region column c and rows s + 3k,
// so its pixel column X and its pixel rows Y_k (mirrored at the image border)
// are fixed for the whole CTA: the rows sit in shared memory (Yc), and per
// plane only the X-dependent part of H*(X, Y, 1) is formed once (COMPENSATED;
// the REFERENCE path keeps the reference's dot-product order).  Cells are processed in
// batches -- coordinates, then all gathers, then the interpolation -- so each
// thread keeps several independent L1/L2 gathers in flight.

// ---- pass B: row sums of one column-sum array --------------------------------------

// The RUN + 2R column sums that thread (b_row, b_seg) reads: 16-byte loads
// when a run is a multiple of 4 (the rows sit at a 16-byte pitch and the runs
// start on multiples of 8 floats; the last word may reach past the region's
// used columns into the row's padding, whose values are never used).
template <int N, int RUN>
__device__ __forceinline__ void load_run(const float *row, float *v)
{
    if constexpr (RUN % 4 == 0) {
        const float4 *q = reinterpret_cast<const float4 *>(row);
#pragma unroll
        for (int i = 0; i < (N + 3) / 4; ++i) {
            const float4 f = q[i];
            v[4 * i] = f.x;
            if (4 * i + 1 < N) v[4 * i + 1] = f.y;
            if (4 * i + 2 < N) v[4 * i + 2] = f.z;
            if (4 * i + 3 < N) v[4 * i + 3] = f.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) v[i] = row[i];
    }
}

template <int WIN, int MOM, int TWS = 0>
__device__ __forceinline__ void row_sums(const float (*CSq)[CSP], float *out)
{
    using G = Geo<WIN, TWS>;
    constexpr int NV = G::RUN + 2 * G::R;
    static_assert(G::RUN % 4 != 0 || 7 * G::RUN + 4 * ((NV + 3) / 4) <= CSP, "run loads stay inside a row");
    float v[NV];
    load_run<NV, G::RUN>(CSq[b_row()] + b_seg() * G::RUN, v);
    if (MOM == MVS_MOMENTS_REFERENCE) {
        // windowed_mean_row_kernel: direct sum in window order, then / winsize
#pragma unroll
        for (int j = 0; j < G::RUN; ++j) {
            float m = 0.f;
#pragma unroll
            for (int i = 0; i < WIN; ++i) m = m + v[j + i];
            out[j] = div_win<WIN>(m);
        }
    } else {
        float m = v[0];
#pragma unroll
        for (int i = 1; i < WIN; ++i) m += v[i];
        out[0] = m;
#pragma unroll
        for (int j = 1; j < G::RUN; ++j) {
            m = (m + v[j + WIN - 1]) - v[j - 1];
            out[j] = m;
        }
    }
}

// Rounding bound of n*Sxx - Sx^2 for the compensated sums, as a multiple of
// Sxx: about 3 n eps per addition, with WIN + 2 (STRIP - 1) additions along
// a column strip and WIN + 2 (RUN - 1) along a row run.  Windows at or below
// it count as flat.
template <int WIN, int TWS = 0>
__device__ __forceinline__ constexpr float flat_kappa()
{
    return 3.f * (float)(WIN * WIN) * (float)(2 * WIN + 2 * (STRIP - 1) + 2 * (Geo<WIN, TWS>::RUN - 1)) * 5.9604645e-8f;
}

// Reference moments of the tile, once per CTA: in REFERENCE mode the mean and
// the naive std (calculate_STD_kernel, kernels.cu:103-120) of the reference
// window; in COMPENSATED mode the shifted sum and n*Syy - Sy^2 (0 if flat),
// or +inf where that is below (st n)^2: the reference window's std is under
// the threshold, and ncc_of's rsqrt(n^2 var_w * inf) = 0 then gives NCC 0
// without a test per view and plane (st > 0; with st = 0 nothing changes).
template <int WIN, int MOM, int TWS = 0>
__device__ void ref_moments(const float (*Rt)[RWMAX], float (*CS)[TH][CSP], float shift, float st, float (*RM)[CSP],
                            float (*RS)[CSP])
{
    using G = Geo<WIN, TWS>;
    if (threadIdx.x < G::COLT) {
        const int c = threadIdx.x % G::RW, s = threadIdx.x / G::RW;
        const int r0 = STRIP * s;
#pragma unroll
        for (int k = 0; k < STRIP; ++k) {
            if (r0 + k >= TH) break;
            float s1 = 0.f, s2 = 0.f;
#pragma unroll
            for (int i = 0; i < WIN; ++i) {
                if (MOM == MVS_MOMENTS_REFERENCE) {
                    const float x = Rt[r0 + k + i][c];
                    s1 = s1 + x;
                    s2 = s2 + x * x;
                } else {
                    const float x = Rt[r0 + k + i][c] - shift;
                    s1 += x;
                    s2 = fmaf(x, x, s2);
                }
            }
            if (MOM == MVS_MOMENTS_REFERENCE) {
                s1 = div_win<WIN>(s1);
                s2 = div_win<WIN>(s2);
            }
            CS[0][r0 + k][c] = s1;
            CS[1][r0 + k][c] = s2;
        }
    }
    __syncthreads();
    float m[G::RUN], q[G::RUN];
    row_sums<WIN, MOM, TWS>(CS[0], m);
    row_sums<WIN, MOM, TWS>(CS[1], q);
    const int y = b_row(), x = b_seg() * G::RUN;
#pragma unroll
    for (int j = 0; j < G::RUN; ++j) {
        if (MOM == MVS_MOMENTS_REFERENCE) {
            const float var = q[j] - m[j] * m[j];
            RM[y][x + j] = m[j];
            RS[y][x + j] = var > 0 ? sqrtf(var) : 0.f;
        } else {
            const float v = fmaf(-m[j], m[j], (float)(WIN * WIN) * q[j]);   // n^2 * var
            const float rs = v > flat_kappa<WIN, TWS>() * q[j] ? v : 0.f;
            const float thr = st * (float)(WIN * WIN);
            RM[y][x + j] = m[j];
            RS[y][x + j] = rs >= thr * thr ? rs : INFINITY;
        }
    }
    __syncthreads();
}

template <int WIN, int MOM, int TWS = 0>
__device__ __forceinline__ float ncc_of(float s1, float s2, float s12, float rm, float rs, float st)
{
    if (MOM == MVS_MOMENTS_REFERENCE) {
        const float var = s2 - s1 * s1;
        const float sd = var > 0 ? sqrtf(var) : 0.f;
        if (rs < st || sd < st) return 0.f;
        return (s12 - rm * s1) / (rs * sd);
    } else {
        constexpr float n = (float)(WIN * WIN);
        const float vx = fmaf(-s1, s1, n * s2);         // n^2 var_w
        const float cv = fmaf(-s1, rm, n * s12);        // n^2 cov
        const float thr = st * n;                        // std >= st  <=>  n^2 var >= (st n)^2
        // rs is +inf where the reference window is under the threshold
        // (ref_moments): vx > 0 here, so the product is +inf and the NCC 0
        if (!(vx >= thr * thr) || !(vx > flat_kappa<WIN, TWS>() * s2)) return 0.f;
        return cv * rsqrtf(vx * rs);
    }
}

// The NCC of a run of RUN outputs against the reference moments, which are
// read in groups of four (one 16-byte load each when RUN is a multiple of 4),
// so at most four of them are live at a time.
template <int WIN, int MOM, int TWS, typename F>
__device__ __forceinline__ void ncc_run(const float *s1, const float *s2, const float *s12, const float *rmrow,
                                        const float *rsrow, float st, F &&use)
{
    using G = Geo<WIN, TWS>;
#pragma unroll
    for (int j0 = 0; j0 < G::RUN; j0 += 4) {
        float rm[4], rs[4];
        if constexpr (G::RUN % 4 == 0) {
            const float4 a = *reinterpret_cast<const float4 *>(rmrow + j0);
            const float4 b = *reinterpret_cast<const float4 *>(rsrow + j0);
            rm[0] = a.x, rm[1] = a.y, rm[2] = a.z, rm[3] = a.w;
            rs[0] = b.x, rs[1] = b.y, rs[2] = b.z, rs[3] = b.w;
        } else {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                rm[i] = j0 + i < G::RUN ? rmrow[j0 + i] : 0.f;
                rs[i] = j0 + i < G::RUN ? rsrow[j0 + i] : 0.f;
            }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (j0 + i < G::RUN) use(j0 + i, ncc_of<WIN, MOM, TWS>(s1[j0 + i], s2[j0 + i], s12[j0 + i], rm[i], rs[i], st));
    }
}

// Shared-memory layout of one CTA.
struct __align__(16) Smem {
    float Wt[RHMAX][RWMAX];        // warped region (reference region at start)
    float CS[3][TH][CSP];          // column sums
    float Hm[2][12];               // homographies of this and the next (plane, view): 9 used, 16-byte rows
    float red[THREADS / 32];
};

// the nine elements of a homography row of Smem::Hm: three 16-byte loads
__device__ __forceinline__ void load_hm(const float *row, float *Hm)
{
    const float4 a = reinterpret_cast<const float4 *>(row)[0], b = reinterpret_cast<const float4 *>(row)[1];
    const float c = row[8];
    Hm[0] = a.x, Hm[1] = a.y, Hm[2] = a.z, Hm[3] = a.w;
    Hm[4] = b.x, Hm[5] = b.y, Hm[6] = b.z, Hm[7] = b.w;
    Hm[8] = c;
}

template <int WIN, int MOM, int TWS = 0>
__device__ __forceinline__ void load_ref_region(Smem &S, const float *__restrict__ ref, int w, int h, int x0,
                                                int y0)
{
    using G = Geo<WIN, TWS>;
    for (int i = threadIdx.x; i < G::RH * RWMAX; i += THREADS) {
        const int ry = i / RWMAX, rx = i % RWMAX;
        if (rx >= G::RW) continue;
        S.Wt[ry][rx] = ldg(ref + (size_t)mirror_idx(y0 - G::R + ry, h) * w + mirror_idx(x0 - G::R + rx, w));
    }
}

// Shift of the compensated sums: the mean of the tile's reference region
// (block reduction; every thread returns the same value).  0 in REFERENCE mode.
template <int WIN, int MOM, int TWS = 0>
__device__ __forceinline__ float tile_shift(Smem &S)
{
    using G = Geo<WIN, TWS>;
    if (MOM == MVS_MOMENTS_REFERENCE) return 0.f;
    float acc = 0.f;
    for (int i = threadIdx.x; i < G::RH * RWMAX; i += THREADS) {
        const int ry = i / RWMAX, rx = i % RWMAX;
        if (rx < G::RW) acc += S.Wt[ry][rx];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) S.red[threadIdx.x >> 5] = acc;
    __syncthreads();
    float t = 0.f;
#pragma unroll
    for (int k = 0; k < THREADS / 32; ++k) t += S.red[k];
    return t / (float)(G::RH * G::RW);
}

// ---- aggregated mode: cost = 1 - mean NCC over views, BF16 WTA -------------------
//
// The per-CTA state that the per-view kernel keeps in registers -- the
// reference column of pass A1, the region row coordinates of pass A0 and the
// reference moments of pass B -- lives in shared memory here (AggSmem), and
// the running best cost and plane are one 32-bit key (bf16 cost bits << 16 |
// plane: non-negative bf16 values order like integers, and equal costs keep
// the earlier plane), so the kernel fits three CTAs per SM.  The arithmetic is
// the per-view kernel's.

struct __align__(16) AggSmem {
    Smem S;
    float Rf[RHMAX][RWMAX];     // reference region (shifted in the compensated mode)
    // reference window sums / means and n^2 var / std per output pixel, at
    // the CSP pitch and 16-byte aligned: pass B reads them as it reads CS
    float RM[TH][CSP];
    float RS[TH][CSP];
    float Yc[RHMAX];            // region row coordinates (1-based, mirrored)
};
// three CTAs per SM: 228 KB of shared memory, 1 KB of it reserved per CTA
static_assert(3 * (sizeof(AggSmem) + 1024) <= 228 * 1024, "three CTAs per SM");
static_assert(offsetof(AggSmem, RM) % 16 == 0 && offsetof(AggSmem, RS) % 16 == 0 &&
                  offsetof(AggSmem, S.CS) % 16 == 0 && offsetof(AggSmem, S.Hm) % 16 == 0 &&
                  (CSP * sizeof(float)) % 16 == 0,
              "16-byte run loads");

// Each source pixel's 2x2 bilinear neighbourhood (x, x+1 on rows y, y+1) as
// one aligned 16-byte word, so that a warp sample is one load instead of four.
// Plain form (REFERENCE moments): the four values d00, d01, d10, d11, so the
// reference's interpolation arithmetic is unchanged.  Difference form
// (COMPENSATED): d00, d01 - d00, d10 - d00 and (d11 - d10) - (d01 - d00),
// so the sample is d00 + a (d01 - d00) + b ((d10 - d00) + a (...)): three
// fused multiply-adds.  Only x <= w-2, y <= h-2 are ever read; the last row
// and column hold zeros.
__device__ __forceinline__ float4 make_quad(const float *r, int w, bool diff)
{
    const float d00 = r[0], d01 = r[1], d10 = r[w], d11 = r[w + 1];
    if (!diff) return make_float4(d00, d01, d10, d11);
    return make_float4(d00, d01 - d00, d10 - d00, (d11 - d10) - (d01 - d00));
}

// make_quad's difference form from four values already in registers
__device__ __forceinline__ float4 make_quad4(float d00, float d01, float d10, float d11)
{
    return make_float4(d00, d01 - d00, d10 - d00, (d11 - d10) - (d01 - d00));
}

__global__ void quad_kernel(const float *__restrict__ src, int V, int w, int h, float4 *__restrict__ quad, int diff)
{
    const size_t n = (size_t)w * h, total = n * V;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t v = i / n, k = i - v * n;
        const int y = (int)(k / w), x = (int)(k - (size_t)y * w);
        float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
        if (x < w - 1 && y < h - 1) q = make_quad(src + v * n + k, w, diff != 0);
        quad[i] = q;
    }
}

// the same for every frame of a batch: grid (blocks, frames)
__global__ void quad_batch_kernel(const BatchFrameDev *__restrict__ frames, int diff)
{
    const BatchFrameDev &f = frames[blockIdx.y];
    float4 *quad = const_cast<float4 *>(f.quad);
    const int w = f.w, h = f.h;
    const size_t n = (size_t)w * h, total = n * f.V;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t v = i / n, k = i - v * n;
        const int y = (int)(k / w), x = (int)(k - (size_t)y * w);
        float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
        if (x < w - 1 && y < h - 1) q = make_quad(f.srcs + v * n + k, w, diff != 0);
        quad[i] = q;
    }
}

// 1.5 * 2^23: for 0 <= x < 2^22, x + C rounded down is C + floor(x) exactly,
// an integer in [2^23, 2^24) whose low mantissa bits are floor(x); the
// subtraction C then gives floor(x) as a float, also exactly.  Floors on the
// FMA pipe instead of the conversion unit (a standard magic-number floor).
constexpr float kFloorMagic = 12582912.f;
constexpr int kFloorMagicBits = 0x4B400000;

// pass A0 with the row coordinates from shared memory; with QUAD, `quad` holds
// the source's 2x2 neighbourhoods (difference form in COMPENSATED), else the
// four samples are gathered from `src`.  COMPENSATED stores the samples
// shifted by `shift`.
template <int WIN, int MOM, bool QUAD, int TWS = 0, bool ROWS_INTERIOR = false>
__device__ __forceinline__ void pass_a0_rows(float (*Wt)[RWMAX], const float *__restrict__ src,
                                             const float4 *__restrict__ quad, int w, int h, const float *Hm, float X,
                                             const float *Yc, float shift)
{
    using G = Geo<WIN, TWS>;
    constexpr int CELLS = G::A0ROWS;
    constexpr int BATCH = 4;
    if (threadIdx.x >= G::COLT) return;
    const int rx = threadIdx.x % G::RW, rb = threadIdx.x / G::RW;
    const float a0 = fmaf(Hm[0], X, Hm[2]), a1 = fmaf(Hm[3], X, Hm[5]), a2 = fmaf(Hm[6], X, Hm[8]);
    // floor(xs) in [0, w - 2] is 0 <= xs < w - 1.  xs is never -0 (a sum
    // x + (-1) that is exactly zero rounds to +0), and non-negative floats,
    // +inf and +NaN order like their bit patterns while negative ones (and
    // -NaN) have the sign bit, so the test is one unsigned compare per axis.
    const unsigned wm1 = __float_as_uint((float)(w - 1)), hm1 = __float_as_uint((float)(h - 1));
#pragma unroll
    for (int k0 = 0; k0 < CELLS; k0 += BATCH) {
        float fa[BATCH], fb[BATCH];
        unsigned off[BATCH];   // read only where ok: unsigned, so the unused values wrap harmlessly
        bool ok[BATCH];
#pragma unroll
        for (int j = 0; j < BATCH; ++j) {
            const int k = k0 + j;
            ok[j] = false;
            fa[j] = fb[j] = 0.f;
            off[j] = 0u;
            if (k < CELLS && rb + 3 * k < G::RH) {
                // ROWS_INTERIOR: no region row is mirrored, so the rows are consecutive
                const float Y = ROWS_INTERIOR ? Yc[rb] + (float)(3 * k) : Yc[rb + 3 * k];
                float xs, ys;
                if (MOM == MVS_MOMENTS_REFERENCE) {
                    const float q0 = Hm[0] * X + Hm[1] * Y + Hm[2] * 1.f;
                    const float q1 = Hm[3] * X + Hm[4] * Y + Hm[5] * 1.f;
                    const float q2 = Hm[6] * X + Hm[7] * Y + Hm[8] * 1.f;
                    xs = q0 / q2 - 1.f;
                    ys = q1 / q2 - 1.f;
                } else {
                    const float q0 = fmaf(Hm[1], Y, a0), q1 = fmaf(Hm[4], Y, a1), q2 = fmaf(Hm[7], Y, a2);
                    float rz;
                    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rz) : "f"(q2));
                    xs = fmaf(q0, rz, -1.f);
                    ys = fmaf(q1, rz, -1.f);
                }
                ok[j] = __float_as_uint(xs) < wm1 && __float_as_uint(ys) < hm1;
                const float tx = __fadd_rd(xs, kFloorMagic), ty = __fadd_rd(ys, kFloorMagic);
                fa[j] = xs - (tx - kFloorMagic);
                fb[j] = ys - (ty - kFloorMagic);
                off[j] = (__float_as_uint(ty) - (unsigned)kFloorMagicBits) * (unsigned)w +
                         (__float_as_uint(tx) - (unsigned)kFloorMagicBits);
            }
        }
        float d00[BATCH], d01[BATCH], d10[BATCH], d11[BATCH];
        if constexpr (QUAD) {
#pragma unroll
            for (int j = 0; j < BATCH; ++j) {
                d00[j] = d01[j] = d10[j] = d11[j] = 0.f;
                if (ok[j]) {
                    const float4 q = __ldg(quad + off[j]);
                    d00[j] = q.x;
                    d01[j] = q.y;
                    d10[j] = q.z;
                    d11[j] = q.w;
                }
            }
        } else {
#pragma unroll
            for (int j = 0; j < BATCH; ++j) {
                d00[j] = d01[j] = d10[j] = d11[j] = 0.f;
                if (ok[j]) {
                    const float *r0 = src + off[j];
                    d00[j] = ldg(r0);
                    d01[j] = ldg(r0 + 1);
                    d10[j] = ldg(r0 + w);
                    d11[j] = ldg(r0 + w + 1);
                }
            }
        }
#pragma unroll
        for (int j = 0; j < BATCH; ++j) {
            const int k = k0 + j;
            if (k >= CELLS || rb + 3 * k >= G::RH) continue;
            const float a = fa[j], b = fb[j];
            float v;
            if (MOM == MVS_MOMENTS_REFERENCE) {
                const float t1 = a * d01[j] + (1 - a) * d00[j];
                const float t2 = a * d11[j] + (1 - a) * d10[j];
                v = ok[j] ? b * t2 + (1 - b) * t1 : 0.f;
            } else {
                // the difference form of the neighbourhood (as quad_kernel
                // stores it), so both sources give the same roundings
                float4 q = make_float4(d00[j], d01[j], d10[j], d11[j]);
                if (!QUAD) q = make_float4(d00[j], d01[j] - d00[j], d10[j] - d00[j], (d11[j] - d10[j]) - (d01[j] - d00[j]));
                v = (ok[j] ? fmaf(b, fmaf(a, q.w, q.z), fmaf(a, q.y, q.x)) : 0.f) - shift;
            }
            Wt[rb + 3 * k][rx] = v;
        }
    }
}

// pass A1 with the reference column read from shared memory: thread (c, s)
// forms the column sums of w, w^2 and ref*w for output rows [11 s, 11 s + 11)
// (COMPENSATED: Wt and Rf hold shifted values already)
template <int WIN, int MOM, int TWS = 0>
__device__ __forceinline__ void pass_a1_rows(const float (*Wt)[RWMAX], float (*CS)[TH][CSP],
                                             const float (*Rf)[RWMAX])
{
    using G = Geo<WIN, TWS>;
    if (threadIdx.x >= G::COLT) return;
    const int c = threadIdx.x % G::RW, s = threadIdx.x / G::RW;
    const int r0 = STRIP * s;
    const bool full = r0 + STRIP <= TH;   // the last strip has TH - 2 STRIP rows
    float wv[G::SROWS];
#pragma unroll
    for (int i = 0; i < G::SROWS; ++i) wv[i] = Wt[r0 + i][c];
    if (MOM == MVS_MOMENTS_REFERENCE) {
#pragma unroll
        for (int k = 0; k < STRIP; ++k) {
            if (k == STRIP - 1 && !full) break;
            float s1 = 0.f, s2 = 0.f, s12 = 0.f;
#pragma unroll
            for (int i = 0; i < WIN; ++i) {
                const float x = wv[k + i];
                s1 = s1 + x;
                s2 = s2 + x * x;
                s12 = s12 + Rf[r0 + k + i][c] * x;
            }
            s1 = div_win<WIN>(s1);
            s2 = div_win<WIN>(s2);
            s12 = div_win<WIN>(s12);
            CS[0][r0 + k][c] = s1;
            CS[1][r0 + k][c] = s2;
            CS[2][r0 + k][c] = s12;
        }
    } else {
        float rf[G::SROWS];
#pragma unroll
        for (int i = 0; i < G::SROWS; ++i) rf[i] = Rf[r0 + i][c];
        // the window's first term starts the sums (0 + x is x, up to the sign
        // of a zero sum, which no NCC sees)
        float s1 = wv[0], s2 = wv[0] * wv[0], s12 = rf[0] * wv[0];
#pragma unroll
        for (int i = 1; i < WIN; ++i) {
            s1 += wv[i];
            s2 = fmaf(wv[i], wv[i], s2);
            s12 = fmaf(rf[i], wv[i], s12);
        }
#pragma unroll
        for (int k = 0; k < STRIP; ++k) {
            if (k == STRIP - 1 && !full) break;
            if (k > 0) {
                const float xn = wv[k + WIN - 1], xo = wv[k - 1];
                s1 = (s1 + xn) - xo;
                s2 = fmaf(-xo, xo, fmaf(xn, xn, s2));
                s12 = fmaf(-rf[k - 1], xo, fmaf(rf[k + WIN - 1], xn, s12));
            }
            CS[0][r0 + k][c] = s1;
            CS[1][r0 + k][c] = s2;
            CS[2][r0 + k][c] = s12;
        }
    }
}

// One CTA's work: tile (tx, ty) of the frame, planes of `chunk`.
// BATCHED: the batched kernel's instantiation, whose seven inlined window
// bodies share one register allocation.  Two choices differ there, each
// measured on the bench's batch of 48 frames: the costs are rounded to BF16
// by f2bf instead of the hardware conversion (the same bits; ptxas spills
// less around it: 59.2 against 61.7 ms), and tiles whose region rows are all
// inside the frame form the row coordinates instead of reading them (58.5
// against 59.1 ms; in the single-frame kernel that form issued 2% more
// instructions and was slower).
template <int WIN, int MOM, int TWS = 0, bool BATCHED = false>
__device__ __forceinline__ void aggregated_tile(AggSmem &A, const SweepArgs &a, int tx, int ty, int chunk)
{
    using G = Geo<WIN, TWS>;
    Smem &S = A.S;
    const int x0 = tx * G::TW, y0 = ty * TH;
    const int w = a.w, h = a.h;
    const size_t n = (size_t)w * h;

    load_ref_region<WIN, MOM, TWS>(S, a.ref, w, h, x0, y0);
    for (int i = threadIdx.x; i < G::RH; i += THREADS) A.Yc[i] = (float)(mirror_idx(y0 - G::R + i, h) + 1);
    __syncthreads();
    const float shift = tile_shift<WIN, MOM, TWS>(S);
    for (int i = threadIdx.x; i < G::RH * RWMAX; i += THREADS) {
        const int ry = i / RWMAX, rx = i % RWMAX;
        const float r = rx < G::RW ? S.Wt[ry][rx] : 0.f;
        A.Rf[ry][rx] = (MOM == MVS_MOMENTS_REFERENCE) ? r : r - shift;
    }
    ref_moments<WIN, MOM, TWS>(S.Wt, S.CS, shift, a.stdthresh, A.RM, A.RS);
    const float Xcol = (float)(mirror_idx(x0 - G::R + (int)(threadIdx.x % G::RW), w) + 1);
    // every region row inside the frame: pass A0 forms the row coordinates
    // instead of reading them (batched kernel only)
    const bool rows_interior = BATCHED && y0 - G::R >= 0 && y0 - G::R + G::RH <= h;

    const int ly = b_row(), lx = b_seg() * G::RUN;
    const int y = y0 + ly, xb = x0 + lx;
    // the run's cost values as one 16-byte store: 8 per run, every row a
    // multiple of 8 values, the run inside the frame, the volume 16-byte aligned
    const bool vec_cost = G::RUN == 8 && a.cost && (w & 7) == 0 && xb + 8 <= w &&
                          ((uintptr_t)a.cost & 15) == 0;
    uint32_t best[G::RUN];   // (bf16 cost bits << 16) | plane
#pragma unroll
    for (int j = 0; j < G::RUN; ++j) best[j] = 0xffffffffu;
    const float invV = 1.f / (float)a.V;
    const float sh = MOM == MVS_MOMENTS_REFERENCE ? 0.f : shift;
    const int p0 = chunk * a.planes_per_chunk, p1 = min(a.P, p0 + a.planes_per_chunk);
    // Homographies double-buffered: thread k < 9 fetches element k of the next
    // (plane, view) during pass A0 and the barrier that ends the pass publishes
    // it, so a view takes two barriers.  Pass A0 of the next view needs no
    // barrier before it: it writes only Wt, which pass A1 has finished reading.
    if (threadIdx.x < 9 && p0 < p1) S.Hm[0][threadIdx.x] = ldg(a.H + (size_t)p0 * 9 + threadIdx.x);
    __syncthreads();
    int hb = 0;
    for (int p = p0; p < p1; ++p) {
        float acc[G::RUN];
#pragma unroll
        for (int j = 0; j < G::RUN; ++j) acc[j] = 0.f;
        for (int view = 0; view < a.V; ++view) {
            float Hm[9];
            load_hm(S.Hm[hb], Hm);
            const bool last_view = view + 1 == a.V;
            const int nv = last_view ? 0 : view + 1, np = last_view ? p + 1 : p;
            float hn = 0.f;
            if (threadIdx.x < 9 && np < p1) hn = ldg(a.H + ((size_t)nv * a.P + np) * 9 + threadIdx.x);
            if (a.quad && rows_interior)
                pass_a0_rows<WIN, MOM, true, TWS, true>(S.Wt, nullptr, a.quad + (size_t)view * n, w, h, Hm, Xcol, A.Yc,
                                                        sh);
            else if (a.quad)
                pass_a0_rows<WIN, MOM, true, TWS>(S.Wt, nullptr, a.quad + (size_t)view * n, w, h, Hm, Xcol, A.Yc, sh);
            else
                pass_a0_rows<WIN, MOM, false, TWS>(S.Wt, a.srcs + (size_t)view * n, nullptr, w, h, Hm, Xcol, A.Yc, sh);
            if (threadIdx.x < 9) S.Hm[hb ^ 1][threadIdx.x] = hn;
            hb ^= 1;
            __syncthreads();
            pass_a1_rows<WIN, MOM, TWS>(S.Wt, S.CS, A.Rf);
            __syncthreads();
            float s1[G::RUN], s2[G::RUN], s12[G::RUN];
            row_sums<WIN, MOM, TWS>(S.CS[0], s1);
            row_sums<WIN, MOM, TWS>(S.CS[1], s2);
            row_sums<WIN, MOM, TWS>(S.CS[2], s12);
            ncc_run<WIN, MOM, TWS>(s1, s2, s12, A.RM[ly] + lx, A.RS[ly] + lx, a.stdthresh,
                              [&](int j, float c) { acc[j] += c; });
        }
        uint16_t cb[G::RUN];
#pragma unroll
        for (int j = 0; j < G::RUN; ++j) {
            // cost = 1 - mean NCC, clamped at 0 (rounding can push a perfect match
            // below 0; the stored bf16 bits then order like unsigned integers)
            float cf = fmaf(-acc[j], invV, 1.f);
            cf = cf > 0.f ? cf : (cf == cf ? 0.f : 3.f);
            cb[j] = BATCHED ? f2bf(cf) : f2bf_num(cf);   // cf is not NaN here
            best[j] = min(best[j], ((uint32_t)cb[j] << 16) | (uint32_t)p);
        }
        if (a.cost && y < h) {
            uint16_t *row = a.cost + (size_t)p * n + (size_t)y * w + xb;
            if (vec_cost) {
                uint4 q;
                q.x = (uint32_t)cb[0] | ((uint32_t)cb[1 % G::RUN] << 16);
                q.y = (uint32_t)cb[2 % G::RUN] | ((uint32_t)cb[3 % G::RUN] << 16);
                q.z = (uint32_t)cb[4 % G::RUN] | ((uint32_t)cb[5 % G::RUN] << 16);
                q.w = (uint32_t)cb[6 % G::RUN] | ((uint32_t)cb[7 % G::RUN] << 16);
                *reinterpret_cast<uint4 *>(row) = q;
            } else {
#pragma unroll
                for (int j = 0; j < G::RUN; ++j)
                    if (xb + j < w) row[j] = cb[j];
            }
        }
    }
    if (y >= h) return;
#pragma unroll
    for (int j = 0; j < G::RUN; ++j) {
        const int x = xb + j;
        if (x >= w) break;
        // (cost bits << 32) | plane: a 64-bit min keeps the lowest cost and,
        // among equal costs, the earliest plane (costs are >= 0).
        const bool any = best[j] != 0xffffffffu;
        const unsigned long long key = !any ? ~0ull
            : ((unsigned long long)__float_as_uint(bf2f((uint16_t)(best[j] >> 16))) << 32) | (best[j] & 0xffffu);
        unsigned long long *o = a.wta + (size_t)y * w + x;
        if (a.n_chunks == 1) *o = key;
        else if (any) atomicMin(o, key);
    }
}

// ---- per-view kernel -------------------------------------------------------------
// grid: (tiles_x, tiles_y, V * n_chunks); dynamic shared memory: sizeof(AggSmem).
// The per-CTA reference state sits in shared memory as in the aggregated
// kernel, so it also runs three CTAs per SM.

template <int WIN, int MOM>
__global__ void __launch_bounds__(THREADS, 3) sweep_view_kernel(SweepArgs a)
{
    using G = Geo<WIN>;
    extern __shared__ __align__(16) unsigned char view_smem[];
    AggSmem &A = *reinterpret_cast<AggSmem *>(view_smem);
    Smem &S = A.S;
    const int view = blockIdx.z / a.n_chunks, chunk = blockIdx.z % a.n_chunks;
    const int x0 = blockIdx.x * G::TW, y0 = blockIdx.y * TH;
    const int w = a.w, h = a.h;
    const size_t n = (size_t)w * h;
    const float *src = a.srcs + (size_t)view * n;
    const float4 *quad = a.quad ? a.quad + (size_t)view * n : nullptr;

    load_ref_region<WIN, MOM>(S, a.ref, w, h, x0, y0);
    for (int i = threadIdx.x; i < G::RH; i += THREADS) A.Yc[i] = (float)(mirror_idx(y0 - G::R + i, h) + 1);
    __syncthreads();
    const float shift = tile_shift<WIN, MOM>(S);
    for (int i = threadIdx.x; i < G::RH * RWMAX; i += THREADS) {
        const int ry = i / RWMAX, rx = i % RWMAX;
        const float r = rx < G::RW ? S.Wt[ry][rx] : 0.f;
        A.Rf[ry][rx] = (MOM == MVS_MOMENTS_REFERENCE) ? r : r - shift;
    }
    ref_moments<WIN, MOM>(S.Wt, S.CS, shift, a.stdthresh, A.RM, A.RS);
    const float Xcol = (float)(mirror_idx(x0 - G::R + (int)(threadIdx.x % G::RW), w) + 1);
    const int ly = b_row(), lx = b_seg() * G::RUN;
    const float sh = MOM == MVS_MOMENTS_REFERENCE ? 0.f : shift;

    float best[G::RUN];
    int lab[G::RUN];
#pragma unroll
    for (int j = 0; j < G::RUN; ++j) {
        best[j] = 0.f;
        lab[j] = -1;
    }
    const int p0 = chunk * a.planes_per_chunk, p1 = min(a.P, p0 + a.planes_per_chunk);
    const float *Hv = a.H + (size_t)view * a.P * 9;
    // homographies double-buffered as in the aggregated tile: two barriers a plane
    if (threadIdx.x < 9 && p0 < p1) S.Hm[0][threadIdx.x] = ldg(Hv + (size_t)p0 * 9 + threadIdx.x);
    __syncthreads();
    int hb = 0;
    for (int p = p0; p < p1; ++p) {
        float Hm[9];
        load_hm(S.Hm[hb], Hm);
        float hn = 0.f;
        if (threadIdx.x < 9 && p + 1 < p1) hn = ldg(Hv + (size_t)(p + 1) * 9 + threadIdx.x);
        if (quad)
            pass_a0_rows<WIN, MOM, true>(S.Wt, nullptr, quad, w, h, Hm, Xcol, A.Yc, sh);
        else
            pass_a0_rows<WIN, MOM, false>(S.Wt, src, nullptr, w, h, Hm, Xcol, A.Yc, sh);
        if (threadIdx.x < 9) S.Hm[hb ^ 1][threadIdx.x] = hn;
        hb ^= 1;
        __syncthreads();   // Wt and the next homography visible; pass B of the previous plane done with CS
        pass_a1_rows<WIN, MOM>(S.Wt, S.CS, A.Rf);
        __syncthreads();
        float s1[G::RUN], s2[G::RUN], s12[G::RUN];
        row_sums<WIN, MOM>(S.CS[0], s1);
        row_sums<WIN, MOM>(S.CS[1], s2);
        row_sums<WIN, MOM>(S.CS[2], s12);
        ncc_run<WIN, MOM, 0>(s1, s2, s12, A.RM[ly] + lx, A.RS[ly] + lx, a.stdthresh, [&](int j, float c) {
            if (c > best[j]) {
                best[j] = c;
                lab[j] = p;
            }
        });
    }
    // results: (ncc bits << 32) | ~plane, so that a 64-bit max keeps the
    // largest NCC and, among equal NCCs, the earliest plane.
    const int y = y0 + ly;
    if (y >= h) return;
    const int xb = x0 + lx;
    unsigned long long *outp = a.packed + (size_t)view * w * h + (size_t)y * w;
#pragma unroll
    for (int j = 0; j < G::RUN; ++j) {
        const int x = xb + j;
        if (x >= w) break;
        unsigned long long key = 0ull;
        if (lab[j] >= 0)
            key = ((unsigned long long)__float_as_uint(best[j]) << 32) | (unsigned long long)(0xffffffffu - (unsigned)lab[j]);
        if (a.n_chunks == 1) outp[x] = key;
        else if (key) atomicMax(outp + x, key);
    }
}

// grid: (tiles_x, tiles_y, n_chunks); dynamic shared memory: sizeof(AggSmem)
template <int WIN, int MOM>
__global__ void __launch_bounds__(THREADS, 3) sweep_aggregated_kernel(SweepArgs a)
{
    extern __shared__ __align__(16) unsigned char agg_smem[];
    AggSmem &A = *reinterpret_cast<AggSmem *>(agg_smem);
    aggregated_tile<WIN, MOM>(A, a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ---- aggregated mode with TMA-staged source regions ------------------------------
//
// The same tile, passes and arithmetic as aggregated_tile, but pass A0 reads
// each sample's 2x2 neighbourhood from a staged copy of the source region in
// shared memory instead of gathering it from L2.  For every (plane, view) the
// tile region's four corners are projected (a homography maps the rectangle
// into the hull of their images when the projective depth stays positive);
// the bounding box, widened by one pixel for rounding and started on a
// 16-byte column, is loaded by one cp.async.bulk.tensor (a plain TMA load of
// this GPU's source stack, no multicast) into one of two staging buffers,
// two (plane, view) steps ahead of its use, and an mbarrier says when it has
// landed.  A box larger than the buffer, a corner behind the camera, or a
// sample outside the box (rounding) falls back to the global gather for that
// step or sample.  The staged values are the source's own bits, and the
// difference form is formed in registers with quad_kernel's operations, so
// the results equal aggregated_tile's bit for bit.  Each staging wait is
// bounded (1 s of %globaltimer): on a timeout the CTA records the error,
// waits (bounded) for its other copy in flight and leaves; the host then
// returns MVS_ERR_TIMEOUT.

constexpr int STG_W = 88, STG_H = 48;     // staged box (floats): every C2 tile region's footprint fits
constexpr uint64_t kStageWaitNs = 1000000000ull;

struct StgCtl {
    uint64_t mbar[2];
    int bx[2], by[2], fits[2];
    int rx0, rx1, ry0, ry1;   // 1-based pixel range the tile region samples
    int abort;
};
constexpr size_t kStgOffset = (sizeof(AggSmem) + 127) / 128 * 128;
constexpr size_t kStgBytes = kStgOffset + 2 * sizeof(float) * STG_W * STG_H + sizeof(StgCtl) + 128;

// the box of (plane, view) pair k of this chunk: bounding box of the region's
// corners under H, or fits = 0 (thread 0)
__device__ __forceinline__ void stage_issue(StgCtl &C, float (*box)[STG_H][STG_W], const CUtensorMap *tmap,
                                            const float *__restrict__ H9, int view, int b)
{
    float H[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) H[i] = ldg(H9 + i);
    float xmin = 3e38f, xmax = -3e38f, ymin = 3e38f, ymax = -3e38f;
    bool ok = true;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float X = (float)((c & 1) ? C.rx1 : C.rx0), Y = (float)((c & 2) ? C.ry1 : C.ry0);
        const float q0 = H[0] * X + H[1] * Y + H[2], q1 = H[3] * X + H[4] * Y + H[5], q2 = H[6] * X + H[7] * Y + H[8];
        ok = ok && q2 > 0.f;
        const float xs = q0 / q2 - 1.f, ys = q1 / q2 - 1.f;
        xmin = fminf(xmin, xs), xmax = fmaxf(xmax, xs), ymin = fminf(ymin, ys), ymax = fmaxf(ymax, ys);
    }
    ok = ok && xmin > -1e6f && xmax < 1e6f && ymin > -1e6f && ymax < 1e6f;   // also false for NaN
    int bx = 0, by = 0;
    if (ok) {
        const int x0 = (int)floorf(xmin) - 1, x1 = (int)floorf(xmax) + 2;
        const int y0 = (int)floorf(ymin) - 1, y1 = (int)floorf(ymax) + 2;
        bx = x0 >= 0 ? x0 & ~3 : -((3 - x0) & ~3);   // down to a multiple of 4 columns (16 bytes)
        by = y0;
        ok = x1 - bx < STG_W && y1 - by < STG_H;
    }
    C.bx[b] = bx;
    C.by[b] = by;
    C.fits[b] = ok;
    const uint32_t bar = smem_u32(&C.mbar[b]);
    if (ok) {
        fence_async_smem();   // the buffer's earlier generic reads before the async write
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                     "r"((uint32_t)(sizeof(float) * STG_W * STG_H))
                     : "memory");
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
            "[%5];" ::"r"(smem_u32(box[b])),
            "l"(tmap), "r"(bx), "r"(by), "r"(view), "r"(bar)
            : "memory");
    } else {
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
    }
}

// pass A0 from a staged box (the gather of pass_a0_rows with QUAD = false
// semantics for the neighbourhood values, then the same interpolation)
template <int WIN, int MOM>
__device__ __forceinline__ void pass_a0_staged(float (*Wt)[RWMAX], const float (*box)[STG_W], int bx, int by,
                                               const float *__restrict__ src, int w, int h, const float *Hm, float X,
                                               const float *Yc, float shift)
{
    using G = Geo<WIN>;
    constexpr int CELLS = G::A0ROWS;
    constexpr int BATCH = 4;
    if (threadIdx.x >= G::COLT) return;
    const int rx = threadIdx.x % G::RW, rb = threadIdx.x / G::RW;
    const float a0 = fmaf(Hm[0], X, Hm[2]), a1 = fmaf(Hm[3], X, Hm[5]), a2 = fmaf(Hm[6], X, Hm[8]);
    const unsigned wm1 = __float_as_uint((float)(w - 1)), hm1 = __float_as_uint((float)(h - 1));
#pragma unroll
    for (int k0 = 0; k0 < CELLS; k0 += BATCH) {
        float fa[BATCH], fb[BATCH], d00[BATCH], d01[BATCH], d10[BATCH], d11[BATCH];
        bool ok[BATCH];
#pragma unroll
        for (int j = 0; j < BATCH; ++j) {
            const int k = k0 + j;
            ok[j] = false;
            fa[j] = fb[j] = 0.f;
            d00[j] = d01[j] = d10[j] = d11[j] = 0.f;
            if (k < CELLS && rb + 3 * k < G::RH) {
                const float Y = Yc[rb + 3 * k];
                float xs, ys;
                if (MOM == MVS_MOMENTS_REFERENCE) {
                    const float q0 = Hm[0] * X + Hm[1] * Y + Hm[2] * 1.f;
                    const float q1 = Hm[3] * X + Hm[4] * Y + Hm[5] * 1.f;
                    const float q2 = Hm[6] * X + Hm[7] * Y + Hm[8] * 1.f;
                    xs = q0 / q2 - 1.f;
                    ys = q1 / q2 - 1.f;
                } else {
                    const float q0 = fmaf(Hm[1], Y, a0), q1 = fmaf(Hm[4], Y, a1), q2 = fmaf(Hm[7], Y, a2);
                    float rz;
                    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rz) : "f"(q2));
                    xs = fmaf(q0, rz, -1.f);
                    ys = fmaf(q1, rz, -1.f);
                }
                ok[j] = __float_as_uint(xs) < wm1 && __float_as_uint(ys) < hm1;
                const float tx = __fadd_rd(xs, kFloorMagic), ty = __fadd_rd(ys, kFloorMagic);
                fa[j] = xs - (tx - kFloorMagic);
                fb[j] = ys - (ty - kFloorMagic);
                if (ok[j]) {
                    const int ix = (int)(__float_as_uint(tx) - (unsigned)kFloorMagicBits);
                    const int iy = (int)(__float_as_uint(ty) - (unsigned)kFloorMagicBits);
                    const unsigned lx = (unsigned)(ix - bx), ly = (unsigned)(iy - by);
                    if (lx <= STG_W - 2u && ly <= STG_H - 2u) {
                        d00[j] = box[ly][lx];
                        d01[j] = box[ly][lx + 1];
                        d10[j] = box[ly + 1][lx];
                        d11[j] = box[ly + 1][lx + 1];
                    } else {   // outside the staged box (rounding): the global gather
                        const float *r0 = src + (size_t)iy * w + ix;
                        d00[j] = ldg(r0);
                        d01[j] = ldg(r0 + 1);
                        d10[j] = ldg(r0 + w);
                        d11[j] = ldg(r0 + w + 1);
                    }
                }
            }
        }
#pragma unroll
        for (int j = 0; j < BATCH; ++j) {
            const int k = k0 + j;
            if (k >= CELLS || rb + 3 * k >= G::RH) continue;
            const float a = fa[j], b = fb[j];
            float v;
            if (MOM == MVS_MOMENTS_REFERENCE) {
                const float t1 = a * d01[j] + (1 - a) * d00[j];
                const float t2 = a * d11[j] + (1 - a) * d10[j];
                v = ok[j] ? b * t2 + (1 - b) * t1 : 0.f;
            } else {
                const float4 q = make_quad4(d00[j], d01[j], d10[j], d11[j]);
                v = (ok[j] ? fmaf(b, fmaf(a, q.w, q.z), fmaf(a, q.y, q.x)) : 0.f) - shift;
            }
            Wt[rb + 3 * k][rx] = v;
        }
    }
}

// grid: (tiles_x, tiles_y, n_chunks); dynamic shared memory: kStgBytes; two CTAs per SM
template <int WIN, int MOM>
__global__ void __launch_bounds__(THREADS, 2) sweep_aggregated_tma_kernel(SweepArgs a,
                                                                          const __grid_constant__ CUtensorMap tmap)
{
    using G = Geo<WIN>;
    extern __shared__ __align__(128) unsigned char stg_smem[];
    unsigned char *base = (unsigned char *)(((uintptr_t)stg_smem + 127) & ~(uintptr_t)127);
    AggSmem &A = *reinterpret_cast<AggSmem *>(base);
    float (*box)[STG_H][STG_W] = reinterpret_cast<float (*)[STG_H][STG_W]>(base + kStgOffset);
    StgCtl &C = *reinterpret_cast<StgCtl *>(base + kStgOffset + 2 * sizeof(float) * STG_W * STG_H);
    Smem &S = A.S;
    const int tx = blockIdx.x, ty = blockIdx.y, chunk = blockIdx.z;
    const int x0 = tx * G::TW, y0 = ty * TH;
    const int w = a.w, h = a.h;
    const size_t n = (size_t)w * h;
    const int p0 = chunk * a.planes_per_chunk, p1 = min(a.P, p0 + a.planes_per_chunk);
    const int K = (p1 - p0) * a.V;   // (plane, view) steps of this CTA
    if (threadIdx.x == 0) {
        mbar_init(&C.mbar[0], 1);
        mbar_init(&C.mbar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        // the clipped pixel range of the region (mirrored coordinates stay inside it)
        C.rx0 = max(x0 - G::R, 0) + 1;
        C.rx1 = min(x0 + G::RW - G::R - 1, w - 1) + 1;
        C.ry0 = max(y0 - G::R, 0) + 1;
        C.ry1 = min(y0 + G::RH - G::R - 1, h - 1) + 1;
        C.abort = 0;
        for (int k = 0; k < 2 && k < K; ++k) {
            const int p = p0 + k / a.V, view = k % a.V;
            stage_issue(C, box, &tmap, a.H + ((size_t)view * a.P + p) * 9, view, k);
        }
    }
    load_ref_region<WIN, MOM>(S, a.ref, w, h, x0, y0);
    for (int i = threadIdx.x; i < G::RH; i += THREADS) A.Yc[i] = (float)(mirror_idx(y0 - G::R + i, h) + 1);
    __syncthreads();
    const float shift = tile_shift<WIN, MOM>(S);
    for (int i = threadIdx.x; i < G::RH * RWMAX; i += THREADS) {
        const int ry = i / RWMAX, rx = i % RWMAX;
        const float r = rx < G::RW ? S.Wt[ry][rx] : 0.f;
        A.Rf[ry][rx] = (MOM == MVS_MOMENTS_REFERENCE) ? r : r - shift;
    }
    ref_moments<WIN, MOM>(S.Wt, S.CS, shift, a.stdthresh, A.RM, A.RS);
    const float Xcol = (float)(mirror_idx(x0 - G::R + (int)(threadIdx.x % G::RW), w) + 1);
    const int ly = b_row(), lx = b_seg() * G::RUN;
    const int y = y0 + ly, xb = x0 + lx;
    const bool vec_cost = G::RUN == 8 && a.cost && (w & 7) == 0 && xb + 8 <= w && ((uintptr_t)a.cost & 15) == 0;
    uint32_t best[G::RUN];
#pragma unroll
    for (int j = 0; j < G::RUN; ++j) best[j] = 0xffffffffu;
    const float invV = 1.f / (float)a.V;
    const float sh = MOM == MVS_MOMENTS_REFERENCE ? 0.f : shift;
    if (threadIdx.x < 9 && p0 < p1) S.Hm[0][threadIdx.x] = ldg(a.H + (size_t)p0 * 9 + threadIdx.x);
    __syncthreads();
    int hb = 0, k = 0;
    for (int p = p0; p < p1; ++p) {
        float acc[G::RUN];
#pragma unroll
        for (int j = 0; j < G::RUN; ++j) acc[j] = 0.f;
        for (int view = 0; view < a.V; ++view, ++k) {
            float Hm[9];
            load_hm(S.Hm[hb], Hm);
            const bool last_view = view + 1 == a.V;
            const int nv = last_view ? 0 : view + 1, np = last_view ? p + 1 : p;
            float hn = 0.f;
            if (threadIdx.x < 9 && np < p1) hn = ldg(a.H + ((size_t)nv * a.P + np) * 9 + threadIdx.x);
            const int b = k & 1;
            if (!mbar_wait_bounded(&C.mbar[b], (uint32_t)((k >> 1) & 1), kStageWaitNs)) C.abort = 1;
            if (C.fits[b])
                pass_a0_staged<WIN, MOM>(S.Wt, box[b], C.bx[b], C.by[b], a.srcs + (size_t)view * n, w, h, Hm, Xcol,
                                         A.Yc, sh);
            else if (a.quad)
                pass_a0_rows<WIN, MOM, true>(S.Wt, nullptr, a.quad + (size_t)view * n, w, h, Hm, Xcol, A.Yc, sh);
            else
                pass_a0_rows<WIN, MOM, false>(S.Wt, a.srcs + (size_t)view * n, nullptr, w, h, Hm, Xcol, A.Yc, sh);
            if (threadIdx.x < 9) S.Hm[hb ^ 1][threadIdx.x] = hn;
            hb ^= 1;
            __syncthreads();   // Wt and the next homography visible; buffer b read
            if (C.abort) {
                if (threadIdx.x == 0) {
                    atomicExch(a.err, 1);
                    // the copies that may still be in flight: this step's and the next one's
                    mbar_wait_bounded(&C.mbar[b], (uint32_t)((k >> 1) & 1), kStageWaitNs);
                    if (k + 1 < K) mbar_wait_bounded(&C.mbar[b ^ 1], (uint32_t)(((k + 1) >> 1) & 1), kStageWaitNs);
                }
                return;
            }
            if (threadIdx.x == 0 && k + 2 < K) {
                const int k2 = k + 2, p2 = p0 + k2 / a.V, v2 = k2 % a.V;
                stage_issue(C, box, &tmap, a.H + ((size_t)v2 * a.P + p2) * 9, v2, b);
            }
            pass_a1_rows<WIN, MOM>(S.Wt, S.CS, A.Rf);
            __syncthreads();
            float s1[G::RUN], s2[G::RUN], s12[G::RUN];
            row_sums<WIN, MOM>(S.CS[0], s1);
            row_sums<WIN, MOM>(S.CS[1], s2);
            row_sums<WIN, MOM>(S.CS[2], s12);
            ncc_run<WIN, MOM, 0>(s1, s2, s12, A.RM[ly] + lx, A.RS[ly] + lx, a.stdthresh,
                                 [&](int j, float c) { acc[j] += c; });
        }
        uint16_t cb[G::RUN];
#pragma unroll
        for (int j = 0; j < G::RUN; ++j) {
            float cf = fmaf(-acc[j], invV, 1.f);
            cf = cf > 0.f ? cf : (cf == cf ? 0.f : 3.f);
            cb[j] = f2bf_num(cf);   // cf is not NaN here
            best[j] = min(best[j], ((uint32_t)cb[j] << 16) | (uint32_t)p);
        }
        if (a.cost && y < h) {
            uint16_t *row = a.cost + (size_t)p * n + (size_t)y * w + xb;
            if (vec_cost) {
                uint4 q;
                q.x = (uint32_t)cb[0] | ((uint32_t)cb[1 % G::RUN] << 16);
                q.y = (uint32_t)cb[2 % G::RUN] | ((uint32_t)cb[3 % G::RUN] << 16);
                q.z = (uint32_t)cb[4 % G::RUN] | ((uint32_t)cb[5 % G::RUN] << 16);
                q.w = (uint32_t)cb[6 % G::RUN] | ((uint32_t)cb[7 % G::RUN] << 16);
                *reinterpret_cast<uint4 *>(row) = q;
            } else {
#pragma unroll
                for (int j = 0; j < G::RUN; ++j)
                    if (xb + j < w) row[j] = cb[j];
            }
        }
    }
    if (y >= h) return;
#pragma unroll
    for (int j = 0; j < G::RUN; ++j) {
        const int x = xb + j;
        if (x >= w) break;
        const bool any = best[j] != 0xffffffffu;
        const unsigned long long key = !any ? ~0ull
            : ((unsigned long long)__float_as_uint(bf2f((uint16_t)(best[j] >> 16))) << 32) | (best[j] & 0xffffu);
        unsigned long long *o = a.wta + (size_t)y * w + x;
        if (a.n_chunks == 1) *o = key;
        else if (any) atomicMin(o, key);
    }
}

// ---- epilogues ----------------------------------------------------------------------

// sum_depthmap_NCC + element_rdivide + set_QNAN_value (kernels.cu:84-101,145-157,
// 331-340), views in order, float accumulation as the reference.
__global__ void sweep_combine_kernel(const unsigned long long *__restrict__ packed, const float *__restrict__ depths,
                                     int n, int V, float nccthresh, float zfar, float *__restrict__ depth,
                                     int32_t *__restrict__ labels, float *__restrict__ best)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float sum = 0.f, cnt = 0.f;
        for (int v = 0; v < V; ++v) {
            const unsigned long long key = packed[(size_t)v * n + i];
            const int lab = key ? (int)(0xffffffffu - (unsigned)(key & 0xffffffffu)) : -1;
            const float b = key ? __uint_as_float((unsigned)(key >> 32)) : 0.f;
            const float d = lab >= 0 ? ldg(depths + lab) : 0.f;
            if (b > nccthresh) {
                sum = sum + d;
                cnt = cnt + 1.f;
            }
            if (labels) labels[(size_t)v * n + i] = lab;
            if (best) best[(size_t)v * n + i] = b;
        }
        float r = cnt != 0.f ? sum / cnt : __int_as_float(0x7fc00000);
        depth[i] = r != r ? zfar : r;
    }
}

__global__ void wta_finish_kernel(const unsigned long long *__restrict__ wta, const float *__restrict__ depths, int n,
                                  float zfar, float *__restrict__ depth, int32_t *__restrict__ labels,
                                  float *__restrict__ best)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned long long key = wta[i];
        const bool ok = key != ~0ull;
        const int lab = ok ? (int)(unsigned)(key & 0xffffffffu) : -1;
        depth[i] = ok ? ldg(depths + lab) : zfar;
        if (labels) labels[i] = lab;
        if (best) best[i] = ok ? __uint_as_float((unsigned)(key >> 32)) : 3.f;
    }
}

// WTA argmin over a stored BF16 cost volume [P][n]: the HBM-bound pass.
// A block owns 32 groups of 8 consecutive pixels; its WTA_WARPS warps split the
// planes into contiguous slices, each lane reading one 16-byte group per plane
// (a warp reads 512 contiguous bytes per plane).  The slices' minima are merged
// in plane order through shared memory, so ties keep the earliest plane.
// 4 warps per block: the 1200 blocks of a 640x480 frame are then all resident
// at once (16 per SM) instead of 1184 plus a 16-block second wave.
constexpr int WTA_WARPS = 4;

__global__ void __launch_bounds__(32 * WTA_WARPS) wta_volume_kernel(const uint16_t *__restrict__ cost, const float *__restrict__ depths,
                                                        int n, int P, float zfar, float *__restrict__ depth,
                                                        int32_t *__restrict__ labels, float *__restrict__ best)
{
    __shared__ uint32_t sk[WTA_WARPS][32][9];
    const int n8 = n / 8;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int g = blockIdx.x * 32 + lane;            // pixel group of this lane
    const int per = (P + WTA_WARPS - 1) / WTA_WARPS;
    const int p0 = wid * per, p1 = min(P, p0 + per);
    // (bf16 bits << 16 | plane): costs are >= 0, so their bf16 bits order like
    // unsigned integers and a 32-bit min gives the lowest cost, then the
    // earliest plane.
    uint32_t key[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) key[j] = 0xffffffffu;
    if (g < n8) {
        const uint4 *col = reinterpret_cast<const uint4 *>(cost) + g;
#pragma unroll 8
        for (int p = p0; p < p1; ++p) {
            const uint4 q = __ldcs(col + (size_t)p * n8);
            const uint32_t wds[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) {
                key[2 * jj] = min(key[2 * jj], (wds[jj] << 16) | (uint32_t)p);
                key[2 * jj + 1] = min(key[2 * jj + 1], (wds[jj] & 0xffff0000u) | (uint32_t)p);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) sk[wid][lane][j] = key[j];
    __syncthreads();
    // each of the block's 256 (group, pixel) results is finalised by one thread
    for (int q = threadIdx.x; q < 32 * 8; q += 32 * WTA_WARPS) {
        const int gl = q >> 3, j = q & 7;
        const int gg = blockIdx.x * 32 + gl;
        if (gg >= n8) continue;
        uint32_t kmin = 0xffffffffu;
#pragma unroll
        for (int k = 0; k < WTA_WARPS; ++k) kmin = min(kmin, sk[k][gl][j]);
        const int l = kmin == 0xffffffffu ? -1 : (int)(kmin & 0xffffu);
        const float c = l >= 0 ? bf2f((uint16_t)(kmin >> 16)) : 3.f;
        const int px = 8 * gg + j;
        depth[px] = l >= 0 ? ldg(depths + l) : zfar;
        if (labels) labels[px] = l;
        if (best) best[px] = c;
    }
}

// FP64 homographies: H = K (Rrel + trel e3^T / d) K^-1, H /= H22, for one
// batch of up to kHomViews views (passed by value: no device allocation).
constexpr int kHomViews = 32;
struct HomCams {
    double K[9], invK[9];
    double Rrel[kHomViews][9];
    double trel[kHomViews][3];
};

__global__ void homography_kernel(HomCams c, const float *__restrict__ depths, int V, int P, float *__restrict__ H)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= V * P) return;
    const int v = idx / P, p = idx % P;
    const double d = (double)depths[p];
    const double *R = c.Rrel[v], *t = c.trel[v];
    double M[9], T[9], O[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) M[i] = R[i];
    M[2] += t[0] / d;
    M[5] += t[1] / d;
    M[8] += t[2] / d;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            T[3 * i + j] = fma(c.K[3 * i], M[j], fma(c.K[3 * i + 1], M[3 + j], c.K[3 * i + 2] * M[6 + j]));
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            O[3 * i + j] = fma(T[3 * i], c.invK[j], fma(T[3 * i + 1], c.invK[3 + j], T[3 * i + 2] * c.invK[6 + j]));
    const double s = O[8];
#pragma unroll
    for (int i = 0; i < 9; ++i) H[(size_t)idx * 9 + i] = (float)(O[i] / s);
}

// ---- batched frames: one persistent launch over a mixed work list ---------------------
//
// Work items (frame, tile, plane chunk) of frames of any size, view and plane
// count and window are handed out by an atomic counter to a grid of
// persistent CTAs, which run the aggregated sweep on each with the frame's
// window (a runtime switch over the compiled windows).  The CTA that
// completes the last chunk of a tile (a per-tile countdown, no waiting)
// finishes that tile -- winner-take-all word -> depth, label, cost -- and
// re-arms its scratch for the next launch; the CTA that finishes the last tile
// of a frame stamps the frame's completion time (%globaltimer).

__device__ __forceinline__ unsigned long long global_timer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__global__ void batch_start_kernel(unsigned int *next, unsigned long long *t_start)
{
    *next = 0u;
    *t_start = global_timer_ns();
}

template <int MOM, int TWS>
__global__ void __launch_bounds__(THREADS, 3) sweep_batch_kernel(const BatchFrameDev *__restrict__ frames,
                                                                  const uint4 *__restrict__ items, int n_items,
                                                                  unsigned int *next)
{
    extern __shared__ __align__(16) unsigned char agg_smem[];
    AggSmem &S = *reinterpret_cast<AggSmem *>(agg_smem);
    __shared__ int s_item, s_last;
    for (;;) {
        if (threadIdx.x == 0) s_item = (int)atomicAdd(next, 1u);
        __syncthreads();
        const int it = s_item;
        if (it >= n_items) break;
        const uint4 item = items[it];   // frame, tile, chunk
        const BatchFrameDev &f = frames[item.x];
        SweepArgs a;
        a.ref = f.ref;
        a.srcs = f.srcs;
        a.H = f.H;
        a.depths = f.depths;
        a.w = f.w;
        a.h = f.h;
        a.V = f.V;
        a.P = f.P;
        a.planes_per_chunk = f.planes_per_chunk;
        a.n_chunks = f.n_chunks;
        a.stdthresh = f.stdthresh;
        a.packed = nullptr;
        a.wta = f.wta;
        a.cost = nullptr;
        a.quad = f.quad;
        const int tx = (int)item.y % f.tiles_x, ty = (int)item.y / f.tiles_x;
        switch (f.win) {
        case 3: aggregated_tile<3, MOM, TWS, true>(S, a, tx, ty, item.z); break;
        case 5: aggregated_tile<5, MOM, TWS, true>(S, a, tx, ty, item.z); break;
        case 7: aggregated_tile<7, MOM, TWS, true>(S, a, tx, ty, item.z); break;
        case 9: aggregated_tile<9, MOM, TWS, true>(S, a, tx, ty, item.z); break;
        case 11: aggregated_tile<11, MOM, TWS, true>(S, a, tx, ty, item.z); break;
        case 13: aggregated_tile<13, MOM, TWS, true>(S, a, tx, ty, item.z); break;
        default: aggregated_tile<15, MOM, TWS, true>(S, a, tx, ty, item.z); break;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();   // this chunk's winner words before the countdown
            s_last = atomicSub(f.tile_left + item.y, 1u) == 1u;
        }
        __syncthreads();
        if (s_last) {
            __threadfence();
            const int tw = f.tile_w, x0 = tx * tw, y0 = ty * TH;
            for (int k = threadIdx.x; k < tw * TH; k += THREADS) {
                const int x = x0 + k % tw, y = y0 + k / tw;
                if (x >= f.w || y >= f.h) continue;
                const size_t i = (size_t)y * f.w + x;
                const unsigned long long key = __ldcg(f.wta + i);
                const bool ok = key != ~0ull;
                const int lab = ok ? (int)(unsigned)(key & 0xffffffffu) : -1;
                f.depth[i] = ok ? ldg(f.depths + lab) : f.zfar;
                if (f.labels) f.labels[i] = lab;
                if (f.best) f.best[i] = ok ? __uint_as_float((unsigned)(key >> 32)) : 3.f;
                __stcg(f.wta + i, ~0ull);   // re-armed for the next launch
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                f.tile_left[item.y] = (unsigned)f.n_chunks;
                __threadfence();
                if (atomicSub(f.frame_left, 1u) == 1u) {
                    *f.done_ns = global_timer_ns();
                    *f.frame_left = (unsigned)f.n_tiles;
                }
            }
        }
        __syncthreads();   // s_item / s_last are rewritten by the next item
    }
}

// FP64 homographies of every (frame, view, plane) of a batch
__global__ void homography_batch_kernel(const BatchCamDev *__restrict__ cams, const int *__restrict__ offsets,
                                        int n_frames)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= offsets[n_frames]) return;
    int f = 0;
    while (offsets[f + 1] <= idx) ++f;   // frames are few
    const BatchCamDev &c = cams[f];
    const int k = idx - offsets[f];
    const int v = k / c.P, p = k % c.P;
    const double d = (double)c.depths[p];
    const double *R = c.Rrel[v], *t = c.trel[v];
    double M[9], T[9], O[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) M[i] = R[i];
    M[2] += t[0] / d;
    M[5] += t[1] / d;
    M[8] += t[2] / d;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            T[3 * i + j] = fma(c.K[3 * i], M[j], fma(c.K[3 * i + 1], M[3 + j], c.K[3 * i + 2] * M[6 + j]));
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            O[3 * i + j] = fma(T[3 * i], c.invK[j], fma(T[3 * i + 1], c.invK[3 + j], T[3 * i + 2] * c.invK[6 + j]));
    const double sc = O[8];
#pragma unroll
    for (int i = 0; i < 9; ++i) c.H[(size_t)k * 9 + i] = (float)(O[i] / sc);
}

template <int MOM>
int launch_window(int win, const SweepArgs &a, int mode, void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
#define MVS_SWEEP_CASE(WIN)                                                                          \
    case WIN: {                                                                                      \
        dim3 grid(ceil_div(a.w, Geo<WIN>::TW), ceil_div(a.h, TH),                                    \
                  mode == MVS_SWEEP_PER_VIEW ? a.V * a.n_chunks : a.n_chunks);                       \
        if (mode == MVS_SWEEP_PER_VIEW) {                                                            \
            MVS_TRY_CUDA(cudaFuncSetAttribute(sweep_view_kernel<WIN, MOM>,                              \
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,              \
                                              (int)sizeof(AggSmem)));                                    \
            sweep_view_kernel<WIN, MOM><<<grid, THREADS, sizeof(AggSmem), st>>>(a);                    \
        } else {                                                                                     \
            MVS_TRY_CUDA(cudaFuncSetAttribute(sweep_aggregated_kernel<WIN, MOM>,                        \
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,              \
                                              (int)sizeof(AggSmem)));                                    \
            sweep_aggregated_kernel<WIN, MOM><<<grid, THREADS, sizeof(AggSmem), st>>>(a);              \
        }                                                                                            \
        return check_launch("sweep kernel");                                                         \
    }
    switch (win) {
        MVS_SWEEP_CASE(3)
        MVS_SWEEP_CASE(5)
        MVS_SWEEP_CASE(7)
        MVS_SWEEP_CASE(9)
        MVS_SWEEP_CASE(11)
        MVS_SWEEP_CASE(13)
        MVS_SWEEP_CASE(15)
    }
#undef MVS_SWEEP_CASE
    return set_error(MVS_ERR_ARG, "window %d not supported (odd, 3..15)", win);
}

// The source stack [V][H][W] as a TMA tensor map (boxes of STG_W x STG_H x 1;
// out-of-range elements read as zero).  false if the driver entry point is
// missing or the layout does not qualify (rows must be whole 16-byte groups).
bool make_source_map(CUtensorMap *m, const float *srcs, int w, int h, int V)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", (void **)&encode, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            encode = nullptr;
        cudaGetLastError();
    }
    if (!encode || (w & 3) || ((uintptr_t)srcs & 15)) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)V};
    const cuuint64_t strides[2] = {(cuuint64_t)w * 4, (cuuint64_t)w * h * 4};
    const cuuint32_t box[3] = {STG_W, STG_H, 1}, es[3] = {1, 1, 1};
    return encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)srcs, dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int MOM>
int launch_window_tma(int win, const SweepArgs &a, const CUtensorMap &tmap, void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
#define MVS_SWEEP_TMA_CASE(WIN)                                                                          \
    case WIN: {                                                                                          \
        dim3 grid(ceil_div(a.w, Geo<WIN>::TW), ceil_div(a.h, TH), a.n_chunks);                           \
        MVS_TRY_CUDA(cudaFuncSetAttribute(sweep_aggregated_tma_kernel<WIN, MOM>,                         \
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStgBytes)); \
        sweep_aggregated_tma_kernel<WIN, MOM><<<grid, THREADS, kStgBytes, st>>>(a, tmap);               \
        return check_launch("sweep kernel (TMA-staged)");                                                \
    }
    switch (win) {
        MVS_SWEEP_TMA_CASE(3)
        MVS_SWEEP_TMA_CASE(5)
        MVS_SWEEP_TMA_CASE(7)
        MVS_SWEEP_TMA_CASE(9)
        MVS_SWEEP_TMA_CASE(11)
        MVS_SWEEP_TMA_CASE(13)
        MVS_SWEEP_TMA_CASE(15)
    }
#undef MVS_SWEEP_TMA_CASE
    return set_error(MVS_ERR_ARG, "window %d not supported (odd, 3..15)", win);
}

// The aggregated sweep with TMA-staged source regions is opt-in: set
// MVS_SWEEP_STAGING=tma in the environment (looked up at every call).  It
// needs a caller workspace (for its error word) and rows of whole 16-byte
// groups; otherwise the gather form runs.
bool staging_requested()
{
    const char *e = getenv("MVS_SWEEP_STAGING");
    return e && strcmp(e, "tma") == 0;
}

int tiles_for(int win, int w, int h)
{
    int tw = ((RWMAX - 2 * (win / 2)) / 8) * 8;
    return ceil_div(w, tw) * ceil_div(h, TH);
}

}  // namespace

// Plane chunking: enough CTAs for a few waves at 2 CTAs per SM, chunks of at
// least 16 planes so the per-CTA start-up (reference moments) stays amortised.
int sweep_pick_chunks(int win, int w, int h, int V, int P, int mode)
{
    const int tiles = tiles_for(win, w, h) * (mode == MVS_SWEEP_PER_VIEW ? V : 1);
    const int target = 4 * 2 * kSMs;
    int chunks = ceil_div(target, tiles);
    chunks = max(1, min(chunks, P / 16 > 0 ? P / 16 : 1));
    return chunks;
}

size_t sweep_scratch_bytes(const mvs_sweep_desc *d)
{
    const size_t n = (size_t)d->width * d->height;
    return (d->mode == MVS_SWEEP_PER_VIEW ? n * d->n_views : n) * sizeof(unsigned long long);
}

size_t sweep_quad_bytes(const mvs_sweep_desc *d)
{
    return (size_t)d->width * d->height * d->n_views * sizeof(float4);
}

int sweep_launch(const mvs_sweep_desc *d, const float *ref, const float *srcs, const float *H, const float *depths,
                 float *depth, int32_t *labels, float *best, uint16_t *cost, unsigned long long *scratch,
                 int n_chunks, void *stream, float4 *quad)
{
    cudaStream_t st = (cudaStream_t)stream;
    const int n = d->width * d->height;
    SweepArgs a;
    a.ref = ref;
    a.srcs = srcs;
    a.H = H;
    a.depths = depths;
    a.w = d->width;
    a.h = d->height;
    a.V = d->n_views;
    a.P = d->n_planes;
    a.n_chunks = n_chunks;
    a.planes_per_chunk = ceil_div(d->n_planes, n_chunks);
    a.n_chunks = ceil_div(d->n_planes, a.planes_per_chunk);
    a.stdthresh = d->std_threshold;
    a.packed = nullptr;
    a.wta = nullptr;
    a.cost = nullptr;
    a.quad = nullptr;
    a.err = nullptr;
    CUtensorMap tmap;
    const bool tma = d->mode == MVS_SWEEP_AGGREGATED && quad && staging_requested() &&
                     make_source_map(&tmap, srcs, d->width, d->height, d->n_views);
    if (tma) {
        // the staged form samples the sources themselves: the quad area holds its error word instead
        a.err = reinterpret_cast<int *>(quad);
        MVS_TRY_CUDA(cudaMemsetAsync(a.err, 0, sizeof(int), st));
        quad = nullptr;
    }
    if (quad) {
        const size_t total = (size_t)n * d->n_views;
        const size_t blocks = (total + 255) / 256 < (size_t)16 * kSMs ? (total + 255) / 256 : (size_t)16 * kSMs;
        quad_kernel<<<(int)blocks, 256, 0, st>>>(srcs, d->n_views, d->width, d->height, quad,
                                                 d->moments == MVS_MOMENTS_COMPENSATED);
        a.quad = quad;
    }
    if (d->mode == MVS_SWEEP_PER_VIEW) {
        a.packed = scratch;
        if (a.n_chunks > 1)
            MVS_TRY_CUDA(cudaMemsetAsync(scratch, 0, sizeof(unsigned long long) * (size_t)n * d->n_views, st));
    } else {
        a.wta = scratch;
        a.cost = cost;
        if (a.n_chunks > 1) MVS_TRY_CUDA(cudaMemsetAsync(scratch, 0xff, sizeof(unsigned long long) * (size_t)n, st));
    }
    int rc;
    if (tma)
        rc = d->moments == MVS_MOMENTS_REFERENCE ? launch_window_tma<MVS_MOMENTS_REFERENCE>(d->window, a, tmap, stream)
                                                 : launch_window_tma<MVS_MOMENTS_COMPENSATED>(d->window, a, tmap, stream);
    else
        rc = d->moments == MVS_MOMENTS_REFERENCE ? launch_window<MVS_MOMENTS_REFERENCE>(d->window, a, d->mode, stream)
                                                 : launch_window<MVS_MOMENTS_COMPENSATED>(d->window, a, d->mode, stream);
    if (rc) return rc;
    const int eb = 256, eg = min(ceil_div(n, eb), 8 * kSMs);
    if (d->mode == MVS_SWEEP_PER_VIEW) {
        sweep_combine_kernel<<<eg, eb, 0, st>>>(scratch, depths, n, d->n_views, d->ncc_threshold, d->zfar, depth,
                                                labels, best);
    } else {
        wta_finish_kernel<<<eg, eb, 0, st>>>(scratch, depths, n, d->zfar, depth, labels, best);
    }
    rc = check_launch("sweep epilogue");
    if (!rc && tma) {
        int h_err = 0;
        MVS_TRY_CUDA(cudaMemcpyAsync(&h_err, a.err, sizeof(int), cudaMemcpyDeviceToHost, st));
        MVS_TRY_CUDA(cudaStreamSynchronize(st));
        if (h_err) rc = set_error(MVS_ERR_TIMEOUT, "sweep: a TMA staging wait gave up");
    }
    return rc;
}

// output columns of a tile for a window and a narrowing step (Geo::TW)
int sweep_tile_width(int win, int tws) { return ((RWMAX - 2 * (win / 2)) / 8 - tws) * 8; }
int sweep_tile_height() { return TH; }

int sweep_batch_launch(const BatchFrameDev *frames, const uint4 *items, int n_items, unsigned int *next,
                       unsigned long long *t_start, const BatchCamDev *cams, const int *hom_offsets, int n_frames,
                       int n_hom, int moments, int ctas, int tws, void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (tws < 0 || tws > 1) return set_error(MVS_ERR_ARG, "tile step %d (0 or 1)", tws);
    batch_start_kernel<<<1, 1, 0, st>>>(next, t_start);
    if (n_hom > 0) homography_batch_kernel<<<ceil_div(n_hom, 128), 128, 0, st>>>(cams, hom_offsets, n_frames);
    quad_batch_kernel<<<dim3(max(1, 4 * kSMs / max(1, n_frames)), n_frames), 256, 0, st>>>(
        frames, moments == MVS_MOMENTS_COMPENSATED);
    const int sm = (int)sizeof(AggSmem);
#define MVS_BATCH_LAUNCH(MOM, TWS)                                                                        \
    do {                                                                                                  \
        MVS_TRY_CUDA(cudaFuncSetAttribute(sweep_batch_kernel<MOM, TWS>,                                   \
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, sm));               \
        sweep_batch_kernel<MOM, TWS><<<ctas, THREADS, sm, st>>>(frames, items, n_items, next);            \
    } while (0)
    if (moments == MVS_MOMENTS_REFERENCE) {
        if (tws == 0) MVS_BATCH_LAUNCH(MVS_MOMENTS_REFERENCE, 0);
        else MVS_BATCH_LAUNCH(MVS_MOMENTS_REFERENCE, 1);
    } else {
        if (tws == 0) MVS_BATCH_LAUNCH(MVS_MOMENTS_COMPENSATED, 0);
        else MVS_BATCH_LAUNCH(MVS_MOMENTS_COMPENSATED, 1);
    }
#undef MVS_BATCH_LAUNCH
    return check_launch("sweep batch");
}

int sweep_wta_volume(const uint16_t *cost, const float *depths, int n, int P, float zfar, float *depth,
                     int32_t *labels, float *best, void *stream)
{
    if (n % 8) return set_error(MVS_ERR_ARG, "WTA over a cost volume needs W*H divisible by 8");
    wta_volume_kernel<<<ceil_div(n / 8, 32), 32 * WTA_WARPS, 0, (cudaStream_t)stream>>>(cost, depths, n, P, zfar,
                                                                                       depth, labels, best);
    return check_launch("wta_volume_kernel");
}

int sweep_homographies(const double *K, const double *invK, const double *Rrel, const double *trel,
                       const float *depths, int V, int P, float *H, void *stream)
{
    for (int v0 = 0; v0 < V; v0 += kHomViews) {
        const int nv = min(kHomViews, V - v0);
        HomCams c;
        for (int i = 0; i < 9; ++i) {
            c.K[i] = K[i];
            c.invK[i] = invK[i];
        }
        for (int v = 0; v < nv; ++v) {
            for (int i = 0; i < 9; ++i) c.Rrel[v][i] = Rrel[9 * (v0 + v) + i];
            for (int i = 0; i < 3; ++i) c.trel[v][i] = trel[3 * (v0 + v) + i];
        }
        const int n = nv * P;
        homography_kernel<<<ceil_div(n, 128), 128, 0, (cudaStream_t)stream>>>(c, depths, nv, P,
                                                                               H + (size_t)v0 * P * 9);
    }
    return check_launch("homography_kernel");
}

}  // namespace mvs
