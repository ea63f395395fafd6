// TV-L1 histogram depthmap fusion for sm_100a (fusion.cu / fusion.h of the
// reference).
//
// Volume layout (structure of arrays, x fastest; n voxels):
//   u[n], v[n]      float primal and over-relaxed primal
//   p[3][n]         float dual, one plane per component
//   hist[n][HS]     uint16 counts, HS = 8 (bins <= 8) or 16, so a voxel's
//                   histogram is one or two 128-bit accesses
// The reference stores an array of 28-byte structs {u, v, float3 p, uint8
// h[N]} (structs.h:131-189), which every pass reads whole.
//
// Kernels:
//   histogram   one voxel pass for a batch of depthmaps: project, sample,
//               vote into registers, store once (FusionUpdateHistogram_kernel
//               + fusionData::updateHist, fusion.cu:5-43, fusion.h:883-907)
//   update_u    FusionUpdateU_kernel (fusion.cu:45-57) with the histogram
//               proximal median computed in closed form (see prox_median)
//   update_p    FusionUpdateP_kernel (fusion.cu:59-70)
// Arithmetic follows the reference statement for statement (-fmad=false).
#include <math.h>

#include <algorithm>

#include "common.cuh"

// With 2 bins the threshold is 0 (fusion.h:888) and the in-between branch,
// reached only by a NaN signed distance, divides by it, as the reference does.
#pragma nv_diag_suppress 39

namespace mvs {

namespace {

template <int BINS>
struct HistStride {
    static constexpr int value = BINS <= 8 ? 8 : 16;
};

struct Dims {
    int vw, vh, vd;
    float ax, ay, az;     // volume corner a
    float sx, sy, sz;     // b - a
};

__device__ __forceinline__ void voxel_xyz(const Dims &D, long i, int &x, int &y, int &z)
{
    x = (int)(i % D.vw);
    y = (int)((i / D.vw) % D.vh);
    z = (int)(i / ((long)D.vw * D.vh));
}

template <int HS>
__device__ __forceinline__ void load_counts(const uint16_t *__restrict__ hist, long i, uint32_t *c)
{
    const uint4 *q = reinterpret_cast<const uint4 *>(hist + (size_t)i * HS);
#pragma unroll
    for (int k = 0; k < HS / 8; ++k) {
        const uint4 v = q[k];
        const uint32_t w4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            c[8 * k + 2 * j] = w4[j] & 0xffffu;
            c[8 * k + 2 * j + 1] = w4[j] >> 16;
        }
    }
}

template <int HS>
__device__ __forceinline__ void store_counts(uint16_t *__restrict__ hist, long i, const uint32_t *c)
{
    uint4 *q = reinterpret_cast<uint4 *>(hist + (size_t)i * HS);
#pragma unroll
    for (int k = 0; k < HS / 8; ++k) {
        uint4 v;
        v.x = (c[8 * k + 0] & 0xffffu) | (c[8 * k + 1] << 16);
        v.y = (c[8 * k + 2] & 0xffffu) | (c[8 * k + 3] << 16);
        v.z = (c[8 * k + 4] & 0xffffu) | (c[8 * k + 5] << 16);
        v.w = (c[8 * k + 6] & 0xffffu) | (c[8 * k + 7] << 16);
        q[k] = v;
    }
}

// Launch shape of the voxel kernels: a (32, 8, 1) block per 32 x 8 patch of
// one z slice; grid (vw/32, vh/8, vd).  No index division anywhere.
constexpr int VX = 32, VY = 8;

template <int BINS>
__global__ void __launch_bounds__(VX *VY) histogram_kernel(Dims D, uint16_t *__restrict__ hist,
                                                          const float *__restrict__ depths, int w, int h, int nmaps,
                                                          const float *__restrict__ cams, float threshold)
{
    constexpr int HS = HistStride<BINS>::value;
    const int x = blockIdx.x * VX + threadIdx.x, y = blockIdx.y * VY + threadIdx.y, z = blockIdx.z;
    if (x >= D.vw || y >= D.vh) return;
    const size_t i = (size_t)z * D.vw * D.vh + (size_t)y * D.vw + x;
    const float thresh = BINS == 2 ? 0.f : threshold;
    // fusionData::worldCoords (fusion.h:360-364): (x + .5) / width in double
    const float wx = (float)((x + .5) / D.vw), wy = (float)((y + .5) / D.vh), wz = (float)((z + .5) / D.vd);
    const float cx = D.ax + D.sx * wx, cy = D.ay + D.sy * wy, cz = D.az + D.sz * wz;
    uint32_t cnt[HS];
    load_counts<HS>(hist, (long)i, cnt);
    for (int m = 0; m < nmaps; ++m) {
        const float *K = cams + kMapCamFloats * m, *R = K + 9, *t = K + 18;
        // c = R c + T; c = K c (fusion.cu:17-20)
        const float r0 = ldg(R + 0) * cx + ldg(R + 1) * cy + ldg(R + 2) * cz + ldg(t + 0);
        const float r1 = ldg(R + 3) * cx + ldg(R + 4) * cy + ldg(R + 5) * cz + ldg(t + 1);
        const float r2 = ldg(R + 6) * cx + ldg(R + 7) * cy + ldg(R + 8) * cz + ldg(t + 2);
        const float k0 = ldg(K + 0) * r0 + ldg(K + 1) * r1 + ldg(K + 2) * r2;
        const float k1 = ldg(K + 3) * r0 + ldg(K + 4) * r1 + ldg(K + 5) * r2;
        const float k2 = ldg(K + 6) * r0 + ldg(K + 7) * r1 + ldg(K + 8) * r2;
        const float px = k0 / k2, py = k1 / k2;
        if ((px < 0) || (px > w - 1) || (py < 0) || (py > h - 1)) continue;
        // The reference's floorf, (int)fmaxf(., 0) and (int)fminf(x0 + 1, w - 1),
        // without the conversion unit: here 0 <= p <= w - 1 < 2^22 (or p is
        // NaN, which fmaxf turns into 0 as the reference's does, and the
        // fraction stays NaN), so p + 1.5 * 2^23 rounded down is 1.5 * 2^23 +
        // floor(p) exactly, whose low bits are floor(p) (a standard
        // magic-number floor).
        const float pxc = fmaxf(px, 0.f), pyc = fmaxf(py, 0.f);
        const float tx = __fadd_rd(pxc, 12582912.f), ty = __fadd_rd(pyc, 12582912.f);
        const float flx = tx - 12582912.f, fly = ty - 12582912.f;
        const int x0 = __float_as_int(tx) - 0x4B400000, y0 = __float_as_int(ty) - 0x4B400000;
        const int x1 = min(x0 + 1, w - 1), y1 = min(y0 + 1, h - 1);
        const float frx = px - flx, fry = py - fly;
        const float *dm = depths + (size_t)m * w * h;
        const float d00 = ldg(dm + x0 + y0 * w), d10 = ldg(dm + x1 + y0 * w);
        const float d01 = ldg(dm + x0 + y1 * w), d11 = ldg(dm + x1 + y1 * w);
        // bilinterp (dev_functions.h:33-38): lerp in y, then in x
        const float l0 = d00 + fry * (d01 - d00), l1 = d10 + fry * (d11 - d10);
        const float depth = l0 + frx * (l1 - l0);
        const float sd = depth - k2;
        int bin;
        if (sd >= thresh) bin = BINS - 1;
        else if (sd <= -thresh) bin = 0;
        else bin = (int)(unsigned char)fminf(roundf((sd + thresh) / (2.f * thresh) * (BINS - 3) + 1), BINS - 2);
#pragma unroll
        for (int k = 0; k < BINS; ++k) cnt[k] += (bin == k);
    }
    store_counts<HS>(hist, (long)i, cnt);
}

// Bin centres (fusion.h:1041-1054).
template <int BINS>
__device__ __forceinline__ float bin_center(int i)
{
    if (i == 0) return -1.f;
    if (i == BINS - 1) return 1.f;
    if (BINS > 3) return 2.f * (float)(i - 1) / (float)(BINS > 3 ? BINS - 3 : 1) - 1.f;
    return 0.f;
}

// fusionData::proxHist (fusion.h:851-858): the element of rank N (0-based)
// after inserting u and the N values u + tau*lambda*W_j into the sorted bin
// centres with sortedHist::insert (structs.h:241-262).  That insertion never
// stores a value below the current first element (the loop ends with the
// first element duplicated instead), and the first element is the lowest bin
// centre, -1; so the result is the rank-N element of
//   A = bin centres (ascending),  B = max(-1, u + tl W_j) (ascending in
//   reverse j: W_j falls with j),  and max(-1, u).
// For two ascending length-N lists the rank N-1 and rank N elements of their
// union are min_i max(A[i-1], B[N-1-i]) and max_i min(A[i], B[N-i]); with the
// single extra value u the answer is u clamped to that pair.
template <int BINS>
__device__ __forceinline__ float prox_median(const uint32_t *cnt, float u, float tl)
{
    int total = 0;
#pragma unroll
    for (int k = 0; k < BINS; ++k) total += (int)cnt[k];
    float Bv[BINS];   // ascending
    // (float)W without the conversion unit: |W| <= total < 2^22, so the bits
    // 0x4B400000 + W are the float 1.5 * 2^23 + W exactly, and subtracting
    // 1.5 * 2^23 leaves W exactly (a standard magic-number conversion)
    const int biased = total + 0x4B400000;
    int pre = 0;
#pragma unroll
    for (int j = 1; j <= BINS; ++j) {
        pre += (int)cnt[j - 1];
        const float W = __int_as_float(biased - 2 * pre) - 12582912.f;   // Wi(j), fusion.h:813-820
        const float pj = u + tl * W;
        Bv[BINS - j] = fmaxf(pj, -1.f);
    }
    const float NEG = -INFINITY, POS = INFINITY;
    float lo = POS, hi = NEG;
#pragma unroll
    for (int i = 0; i <= BINS; ++i) {
        const float a_lo = i > 0 ? bin_center<BINS>(i - 1) : NEG;
        const float b_lo = (BINS - 1 - i) >= 0 ? Bv[BINS - 1 - i] : NEG;
        lo = fminf(lo, fmaxf(a_lo, b_lo));
        const float a_hi = i < BINS ? bin_center<BINS>(i) : POS;
        const float b_hi = (BINS - i) < BINS ? Bv[BINS - i] : POS;
        hi = fmaxf(hi, fminf(a_hi, b_hi));
    }
    const float uc = fmaxf(u, -1.f);
    return fminf(fmaxf(uc, lo), hi);
}

// The U step of one voxel (FusionUpdateU_kernel, fusion.cu:45-57): u + tau
// div p, the histogram proximal median, and v = 2 u_new - u_old.
template <int BINS>
__device__ __forceinline__ float u_step(float div, float u_old, const uint32_t *cnt, double tau, float tl, float &v_new)
{
    const double un = u_old;
    const double uu = un - tau * (-(double)div);
    const float m = prox_median<BINS>(cnt, (float)uu, tl);
    v_new = (float)((double)(2 * m) - un);
    return m;
}

// The P step of one voxel (FusionUpdateP_kernel, fusion.cu:59-70): p + sigma
// grad v with the forward differences of gradVFwd (fusion.h:773-781, zero at
// the far faces: hx, hy, hz say whether the +x, +y, +z neighbour exists),
// then projectUnitBall (fusion.h:866-870; dividing by exactly 1 is the identity).
__device__ __forceinline__ void p_step(float px, float py, float pz, float vi, float vx1, float vy1, float vz1, bool hx,
                                       bool hy, bool hz, float sigma, float &qx, float &qy, float &qz)
{
    const float gx = hx ? vx1 - vi : 0.f;
    const float gy = hy ? vy1 - vi : 0.f;
    const float gz = hz ? vz1 - vi : 0.f;
    qx = px + sigma * gx;
    qy = py + sigma * gy;
    qz = pz + sigma * gz;
    const float d = fmaxf(1.f, sqrtf(qx * qx + qy * qy + qz * qz));
    if (d != 1.f) {
        qx = qx / d;
        qy = qy / d;
        qz = qz / d;
    }
}

template <int BINS>
__global__ void __launch_bounds__(VX *VY) update_u_kernel(Dims D, const uint16_t *__restrict__ hist,
                                                         float *__restrict__ u, float *__restrict__ v,
                                                         const float *__restrict__ p, double tau, double lambda)
{
    wait_for_previous_grid();   // launched as a dependent launch: the previous step is complete
    allow_next_grid();
    constexpr int HS = HistStride<BINS>::value;
    const int x = blockIdx.x * VX + threadIdx.x, y = blockIdx.y * VY + threadIdx.y, z = blockIdx.z;
    if (x >= D.vw || y >= D.vh) return;
    const size_t sz = (size_t)D.vw * D.vh, n = sz * D.vd;
    const size_t i = (size_t)z * sz + (size_t)y * D.vw + x;
    const float *px = p, *py = p + n, *pz = p + 2 * n;
    const float tl = (float)tau * (float)lambda;
    // divPBwd (fusion.h:793-802)
    float div = px[i] + py[i] + pz[i];
    if (x > 0) div -= px[i - 1];
    if (y > 0) div -= py[i - D.vw];
    if (z > 0) div -= pz[i - sz];
    uint32_t cnt[HS];
    load_counts<HS>(hist, (long)i, cnt);
    float vn;
    u[i] = u_step<BINS>(div, u[i], cnt, tau, tl, vn);
    v[i] = vn;
}

__global__ void __launch_bounds__(VX *VY) update_p_kernel(Dims D, const float *__restrict__ v, float *__restrict__ p,
                                                         float sigma)
{
    wait_for_previous_grid();   // launched as a dependent launch: the previous step is complete
    allow_next_grid();
    const int x = blockIdx.x * VX + threadIdx.x, y = blockIdx.y * VY + threadIdx.y, z = blockIdx.z;
    if (x >= D.vw || y >= D.vh) return;
    const size_t sz = (size_t)D.vw * D.vh, n = sz * D.vd;
    const size_t i = (size_t)z * sz + (size_t)y * D.vw + x;
    float *px = p, *py = p + n, *pz = p + 2 * n;
    const bool hx = x < D.vw - 1, hy = y < D.vh - 1, hz = z < D.vd - 1;
    const float vi = v[i];
    float qx, qy, qz;
    p_step(px[i], py[i], pz[i], vi, hx ? v[i + 1] : 0.f, hy ? v[i + D.vw] : 0.f, hz ? v[i + sz] : 0.f, hx, hy, hz,
           sigma, qx, qy, qz);
    px[i] = qx;
    py[i] = qy;
    pz[i] = qz;
}

__global__ void extract_count_kernel(const float *__restrict__ u, long n, float lo, float hi,
                                     unsigned long long *__restrict__ block_counts)
{
    __shared__ unsigned int c;
    if (threadIdx.x == 0) c = 0;
    __syncthreads();
    const long base = (long)blockIdx.x * 4096;
    unsigned int mine = 0;
    for (int k = threadIdx.x; k < 4096; k += blockDim.x) {
        const long i = base + k;
        if (i < n && u[i] > lo && u[i] < hi) ++mine;
    }
    atomicAdd(&c, mine);
    __syncthreads();
    if (threadIdx.x == 0) block_counts[blockIdx.x] = c;
}

// Second pass: block b writes its voxels in index order starting at offs[b].
__global__ void extract_write_kernel(Dims D, const float *__restrict__ u, long n, float lo, float hi,
                                     const unsigned long long *__restrict__ offs, float *__restrict__ xyz,
                                     long capacity)
{
    __shared__ unsigned int scan[256];
    const long base = (long)blockIdx.x * 4096;
    unsigned long long o = offs[blockIdx.x];
    for (int chunk = 0; chunk < 4096; chunk += 256) {
        const long i = base + chunk + threadIdx.x;
        const bool keep = i < n && u[i] > lo && u[i] < hi;
        scan[threadIdx.x] = keep;
        __syncthreads();
        for (int s = 1; s < 256; s <<= 1) {
            unsigned int t = threadIdx.x >= s ? scan[threadIdx.x - s] : 0;
            __syncthreads();
            scan[threadIdx.x] += t;
            __syncthreads();
        }
        const unsigned int incl = scan[threadIdx.x], total = scan[255];
        if (keep) {
            const unsigned long long k = o + incl - 1;
            if ((long)k < capacity) {
                int x, y, z;
                voxel_xyz(D, i, x, y, z);
                xyz[3 * k + 0] = D.ax + D.sx * (float)((x + .5) / D.vw);
                xyz[3 * k + 1] = D.ay + D.sy * (float)((y + .5) / D.vh);
                xyz[3 * k + 2] = D.az + D.sz * (float)((z + .5) / D.vd);
            }
        }
        o += total;
        __syncthreads();
    }
}

Dims dims_of(int vw, int vh, int vd, const float *a, const float *b)
{
    Dims D;
    D.vw = vw;
    D.vh = vh;
    D.vd = vd;
    D.ax = a[0];
    D.ay = a[1];
    D.az = a[2];
    D.sx = b[0] - a[0];
    D.sy = b[1] - a[1];
    D.sz = b[2] - a[2];
    return D;
}

const float kZero3[3] = {0.f, 0.f, 0.f};

dim3 voxel_grid(int vw, int vh, int vd) { return dim3((vw + VX - 1) / VX, (vh + VY - 1) / VY, vd); }

}  // namespace

int fusion_hist_stride(int bins) { return bins <= 8 ? 8 : 16; }

#define MVS_BINS(X) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10)

int fusion_histogram(int vw, int vh, int vd, int bins, const float *a, const float *b, uint16_t *hist,
                     const float *depths, int nmaps, int w, int h, const float *d_cams, float thr, cudaStream_t st)
{
    const Dims D = dims_of(vw, vh, vd, a, b);
    switch (bins) {
#define H(N) case N: histogram_kernel<N><<<voxel_grid(vw, vh, vd), dim3(VX, VY), 0, st>>>(D, hist, depths, w, h, nmaps, d_cams, thr); break;
        MVS_BINS(H)
#undef H
    default: return set_error(MVS_ERR_ARG, "bins %d not supported (2..10)", bins);
    }
    return check_launch("fusion histogram_kernel");
}

int fusion_update_u(int vw, int vh, int vd, int bins, const uint16_t *hist, float *u, float *v, const float *p,
                    double tau, double lambda, cudaStream_t st)
{
    const Dims D = dims_of(vw, vh, vd, kZero3, kZero3);
    switch (bins) {
#define U(N) case N: MVS_TRY_CUDA(launch_dependent(update_u_kernel<N>, voxel_grid(vw, vh, vd), dim3(VX, VY), 0, st, D, hist, u, v, p, tau, lambda)); break;
        MVS_BINS(U)
#undef U
    default: return set_error(MVS_ERR_ARG, "bins %d not supported (2..10)", bins);
    }
    return check_launch("fusion update_u_kernel");
}

int fusion_update_p(int vw, int vh, int vd, const float *v, float *p, double sigma, cudaStream_t st)
{
    const Dims D = dims_of(vw, vh, vd, kZero3, kZero3);
    MVS_TRY_CUDA(launch_dependent(update_p_kernel, voxel_grid(vw, vh, vd), dim3(VX, VY), 0, st, D, v, p, (float)sigma));
    return check_launch("fusion update_p_kernel");
}

long fusion_extract_blocks(long n) { return (n + 4095) / 4096; }

int fusion_extract(int vw, int vh, int vd, const float *a, const float *b, const float *u, float lo, float hi,
                   unsigned long long *d_counts, unsigned long long *h_counts, float *d_xyz, long capacity,
                   long *total, cudaStream_t st)
{
    const Dims D = dims_of(vw, vh, vd, a, b);
    const long n = (long)vw * vh * vd;
    const long nb = fusion_extract_blocks(n);
    extract_count_kernel<<<(unsigned)nb, 256, 0, st>>>(u, n, lo, hi, d_counts);
    MVS_TRY_CUDA(cudaMemcpyAsync(h_counts, d_counts, nb * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    MVS_TRY_CUDA(cudaStreamSynchronize(st));
    unsigned long long acc = 0;
    for (long k = 0; k < nb; ++k) {
        const unsigned long long c = h_counts[k];
        h_counts[k] = acc;
        acc += c;
    }
    *total = (long)acc;
    if (d_xyz && capacity > 0 && acc > 0) {
        MVS_TRY_CUDA(cudaMemcpyAsync(d_counts, h_counts, nb * sizeof(unsigned long long), cudaMemcpyHostToDevice, st));
        extract_write_kernel<<<(unsigned)nb, 256, 0, st>>>(D, u, n, lo, hi, d_counts, d_xyz, capacity);
    }
    return check_launch("fusion extract");
}

}  // namespace mvs
