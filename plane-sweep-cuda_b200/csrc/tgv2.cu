// TGV2-L1 multiview refinement for sm_100a.
//
// The reference runs one full-image launch per update per view
// (planesweep.cpp:442-509: updateP, updateQ, prodsum reset, V x updateR,
// updateU, i.e. 4 + V passes per iteration).  Here one launch does a whole
// iteration: a 32 x 8 tile recomputes the new dual variables p, q on a
// one-pixel halo to its left and top (the backward differences of the primal
// step read them there), updates every view's r and the running sum
// sum_i r_i Iu_i in registers, and writes u, v, ubar, vbar.  Variables that
// are read at neighbouring pixels (ubar, vbar, p, q) are double-buffered, so
// one launch never reads what another CTA of the same launch writes.
//
// Arithmetic is the reference's, statement for statement (float storage, the
// double intermediates it uses, the same order; the file is compiled with
// -fmad=false), so the iteration reproduces the reference's roundings.  The
// qw component is not stored: the reference updates qz and qw with the same
// expression from the same inputs, so they are always equal
// (TGV2_kernels.cu:77-78).  T21 == T12 likewise (TGV2_kernels.cu:286-287).
#include <math.h>

#include "common.cuh"

namespace mvs {
namespace {

constexpr float kInv255 = 1.f / 255.f;
constexpr int TX = 32, TY = 8;
constexpr int kMaxViews = 32;

struct Cams {
    float K[9], invK[9];
    float Rrel[kMaxViews][9];
    float trel[kMaxViews][3];
};

__device__ __forceinline__ void matvec(const float *M, float x, float y, float z, float &a, float &b, float &c)
{
    a = M[0] * x + M[1] * y + M[2] * z;
    b = M[3] * x + M[4] * y + M[5] * z;
    c = M[6] * x + M[7] * y + M[8] * z;
}

// Anisotropic_diffusion_tensor_kernel (TGV2_kernels.cu:257-298) on ref/255,
// which is also stored (element_scale, planesweep.cpp:419).
__global__ void tensor_kernel(const float *__restrict__ ref255, int w, int h, float beta, float gamma,
                              float *__restrict__ ref01, float *__restrict__ T11, float *__restrict__ T12,
                              float *__restrict__ T22)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const int i = y * w + x, xn = min(x + 1, w - 1), yn = min(y + 1, h - 1);
    const float r = ref255[i] * kInv255;
    float gx = ref255[y * w + xn] * kInv255 - r;
    float gy = ref255[yn * w + x] * kInv255 - r;
    const float d = sqrtf(gx * gx + gy * gy);
    ref01[i] = r;
    if (d > 0.f) {
        gx = gx / d;
        gy = gy / d;
        const float k = expf(-beta * powf(d, gamma));
        T11[i] = k * gx * gx + gy * gy;
        T12[i] = (k - 1) * gx * gy;
        T22[i] = k * gy * gy + gx * gx;
    } else {
        T11[i] = 1.f;
        T12[i] = 0.f;
        T22[i] = 1.f;
    }
}

// The per-view arrays r, It and Iu are stored view-interleaved, [pixel][VS]
// with VS = V rounded up to a multiple of 4, so a pixel's views are whole
// 16-byte words (the padding entries are never used).
__host__ __device__ constexpr int view_stride(int V) { return (V + 3) & ~3; }

// Start of a linearisation (planesweep.cpp:445-458,482): u0 = ubar = u, the
// other primal/dual variables and r to zero.
__global__ void warp_init_kernel(int n, int V, const float *__restrict__ u, float *__restrict__ u0,
                                 float *__restrict__ ubar, float *__restrict__ u1x, float *__restrict__ u1y,
                                 float *__restrict__ u1xbar, float *__restrict__ u1ybar, float *__restrict__ Px,
                                 float *__restrict__ Py, float *__restrict__ Qx, float *__restrict__ Qy,
                                 float *__restrict__ Qz, float *__restrict__ r)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float v = u[i];
        u0[i] = v;
        ubar[i] = v;
        u1x[i] = u1y[i] = u1xbar[i] = u1ybar[i] = 0.f;
        Px[i] = Py[i] = Qx[i] = Qy[i] = Qz[i] = 0.f;
        const int VS = view_stride(V);
        for (int k = 0; k < VS; ++k) r[(size_t)i * VS + k] = 0.f;
    }
}

// Start of a warm-started linearisation: the data term is linearised at
// u_lin while the primal starts at (u, v) -- e.g. a learned prediction of the
// converged solution; dual variables and r start at zero.
__global__ void warm_init_kernel(int n, int V, const float *__restrict__ u_lin, const float *__restrict__ u,
                                 const float *__restrict__ vx, const float *__restrict__ vy, float *__restrict__ u0,
                                 float *__restrict__ ubar, float *__restrict__ u1x, float *__restrict__ u1y,
                                 float *__restrict__ u1xbar, float *__restrict__ u1ybar, float *__restrict__ Px,
                                 float *__restrict__ Py, float *__restrict__ Qx, float *__restrict__ Qy,
                                 float *__restrict__ Qz, float *__restrict__ r, const float *__restrict__ pq_in,
                                 const float *__restrict__ r_in)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        u0[i] = u_lin[i];
        ubar[i] = u[i];
        const float a = vx ? vx[i] : 0.f, c = vy ? vy[i] : 0.f;
        u1x[i] = u1xbar[i] = a;
        u1y[i] = u1ybar[i] = c;
        if (pq_in) {
            Px[i] = pq_in[i];
            Py[i] = pq_in[(size_t)n + i];
            Qx[i] = pq_in[2 * (size_t)n + i];
            Qy[i] = pq_in[3 * (size_t)n + i];
            Qz[i] = pq_in[4 * (size_t)n + i];
        } else {
            Px[i] = Py[i] = Qx[i] = Qy[i] = Qz[i] = 0.f;
        }
        // r_in: the caller's [V][n] planes
        const int VS = view_stride(V);
        for (int k = 0; k < VS; ++k) r[(size_t)i * VS + k] = r_in && k < V ? r_in[(size_t)k * n + i] : 0.f;
    }
}

// view-interleaved r ([pixel][VS]) to [V][n] planes
__global__ void r_planes_kernel(const float *__restrict__ r, int n, int V, float *__restrict__ out)
{
    const int VS = view_stride(V);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int v = 0; v < V; ++v) out[(size_t)v * n + i] = r[(size_t)i * VS + v];
}

__global__ void fill_kernel(float *__restrict__ p, int n, float v)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

// TGV2_transform_coordinates_kernel (TGV2_kernels.cu:141-179) then
// bilinear_interpolation_kernel_GPU (kernels.cu:4-29) of source/255.
__device__ __forceinline__ float warped_at(const Cams &c, int v, const float *__restrict__ src255, int w, int h,
                                           int x, int y, float u0, float &X, float &Y, float &Z)
{
    float ka, kb, kc;
    matvec(c.invK, (float)(x + 1), (float)(y + 1), 1.f, ka, kb, kc);
    const float x1a = u0 * ka, x1b = u0 * kb, x1c = u0 * kc;
    float a2, b2, c2;
    matvec(c.Rrel[v], x1a, x1b, x1c, a2, b2, c2);
    X = a2 + c.trel[v][0];
    Y = b2 + c.trel[v][1];
    Z = c2 + c.trel[v][2];
    float p0, p1, p2;
    matvec(c.K, X, Y, Z, p0, p1, p2);
    const float xs = p0 / p2 - 1, ys = p1 / p2 - 1;
    const float fx = floorf(xs), fy = floorf(ys);
    if (!(fx >= 0.f && fy >= 0.f && fx + 1.f <= (float)(w - 1) && fy + 1.f <= (float)(h - 1))) return 0.f;
    const int ix = (int)fx, iy = (int)fy;
    const float a = xs - (float)ix, b = ys - (float)iy;
    const float *r0 = src255 + (size_t)iy * w + ix;
    const float d00 = ldg(r0) * kInv255, d01 = ldg(r0 + 1) * kInv255;
    const float d10 = ldg(r0 + w) * kInv255, d11 = ldg(r0 + w + 1) * kInv255;
    const float t1 = a * d01 + (1 - a) * d00;
    const float t2 = a * d11 + (1 - a) * d10;
    return b * t2 + (1 - b) * t1;
}

// One view's linearisation at u0 (planesweep.cpp:460-483) in one pass:
// coordinates, their derivatives (TGV2_calculate_coordinate_derivatives_kernel,
// :194-219), df/du (TGV2_calculate_derivativeF_kernel, :221-236), the warped
// source here and at the right and lower neighbours (the forward differences
// of TGV2_calculate_Iu_kernel, :238-255, are taken on the warped image), It.
__global__ void linearize_kernel(Cams c, const float *__restrict__ srcs255, const float *__restrict__ ref01,
                                 const float *__restrict__ u0, int w, int h, float *__restrict__ It,
                                 float *__restrict__ Iu)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    const int v = blockIdx.z;
    if (x >= w || y >= h) return;
    const size_t n = (size_t)w * h;
    const float *src = srcs255 + (size_t)v * n;
    const int i = y * w + x, xn = min(x + 1, w - 1), yn = min(y + 1, h - 1);
    float X, Y, Z, Xd, Yd, Zd;
    const float Iw = warped_at(c, v, src, w, h, x, y, u0[i], X, Y, Z);
    const float Ixn = warped_at(c, v, src, w, h, xn, y, u0[y * w + xn], Xd, Yd, Zd);
    const float Iyn = warped_at(c, v, src, w, h, x, yn, u0[yn * w + x], Xd, Yd, Zd);
    // (Rrel * invK) * (x+1, y+1, 1): the matrix product first, as the reference
    float RK[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q)
            RK[3 * r + q] = c.Rrel[v][3 * r] * c.invK[q] + c.Rrel[v][3 * r + 1] * c.invK[3 + q] +
                            c.Rrel[v][3 * r + 2] * c.invK[6 + q];
    float dX, dY, dZ;
    matvec(RK, (float)(x + 1), (float)(y + 1), 1.f, dX, dY, dZ);
    const float fx = c.K[0], fy = c.K[4];
    const float dfx = fx * (dX * Z - X * dZ) / (Z * Z);
    const float dfy = fy * (dY * Z - Y * dZ) / (Z * Z);
    const double gx = Ixn - Iw, gy = Iyn - Iw;
    const int VS = view_stride((int)gridDim.z);   // one grid layer per view
    Iu[(size_t)i * VS + v] = (float)(gx * (double)dfx + gy * (double)dfy);
    It[(size_t)i * VS + v] = Iw - ref01[i];
}

// Stopping state of a launch-per-iteration run, in device memory.  The energy
// check sets `done` once the tolerance is met; iterations and checks launched
// after that return at once, so the host only polls the flag now and then
// instead of waiting for every energy, and the result is the one of stopping
// at that check.
struct IterCtl {
    int done;          // the tolerance was met
    int n_hist;        // energies evaluated in this linearisation
    int have_energy;   // last_e holds an energy
    int stop_total;    // iteration count at which the tolerance was met
    int energy_at;     // iteration count at which last_e was evaluated
    unsigned int blocks_done;   // energy_kernel blocks finished (the last one resets it)
    double last_e;
    double hist[MVS_TGV2_STOP_WINDOW_MAX];   // the last energies, hist[j % MAX] = E_j
};

// The stopping test at check j of a linearisation (E_j = E, `hist` holding
// E_{j-W} .. E_{j-1} in ring order, `n` = j): the mean relative change per
// check over the last W checks is at most tol.  Records E_j.  W <= MAX, so
// E_{j-W} is read before E_j replaces it in the ring.
__device__ __forceinline__ bool stop_test(double *hist, int n, double E, double tol, int W)
{
    bool met = false;
    if (n >= W) {
        const double old = hist[(n - W) % MVS_TGV2_STOP_WINDOW_MAX];
        met = fabs(old - E) <= tol * (double)W * fabs(old);
    }
    hist[n % MVS_TGV2_STOP_WINDOW_MAX] = E;
    return met;
}

struct IterBufs {
    const IterCtl *ctl;   // null: no stopping test
    const float *T11, *T12, *T22, *u0, *It, *Iu;
    float *u, *u1x, *u1y, *r;
    const float *ubar_in, *u1xbar_in, *u1ybar_in, *Px_in, *Py_in, *Qx_in, *Qy_in, *Qz_in;
    float *ubar_out, *u1xbar_out, *u1ybar_out, *Px_out, *Py_out, *Qx_out, *Qy_out, *Qz_out;
    int w, h, V;
    float lambda, alpha0, alpha1, tau, sigma;
};

// fmaxf(1.f, (float)sqrt(s)) of the reference's projections, without the
// FP64 square root when s <= 1 (then the result is exactly 1).
__device__ __forceinline__ double proj_norm(double s) { return s > 1.0 ? (double)fmaxf(1.f, (float)sqrt(s)) : 1.0; }

// r / fmaxf(1, |r|) of TGV2_updateR (TGV2_kernels.cu:99-101) without the
// division: |r| <= 1 divides by 1 and |r| > 1 divides r by its own magnitude,
// exactly +-1 in IEEE arithmetic (NaN stays NaN, as in the division).
__device__ __forceinline__ float proj_unit(float r) { return fabsf(r) > 1.f ? copysignf(1.f, r) : r; }

// (float)(v / d) for the reference's projections with d = proj_norm(s): the
// square root and the FP64 divisions sit behind real branches, so warps whose
// projections are all the identity skip them.
__device__ __forceinline__ void proj2(double s, double &a, double &b)
{
    if (s > 1.0) {
        const double d = (double)fmaxf(1.f, (float)sqrt(s));
        if (d != 1.0) {
            a = a / d;
            b = b / d;
        }
    }
}

__device__ __forceinline__ void proj3(double s, double &a, double &b, double &c)
{
    if (s > 1.0) {
        const double d = (double)fmaxf(1.f, (float)sqrt(s));
        if (d != 1.0) {
            a = a / d;
            b = b / d;
            c = c / d;
        }
    }
}

// ---- the TGV2 energy (no reference symbol: the reference runs a fixed count) ----
//
// alpha1 |T (grad u - v)|_2 + alpha0 |eps(v)| + lambda sum_i |It_i + (u - u0) Iu_i|
// per pixel, in double, with the forward differences of the P and Q updates
// (clamped at the last column / row).  `r`, `d` are the right and lower
// neighbours; `data(du)` adds the views' |It_i + du Iu_i| in view order.
template <typename DataTerm>
__device__ __forceinline__ double pixel_energy(float uc, float ur, float ud, float vxc, float vyc, float vxr,
                                               float vyr, float vxd, float vyd, float t11, float t12, float t22,
                                               float u0v, double lambda, double alpha0, double alpha1, DataTerm &&data)
{
    const double gx = (double)ur - uc - vxc;
    const double gy = (double)ud - uc - vyc;
    const double tx = t11 * gx + t12 * gy, ty = t12 * gx + t22 * gy;
    double ei = alpha1 * sqrt(tx * tx + ty * ty);
    const double a = (double)vxr - vxc, bb = (double)vyd - vyc;
    const double c = 0.5 * (((double)vxd - vxc) + ((double)vyr - vyc));
    ei += alpha0 * sqrt(a * a + bb * bb + 2 * c * c);
    const double du = (double)uc - u0v;
    return ei + lambda * data(du);
}

// Threads of an energy_kernel block (one TX x TY tile).
constexpr int EB = 256;

// A block's share of the energy, first step (every thread): each warp's sum
// of `e` into red[warp] (EB / 32 doubles).
__device__ __forceinline__ void energy_warp_sum(double e, double *red)
{
    for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
    if ((threadIdx.x + threadIdx.y * blockDim.x) % 32 == 0) red[(threadIdx.x + threadIdx.y * blockDim.x) / 32] = e;
}

// Second step (thread 0, after a barrier): the warps' sums in warp order,
// written to partial[block] and fenced before the block counts itself done on
// the completion counter; true for the block that finished last.
__device__ __forceinline__ bool energy_block_done(const double *red, double *partial, int block, unsigned nblocks,
                                                  IterCtl *ctl)
{
    double s = 0.0;
    for (int k = 0; k < EB / 32; ++k) s += red[k];
    partial[block] = s;
    __threadfence();   // the partial is visible before the block counts as done
    return atomicAdd(&ctl->blocks_done, 1u) == nblocks - 1;
}

// The block that finished last: adds the partial sums in block order, writes
// the energy and, with tol > 0, applies the stopping test of the launch path
// (stop_test over the checks of one linearisation); re-arms the counter.
// Every thread of that block calls it.
__device__ __forceinline__ void energy_finish(const double *partial, int nblocks, double *red, double *out,
                                              IterCtl *ctl, double tol, int total, int window)
{
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    __threadfence();   // every partial is written (each was fenced before its count)
    double t = 0.0;
    for (int k = tid; k < nblocks; k += EB) t += __ldcg(partial + k);
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    __syncthreads();
    if (tid % 32 == 0) red[tid / 32] = t;
    __syncthreads();
    if (tid == 0) {
        double E = 0.0;
        for (int k = 0; k < EB / 32; ++k) E += red[k];
        *out = E;
        if (tol > 0) {
            if (stop_test(ctl->hist, ctl->n_hist, E, tol, window)) {
                ctl->done = 1;
                ctl->stop_total = total;
            }
            ++ctl->n_hist;
            ctl->last_e = E;
            ctl->have_energy = 1;
            ctl->energy_at = total;
        }
        ctl->blocks_done = 0;   // ready for the next evaluation
    }
}

// New p (TGV2_updateP_tensor_weighed_kernel, TGV2_kernels.cu:340-365) and q
// (TGV2_updateQ_kernel, :54-85) at one cell (rx, ry) of the tile's p/q region,
// from the ubar / vbar halo in shared memory and the cell's T, p, q operands.
__device__ __forceinline__ void pq_cell(const float (*sU)[TX + 2], const float (*sVX)[TX + 2],
                                        const float (*sVY)[TX + 2], float (*sPx)[TX + 1], float (*sPy)[TX + 1],
                                        float (*sQx)[TX + 1], float (*sQy)[TX + 1], float (*sQz)[TX + 1], int rx,
                                        int ry, int nx, int ny, float t11, float t12, float t22, float pxin,
                                        float pyin, float qxin, float qyin, float qzin, float a1s, float a0s)
{
    {
        const double xg = sU[ry][nx] - sU[ry][rx] - sVX[ry][rx];
        const double yg = sU[ny][rx] - sU[ry][rx] - sVY[ry][rx];
        const double c11 = t11, c12 = t12, c22 = t22;
        double dx = (double)pxin + (double)a1s * (c11 * xg + c12 * yg);
        double dy = (double)pyin + (double)a1s * (c12 * xg + c22 * yg);
        proj2(dx * dx + dy * dy, dx, dy);
        sPx[ry][rx] = (float)dx;
        sPy[ry][rx] = (float)dy;
    }
    {
        const float dx_u1x = sVX[ry][nx] - sVX[ry][rx];
        const float dy_u1x = sVX[ny][rx] - sVX[ry][rx];
        const float dx_u1y = sVY[ry][nx] - sVY[ry][rx];
        const float dy_u1y = sVY[ny][rx] - sVY[ry][rx];
        double dx = qxin + a0s * dx_u1x;
        double dy = qyin + a0s * dy_u1y;
        double dz = qzin + a0s * (dy_u1x + dx_u1y) / 2.0f;
        proj3(dx * dx + dy * dy + dz * dz + dz * dz, dx, dy, dz);
        sQx[ry][rx] = (float)dx;
        sQy[ry][rx] = (float)dy;
        sQz[ry][rx] = (float)dz;
    }
}

// One full TGV2 iteration (planesweep.cpp:485-509).  A 32 x 8 tile computes p
// and q on the 33 x 9 cells [x0-1, x0+32) x [y0-1, y0+8): thread (tx, ty)
// takes the cell of its own pixel, threads 0..40 also one of the 41 halo
// cells (the top row, then the left column).  Every global operand of the
// iteration -- the pixel's r, It, Iu, T, u, u0, v, p, q, the halo cell's T,
// p, q and the ubar / vbar halo -- is loaded at the start, one round of loads
// per CTA; the data duals r and their sum (which read no neighbour) are
// updated while the halo is stored, so their 3V registers are free before
// the p / q phase.  The arithmetic and its order are the reference's.
template <int VMAX>
__global__ void __launch_bounds__(TX *TY) iteration_kernel(IterBufs b)
{
    __shared__ float sU[TY + 2][TX + 2], sVX[TY + 2][TX + 2], sVY[TY + 2][TX + 2];
    __shared__ float sPx[TY + 1][TX + 1], sPy[TY + 1][TX + 1];
    __shared__ float sQx[TY + 1][TX + 1], sQy[TY + 1][TX + 1], sQz[TY + 1][TX + 1];
    constexpr int HALO = (TX + 2) * (TY + 2);    // ubar / vbar halo cells: 340
    constexpr int HCELLS = TX + 1 + TY;           // p / q cells outside the tile: 41
    static_assert(HALO <= 2 * TX * TY && HCELLS <= TX * TY, "two halo cells and one p/q halo cell per thread");
    wait_for_previous_grid();   // launched as a dependent launch: the previous iteration is complete
    allow_next_grid();
    if (b.ctl && b.ctl->done) return;   // the run stopped at an earlier energy check
    const int w = b.w, h = b.h;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int tid = threadIdx.y * TX + threadIdx.x;
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    const bool own = x < w && y < h;
    const int i = own ? y * w + x : 0;
    const int V = b.V;   // <= VMAX (the launch picks VMAX)

    // ---- loads ----
    const int VS = view_stride(V);
    float rv[VMAX], itv[VMAX], iuv[VMAX];
    if (own) {
        const float4 *r4 = reinterpret_cast<const float4 *>(b.r + (size_t)i * VS);
        const float4 *t4 = reinterpret_cast<const float4 *>(b.It + (size_t)i * VS);
        const float4 *d4 = reinterpret_cast<const float4 *>(b.Iu + (size_t)i * VS);
#pragma unroll
        for (int q = 0; q < VMAX / 4; ++q) {
            if (4 * q < V) {
                const float4 a = r4[q], c = t4[q], d = d4[q];
                rv[4 * q] = a.x, rv[4 * q + 1] = a.y, rv[4 * q + 2] = a.z, rv[4 * q + 3] = a.w;
                itv[4 * q] = c.x, itv[4 * q + 1] = c.y, itv[4 * q + 2] = c.z, itv[4 * q + 3] = c.w;
                iuv[4 * q] = d.x, iuv[4 * q + 1] = d.y, iuv[4 * q + 2] = d.z, iuv[4 * q + 3] = d.w;
            }
        }
    }
    float t11 = 0.f, t12 = 0.f, t22 = 0.f, uold = 0.f, u0v = 0.f, u1xprev = 0.f, u1yprev = 0.f;
    float pxin = 0.f, pyin = 0.f, qxin = 0.f, qyin = 0.f, qzin = 0.f;
    if (own) {
        t11 = b.T11[i];
        t12 = b.T12[i];
        t22 = b.T22[i];
        uold = b.u[i];
        u0v = b.u0[i];
        u1xprev = b.u1x[i];
        u1yprev = b.u1y[i];
        pxin = b.Px_in[i];
        pyin = b.Py_in[i];
        qxin = b.Qx_in[i];
        qyin = b.Qy_in[i];
        qzin = b.Qz_in[i];
    }
    // the halo p / q cell of threads 0..40: (rx, 0) for rx = tid <= TX, then (0, tid - TX)
    const int hrx = tid <= TX ? tid : 0, hry = tid <= TX ? 0 : tid - TX;
    const int hpx = x0 - 1 + hrx, hpy = y0 - 1 + hry;
    const bool hcell = tid < HCELLS && hpx >= 0 && hpy >= 0 && hpx < w && hpy < h;
    float ht11 = 0.f, ht12 = 0.f, ht22 = 0.f, hpxin = 0.f, hpyin = 0.f, hqxin = 0.f, hqyin = 0.f, hqzin = 0.f;
    if (hcell) {
        const int j = hpy * w + hpx;
        ht11 = b.T11[j];
        ht12 = b.T12[j];
        ht22 = b.T22[j];
        hpxin = b.Px_in[j];
        hpyin = b.Py_in[j];
        hqxin = b.Qx_in[j];
        hqyin = b.Qy_in[j];
        hqzin = b.Qz_in[j];
    }
    // ubar, vbar on [x0-1, x0+TX] x [y0-1, y0+TY] (clamped; cells outside the
    // image are never read): cells tid and tid + TX*TY
    float hu[2], hvx[2], hvy[2];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        const int k = tid + c * TX * TY;
        hu[c] = hvx[c] = hvy[c] = 0.f;
        if (k < HALO) {
            const int ry = k / (TX + 2), rx = k % (TX + 2);
            const int px = min(max(x0 - 1 + rx, 0), w - 1), py = min(max(y0 - 1 + ry, 0), h - 1);
            const int j = py * w + px;
            hu[c] = b.ubar_in[j];
            hvx[c] = b.u1xbar_in[j];
            hvy[c] = b.u1ybar_in[j];
        }
    }

    // ---- r and prodsum (TGV2_updateR_kernel, TGV2_kernels.cu:87-105), views in order ----
    const float du = uold - u0v;
    const float sl = b.sigma * b.lambda;
    float prodsum = 0.f;
    if (own) {
        float rn[VMAX];
#pragma unroll
        for (int v = 0; v < VMAX; ++v) {
            rn[v] = 0.f;
            if (v < V) {
                const float r = proj_unit(rv[v] + sl * (itv[v] + du * iuv[v]));
                rn[v] = r;
                prodsum += r * iuv[v];
            }
        }
        float4 *r4 = reinterpret_cast<float4 *>(b.r + (size_t)i * VS);
#pragma unroll
        for (int q = 0; q < VMAX / 4; ++q)
            if (4 * q < V) r4[q] = make_float4(rn[4 * q], rn[4 * q + 1], rn[4 * q + 2], rn[4 * q + 3]);
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        const int k = tid + c * TX * TY;
        if (k < HALO) {
            const int ry = k / (TX + 2), rx = k % (TX + 2);
            sU[ry][rx] = hu[c];
            sVX[ry][rx] = hvx[c];
            sVY[ry][rx] = hvy[c];
        }
    }
    __syncthreads();

    // ---- p, q on the tile and its left / top halo ----
    const float a1s = b.alpha1 * b.sigma, a0s = b.alpha0 * b.sigma;
    const int lx = threadIdx.x + 1, ly = threadIdx.y + 1;
    if (own) {
        const int nx = x + 1 <= w - 1 ? lx + 1 : lx, ny = y + 1 <= h - 1 ? ly + 1 : ly;
        pq_cell(sU, sVX, sVY, sPx, sPy, sQx, sQy, sQz, lx, ly, nx, ny, t11, t12, t22, pxin, pyin, qxin, qyin, qzin,
                a1s, a0s);
    }
    if (hcell) {
        const int nx = hpx + 1 <= w - 1 ? hrx + 1 : hrx, ny = hpy + 1 <= h - 1 ? hry + 1 : hry;
        pq_cell(sU, sVX, sVY, sPx, sPy, sQx, sQy, sQz, hrx, hry, nx, ny, ht11, ht12, ht22, hpxin, hpyin, hqxin,
                hqyin, hqzin, a1s, a0s);
    }
    __syncthreads();
    if (!own) return;

    // ---- primal step (TGV2_updateU_tensor_weighed_kernel, TGV2_kernels.cu:300-338) ----
    const int xp = max(x - 1, 0), yp = max(y - 1, 0);
    const int lxp = lx - (x - xp), lyp = ly - (y - yp);
    const float c_px = sPx[ly][lx], c_py = sPy[ly][lx];
    const float xp_px = sPx[ly][lxp], yp_px = sPx[lyp][lx];
    const float xp_py = sPy[ly][lxp], yp_py = sPy[lyp][lx];
    const float unew = uold - b.tau * (-b.alpha1 * (t11 * (c_px - xp_px) + t12 * (c_py - xp_py) +
                                                   t12 * (c_px - yp_px) + t22 * (c_py - yp_py)) +
                                       b.lambda * prodsum);
    const float qx = sQx[ly][lx], qy = sQy[ly][lx], qz = sQz[ly][lx];
    const float u1xn = u1xprev - b.tau * (-b.alpha1 * (t11 * c_px + t12 * c_py) -
                                          b.alpha0 * (qx - sQx[ly][lxp] + qz - sQz[lyp][lx]));
    const float u1yn = u1yprev - b.tau * (-b.alpha1 * (t12 * c_px + t22 * c_py) -
                                          b.alpha0 * (qz - sQz[ly][lxp] + qy - sQy[lyp][lx]));
    b.u[i] = unew;
    b.u1x[i] = u1xn;
    b.u1y[i] = u1yn;
    b.ubar_out[i] = 2 * unew - uold;
    b.u1xbar_out[i] = 2 * u1xn - u1xprev;
    b.u1ybar_out[i] = 2 * u1yn - u1yprev;
    b.Px_out[i] = c_px;
    b.Py_out[i] = c_py;
    b.Qx_out[i] = qx;
    b.Qy_out[i] = qy;
    b.Qz_out[i] = qz;
}

// The energy of the current iterate (the energy checks of the launch path and
// the final energy).  One TX x TY tile per block, one pixel per thread: the
// iteration's grid, at full occupancy (32 registers), so the pixels' loads
// are all in flight at once; per warp, then per block in warp order, then
// the blocks' partial sums in block order by the block that finishes last (a
// completion counter, nothing waits).  With tol > 0 the last block applies
// the stopping test.  Launches after a met tolerance return at once.
__global__ void __launch_bounds__(TX *TY) energy_kernel(const float *__restrict__ T11, const float *__restrict__ T12,
                                                        const float *__restrict__ T22, const float *__restrict__ It,
                                                        const float *__restrict__ Iu, const float *__restrict__ u0,
                                                        const float *__restrict__ u, const float *__restrict__ u1x,
                                                        const float *__restrict__ u1y, int w, int h, int V,
                                                        double lambda, double alpha0, double alpha1,
                                                        double *__restrict__ partial, double *__restrict__ out,
                                                        IterCtl *ctl, double tol, int total, int window)
{
    __shared__ double red[EB / 32];
    __shared__ int last;
    wait_for_previous_grid();   // also launched as a dependent launch after the iterations
    allow_next_grid();
    if (ctl->done) return;
    const int x = blockIdx.x * TX + threadIdx.x, y = blockIdx.y * TY + threadIdx.y;
    double e = 0.0;
    if (x < w && y < h) {
        const int i = y * w + x, jr = y * w + min(x + 1, w - 1), jd = min(y + 1, h - 1) * w + x;
        e = pixel_energy(u[i], u[jr], u[jd], u1x[i], u1y[i], u1x[jr], u1y[jr], u1x[jd], u1y[jd], T11[i], T12[i],
                         T22[i], u0[i], lambda, alpha0, alpha1, [&](double du) {
                             double ed = 0.0;
                             // the pixel's views as 16-byte words, added in view order
                             const int VS = view_stride(V);
                             const float4 *t4 = reinterpret_cast<const float4 *>(It + (size_t)i * VS);
                             const float4 *d4 = reinterpret_cast<const float4 *>(Iu + (size_t)i * VS);
                             for (int q = 0; 4 * q < V; ++q) {
                                 const float4 a = t4[q], c = d4[q];
                                 const float tv[4] = {a.x, a.y, a.z, a.w}, dv[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
                                 for (int e = 0; e < 4; ++e)
                                     if (4 * q + e < V) ed += fabs((double)tv[e] + du * dv[e]);
                             }
                             return ed;
                         });
    }
    energy_warp_sum(e, red);
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0)
        last = energy_block_done(red, partial, blockIdx.y * gridDim.x + blockIdx.x, gridDim.x * gridDim.y, ctl);
    __syncthreads();
    if (last) energy_finish(partial, gridDim.x * gridDim.y, red, out, ctl, tol, total, window);
}

// Dual start for a warm-started primal: one dual step from zero, of size sd
// for the regulariser's duals and sdr for the data duals:
// p = P(a1 sd T(grad u - v)), q = P(a0 sd e(v)), r_i = P(sdr lambda (It_i +
// (u - u0) Iu_i)), with the iteration's projections.  A large step puts a dual
// variable at the unit direction of its term, its value at the saddle point
// wherever that term is non-zero (for r: the sign of the residual).
__global__ void dual_init_kernel(const float *__restrict__ T11, const float *__restrict__ T12,
                                 const float *__restrict__ T22, const float *__restrict__ It,
                                 const float *__restrict__ Iu, const float *__restrict__ u0,
                                 const float *__restrict__ u, const float *__restrict__ u1x,
                                 const float *__restrict__ u1y, int w, int h, int V, float lambda, float alpha0,
                                 float alpha1, float sd, float sdr, float *__restrict__ Px, float *__restrict__ Py,
                                 float *__restrict__ Qx, float *__restrict__ Qy, float *__restrict__ Qz,
                                 float *__restrict__ r, int do_pq, int do_r)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const int i = y * w + x, xn = min(x + 1, w - 1), yn = min(y + 1, h - 1);
    const int ix = y * w + xn, iy = yn * w + x;
    if (do_pq) {
        const double xg = (double)u[ix] - u[i] - u1x[i];
        const double yg = (double)u[iy] - u[i] - u1y[i];
        const double s = (double)alpha1 * sd;
        const double dx = s * (T11[i] * xg + T12[i] * yg), dy = s * (T12[i] * xg + T22[i] * yg);
        const double d = proj_norm(dx * dx + dy * dy);
        Px[i] = (float)(dx / d);
        Py[i] = (float)(dy / d);
    }
    if (do_pq) {
        const double s = (double)alpha0 * sd;
        const double dx = s * ((double)u1x[ix] - u1x[i]);
        const double dy = s * ((double)u1y[iy] - u1y[i]);
        const double dz = s * (((double)u1x[iy] - u1x[i]) + ((double)u1y[ix] - u1y[i])) / 2.0;
        const double d = proj_norm(dx * dx + dy * dy + dz * dz + dz * dz);
        Qx[i] = (float)(dx / d);
        Qy[i] = (float)(dy / d);
        Qz[i] = (float)(dz / d);
    }
    if (!do_r) return;
    const float du = u[i] - u0[i];
    for (int v = 0; v < V; ++v) {
        const size_t k = (size_t)i * view_stride(V) + v;
        float q = sdr * lambda * (It[k] + du * Iu[k]);
        r[k] = q / fmaxf(1.f, fabsf(q));
    }
}


// A pixel's It and Iu of views 0 .. V-1 (view-interleaved, view_stride) as
// 16-byte words.
template <int VMAX>
__device__ __forceinline__ void load_views(const float *__restrict__ It, const float *__restrict__ Iu, size_t i, int V,
                                           float *itv, float *iuv)
{
    const int VS = view_stride(V);
    const float4 *t4 = reinterpret_cast<const float4 *>(It + i * VS);
    const float4 *d4 = reinterpret_cast<const float4 *>(Iu + i * VS);
#pragma unroll
    for (int q = 0; q < VMAX / 4; ++q) {
        if (4 * q < V) {
            const float4 c = __ldg(t4 + q), d = __ldg(d4 + q);
            itv[4 * q] = c.x, itv[4 * q + 1] = c.y, itv[4 * q + 2] = c.z, itv[4 * q + 3] = c.w;
            iuv[4 * q] = d.x, iuv[4 * q + 1] = d.y, iuv[4 * q + 2] = d.z, iuv[4 * q + 3] = d.w;
        }
    }
}

// ---- persistent iteration: the state stays on chip -----------------------------------
//
// One CTA per SM owns a 64 x TH tile for a whole linearisation: u, v, their
// over-relaxations, p, q, r of every view and the tensor T live in shared
// memory (about 200 KB at 64 x 35 pixels and 8 views); u0, It and Iu stream
// from L2.  An iteration is the fused kernel's arithmetic, statement for
// statement, with one grid-wide barrier: every CTA publishes its edge pixels
// (ubar, vbar on all four edges; p, q on the right column and bottom row) to a
// double-buffered exchange array, waits at the barrier, and reads its halo.
// Energy checks (every check_every iterations) evaluate the same energy as
// energy_kernel: each CTA writes its partial sum, and after a second barrier
// every CTA adds the partials in CTA order, so all reach the same stopping
// decision without the host.  Co-residency comes from a cooperative launch;
// each barrier wait gives up after 1 s (then every CTA leaves and the host
// reports MVS_ERR_TIMEOUT).

constexpr int PT_THREADS = 768;
constexpr int PT_TW = 64;
constexpr int PT_VMAX = 8;
constexpr unsigned long long kBarrierNs = 1000000000ull;

struct PersistResult {
    int iters, energy_at, done, err;
    double energy;
};

struct PersistBufs {
    const float *T11, *T12, *T22, *u0, *It, *Iu;
    float *u, *u1x, *u1y, *r;                  // state in / out
    const float *ubar0, *u1xbar0, *u1ybar0;    // start of the over-relaxations
    float *Px, *Py, *Qx, *Qy, *Qz;             // p, q in / out
    float *exb[2], *exq[2], *exu;              // edge exchange: [3][n], [5][n], [3][n]
    double *partial;                           // [grid]
    unsigned int *bar;                         // count, generation, abort
    PersistResult *res;
    int w, h, V, tiles_x, th, niters, cap_left, check_every, stop_window;
    double tol;
    float lambda, alpha0, alpha1, tau, sigma;
    double dlambda, dalpha0, dalpha1;
};

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long now_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid-wide barrier with a bounded wait; false (for every thread of the CTA)
// if it gave up or another CTA did.  Thread 0 arrives with an acquire-release
// add (after the CTA barrier, so the CTA's earlier writes are released with
// it); the last to arrive resets the count and publishes the next generation
// with a release store, the others poll it with acquire loads.
__device__ bool grid_barrier(unsigned int *bar, unsigned int nblocks, unsigned int &gen)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned int g = gen;
        unsigned int old;
        asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], 1;" : "=r"(old) : "l"(bar) : "memory");
        if (old == nblocks - 1) {
            asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(bar), "r"(0u) : "memory");
            asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(bar + 1), "r"(g + 1u) : "memory");
        } else {
            // the clock and the abort flag are looked at every 1024 polls
            const unsigned long long t0 = now_ns();
            unsigned int polls = 0;
            while (ld_acquire_u32(&bar[1]) == g) {
                if ((++polls & 1023u) == 0u &&
                    (ld_acquire_u32(&bar[2]) != 0u || now_ns() - t0 > kBarrierNs)) {
                    ok = 0;
                    break;
                }
            }
        }
        if (!ok) atomicExch(&bar[2], 1u);
        s_ok = ok && ld_acquire_u32(&bar[2]) == 0u;
    }
    __syncthreads();
    gen += 1u;
    return s_ok != 0;
}

__global__ void __launch_bounds__(PT_THREADS, 1) tgv2_persistent_kernel(PersistBufs b)
{
    extern __shared__ __align__(16) float sm[];
    __shared__ double red[PT_THREADS / 32];
    __shared__ double s_e;
    const int TW = PT_TW, TH = b.th, V = b.V, w = b.w, h = b.h;
    const int PW = TW + 2, QW = TW + 1;
    const int NB = (TH + 2) * PW, NQ = (TH + 1) * QW, NP = TH * TW;
    float *sUb = sm, *sVxb = sUb + NB, *sVyb = sVxb + NB;
    float *sPx = sVyb + NB, *sPy = sPx + NQ, *sQx = sPy + NQ, *sQy = sQx + NQ, *sQz = sQy + NQ;
    float *sU = sQz + NQ, *sVx = sU + NQ, *sVy = sVx + NQ;
    float *sR = sVy + NQ, *sT11 = sR + V * NP, *sT12 = sT11 + NP, *sT22 = sT12 + NP;
    // bar arrays: (ly, lx) in [-1, TH] x [-1, TW]; p/q: [-1, TH-1] x [-1, TW-1];
    // u/v: [0, TH] x [0, TW]
#define BI(ly, lx) (((ly) + 1) * PW + (lx) + 1)
#define QI(ly, lx) (((ly) + 1) * QW + (lx) + 1)
#define UI(ly, lx) ((ly) * QW + (lx))
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int x0 = (blockIdx.x % b.tiles_x) * TW, y0 = (blockIdx.x / b.tiles_x) * TH;
    const size_t n = (size_t)w * h;
    const unsigned int nblocks = gridDim.x;
    unsigned int gen = 0;

    // load the tile's state
    for (int k = tid; k < NP; k += nthr) {
        const int ly = k / TW, lx = k - ly * TW, x = x0 + lx, y = y0 + ly;
        if (x >= w || y >= h) continue;
        const size_t i = (size_t)y * w + x;
        sU[UI(ly, lx)] = b.u[i];
        sVx[UI(ly, lx)] = b.u1x[i];
        sVy[UI(ly, lx)] = b.u1y[i];
        sUb[BI(ly, lx)] = b.ubar0[i];
        sVxb[BI(ly, lx)] = b.u1xbar0[i];
        sVyb[BI(ly, lx)] = b.u1ybar0[i];
        sPx[QI(ly, lx)] = b.Px[i];
        sPy[QI(ly, lx)] = b.Py[i];
        sQx[QI(ly, lx)] = b.Qx[i];
        sQy[QI(ly, lx)] = b.Qy[i];
        sQz[QI(ly, lx)] = b.Qz[i];
        sT11[k] = b.T11[i];
        sT12[k] = b.T12[i];
        sT22[k] = b.T22[i];
        for (int v = 0; v < V; ++v) sR[v * NP + k] = b.r[(size_t)i * view_stride(V) + v];
    }
    __syncthreads();

    const float a1s = b.alpha1 * b.sigma, a0s = b.alpha0 * b.sigma, sl = b.sigma * b.lambda;
    const int limit = min(b.niters, b.cap_left);
    int k = 0, energy_at = -1, n_hist = 0, done = 0;
    double last_e = 0.0;
    __shared__ double s_hist[MVS_TGV2_STOP_WINDOW_MAX];   // energies of this launch's checks (thread 0)
    __shared__ int s_met;
    bool ok = true;
    while (k < limit) {
        const int par = k & 1;
        float *exb = b.exb[par], *exq = b.exq[par];
        // (1) publish edges
        for (int q = tid; q < NP; q += nthr) {
            const int ly = q / TW, lx = q - ly * TW, x = x0 + lx, y = y0 + ly;
            if (x >= w || y >= h) continue;
            const bool right = lx == TW - 1 || x == w - 1, bottom = ly == TH - 1 || y == h - 1;
            if (!(lx == 0 || ly == 0 || right || bottom)) continue;
            const size_t i = (size_t)y * w + x;
            exb[i] = sUb[BI(ly, lx)];
            exb[n + i] = sVxb[BI(ly, lx)];
            exb[2 * n + i] = sVyb[BI(ly, lx)];
            if (right || bottom) {
                exq[i] = sPx[QI(ly, lx)];
                exq[n + i] = sPy[QI(ly, lx)];
                exq[2 * n + i] = sQx[QI(ly, lx)];
                exq[3 * n + i] = sQy[QI(ly, lx)];
                exq[4 * n + i] = sQz[QI(ly, lx)];
            }
        }
        // (2) barrier
        if (!(ok = grid_barrier(b.bar, nblocks, gen))) break;
        // (3) halo: the over-relaxations on the ring (clamped at the image
        // border), p and q left of and above the tile
        const int ring = 2 * (TW + 2) + 2 * TH;
        for (int q = tid; q < ring; q += nthr) {
            int ly, lx;
            if (q < TW + 2) { ly = -1; lx = q - 1; }
            else if (q < 2 * (TW + 2)) { ly = TH; lx = q - (TW + 2) - 1; }
            else if (q < 2 * (TW + 2) + TH) { ly = q - 2 * (TW + 2); lx = -1; }
            else { ly = q - 2 * (TW + 2) - TH; lx = TW; }
            const int px = min(max(x0 + lx, 0), w - 1), py = min(max(y0 + ly, 0), h - 1);
            const size_t i = (size_t)py * w + px;
            sUb[BI(ly, lx)] = __ldcg(exb + i);
            sVxb[BI(ly, lx)] = __ldcg(exb + n + i);
            sVyb[BI(ly, lx)] = __ldcg(exb + 2 * n + i);
        }
        // tile cells beyond the image read their clamped in-image neighbour, as
        // the fused kernel's clamped tile load does
        for (int q = tid; q < NP; q += nthr) {
            const int ly = q / TW, lx = q - ly * TW, x = x0 + lx, y = y0 + ly;
            if (x < w && y < h) continue;
            const int px = min(x, w - 1), py = min(y, h - 1);
            const size_t i = (size_t)py * w + px;
            sUb[BI(ly, lx)] = __ldcg(exb + i);
            sVxb[BI(ly, lx)] = __ldcg(exb + n + i);
            sVyb[BI(ly, lx)] = __ldcg(exb + 2 * n + i);
        }
        for (int q = tid; q < TW + TH + 1; q += nthr) {
            const int ly = q <= TW ? -1 : q - TW - 1, lx = q <= TW ? q - 1 : -1;
            const int px = x0 + lx, py = y0 + ly;
            if (px < 0 || py < 0 || px >= w || py >= h) continue;
            const size_t i = (size_t)py * w + px;
            sPx[QI(ly, lx)] = __ldcg(exq + i);
            sPy[QI(ly, lx)] = __ldcg(exq + n + i);
            sQx[QI(ly, lx)] = __ldcg(exq + 2 * n + i);
            sQy[QI(ly, lx)] = __ldcg(exq + 3 * n + i);
            sQz[QI(ly, lx)] = __ldcg(exq + 4 * n + i);
        }
        __syncthreads();
        // (4) p and q on the tile and its left / top halo (TGV2_updateP_tensor_weighed,
        // TGV2_kernels.cu:340-365; TGV2_updateQ, :54-85), in place
        for (int q = tid; q < (TH + 1) * (TW + 1); q += nthr) {
            const int ly = q / (TW + 1) - 1, lx = q % (TW + 1) - 1;
            const int px = x0 + lx, py = y0 + ly;
            if (px < 0 || py < 0 || px >= w || py >= h) continue;
            const int nx = px + 1 <= w - 1 ? lx + 1 : lx, ny = py + 1 <= h - 1 ? ly + 1 : ly;
            float c11f, c12f, c22f;
            if (lx >= 0 && ly >= 0) {
                c11f = sT11[ly * TW + lx];
                c12f = sT12[ly * TW + lx];
                c22f = sT22[ly * TW + lx];
            } else {
                const size_t j = (size_t)py * w + px;
                c11f = b.T11[j];
                c12f = b.T12[j];
                c22f = b.T22[j];
            }
            const int c = BI(ly, lx);
            {
                const double xg = sUb[BI(ly, nx)] - sUb[c] - sVxb[c];
                const double yg = sUb[BI(ny, lx)] - sUb[c] - sVyb[c];
                const double c11 = c11f, c12 = c12f, c22 = c22f;
                double dx = (double)sPx[QI(ly, lx)] + (double)a1s * (c11 * xg + c12 * yg);
                double dy = (double)sPy[QI(ly, lx)] + (double)a1s * (c12 * xg + c22 * yg);
                proj2(dx * dx + dy * dy, dx, dy);
                sPx[QI(ly, lx)] = (float)dx;
                sPy[QI(ly, lx)] = (float)dy;
            }
            {
                const float dx_u1x = sVxb[BI(ly, nx)] - sVxb[c];
                const float dy_u1x = sVxb[BI(ny, lx)] - sVxb[c];
                const float dx_u1y = sVyb[BI(ly, nx)] - sVyb[c];
                const float dy_u1y = sVyb[BI(ny, lx)] - sVyb[c];
                double dx = sQx[QI(ly, lx)] + a0s * dx_u1x;
                double dy = sQy[QI(ly, lx)] + a0s * dy_u1y;
                double dz = sQz[QI(ly, lx)] + a0s * (dy_u1x + dx_u1y) / 2.0f;
                proj3(dx * dx + dy * dy + dz * dz + dz * dz, dx, dy, dz);
                sQx[QI(ly, lx)] = (float)dx;
                sQy[QI(ly, lx)] = (float)dy;
                sQz[QI(ly, lx)] = (float)dz;
            }
        }
        __syncthreads();
        // (5) r, u, v (TGV2_updateR, TGV2_kernels.cu:87-105; TGV2_updateU_tensor_weighed, :300-338)
        for (int q = tid; q < NP; q += nthr) {
            const int ly = q / TW, lx = q - ly * TW, x = x0 + lx, y = y0 + ly;
            if (x >= w || y >= h) continue;
            const size_t i = (size_t)y * w + x;
            // this pixel's L2 operands, all requested before the first use
            float itv[PT_VMAX], iuv[PT_VMAX];
            load_views<PT_VMAX>(b.It, b.Iu, i, V, itv, iuv);
            const float u0v = __ldg(b.u0 + i);
            const float uold = sU[UI(ly, lx)], u1xprev = sVx[UI(ly, lx)], u1yprev = sVy[UI(ly, lx)];
            const float du = uold - u0v;
            float prodsum = 0.f;
#pragma unroll
            for (int v = 0; v < PT_VMAX; ++v) {
                if (v < V) {
                    const float r = proj_unit(sR[v * NP + q] + sl * (itv[v] + du * iuv[v]));
                    sR[v * NP + q] = r;
                    prodsum += r * iuv[v];
                }
            }
            const int lxp = x > 0 ? lx - 1 : lx, lyp = y > 0 ? ly - 1 : ly;
            const float t11 = sT11[q], t12 = sT12[q], t22 = sT22[q];
            const float c_px = sPx[QI(ly, lx)], c_py = sPy[QI(ly, lx)];
            const float xp_px = sPx[QI(ly, lxp)], yp_px = sPx[QI(lyp, lx)];
            const float xp_py = sPy[QI(ly, lxp)], yp_py = sPy[QI(lyp, lx)];
            const float unew = uold - b.tau * (-b.alpha1 * (t11 * (c_px - xp_px) + t12 * (c_py - xp_py) +
                                                            t12 * (c_px - yp_px) + t22 * (c_py - yp_py)) +
                                                b.lambda * prodsum);
            const float qx = sQx[QI(ly, lx)], qy = sQy[QI(ly, lx)], qz = sQz[QI(ly, lx)];
            const float u1xn = u1xprev - b.tau * (-b.alpha1 * (t11 * c_px + t12 * c_py) -
                                                  b.alpha0 * (qx - sQx[QI(ly, lxp)] + qz - sQz[QI(lyp, lx)]));
            const float u1yn = u1yprev - b.tau * (-b.alpha1 * (t12 * c_px + t22 * c_py) -
                                                  b.alpha0 * (qz - sQz[QI(ly, lxp)] + qy - sQy[QI(lyp, lx)]));
            sU[UI(ly, lx)] = unew;
            sVx[UI(ly, lx)] = u1xn;
            sVy[UI(ly, lx)] = u1yn;
            sUb[BI(ly, lx)] = 2 * unew - uold;
            sVxb[BI(ly, lx)] = 2 * u1xn - u1xprev;
            sVyb[BI(ly, lx)] = 2 * u1yn - u1yprev;
        }
        __syncthreads();
        ++k;
        // (6) energy check (energy_kernel's terms; partials summed in CTA order)
        if (b.tol > 0 && k % b.check_every == 0) {
            for (int q = tid; q < NP; q += nthr) {
                const int ly = q / TW, lx = q - ly * TW, x = x0 + lx, y = y0 + ly;
                if (x >= w || y >= h || (lx != 0 && ly != 0)) continue;
                const size_t i = (size_t)y * w + x;
                b.exu[i] = sU[UI(ly, lx)];
                b.exu[n + i] = sVx[UI(ly, lx)];
                b.exu[2 * n + i] = sVy[UI(ly, lx)];
            }
            if (!(ok = grid_barrier(b.bar, nblocks, gen))) break;
            for (int q = tid; q < TW + TH + 1; q += nthr) {
                // right column (x0 + TW) and bottom row (y0 + TH), clamped
                const int ly = q <= TH ? q : TH, lx = q <= TH ? TW : q - TH - 1;
                const int px = min(x0 + lx, w - 1), py = min(y0 + ly, h - 1);
                const size_t i = (size_t)py * w + px;
                sU[UI(ly, lx)] = __ldcg(b.exu + i);
                sVx[UI(ly, lx)] = __ldcg(b.exu + n + i);
                sVy[UI(ly, lx)] = __ldcg(b.exu + 2 * n + i);
            }
            __syncthreads();
            double e = 0.0;
            for (int q = tid; q < NP; q += nthr) {
                const int ly = q / TW, lx = q - ly * TW, x = x0 + lx, y = y0 + ly;
                if (x >= w || y >= h) continue;
                const size_t i = (size_t)y * w + x;
                const int lxn = x + 1 <= w - 1 ? lx + 1 : lx, lyn = y + 1 <= h - 1 ? ly + 1 : ly;
                const float uc = sU[UI(ly, lx)], ux = sU[UI(ly, lxn)], uy = sU[UI(lyn, lx)];
                const float vxc = sVx[UI(ly, lx)], vyc = sVy[UI(ly, lx)];
                const double gx = (double)ux - uc - vxc;
                const double gy = (double)uy - uc - vyc;
                const double tx = sT11[q] * gx + sT12[q] * gy, ty = sT12[q] * gx + sT22[q] * gy;
                double ei = b.dalpha1 * sqrt(tx * tx + ty * ty);
                const double a = (double)sVx[UI(ly, lxn)] - vxc, bb = (double)sVy[UI(lyn, lx)] - vyc;
                const double cc = 0.5 * (((double)sVx[UI(lyn, lx)] - vxc) + ((double)sVy[UI(ly, lxn)] - vyc));
                ei += b.dalpha0 * sqrt(a * a + bb * bb + 2 * cc * cc);
                float itv[PT_VMAX], iuv[PT_VMAX];
                load_views<PT_VMAX>(b.It, b.Iu, i, V, itv, iuv);
                const double du = (double)uc - __ldg(b.u0 + i);
                double ed = 0.0;
#pragma unroll
                for (int v = 0; v < PT_VMAX; ++v)
                    if (v < V) ed += fabs((double)itv[v] + du * iuv[v]);
                e += ei + b.dlambda * ed;
            }
            for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
            if ((tid & 31) == 0) red[tid >> 5] = e;
            __syncthreads();
            if (tid == 0) {
                double t = 0.0;
                for (int q = 0; q < PT_THREADS / 32; ++q) t += red[q];
                b.partial[blockIdx.x] = t;
            }
            if (!(ok = grid_barrier(b.bar, nblocks, gen))) break;
            if (tid == 0) {
                double t = 0.0;
                for (unsigned int q = 0; q < nblocks; ++q) t += __ldcg(b.partial + q);
                s_e = t;
                s_met = stop_test(s_hist, n_hist, t, b.tol, b.stop_window);
            }
            __syncthreads();
            last_e = s_e;
            energy_at = k;
            ++n_hist;
            if (s_met) {
                done = 1;
                break;
            }
        }
    }
    if (ok) {
        // write the state back
        for (int q = tid; q < NP; q += nthr) {
            const int ly = q / TW, lx = q - ly * TW, x = x0 + lx, y = y0 + ly;
            if (x >= w || y >= h) continue;
            const size_t i = (size_t)y * w + x;
            b.u[i] = sU[UI(ly, lx)];
            b.u1x[i] = sVx[UI(ly, lx)];
            b.u1y[i] = sVy[UI(ly, lx)];
            b.Px[i] = sPx[QI(ly, lx)];
            b.Py[i] = sPy[QI(ly, lx)];
            b.Qx[i] = sQx[QI(ly, lx)];
            b.Qy[i] = sQy[QI(ly, lx)];
            b.Qz[i] = sQz[QI(ly, lx)];
            for (int v = 0; v < V; ++v) b.r[(size_t)i * view_stride(V) + v] = sR[v * NP + q];
        }
    }
    if (blockIdx.x == 0 && tid == 0) {
        b.res->iters = k;
        b.res->energy_at = energy_at;
        b.res->done = done;
        b.res->err = ok ? 0 : 1;
        b.res->energy = last_e;
    }
#undef BI
#undef QI
#undef UI
}

size_t persist_smem_bytes(int th, int V)
{
    const int TW = PT_TW, NB = (th + 2) * (TW + 2), NQ = (th + 1) * (TW + 1), NP = th * TW;
    return sizeof(float) * ((size_t)3 * NB + 5 * (size_t)NQ + 3 * (size_t)NQ + (size_t)V * NP + 3 * (size_t)NP);
}

struct Layout {
    float *ref01, *T11, *T12, *T22, *u0, *u1x, *u1y, *ubar[2], *u1xbar[2], *u1ybar[2], *Px[2], *Py[2], *Qx[2],
        *Qy[2], *Qz[2], *It, *Iu, *r;
    double *partial, *energy;   // energy_kernel's per-block partial sums (one per tile) and result
    IterCtl *ctl;
    float *exb[2], *exq[2], *exu;
    double *ppartial;
    unsigned int *bar;
    PersistResult *res;
    size_t bytes;
};

Layout layout(void *base, int w, int h, int V)
{
    Layout L{};
    const size_t n = (size_t)w * h;
    char *p = (char *)base;
    size_t off = 0;
    auto take = [&](size_t count) {
        float *q = (float *)(p + off);
        off += ((count * sizeof(float) + 255) / 256) * 256;
        return q;
    };
    L.ref01 = take(n);
    L.T11 = take(n);
    L.T12 = take(n);
    L.T22 = take(n);
    L.u0 = take(n);
    L.u1x = take(n);
    L.u1y = take(n);
    for (int k = 0; k < 2; ++k) {
        L.ubar[k] = take(n);
        L.u1xbar[k] = take(n);
        L.u1ybar[k] = take(n);
        L.Px[k] = take(n);
        L.Py[k] = take(n);
        L.Qx[k] = take(n);
        L.Qy[k] = take(n);
        L.Qz[k] = take(n);
    }
    L.It = take(n * view_stride(V));   // [pixel][VS] (view_stride)
    L.Iu = take(n * view_stride(V));
    L.r = take(n * view_stride(V));
    L.partial = (double *)take(2 * (size_t)ceil_div(w, TX) * ceil_div(h, TY));
    L.energy = (double *)take(2);
    L.ctl = (IterCtl *)take(sizeof(IterCtl) / sizeof(float));
    for (int k = 0; k < 2; ++k) {
        L.exb[k] = take(3 * n);
        L.exq[k] = take(5 * n);
    }
    L.exu = take(3 * n);
    L.ppartial = (double *)take(2 * 1024);
    L.bar = (unsigned int *)take(64);
    L.res = (PersistResult *)take(16);
    L.bytes = off;
    return L;
}

// Tile height for the persistent kernel, or 0 when the image does not fit on
// chip (one 64-column tile per SM) or has more views than it keeps.
int persist_tile_height(int w, int h, int V, int sms, size_t smem_limit)
{
    if (V > PT_VMAX) return 0;
    const int tx = ceil_div(w, PT_TW);
    if (tx > sms) return 0;
    const int rows = sms / tx;
    // as few rows per tile as the SM count allows, but not below 16 (small
    // images then use fewer CTAs than SMs)
    const int th = max(ceil_div(h, rows), min(h, 16));
    if (th < 2 || persist_smem_bytes(th, V) > smem_limit) return 0;
    return th;
}

// ---- TGV2 towards a sparse depth (PlaneSweep::TGVdenoiseFromSparse) ----------------
//
// planesweep.cpp:596-674 with TGV2_kernels.cu:340-445: P from u itself (the
// call passes d_depthmap, not ubar), Q from v, and the update of
// TGV2_updateU_sparseDepthTensor_kernel, whose call at planesweep.cpp:645
// passes vxbar / vybar as both v and its over-relaxation, so the in-place
// update leaves vbar == v.  ubar is written there but never read (P takes u),
// so it does not change the result and is not kept here; neither is theta,
// which only enters ubar.  One fused launch per iteration, P and Q recomputed
// on the left / top halo as in iteration_kernel; u, v, p, q are
// double-buffered because neighbouring CTAs read them.

struct SparseBufs {
    const float *T11, *T12, *T22, *wgt, *Ds;
    const float *u_in, *vx_in, *vy_in, *Px_in, *Py_in, *Qx_in, *Qy_in, *Qz_in;
    float *u_out, *vx_out, *vy_out, *Px_out, *Py_out, *Qx_out, *Qy_out, *Qz_out;
    int w, h;
    float alpha0, alpha1, tau, sigma;
};

// Tile of SX x SY pixels per CTA of SNT threads, two rows per thread in the
// primal step (the p, q halo is then 6% of the tile instead of 16%).  The
// iterations are dependent launches (launch_dependent): each waits for the
// previous one before its first global access, and its launch overlaps the
// previous one's tail.
constexpr int SX = 32, SY = 16, SNT = 256;

__global__ void __launch_bounds__(SNT) sparse_iteration_kernel(SparseBufs b)
{
    __shared__ float sU[SY + 2][SX + 2], sVX[SY + 2][SX + 2], sVY[SY + 2][SX + 2];
    __shared__ float sPx[SY + 1][SX + 1], sPy[SY + 1][SX + 1];
    __shared__ float sQx[SY + 1][SX + 1], sQy[SY + 1][SX + 1], sQz[SY + 1][SX + 1];
    const int w = b.w, h = b.h;
    const int x0 = blockIdx.x * SX, y0 = blockIdx.y * SY;
    const int tid = threadIdx.x;
    wait_for_previous_grid();   // the previous iteration's state (or the set-up) is complete
    allow_next_grid();          // the next iteration may be scheduled; it waits the same way
    for (int k = tid; k < (SX + 2) * (SY + 2); k += SNT) {
        const int ry = k / (SX + 2), rx = k % (SX + 2);
        const int px = min(max(x0 - 1 + rx, 0), w - 1), py = min(max(y0 - 1 + ry, 0), h - 1);
        const int j = py * w + px;
        sU[ry][rx] = b.u_in[j];
        sVX[ry][rx] = b.vx_in[j];
        sVY[ry][rx] = b.vy_in[j];
    }
    __syncthreads();
    // TGV2_updateP_tensor_weighed (TGV2_kernels.cu:340-365) on u and v, TGV2_updateQ (:54-85) on v
    const float a1s = b.alpha1 * b.sigma, a0s = b.alpha0 * b.sigma;
    for (int k = tid; k < (SX + 1) * (SY + 1); k += SNT) {
        const int ry = k / (SX + 1), rx = k % (SX + 1);
        const int px = x0 - 1 + rx, py = y0 - 1 + ry;
        if (px < 0 || py < 0 || px >= w || py >= h) continue;
        const int j = py * w + px;
        const int nx = px + 1 <= w - 1 ? rx + 1 : rx, ny = py + 1 <= h - 1 ? ry + 1 : ry;
        {
            const double xg = sU[ry][nx] - sU[ry][rx] - sVX[ry][rx];
            const double yg = sU[ny][rx] - sU[ry][rx] - sVY[ry][rx];
            const double c11 = b.T11[j], c12 = b.T12[j], c22 = b.T22[j];
            double dx = (double)b.Px_in[j] + (double)a1s * (c11 * xg + c12 * yg);
            double dy = (double)b.Py_in[j] + (double)a1s * (c12 * xg + c22 * yg);
            proj2(dx * dx + dy * dy, dx, dy);
            sPx[ry][rx] = (float)dx;
            sPy[ry][rx] = (float)dy;
        }
        {
            const float dx_u1x = sVX[ry][nx] - sVX[ry][rx];
            const float dy_u1x = sVX[ny][rx] - sVX[ry][rx];
            const float dx_u1y = sVY[ry][nx] - sVY[ry][rx];
            const float dy_u1y = sVY[ny][rx] - sVY[ry][rx];
            double dx = b.Qx_in[j] + a0s * dx_u1x;
            double dy = b.Qy_in[j] + a0s * dy_u1y;
            double dz = b.Qz_in[j] + a0s * (dy_u1x + dx_u1y) / 2.0f;
            proj3(dx * dx + dy * dy + dz * dz + dz * dz, dx, dy, dz);
            sQx[ry][rx] = (float)dx;
            sQy[ry][rx] = (float)dy;
            sQz[ry][rx] = (float)dz;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < SY * SX / SNT; ++r) {
        const int tx = tid % SX, ty = tid / SX + r * (SNT / SX);
        const int x = x0 + tx, y = y0 + ty;
        if (x >= w || y >= h) continue;
        const int i = y * w + x, lx = tx + 1, ly = ty + 1;
        const int lxp = x > 0 ? lx - 1 : lx, lyp = y > 0 ? ly - 1 : ly;
        // TGV2_updateU_sparseDepthTensor_kernel (TGV2_kernels.cu:399-430)
        const float t11 = b.T11[i], t12 = b.T12[i], t22 = b.T22[i], wi = b.wgt[i];
        const float c_px = sPx[ly][lx], c_py = sPy[ly][lx];
        const float xp_px = sPx[ly][lxp], yp_px = sPx[lyp][lx];
        const float xp_py = sPy[ly][lxp], yp_py = sPy[lyp][lx];
        const float uold = sU[ly][lx];
        const float unew = (uold + b.tau * (b.alpha1 * (t11 * (c_px - xp_px) + t12 * (c_py - xp_py) +
                                                        t12 * (c_px - yp_px) + t22 * (c_py - yp_py)) +
                                            wi * b.Ds[i])) /
                           (1 + b.tau * wi);
        const float qx = sQx[ly][lx], qy = sQy[ly][lx], qz = sQz[ly][lx];
        const float vxn = sVX[ly][lx] - b.tau * (-b.alpha1 * (t11 * c_px + t12 * c_py) -
                                                 b.alpha0 * (qx - sQx[ly][lxp] + qz - sQz[lyp][lx]));
        const float vyn = sVY[ly][lx] - b.tau * (-b.alpha1 * (t12 * c_px + t22 * c_py) -
                                                 b.alpha0 * (qz - sQz[ly][lxp] + qy - sQy[lyp][lx]));
        b.u_out[i] = unew;
        b.vx_out[i] = vxn;   // v and its over-relaxation are the same array in the reference
        b.vy_out[i] = vyn;
        b.Px_out[i] = c_px;
        b.Py_out[i] = c_py;
        b.Qx_out[i] = qx;
        b.Qy_out[i] = qy;
        b.Qz_out[i] = qz;
    }
}

// setup: weights (calculateWeights_sparseDepth_kernel, TGV2_kernels.cu:432-445),
// Ds / zfar, u = depthmap / zfar (element_scale: x * (1.f / zfar)), the other
// state at zero
__global__ void sparse_setup_kernel(const float *__restrict__ depthmap, const float *__restrict__ sparse, int n,
                                    float inv_zfar, float *__restrict__ wgt, float *__restrict__ Ds,
                                    float *__restrict__ u, float *__restrict__ vx,
                                    float *__restrict__ vy, float *__restrict__ Px, float *__restrict__ Py,
                                    float *__restrict__ Qx, float *__restrict__ Qy, float *__restrict__ Qz)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float s = sparse[i];
        wgt[i] = s > 0 ? 1.f : 0.f;
        Ds[i] = s * inv_zfar;
        u[i] = depthmap[i] * inv_zfar;
        vx[i] = vy[i] = Px[i] = Py[i] = Qx[i] = Qy[i] = Qz[i] = 0.f;
    }
}

__global__ void scale_kernel(const float *__restrict__ in, int n, float s, float *__restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = in[i] * s;
}

struct SparseLayout {
    float *ref01, *T11, *T12, *T22, *wgt, *Ds, *u[2], *vx[2], *vy[2], *Px[2], *Py[2], *Qx[2], *Qy[2], *Qz[2];
    size_t bytes;
};

SparseLayout sparse_layout(void *base, int w, int h)
{
    SparseLayout L{};
    const size_t n = (size_t)w * h;
    char *p = (char *)base;
    size_t off = 0;
    auto take = [&]() {
        float *q = (float *)(p + off);
        off += ((n * sizeof(float) + 255) / 256) * 256;
        return q;
    };
    L.ref01 = take();
    L.T11 = take();
    L.T12 = take();
    L.T22 = take();
    L.wgt = take();
    L.Ds = take();
    for (int k = 0; k < 2; ++k) {
        L.u[k] = take();
        L.vx[k] = take();
        L.vy[k] = take();
        L.Px[k] = take();
        L.Py[k] = take();
        L.Qx[k] = take();
        L.Qy[k] = take();
        L.Qz[k] = take();
    }
    L.bytes = off;
    return L;
}

}  // namespace

size_t tgv2_sparse_workspace_bytes(int w, int h) { return sparse_layout(nullptr, w, h).bytes; }

int tgv2_sparse_run(int w, int h, const float *ref255, const float *depthmap, const float *sparse, float zfar,
                    int niters, double alpha0, double alpha1, double tau, double sigma, double beta, double gamma,
                    float *out, void *ws, cudaStream_t st)
{
    SparseLayout L = sparse_layout(ws, w, h);
    const int n = w * h;
    const dim3 b2(32, 8), g2(ceil_div(w, 32), ceil_div(h, 8));
    const int eg = min(ceil_div(n, 256), 8 * kSMs);
    // the reference passes its double parameters to float kernel arguments
    tensor_kernel<<<g2, b2, 0, st>>>(ref255, w, h, (float)beta, (float)gamma, L.ref01, L.T11, L.T12, L.T22);
    sparse_setup_kernel<<<eg, 256, 0, st>>>(depthmap, sparse, n, 1.f / zfar, L.wgt, L.Ds, L.u[0], L.vx[0],
                                           L.vy[0], L.Px[0], L.Py[0], L.Qx[0], L.Qy[0], L.Qz[0]);
    SparseBufs b;
    b.T11 = L.T11;
    b.T12 = L.T12;
    b.T22 = L.T22;
    b.wgt = L.wgt;
    b.Ds = L.Ds;
    b.w = w;
    b.h = h;
    b.alpha0 = (float)alpha0;
    b.alpha1 = (float)alpha1;
    b.tau = (float)tau;
    b.sigma = (float)sigma;
    int cur = 0;
    const dim3 gi(ceil_div(w, SX), ceil_div(h, SY)), bi(SNT);
    for (int it = 0; it < niters; ++it) {
        b.u_in = L.u[cur];
        b.vx_in = L.vx[cur];
        b.vy_in = L.vy[cur];
        b.Px_in = L.Px[cur];
        b.Py_in = L.Py[cur];
        b.Qx_in = L.Qx[cur];
        b.Qy_in = L.Qy[cur];
        b.Qz_in = L.Qz[cur];
        b.u_out = L.u[cur ^ 1];
        b.vx_out = L.vx[cur ^ 1];
        b.vy_out = L.vy[cur ^ 1];
        b.Px_out = L.Px[cur ^ 1];
        b.Py_out = L.Py[cur ^ 1];
        b.Qx_out = L.Qx[cur ^ 1];
        b.Qy_out = L.Qy[cur ^ 1];
        b.Qz_out = L.Qz[cur ^ 1];
        MVS_TRY_CUDA(launch_dependent(sparse_iteration_kernel, gi, bi, 0, st, b));
        cur ^= 1;
    }
    scale_kernel<<<eg, 256, 0, st>>>(L.u[cur], n, zfar, out);
    return check_launch("tgv2 sparse");
}

size_t tgv2_workspace_bytes(int w, int h, int V) { return layout(nullptr, w, h, V).bytes; }

// Reads of the stopping flag that do not drain the launch stream.  After each
// energy check the launch path records an event; once kPollLead more
// iterations are queued behind it, a side stream waits for that event and
// copies the flag to the host, so the host learns of a met tolerance while
// the GPU still has those iterations to run (a copy on the launching stream
// would wait for all of them, leaving the GPU idle until the next launch
// arrives).  Iterations queued after a met tolerance return at once.  Only
// the flag is read this way: the rest of the state is read in stream order at
// the end of the linearisation.
constexpr int kPollLead = 20;
constexpr int kPollRing = 32;
constexpr int kPollDevices = 64;

// The side stream and events of one device, made on a thread's first checked
// run on it and kept for the thread's lifetime (making them costs more than a
// short run's polls save).
struct PollResources {
    cudaStream_t s = nullptr;
    cudaEvent_t ev[kPollRing] = {};
    bool tried = false, ok = false;
    ~PollResources()
    {
        for (int k = 0; k < kPollRing; ++k)
            if (ev[k]) cudaEventDestroy(ev[k]);
        if (s) cudaStreamDestroy(s);
    }
};

PollResources *poll_resources()
{
    thread_local PollResources res[kPollDevices];
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kPollDevices) {
        cudaGetLastError();
        return nullptr;
    }
    PollResources &r = res[dev];
    if (!r.tried) {
        r.tried = true;
        r.ok = cudaStreamCreateWithFlags(&r.s, cudaStreamNonBlocking) == cudaSuccess;
        for (int k = 0; r.ok && k < kPollRing; ++k)
            r.ok = cudaEventCreateWithFlags(&r.ev[k], cudaEventDisableTiming) == cudaSuccess;
        if (!r.ok) cudaGetLastError();   // the launch path then polls on its own stream
    }
    return r.ok ? &r : nullptr;
}

struct SidePoll {
    PollResources *res = nullptr;
    int at[kPollRing] = {};   // launch count when each check was recorded
    int head = 0, count = 0;
    bool ok = false;
    void open()
    {
        res = poll_resources();
        ok = res != nullptr;
    }
    // after a check launch on `st`
    cudaError_t record(cudaStream_t st, int launched)
    {
        const int slot = (head + count) % kPollRing;
        at[slot] = launched;
        ++count;
        return cudaEventRecord(res->ev[slot], st);
    }
    // the oldest check's flag, if kPollLead launches are queued behind it (or
    // the ring is full); `*read` says whether a flag was read
    cudaError_t due(int launched, const int *d_done, int *h_done, bool *read)
    {
        *read = false;
        if (!count || (launched - at[head] < kPollLead && count < kPollRing)) return cudaSuccess;
        cudaError_t e = cudaStreamWaitEvent(res->s, res->ev[head], 0);
        if (e == cudaSuccess) e = cudaMemcpyAsync(h_done, d_done, sizeof(int), cudaMemcpyDeviceToHost, res->s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(res->s);
        head = (head + 1) % kPollRing;
        --count;
        *read = e == cudaSuccess;
        return e;
    }
    void reset() { head = count = 0; }
    // a failed side call (say, a context reset since the resources were made):
    // clear the error, remake them on the next run, poll in order for the rest
    // of this one
    void fail()
    {
        cudaGetLastError();
        *res = PollResources{};   // the old handles may be stale: dropped, not destroyed
        ok = false;
    }
};

// One iteration launch for V views (the smallest compiled view count >= V).
cudaError_t launch_iteration(int V, dim3 grid, dim3 block, cudaStream_t st, const IterBufs &ib)
{
    if (V <= 4) return launch_dependent(iteration_kernel<4>, grid, block, 0, st, ib);
    if (V <= 8) return launch_dependent(iteration_kernel<8>, grid, block, 0, st, ib);
    if (V <= 16) return launch_dependent(iteration_kernel<16>, grid, block, 0, st, ib);
    return launch_dependent(iteration_kernel<32>, grid, block, 0, st, ib);
}

int tgv2_run(int w, int h, int V, const float *ref255, const float *srcs255, const float *K9, const float *invK9,
             const float *Rrel, const float *trel, const mvs_tgv2_params *prm, int u_from_input, float u_init,
             float *u, int *iters_out, double *energy_out, void *ws, cudaStream_t st, const TGV2Warm *warm)
{
    if (V > kMaxViews) return set_error(MVS_ERR_ARG, "at most %d views", kMaxViews);
    if (prm->stop_window < 0 || prm->stop_window > MVS_TGV2_STOP_WINDOW_MAX)
        return set_error(MVS_ERR_ARG, "stop_window %d: 0 (default) or 1..%d", prm->stop_window,
                         MVS_TGV2_STOP_WINDOW_MAX);
    Layout L = layout(ws, w, h, V);
    const int n = w * h;
    Cams cams;
    for (int k = 0; k < 9; ++k) {
        cams.K[k] = K9[k];
        cams.invK[k] = invK9[k];
    }
    for (int v = 0; v < V; ++v) {
        for (int k = 0; k < 9; ++k) cams.Rrel[v][k] = Rrel[9 * v + k];
        for (int k = 0; k < 3; ++k) cams.trel[v][k] = trel[3 * v + k];
    }
    const dim3 b2(32, 8), g2(ceil_div(w, 32), ceil_div(h, 8));
    const int eg = min(ceil_div(n, 256), 8 * kSMs);
    tensor_kernel<<<g2, b2, 0, st>>>(ref255, w, h, prm->beta, prm->gamma, L.ref01, L.T11, L.T12, L.T22);
    if (!u_from_input) fill_kernel<<<eg, 256, 0, st>>>(u, n, u_init);
    int rc = check_launch("tgv2 setup");
    if (rc) return rc;

    const int cap = prm->max_iters > 0 ? prm->max_iters : prm->warps * prm->niters;
    const int check_every = prm->check_every > 0 ? prm->check_every : 10;
    const int stop_window = prm->stop_window > 0 ? prm->stop_window : MVS_TGV2_STOP_WINDOW_DEFAULT;
    // the energy is read back into pageable host memory: a synchronous 8-byte
    // copy needs no pinned staging (allocating one per call costs milliseconds)
    double host_energy = 0.0;
    double *h_energy = &host_energy;
    int total = 0;
    double last_e = 0.0;
    int energy_at = -1;   // iteration count at which last_e was evaluated
    int cur = 0;          // ping-pong buffer holding the current p, q
    bool done = false;
    IterBufs ib;
    ib.ctl = prm->tol > 0 ? L.ctl : nullptr;
    ib.T11 = L.T11;
    ib.T12 = L.T12;
    ib.T22 = L.T22;
    ib.u0 = L.u0;
    ib.It = L.It;
    ib.Iu = L.Iu;
    ib.u = u;
    ib.u1x = L.u1x;
    ib.u1y = L.u1y;
    ib.r = L.r;
    ib.w = w;
    ib.h = h;
    ib.V = V;
    ib.lambda = prm->lambda;
    ib.alpha0 = prm->alpha0;
    ib.alpha1 = prm->alpha1;
    ib.tau = prm->tau;
    ib.sigma = prm->sigma;
    const dim3 gi(ceil_div(w, TX), ceil_div(h, TY)), bi(TX, TY);

    // on-chip persistent iterations when the image fits one tile per SM
    int pth = 0, ptiles = 0;
    size_t psmem = 0;
    // (one launch per iteration with dependent launches and the stopping test on
    // the device is faster at every measured size: 14.3 vs 15.9 us per
    // iteration at 640x480 with 8 views, equal at 320x240)
    if (prm->iteration_kernel == MVS_TGV2_ITER_PERSISTENT) {
        int dev = 0, sms = 0, coop = 0, optin = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        const size_t limit = optin > 4096 ? (size_t)optin - 4096 : 0;   // room for the static shared memory
        pth = coop ? persist_tile_height(w, h, V, sms, limit) : 0;
        if (pth) {
            psmem = persist_smem_bytes(pth, V);
            ptiles = ceil_div(w, PT_TW) * ceil_div(h, pth);
            int per_sm = 0;
            if (cudaFuncSetAttribute(tgv2_persistent_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)psmem) != cudaSuccess ||
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tgv2_persistent_kernel, PT_THREADS, psmem) !=
                    cudaSuccess ||
                per_sm * sms < ptiles)
                pth = 0;
            cudaGetLastError();   // a refused attribute or query is not an error of this call
        }
    }
    // launch path: the stopping state lives on the device (IterCtl); the host
    // reads its flag after each check (SidePoll; on the launching stream every
    // kPoll iterations if no side stream could be made) and all of it at the
    // end of each linearisation
    constexpr int kPoll = 50;
    SidePoll sp;
    if (!pth && prm->tol > 0) sp.open();
    IterCtl hc{};
    int launched = 0;
    auto poll = [&]() -> int {
        MVS_TRY_CUDA(cudaMemcpyAsync(&hc, L.ctl, sizeof(IterCtl), cudaMemcpyDeviceToHost, st));
        MVS_TRY_CUDA(cudaStreamSynchronize(st));
        return MVS_OK;
    };
    // (also clears energy_kernel's completion counter, which every run's final energy uses)
    MVS_TRY_CUDA(cudaMemsetAsync(L.ctl, 0, sizeof(IterCtl), st));
    for (int l = 0; l < prm->warps && !done; ++l) {
        if (!pth && prm->tol > 0 && l > 0)   // a new linearisation has no previous energy
            MVS_TRY_CUDA(cudaMemsetAsync(&L.ctl->n_hist, 0, sizeof(int), st));
        if (warm && l == 0)
            warm_init_kernel<<<eg, 256, 0, st>>>(n, V, warm->u_lin, u, warm->v, warm->v ? warm->v + n : nullptr, L.u0,
                                                L.ubar[0], L.u1x, L.u1y, L.u1xbar[0], L.u1ybar[0], L.Px[0], L.Py[0],
                                                L.Qx[0], L.Qy[0], L.Qz[0], L.r, warm->pq, warm->r);
        else
            warp_init_kernel<<<eg, 256, 0, st>>>(n, V, u, L.u0, L.ubar[0], L.u1x, L.u1y, L.u1xbar[0], L.u1ybar[0],
                                                L.Px[0], L.Py[0], L.Qx[0], L.Qy[0], L.Qz[0], L.r);
        linearize_kernel<<<dim3(g2.x, g2.y, V), b2, 0, st>>>(cams, srcs255, L.ref01, L.u0, w, h, L.It, L.Iu);
        if (warm && l == 0) {
            const int do_pq = !warm->pq && warm->dual_sigma > 0, do_r = !warm->r && warm->dual_sigma_r > 0;
            if (do_pq || do_r)
                dual_init_kernel<<<g2, b2, 0, st>>>(L.T11, L.T12, L.T22, L.It, L.Iu, L.u0, u, L.u1x, L.u1y, w, h, V,
                                                   prm->lambda, prm->alpha0, prm->alpha1, (float)warm->dual_sigma,
                                                   (float)warm->dual_sigma_r, L.Px[0], L.Py[0], L.Qx[0], L.Qy[0],
                                                   L.Qz[0], L.r, do_pq, do_r);
        }
        rc = check_launch("tgv2 linearisation");
        if (rc) break;
        cur = 0;
        if (pth) {
            // the whole linearisation in one cooperative launch
            PersistBufs pb;
            pb.T11 = L.T11;
            pb.T12 = L.T12;
            pb.T22 = L.T22;
            pb.u0 = L.u0;
            pb.It = L.It;
            pb.Iu = L.Iu;
            pb.u = u;
            pb.u1x = L.u1x;
            pb.u1y = L.u1y;
            pb.r = L.r;
            pb.ubar0 = L.ubar[0];
            pb.u1xbar0 = L.u1xbar[0];
            pb.u1ybar0 = L.u1ybar[0];
            pb.Px = L.Px[0];
            pb.Py = L.Py[0];
            pb.Qx = L.Qx[0];
            pb.Qy = L.Qy[0];
            pb.Qz = L.Qz[0];
            for (int q = 0; q < 2; ++q) {
                pb.exb[q] = L.exb[q];
                pb.exq[q] = L.exq[q];
            }
            pb.exu = L.exu;
            pb.partial = L.ppartial;
            pb.bar = L.bar;
            pb.res = L.res;
            pb.w = w;
            pb.h = h;
            pb.V = V;
            pb.tiles_x = ceil_div(w, PT_TW);
            pb.th = pth;
            pb.niters = prm->niters;
            pb.cap_left = cap - total;
            pb.check_every = check_every;
            pb.stop_window = stop_window;
            pb.tol = prm->tol;
            pb.lambda = prm->lambda;
            pb.alpha0 = prm->alpha0;
            pb.alpha1 = prm->alpha1;
            pb.tau = prm->tau;
            pb.sigma = prm->sigma;
            pb.dlambda = prm->lambda;
            pb.dalpha0 = prm->alpha0;
            pb.dalpha1 = prm->alpha1;
            cudaMemsetAsync(L.bar, 0, 64, st);
            void *args[] = {&pb};
            cudaError_t e = cudaLaunchCooperativeKernel((const void *)tgv2_persistent_kernel, dim3(ptiles),
                                                        dim3(PT_THREADS), args, psmem, st);
            PersistResult hr{};
            if (e == cudaSuccess) e = cudaMemcpyAsync(&hr, L.res, sizeof(hr), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) {
                rc = set_error(MVS_ERR_CUDA, "tgv2 persistent iteration: %s", cudaGetErrorString(e));
                break;
            }
            if (hr.err) {
                rc = set_error(MVS_ERR_TIMEOUT, "tgv2 persistent iteration: a grid barrier wait gave up");
                break;
            }
            if (hr.energy_at >= 0) {
                last_e = hr.energy;
                energy_at = total + hr.energy_at;
            }
            total += hr.iters;
            done = hr.done || total >= cap;
            continue;
        }
        const int warp_start = launched;
        for (int k = 0; k < prm->niters; ++k) {
            ib.ubar_in = L.ubar[cur];
            ib.u1xbar_in = L.u1xbar[cur];
            ib.u1ybar_in = L.u1ybar[cur];
            ib.Px_in = L.Px[cur];
            ib.Py_in = L.Py[cur];
            ib.Qx_in = L.Qx[cur];
            ib.Qy_in = L.Qy[cur];
            ib.Qz_in = L.Qz[cur];
            ib.ubar_out = L.ubar[cur ^ 1];
            ib.u1xbar_out = L.u1xbar[cur ^ 1];
            ib.u1ybar_out = L.u1ybar[cur ^ 1];
            ib.Px_out = L.Px[cur ^ 1];
            ib.Py_out = L.Py[cur ^ 1];
            ib.Qx_out = L.Qx[cur ^ 1];
            ib.Qy_out = L.Qy[cur ^ 1];
            ib.Qz_out = L.Qz[cur ^ 1];
            // dependent launches: each iteration's launch overlaps the previous one's tail
            MVS_TRY_CUDA(launch_iteration(V, gi, bi, st, ib));
            cur ^= 1;
            ++launched;
            const bool check = prm->tol > 0 && (k + 1) % check_every == 0;
            if (check)
                MVS_TRY_CUDA(launch_dependent(energy_kernel, gi, bi, 0, st, L.T11, L.T12, L.T22, L.It, L.Iu, L.u0, u,
                                              L.u1x, L.u1y, w, h, V, prm->lambda, prm->alpha0, prm->alpha1, L.partial,
                                              L.energy, L.ctl, prm->tol, launched, stop_window));
            if (launched >= cap) {
                done = true;
                break;
            }
            if (sp.ok) {
                cudaError_t e = check ? sp.record(st, launched) : cudaSuccess;
                bool read = false;
                if (e == cudaSuccess) e = sp.due(launched, &L.ctl->done, &hc.done, &read);
                if (e != cudaSuccess) sp.fail();
                else if (read && hc.done) break;
            } else if (prm->tol > 0 && launched % kPoll == 0) {
                if ((rc = poll())) break;
                if (hc.done) break;
            }
        }
        sp.reset();
        if (!rc && prm->tol > 0) {
            rc = poll();
            if (!rc && hc.done) {
                done = true;
                cur = (hc.stop_total - warp_start) & 1;   // p, q of the last iteration that ran
            }
        }
        if (!rc) rc = check_launch("tgv2 iteration");
        if (rc) break;
    }
    if (!pth) {
        // launch path: iterations after a met tolerance did nothing
        total = prm->tol > 0 && hc.done ? hc.stop_total : launched;
        if (prm->tol > 0 && hc.have_energy) {
            last_e = hc.last_e;
            energy_at = hc.energy_at;
        }
    }
    if (!rc && warm && warm->v) {
        cudaMemcpyAsync(warm->v, L.u1x, n * sizeof(float), cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(warm->v + n, L.u1y, n * sizeof(float), cudaMemcpyDeviceToDevice, st);
        rc = check_launch("tgv2 v readout");
    }
    if (!rc && warm && warm->pq) {
        float *const src[5] = {L.Px[cur], L.Py[cur], L.Qx[cur], L.Qy[cur], L.Qz[cur]};
        for (int k = 0; k < 5; ++k)
            cudaMemcpyAsync(warm->pq + (size_t)k * n, src[k], n * sizeof(float), cudaMemcpyDeviceToDevice, st);
        rc = check_launch("tgv2 dual readout");
    }
    if (!rc && warm && warm->r) {   // the caller's [V][n] planes
        r_planes_kernel<<<eg, 256, 0, st>>>(L.r, n, V, warm->r);
        rc = check_launch("tgv2 dual readout");
    }
    if (!rc && energy_out && energy_at != total) {
        // energy of the final iterate for callers that ask for it
        energy_kernel<<<gi, bi, 0, st>>>(L.T11, L.T12, L.T22, L.It, L.Iu, L.u0, u, L.u1x, L.u1y, w, h, V, prm->lambda,
                                         prm->alpha0, prm->alpha1, L.partial, L.energy, L.ctl, 0.0, total, 1);
        cudaMemcpyAsync(h_energy, L.energy, sizeof(double), cudaMemcpyDeviceToHost, st);
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = set_error(MVS_ERR_CUDA, "tgv2 energy: %s", cudaGetErrorString(e));
        last_e = *h_energy;
    }
    if (iters_out) *iters_out = total;
    if (energy_out) *energy_out = last_e;
    return rc;
}

}  // namespace mvs
