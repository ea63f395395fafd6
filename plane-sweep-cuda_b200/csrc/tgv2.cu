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
        for (int k = 0; k < V; ++k) r[(size_t)k * n + i] = 0.f;
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
        for (int k = 0; k < V; ++k) r[(size_t)k * n + i] = r_in ? r_in[(size_t)k * n + i] : 0.f;
    }
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
    Iu[(size_t)v * n + i] = (float)(gx * (double)dfx + gy * (double)dfy);
    It[(size_t)v * n + i] = Iw - ref01[i];
}

struct IterBufs {
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

// One full TGV2 iteration (planesweep.cpp:485-509).  The pixel's own operands
// (r, It, Iu of every view, T, u, u0, v) are loaded before the shared-memory
// phase so their latency overlaps the halo work.
template <int VMAX>
__global__ void __launch_bounds__(TX *TY) iteration_kernel(IterBufs b)
{
    __shared__ float sU[TY + 2][TX + 2], sVX[TY + 2][TX + 2], sVY[TY + 2][TX + 2];
    __shared__ float sPx[TY + 1][TX + 1], sPy[TY + 1][TX + 1];
    __shared__ float sQx[TY + 1][TX + 1], sQy[TY + 1][TX + 1], sQz[TY + 1][TX + 1];
    const int w = b.w, h = b.h;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int tid = threadIdx.y * TX + threadIdx.x;
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    const bool own = x < w && y < h;
    const int i = own ? y * w + x : 0;
    const size_t n = (size_t)w * h;

    // own-pixel operands, prefetched
    float rv[VMAX], itv[VMAX], iuv[VMAX];
    const int V = b.V;   // <= VMAX (the launch picks VMAX)
#pragma unroll
    for (int v = 0; v < VMAX; ++v) {
        if (v < V && own) {
            const size_t k = (size_t)v * n + i;
            rv[v] = b.r[k];
            itv[v] = b.It[k];
            iuv[v] = b.Iu[k];
        }
    }
    float t11 = 0.f, t12 = 0.f, t22 = 0.f, uold = 0.f, u0v = 0.f, u1xprev = 0.f, u1yprev = 0.f;
    if (own) {
        t11 = b.T11[i];
        t12 = b.T12[i];
        t22 = b.T22[i];
        uold = b.u[i];
        u0v = b.u0[i];
        u1xprev = b.u1x[i];
        u1yprev = b.u1y[i];
    }

    // ubar, vbar on [x0-1, x0+TX] x [y0-1, y0+TY] (clamped; cells outside the
    // image are never read)
    for (int k = tid; k < (TX + 2) * (TY + 2); k += TX * TY) {
        const int ry = k / (TX + 2), rx = k % (TX + 2);
        const int px = min(max(x0 - 1 + rx, 0), w - 1), py = min(max(y0 - 1 + ry, 0), h - 1);
        const int j = py * w + px;
        sU[ry][rx] = b.ubar_in[j];
        sVX[ry][rx] = b.u1xbar_in[j];
        sVY[ry][rx] = b.u1ybar_in[j];
    }
    __syncthreads();

    // new p (TGV2_updateP_tensor_weighed_kernel, TGV2_kernels.cu:340-365) and
    // q (TGV2_updateQ_kernel, :54-85) on [x0-1, x0+TX) x [y0-1, y0+TY)
    const float a1s = b.alpha1 * b.sigma, a0s = b.alpha0 * b.sigma;
    for (int k = tid; k < (TX + 1) * (TY + 1); k += TX * TY) {
        const int ry = k / (TX + 1), rx = k % (TX + 1);
        const int px = x0 - 1 + rx, py = y0 - 1 + ry;
        if (px < 0 || py < 0 || px >= w || py >= h) continue;
        const int j = py * w + px;
        const int nx = px + 1 <= w - 1 ? rx + 1 : rx, ny = py + 1 <= h - 1 ? ry + 1 : ry;
        {
            const double xg = sU[ry][nx] - sU[ry][rx] - sVX[ry][rx];
            const double yg = sU[ny][rx] - sU[ry][rx] - sVY[ry][rx];
            const double c11 = b.T11[j], c12 = b.T12[j], c22 = b.T22[j];
            const double dx = (double)b.Px_in[j] + (double)a1s * (c11 * xg + c12 * yg);
            const double dy = (double)b.Py_in[j] + (double)a1s * (c12 * xg + c22 * yg);
            const double d = proj_norm(dx * dx + dy * dy);
            sPx[ry][rx] = (float)(d == 1.0 ? dx : dx / d);
            sPy[ry][rx] = (float)(d == 1.0 ? dy : dy / d);
        }
        {
            const float dx_u1x = sVX[ry][nx] - sVX[ry][rx];
            const float dy_u1x = sVX[ny][rx] - sVX[ry][rx];
            const float dx_u1y = sVY[ry][nx] - sVY[ry][rx];
            const float dy_u1y = sVY[ny][rx] - sVY[ry][rx];
            const double dx = b.Qx_in[j] + a0s * dx_u1x;
            const double dy = b.Qy_in[j] + a0s * dy_u1y;
            const double dz = b.Qz_in[j] + a0s * (dy_u1x + dx_u1y) / 2.0f;
            const double d = proj_norm(dx * dx + dy * dy + dz * dz + dz * dz);
            sQx[ry][rx] = (float)(d == 1.0 ? dx : dx / d);
            sQy[ry][rx] = (float)(d == 1.0 ? dy : dy / d);
            sQz[ry][rx] = (float)(d == 1.0 ? dz : dz / d);
        }
    }
    __syncthreads();

    if (!own) return;
    const int lx = threadIdx.x + 1, ly = threadIdx.y + 1;

    // r and prodsum (TGV2_updateR_kernel, TGV2_kernels.cu:87-105), views in order
    const float du = uold - u0v;
    const float sl = b.sigma * b.lambda;
    float prodsum = 0.f;
#pragma unroll
    for (int v = 0; v < VMAX; ++v) {
        if (v < V) {
            float r = rv[v] + sl * (itv[v] + du * iuv[v]);
            r = r / fmaxf(1.f, fabsf(r));
            b.r[(size_t)v * n + i] = r;
            prodsum += r * iuv[v];
        }
    }

    // primal step (TGV2_updateU_tensor_weighed_kernel, TGV2_kernels.cu:300-338)
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

// Energy of the current iterate (the functional the updates minimise; the
// reference has none): per-block FP64 partial sums, then one block adds them.
constexpr int EB = 256;

__global__ void __launch_bounds__(EB) energy_kernel(const float *__restrict__ T11, const float *__restrict__ T12,
                                                    const float *__restrict__ T22, const float *__restrict__ It,
                                                    const float *__restrict__ Iu, const float *__restrict__ u0,
                                                    const float *__restrict__ u, const float *__restrict__ u1x,
                                                    const float *__restrict__ u1y, int w, int h, int V, double lambda,
                                                    double alpha0, double alpha1, double *__restrict__ partial)
{
    __shared__ double red[EB / 32];
    const int n = w * h;
    double e = 0.0;
    for (int i = blockIdx.x * EB + threadIdx.x; i < n; i += gridDim.x * EB) {
        const int y = i / w, x = i - y * w;
        const int xn = min(x + 1, w - 1), yn = min(y + 1, h - 1);
        const double gx = (double)u[y * w + xn] - u[i] - u1x[i];
        const double gy = (double)u[yn * w + x] - u[i] - u1y[i];
        const double tx = T11[i] * gx + T12[i] * gy, ty = T12[i] * gx + T22[i] * gy;
        double ei = alpha1 * sqrt(tx * tx + ty * ty);
        const double a = (double)u1x[y * w + xn] - u1x[i], bb = (double)u1y[yn * w + x] - u1y[i];
        const double c = 0.5 * (((double)u1x[yn * w + x] - u1x[i]) + ((double)u1y[y * w + xn] - u1y[i]));
        ei += alpha0 * sqrt(a * a + bb * bb + 2 * c * c);
        const double du = (double)u[i] - u0[i];
        double ed = 0.0;
        for (int v = 0; v < V; ++v) ed += fabs((double)It[(size_t)v * n + i] + du * Iu[(size_t)v * n + i]);
        e += ei + lambda * ed;
    }
    for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < EB / 32; ++k) s += red[k];
        partial[blockIdx.x] = s;
    }
}

__global__ void sum_partials_kernel(const double *__restrict__ partial, int m, double *__restrict__ out)
{
    __shared__ double red[EB / 32];
    double s = 0.0;
    for (int k = threadIdx.x; k < m; k += EB) s += partial[k];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < EB / 32; ++k) t += red[k];
        *out = t;
    }
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
    const size_t n = (size_t)w * h;
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
        const size_t k = (size_t)v * n + i;
        float q = sdr * lambda * (It[k] + du * Iu[k]);
        r[k] = q / fmaxf(1.f, fabsf(q));
    }
}

constexpr int kEnergyBlocks = 2 * kSMs;

struct Layout {
    float *ref01, *T11, *T12, *T22, *u0, *u1x, *u1y, *ubar[2], *u1xbar[2], *u1ybar[2], *Px[2], *Py[2], *Qx[2],
        *Qy[2], *Qz[2], *It, *Iu, *r;
    double *partial, *energy;
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
    L.It = take(n * V);
    L.Iu = take(n * V);
    L.r = take(n * V);
    L.partial = (double *)take(2 * kEnergyBlocks);
    L.energy = (double *)take(2);
    L.bytes = off;
    return L;
}

}  // namespace

size_t tgv2_workspace_bytes(int w, int h, int V) { return layout(nullptr, w, h, V).bytes; }

int tgv2_run(int w, int h, int V, const float *ref255, const float *srcs255, const float *K9, const float *invK9,
             const float *Rrel, const float *trel, const mvs_tgv2_params *prm, int u_from_input, float u_init,
             float *u, int *iters_out, double *energy_out, void *ws, cudaStream_t st, const TGV2Warm *warm)
{
    if (V > kMaxViews) return set_error(MVS_ERR_ARG, "at most %d views", kMaxViews);
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
    for (int l = 0; l < prm->warps && !done; ++l) {
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
        bool have_prev = false;
        double prev = 0.0;
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
            if (V <= 4) iteration_kernel<4><<<gi, bi, 0, st>>>(ib);
            else if (V <= 8) iteration_kernel<8><<<gi, bi, 0, st>>>(ib);
            else if (V <= 16) iteration_kernel<16><<<gi, bi, 0, st>>>(ib);
            else iteration_kernel<32><<<gi, bi, 0, st>>>(ib);
            cur ^= 1;
            ++total;
            if (prm->tol > 0 && (k + 1) % check_every == 0) {
                energy_kernel<<<kEnergyBlocks, EB, 0, st>>>(L.T11, L.T12, L.T22, L.It, L.Iu, L.u0, u, L.u1x, L.u1y, w,
                                                           h, V, prm->lambda, prm->alpha0, prm->alpha1, L.partial);
                sum_partials_kernel<<<1, EB, 0, st>>>(L.partial, kEnergyBlocks, L.energy);
                cudaMemcpyAsync(h_energy, L.energy, sizeof(double), cudaMemcpyDeviceToHost, st);
                cudaError_t e = cudaStreamSynchronize(st);
                if (e != cudaSuccess) {
                    rc = set_error(MVS_ERR_CUDA, "tgv2 energy: %s", cudaGetErrorString(e));
                    done = true;
                    break;
                }
                last_e = *h_energy;
                energy_at = total;
                if (have_prev && fabs(prev - last_e) <= prm->tol * fabs(prev)) {
                    done = true;
                    break;
                }
                prev = last_e;
                have_prev = true;
            }
            if (total >= cap) {
                done = true;
                break;
            }
        }
        if (!rc) rc = check_launch("tgv2 iteration");
        if (rc) break;
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
    if (!rc && warm && warm->r) {
        cudaMemcpyAsync(warm->r, L.r, (size_t)V * n * sizeof(float), cudaMemcpyDeviceToDevice, st);
        rc = check_launch("tgv2 dual readout");
    }
    if (!rc && energy_out && energy_at != total) {
        // energy of the final iterate for callers that ask for it
        energy_kernel<<<kEnergyBlocks, EB, 0, st>>>(L.T11, L.T12, L.T22, L.It, L.Iu, L.u0, u, L.u1x, L.u1y, w, h, V,
                                                   prm->lambda, prm->alpha0, prm->alpha1, L.partial);
        sum_partials_kernel<<<1, EB, 0, st>>>(L.partial, kEnergyBlocks, L.energy);
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
