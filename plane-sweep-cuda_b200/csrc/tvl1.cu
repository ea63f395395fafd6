// TV-L1 depth denoising (PlaneSweep::CudaDenoise, planesweep.cpp:297-379) for
// sm_100a.
//
// The reference alternates two full-image launches per iteration:
// denoising_TVL1_calculateP_tensor_weighed (kernels.cu:283-307) and
// denoising_TVL1_update (kernels.cu:342-370).  Here one launch per iteration
// recomputes the new dual p on a one-pixel halo to the left and top of a
// 32 x 8 tile (the primal update reads p at x-1 and y-1) and then updates
// the primal in place; p and the primal (read at x+1, y+1) are
// double-buffered.  Arithmetic follows the reference statement for
// statement (compiled with -fmad=false).
#include <math.h>

#include "common.cuh"

namespace mvs {
namespace {

constexpr float kInv255 = 1.f / 255.f;
constexpr int TX = 32, TY = 8;

// ref/255 and its diffusion tensor (Anisotropic_diffusion_tensor_kernel,
// TGV2_kernels.cu:257-298), and the scaled start (planesweep.cpp:334-344):
// out = (d - znear) * xscale, raw = (d - znear) * inputscale.
__global__ void tvl1_setup_kernel(const float *__restrict__ ref255, const float *__restrict__ depth, int w, int h,
                                  float beta, float gamma, float znear, float xscale, float inputscale,
                                  float *__restrict__ T11, float *__restrict__ T12, float *__restrict__ T22,
                                  float *__restrict__ out, float *__restrict__ raw, float *__restrict__ R,
                                  float *__restrict__ Px, float *__restrict__ Py)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const int i = y * w + x, xn = min(x + 1, w - 1), yn = min(y + 1, h - 1);
    const float r = ref255[i] * kInv255;
    float gx = ref255[y * w + xn] * kInv255 - r;
    float gy = ref255[yn * w + x] * kInv255 - r;
    const float d = sqrtf(gx * gx + gy * gy);
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
    const float s = depth[i] + -znear;
    out[i] = s * xscale;
    raw[i] = s * inputscale;
    R[i] = 0.f;
    Px[i] = 0.f;
    Py[i] = 0.f;
}

struct Bufs {
    const float *T11, *T12, *T22, *raw;
    const float *in, *Px_in, *Py_in;
    float *out, *Px_out, *Py_out, *R;
    int w, h;
    float sigma_p, tau, theta, lambda, sigma;
};

__global__ void __launch_bounds__(TX *TY) tvl1_iteration_kernel(Bufs b)
{
    __shared__ float sD[TY + 2][TX + 2];
    __shared__ float sPx[TY + 1][TX + 1], sPy[TY + 1][TX + 1];
    wait_for_previous_grid();   // launched as a dependent launch: the previous iteration is complete
    allow_next_grid();
    const int w = b.w, h = b.h;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int tid = threadIdx.y * TX + threadIdx.x;
    for (int k = tid; k < (TX + 2) * (TY + 2); k += TX * TY) {
        const int ry = k / (TX + 2), rx = k % (TX + 2);
        const int px = min(max(x0 - 1 + rx, 0), w - 1), py = min(max(y0 - 1 + ry, 0), h - 1);
        sD[ry][rx] = b.in[py * w + px];
    }
    __syncthreads();
    // denoising_TVL1_calculateP_tensor_weighed_kernel (kernels.cu:283-307)
    for (int k = tid; k < (TX + 1) * (TY + 1); k += TX * TY) {
        const int ry = k / (TX + 1), rx = k % (TX + 1);
        const int px = x0 - 1 + rx, py = y0 - 1 + ry;
        if (px < 0 || py < 0 || px >= w || py >= h) continue;
        const int j = py * w + px;
        const int nx = px + 1 <= w - 1 ? rx + 1 : rx, ny = py + 1 <= h - 1 ? ry + 1 : ry;
        const double x = sD[ry][nx] - sD[ry][rx];
        const double y = sD[ny][rx] - sD[ry][rx];
        const double t11 = b.T11[j], t12 = b.T12[j], t22 = b.T22[j];
        const double dx = (double)b.Px_in[j] + (double)b.sigma_p * (t11 * x + t12 * y);
        const double dy = (double)b.Py_in[j] + (double)b.sigma_p * (t12 * x + t22 * y);
        // fmaxf(1, sqrt(s)) is exactly 1 for s <= 1, and dividing by 1 is the identity
        const double s2 = dx * dx + dy * dy;
        const double d = s2 > 1.0 ? (double)fmaxf(1.f, (float)sqrt(s2)) : 1.0;
        sPx[ry][rx] = (float)(d == 1.0 ? dx : dx / d);
        sPy[ry][rx] = (float)(d == 1.0 ? dy : dy / d);
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    if (x >= w || y >= h) return;
    const int i = y * w + x, lx = threadIdx.x + 1, ly = threadIdx.y + 1;
    const int lyp = y > 0 ? ly - 1 : ly;
    // denoising_TVL1_update_kernel (kernels.cu:342-370)
    float r = b.R[i];
    r += b.raw[i];
    const float o = sD[ly][lx];
    r += b.sigma * o;
    if (r > b.lambda) r = b.lambda;
    if (r < -b.lambda) r = -b.lambda;
    b.R[i] = r;
    const float cpx = sPx[ly][lx], cpy = sPy[ly][lx];
    double x_new;
    if (x == 0) x_new = o + b.tau * (cpy - sPy[lyp][lx]) - b.tau * r;
    else x_new = o + b.tau * (cpx - sPx[ly][lx - 1] + cpy - sPy[lyp][lx]) - b.tau * r;
    b.out[i] = (float)(x_new + (double)b.theta * (x_new - (double)o));
    b.Px_out[i] = cpx;
    b.Py_out[i] = cpy;
}

// element_scale(d, zfar - znear) then element_add(d, znear) (planesweep.cpp:355-356)
__global__ void tvl1_finish_kernel(const float *__restrict__ in, int n, float scale, float znear, float *__restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = in[i] * scale + znear;
}

struct Layout {
    float *T11, *T12, *T22, *raw, *R, *D[2], *Px[2], *Py[2];
    size_t bytes;
};

Layout layout(void *base, int w, int h)
{
    Layout L{};
    const size_t n = (size_t)w * h;
    char *p = (char *)base;
    size_t off = 0;
    auto take = [&]() {
        float *q = (float *)(p + off);
        off += ((n * sizeof(float) + 255) / 256) * 256;
        return q;
    };
    L.T11 = take();
    L.T12 = take();
    L.T22 = take();
    L.raw = take();
    L.R = take();
    for (int k = 0; k < 2; ++k) {
        L.D[k] = take();
        L.Px[k] = take();
        L.Py[k] = take();
    }
    L.bytes = off;
    return L;
}

}  // namespace

size_t tvl1_workspace_bytes(int w, int h) { return layout(nullptr, w, h).bytes; }

int tvl1_run(int w, int h, const float *ref255, float *depth, float znear, float zfar, const mvs_tvl1_params *prm,
             void *ws, cudaStream_t st)
{
    Layout L = layout(ws, w, h);
    const int n = w * h;
    // xscale = 1.f/(zfar - znear) in float; inputscale = -sigma/(zfar - znear)
    // in double, both handed to float kernel parameters (planesweep.cpp:340-344)
    const float xscale = 1.f / (zfar - znear);
    const float inputscale = (float)(-(double)prm->sigma / (double)(zfar - znear));
    const dim3 b2(TX, TY), g2(ceil_div(w, TX), ceil_div(h, TY));
    tvl1_setup_kernel<<<g2, b2, 0, st>>>(ref255, depth, w, h, prm->beta, prm->gamma, znear, xscale, inputscale, L.T11,
                                        L.T12, L.T22, L.D[0], L.raw, L.R, L.Px[0], L.Py[0]);
    int cur = 0;
    Bufs b;
    b.T11 = L.T11;
    b.T12 = L.T12;
    b.T22 = L.T22;
    b.raw = L.raw;
    b.R = L.R;
    b.w = w;
    b.h = h;
    b.tau = prm->tau;
    b.theta = prm->theta;
    b.lambda = prm->lambda;
    b.sigma = prm->sigma;
    for (int it = 0; it < prm->niters; ++it) {
        // first dual step uses sigma + 1 (planesweep.cpp:347)
        b.sigma_p = (float)(it == 0 ? 1.0 + (double)prm->sigma : (double)prm->sigma);
        b.in = L.D[cur];
        b.Px_in = L.Px[cur];
        b.Py_in = L.Py[cur];
        b.out = L.D[cur ^ 1];
        b.Px_out = L.Px[cur ^ 1];
        b.Py_out = L.Py[cur ^ 1];
        MVS_TRY_CUDA(launch_dependent(tvl1_iteration_kernel, g2, b2, 0, st, b));
        cur ^= 1;
    }
    tvl1_finish_kernel<<<min(ceil_div(n, 256), 8 * kSMs), 256, 0, st>>>(L.D[cur], n, zfar - znear, znear, depth);
    return check_launch("tvl1 denoise");
}

}  // namespace mvs
