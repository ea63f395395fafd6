// Shared device/host helpers for the sm_100a kernels of libmvs_b200.
//
// Every .cu file of the library is compiled with -fmad=false: a plain `a*b+c`
// is two IEEE roundings, exactly as the reference's arithmetic when it is run
// on the CPU.  Kernels that want fused multiply-adds on their fast paths ask
// for them explicitly with fmaf()/__fmaf_rn().
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/mvs_b200.h"

namespace mvs {

constexpr int kSMs = 148;          // B200: 2 dies x 74 SMs
constexpr int kMapCamFloats = 21;  // per fusion depthmap: K[9] R[9] t[3]

// Last-error bookkeeping shared by every entry point (defined in capi.cu).
int set_error(int code, const char *fmt, ...);
int check_launch(const char *what);
void clear_error();
// Validates a sweep descriptor; MVS_OK or MVS_ERR_ARG with the message set.
int check_sweep_desc(const mvs_sweep_desc *d);

#define MVS_TRY_CUDA(expr)                                                              \
    do {                                                                                \
        cudaError_t e__ = (expr);                                                       \
        if (e__ != cudaSuccess)                                                         \
            return ::mvs::set_error(MVS_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e__)); \
    } while (0)

// ---- mbarrier helpers (inline PTX, sm_100a) ----
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait for one phase of an mbarrier: false after `limit_ns`.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint64_t limit_ns)
{
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > limit_ns) return false;
    return true;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Boundary mirror of windowed_mean_row/column_kernel (kernels.cu:203-204,
// 228-229): k < 0 -> -k, k > n-1 -> 2(n-1)-k.  The final clamp only matters
// for cells that no in-image output reads (entry points reject images
// narrower than the window, the one case where the reference itself reads
// out of bounds).
__device__ __forceinline__ int mirror_idx(int k, int n)
{
    if (k < 0) k = -k;
    if (k > n - 1) k = 2 * (n - 1) - k;
    return min(max(k, 0), n - 1);
}

__device__ __forceinline__ float ldg(const float *p) { return __ldg(p); }

// Round-to-nearest-even float -> bf16 bits (finite inputs; NaN stays NaN).
__device__ __forceinline__ uint16_t f2bf(float f)
{
    uint32_t u = __float_as_uint(f);
    if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40);
    u += 0x7fffu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

// f2bf for a value that is not NaN: the hardware's round-to-nearest-even
// conversion, one instruction, the same bits as f2bf for every other input.
__device__ __forceinline__ uint16_t f2bf_num(float f)
{
    uint16_t b;
    asm("cvt.rn.bf16.f32 %0, %1;" : "=h"(b) : "f"(f));
    return b;
}

__device__ __forceinline__ float bf2f(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }

inline int ceil_div(int a, int b) { return (a + b - 1) / b; }

// Programmatic dependent launch, for loops of short dependent launches (one
// launch per iteration).  A kernel launched with launch_dependent() may be
// scheduled while the previous kernel of its stream is still finishing, which
// hides the gap between the two launches (about 2.6 us per launch measured on
// the B200).  Such a kernel calls wait_for_previous_grid() before it reads or
// writes any global memory that the previous kernels of the stream touch: the
// wait returns once those grids have completed and their writes are visible.
// Without the launch attribute the wait returns at once.
__device__ __forceinline__ void wait_for_previous_grid() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void allow_next_grid() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
cudaError_t launch_dependent(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                             Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, ((KArgs)args)...);
}

// One frame of a batched sweep (device copy; see sweep_batch_kernel).
struct BatchFrameDev {
    const float *ref, *srcs, *H, *depths;
    float *depth;
    int32_t *labels;
    float *best;
    unsigned long long *wta;      // [w*h] winner words, ~0 between launches
    unsigned int *tile_left;      // [n_tiles] chunks still running
    unsigned int *frame_left;     // tiles still running
    unsigned long long *done_ns;  // completion time of the last launch
    const float4 *quad;           // [V][w*h] 2x2 source neighbourhoods, or null
    int w, h, V, P, win, planes_per_chunk, n_chunks, tiles_x, n_tiles, tile_w;
    float stdthresh, zfar;
};

constexpr int kBatchMaxViews = 16;
struct BatchCamDev {
    double K[9], invK[9];
    double Rrel[kBatchMaxViews][9];
    double trel[kBatchMaxViews][3];
    const float *depths;
    float *H;
    int V, P;
};

// Warm start of a TGV2 run: the data term is linearised at u_lin (first
// linearisation) while the primal starts at the caller's u and at v (2 planes,
// vx then vy; NULL = 0), which also receives the final v.  dual_sigma > 0
// (dual_sigma_r > 0) starts the regulariser's (the data term's) dual
// variables one dual step of that size from zero.  pq (5 planes: px, py, qx,
// qy, qz) and r (one plane per view), when given, are the duals' start
// instead and receive their final values.
struct TGV2Warm {
    const float *u_lin;
    float *v;
    double dual_sigma, dual_sigma_r;
    float *pq, *r;
};

}  // namespace mvs
