// mvs_sweep_noalloc: the fused plane sweep with its scratch in a fixed,
// library-owned device array instead of caller-allocated workspace.
//
// Some callers cannot allocate device memory when they run the sweep: host
// frameworks and plugin hosts that hand a library all the device memory it may
// use up front and forbid allocations afterwards, and real-time loops that
// cannot afford cudaMalloc's latency and implicit device synchronisation.
// They still pass their own inputs and outputs; the only memory the sweep
// needs beyond those -- the per-pixel best-match words that the sweep kernel
// and its epilogue exchange -- lives in `g_sweep_scratch` below.
//
// The array is a file-scope __device__ variable of this file's CUDA module.
// CUDA loads a module lazily (the default since CUDA 12.2): the first time
// host code touches it on a device, here the first cudaGetSymbolAddress of a
// call on that device.  That load reserves the array's 32 MiB on the device,
// which then holds it until the process exits.  Host code must not pass the
// array's name to a kernel (on the host that name is a stand-in, not a device
// address), so every call looks the device address up with
// cudaGetSymbolAddress for the current device and context; once the module is
// loaded the lookup is cheap, and it stays right after a device reset or when
// a caller's own context is current.
#include "common.cuh"

namespace mvs {

int sweep_pick_chunks(int win, int w, int h, int V, int P, int mode);
int sweep_launch(const mvs_sweep_desc *d, const float *ref, const float *srcs, const float *H, const float *depths,
                 float *depth, int32_t *labels, float *best, uint16_t *cost, unsigned long long *scratch,
                 int n_chunks, void *stream, float4 *quad);
size_t sweep_scratch_bytes(const mvs_sweep_desc *d);

// 32 MiB: 4 Mi 64-bit words, one per pixel and source view in the per-view
// mode (a 640x480 frame with up to 13 views) or one per pixel in the
// aggregated mode (up to 4 Mi pixels).
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
static __device__ __align__(256) unsigned long long g_sweep_scratch[kNoAllocScratchBytes / 8];

}  // namespace mvs

extern "C" {

size_t mvs_sweep_noalloc_scratch_bytes(void) { return mvs::kNoAllocScratchBytes; }

int mvs_sweep_noalloc(const mvs_sweep_desc *d, const float *ref, const float *srcs, const float *H,
                      const float *depths, float *depth, int32_t *labels, float *best, uint16_t *cost, void *stream)
{
    using namespace mvs;
    clear_error();
    if (int rc = check_sweep_desc(d)) return rc;
    // only the winner words: the fixed array holds no 2x2 source neighbourhoods
    // (the kernel then gathers the four samples itself)
    const size_t need = sweep_scratch_bytes(d);
    if (need > kNoAllocScratchBytes)
        return set_error(MVS_ERR_ARG,
                         "mvs_sweep_noalloc: this sweep needs %zu bytes of scratch, the fixed array holds %zu "
                         "(at most %zu pixel-view words); use mvs_sweep with a caller workspace",
                         need, kNoAllocScratchBytes, kNoAllocScratchBytes / 8);
    if (!ref || !srcs || !H || !depths || !depth) return set_error(MVS_ERR_ARG, "null input/output pointer");
    if (d->mode == MVS_SWEEP_PER_VIEW && cost) return set_error(MVS_ERR_ARG, "cost volume is an aggregated-mode output");
    void *scratch = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&scratch, g_sweep_scratch);
    if (e != cudaSuccess)
        return set_error(MVS_ERR_CUDA, "cudaGetSymbolAddress(sweep scratch): %s", cudaGetErrorString(e));
    const int chunks = sweep_pick_chunks(d->window, d->width, d->height, d->n_views, d->n_planes, d->mode);
    return sweep_launch(d, ref, srcs, H, depths, depth, labels, best, cost, (unsigned long long *)scratch, chunks,
                        stream, nullptr);
}

}  // extern "C"
