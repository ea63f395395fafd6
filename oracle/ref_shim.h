/* Host shim that lets the reference's CUDA kernel sources run on the CPU.
 *
 * Test infrastructure only: this header is force-included when the oracle
 * recipe compiles the reference's own kernels.cu, TGV2_kernels.cu and
 * fusion.cu with g++ (after the recipe rewrites each `k<<<g, b>>>(args)`
 * launch into `shim_launch(g, b, k, args)`).  Every reference kernel is one
 * thread per output element with no shared memory and no barriers
 * (kernels.cu:4-429, TGV2_kernels.cu:31-445, fusion.cu:5-70), so running the
 * (block, thread) grid as plain loops, blocks spread over OpenMP threads,
 * computes exactly what each CUDA thread computes.
 */
#ifndef MVS_REF_SHIM_H
#define MVS_REF_SHIM_H

#include <cuda_runtime.h>
#include <device_launch_parameters.h>
#include <iostream>
#include <stdexcept>
#include <string>

/* The reference's exception.h overrides std::exception::what() without
 * noexcept, which current g++ rejects; it is not on the compute path, so the
 * recipe defines its guard and this shim supplies the one macro the memory
 * helpers need. */
#define EXCEPTION_H
#define THROW_EXCEP(msg) throw std::runtime_error(std::string("reference shim: ") + (msg))

struct shim_dim { unsigned x, y, z; };
extern thread_local uint3 shim_threadIdx;
extern thread_local uint3 shim_blockIdx;
extern dim3 shim_blockDim;
extern dim3 shim_gridDim;

#define threadIdx shim_threadIdx
#define blockIdx shim_blockIdx
#define blockDim shim_blockDim
#define gridDim shim_gridDim

template <typename Kernel, typename... Args>
static void shim_launch(dim3 grid, dim3 block, Kernel kernel, Args... args)
{
    shim_gridDim = grid;
    shim_blockDim = block;
    const long nb = (long)grid.x * grid.y * grid.z;
#pragma omp parallel for schedule(dynamic, 4)
    for (long b = 0; b < nb; ++b) {
        shim_blockIdx.x = (unsigned)(b % grid.x);
        shim_blockIdx.y = (unsigned)((b / grid.x) % grid.y);
        shim_blockIdx.z = (unsigned)(b / ((long)grid.x * grid.y));
        for (unsigned tz = 0; tz < block.z; ++tz)
            for (unsigned ty = 0; ty < block.y; ++ty)
                for (unsigned tx = 0; tx < block.x; ++tx) {
                    shim_threadIdx.x = tx;
                    shim_threadIdx.y = ty;
                    shim_threadIdx.z = tz;
                    kernel(args...);
                }
    }
}

#endif
