// Exhaustive check of mvs::div_win<WIN> (the reference-arithmetic sweep's
// division of a window sum by the window side) against the IEEE division
// x / WIN, for every float bit pattern (both signs, zeros, subnormals,
// infinities; NaN results only have to be NaN on both sides) and every
// window side 3..15.  Prints one line per window side and exits 1 on any
// difference.
#include <cstdio>
#include <cstdint>

#include "../../plane-sweep-cuda_b200/csrc/div_win.cuh"

template <int WIN>
__global__ void check(unsigned long long *bad, unsigned int *first)
{
    // u runs over the 2^31 magnitudes; both signs per u
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < (1ull << 31);
         u += (uint64_t)gridDim.x * blockDim.x) {
        for (int s = 0; s < 2; ++s) {
            const float x = __uint_as_float((uint32_t)u | (s ? 0x80000000u : 0u));
            const float a = mvs::div_win<WIN>(x), b = __fdiv_rn(x, (float)WIN);
            const bool both_nan = a != a && b != b;
            if (!both_nan && __float_as_uint(a) != __float_as_uint(b)) {
                atomicAdd(bad, 1ull);
                atomicMin(first, (uint32_t)u);
            }
        }
    }
}

template <int WIN>
unsigned long long run(unsigned long long *bad, unsigned int *first)
{
    cudaMemset(bad, 0, sizeof(*bad));
    cudaMemset(first, 0xff, sizeof(*first));
    check<WIN><<<148 * 16, 256>>>(bad, first);
    unsigned long long hb = ~0ull;
    unsigned int hf = 0;
    cudaMemcpy(&hb, bad, sizeof(hb), cudaMemcpyDeviceToHost);
    cudaMemcpy(&hf, first, sizeof(hf), cudaMemcpyDeviceToHost);
    const cudaError_t e = cudaGetLastError();
    printf("window %2d: %llu differences (first magnitude bits 0x%08x) %s\n", WIN, hb, hf, cudaGetErrorString(e));
    return e == cudaSuccess ? hb : ~0ull;
}

int main()
{
    unsigned long long *bad = nullptr;
    unsigned int *first = nullptr;
    if (cudaMalloc(&bad, sizeof(*bad)) != cudaSuccess || cudaMalloc(&first, sizeof(*first)) != cudaSuccess) return 2;
    unsigned long long total = run<3>(bad, first);
    total += run<5>(bad, first);
    total += run<7>(bad, first);
    total += run<9>(bad, first);
    total += run<11>(bad, first);
    total += run<13>(bad, first);
    total += run<15>(bad, first);
    cudaFree(bad);
    cudaFree(first);
    return total == 0 ? 0 : 1;
}
