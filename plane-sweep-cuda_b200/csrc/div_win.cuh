// Division of a window sum by the window side, for the reference-arithmetic
// sweep (sweep.cu) and its exhaustive check (tests/cuda/div_win_check.cu).
#pragma once

#include <math.h>

namespace mvs {

// x / WIN rounded to nearest, as the reference divides its window sums by the
// window side, in three instructions instead of a division: with
// y = RN(1 / WIN), q = RN(x y) is within one ulp of x / WIN, the residual
// x - q WIN is exact in one fused multiply-add, and RN(q + residual * y) is
// the correctly rounded quotient (Markstein's correction: P. W. Markstein,
// IBM J. Res. Dev. 34(1), 1990).  Zero, infinite and NaN x keep q, which is
// then exact (the correction would turn -0 into +0 and inf into NaN).
// tests/test_div_win_gpu.py compares it with the IEEE division for every
// float bit pattern and every window side 3..15: no difference.
template <int WIN>
__device__ __forceinline__ float div_win(float x)
{
    constexpr float d = (float)WIN, y = 1.f / (float)WIN;
    const float q = __fmul_rn(x, y);
    const float r = __fmaf_rn(-q, d, x);
    return isfinite(x) && x != 0.f ? __fmaf_rn(r, y, q) : q;
}

}  // namespace mvs
