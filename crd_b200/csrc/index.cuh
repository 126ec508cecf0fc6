#pragma once

// Integer quotients of line and element indices by run-time sizes. The kernels index with 64-bit integers, but a
// 64-bit division by a run-time value is a long software sequence: at the start of a CTA it delays the first loads
// by hundreds of cycles of dependent instructions (measured: the 4096-point line kernel ran 25 % slower with one in
// its prologue). The values nearly always fit 31 bits, where the 32-bit division is a short sequence, and a divisor
// of 1 (one line a group, no row divisor) needs none.

#include <cuda_runtime.h>

namespace crdfft
{

__device__ __forceinline__ long long idiv(long long a, long long b)
{
    if (b == 1)
        return a;
    if (((a | b) >> 31) == 0)
        return static_cast<long long>(static_cast<unsigned>(a) / static_cast<unsigned>(b));
    return a / b;
}

// a mod b for a >= 0, b >= 1
__device__ __forceinline__ long long imod(long long a, long long b) { return a - idiv(a, b) * b; }

} // namespace crdfft
