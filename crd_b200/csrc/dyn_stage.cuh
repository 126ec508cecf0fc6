// Stages of a run-time radix schedule on one line held in shared memory (the classic padded layout, line_fft.cuh
// LayRow<1>): what a kernel runs when no compile-time schedule exists for its line length. Each radix is its own
// out-of-line function with scalar arguments only, so each gets its own register allocation; a single inlined body
// holding every radix's variants does not fit the register file and spills.

#pragma once

#include "codelets.cuh"

#include <cuda_runtime.h>

namespace crdfft
{
namespace lfft
{
namespace
{

// Shared-memory slot of element e of a line: one pad slot every 16 complex.
__device__ __forceinline__ int spad(int e) { return e + (e >> 4); }

// One Stockham stage (the line-FFT kernel's formula, line_fft.cuh) over a line of n points, 16 points a thread,
// T threads a line. j / L comes from a multiply-high by ceil(2^32 / L) (exact for j < 2^13 and L < 2^19).
// Every thread of the CTA calls it (it holds two barriers); `ok` false idles a thread.
template <int R>
__device__ __noinline__ void dstage(float2* sl, const float2* tw, int n, int L, unsigned magic, int jt, int T, bool ok)
{
    constexpr int B = (16 + R - 1) / R;
    const int nb = n / R;
    float2 v[B][R];
#pragma unroll
    for (int b = 0; b < B; ++b)
    {
        const int j = jt + b * T;
        if (ok && j < nb)
        {
#pragma unroll
            for (int r = 0; r < R; ++r)
                v[b][r] = sl[spad(j + r * nb)];
        }
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < B; ++b)
    {
        const int j = jt + b * T;
        if (ok && j < nb)
        {
            const int q = L == 1 ? j : static_cast<int>(__umulhi(static_cast<unsigned>(j), magic));
            const int k = j - q * L;
            if (L > 1)
            {
#pragma unroll
                for (int r = 1; r < R; ++r)
                    v[b][r] = cmul(v[b][r], __ldg(tw + (r - 1) * L + k));
            }
            Dft<R>::run(v[b]);
            const int base = q * L * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r)
                sl[spad(base + r * L)] = v[b][r];
        }
    }
    __syncthreads();
}

// All stages of a schedule (radix[0 .. nstages)), twiddles from the stage-ordered table tw.
__device__ __forceinline__ void dyn_stages(const int* radix, int nstages, const float2* tw, int n, float2* sl, int jt,
                                           int T, bool ok)
{
    int L = 1;
    for (int st = 0; st < nstages; ++st)
    {
        const int R = radix[st];
        const unsigned magic = L == 1 ? 0u : (0xFFFFFFFFu / static_cast<unsigned>(L)) + 1u;
        switch (R)
        {
            case 2: dstage<2>(sl, tw, n, L, magic, jt, T, ok); break;
            case 3: dstage<3>(sl, tw, n, L, magic, jt, T, ok); break;
            case 4: dstage<4>(sl, tw, n, L, magic, jt, T, ok); break;
            case 5: dstage<5>(sl, tw, n, L, magic, jt, T, ok); break;
            case 7: dstage<7>(sl, tw, n, L, magic, jt, T, ok); break;
            case 8: dstage<8>(sl, tw, n, L, magic, jt, T, ok); break;
            case 32: dstage<32>(sl, tw, n, L, magic, jt, T, ok); break;
            default: dstage<16>(sl, tw, n, L, magic, jt, T, ok); break;
        }
        if (L > 1)
            tw += (R - 1) * L;
        L *= R;
    }
}

} // namespace
} // namespace lfft
} // namespace crdfft
