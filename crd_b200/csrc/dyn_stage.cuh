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
            case 9: dstage<9>(sl, tw, n, L, magic, jt, T, ok); break;
            case 25: dstage<25>(sl, tw, n, L, magic, jt, T, ok); break;
            case 8: dstage<8>(sl, tw, n, L, magic, jt, T, ok); break;
            case 32: dstage<32>(sl, tw, n, L, magic, jt, T, ok); break;
            default: dstage<16>(sl, tw, n, L, magic, jt, T, ok); break;
        }
        if (L > 1)
            tw += (R - 1) * L;
        L *= R;
    }
}

// Visits (line a < lpc, element e < n) of a CTA's tile, each thread at most 16 of them (the CTA has at least
// lpc * ceil(n / 16) threads), K at a time: first `load` for K of a thread's elements into registers, then `put`
// for each, so K global loads of a thread are in flight at once (a loop that loads and stores one element at a
// time waits a full memory latency per element). Consecutive threads run along e (along_e) or along the lines.
template <int K, class Load, class Put>
__device__ __forceinline__ void tile_load(int n, int lpc, bool along_e, Load&& load, Put&& put)
{
    static_assert(16 % K == 0, "rounds of K cover the 16 elements a thread");
    const int tid = threadIdx.x;
    const int nt = blockDim.x;
    float2 v[K];
    if (along_e)
    {
        const int total = n * lpc;
        // idx / n by multiply-high with ceil(2^32 / n): exact for idx < 2^32 / n, and idx < 16 * 512 here
        const unsigned magic = n > 1 ? 0xFFFFFFFFu / static_cast<unsigned>(n) + 1u : 0u;
#pragma unroll 1
        for (int k0 = 0; k0 < 16; k0 += K)
        {
#pragma unroll
            for (int k = 0; k < K; ++k)
            {
                const int idx = tid + (k0 + k) * nt;
                if (idx < total)
                {
                    const int a = n > 1 ? static_cast<int>(__umulhi(static_cast<unsigned>(idx), magic)) : idx;
                    v[k] = load(a, idx - a * n);
                }
            }
#pragma unroll
            for (int k = 0; k < K; ++k)
            {
                const int idx = tid + (k0 + k) * nt;
                if (idx < total)
                {
                    const int a = n > 1 ? static_cast<int>(__umulhi(static_cast<unsigned>(idx), magic)) : idx;
                    put(a, idx - a * n, v[k]);
                }
            }
        }
    }
    else
    {
        const int a = tid % lpc;
        const int e0 = tid / lpc;
        const int step = nt / lpc;
#pragma unroll 1
        for (int k0 = 0; k0 < 16; k0 += K)
        {
#pragma unroll
            for (int k = 0; k < K; ++k)
            {
                const int e = e0 + (k0 + k) * step;
                if (e < n)
                    v[k] = load(a, e);
            }
#pragma unroll
            for (int k = 0; k < K; ++k)
            {
                const int e = e0 + (k0 + k) * step;
                if (e < n)
                    put(a, e, v[k]);
            }
        }
    }
}

// One stage out of place, src -> dst (two buffers of the same layout), one butterfly at a time: with no barrier
// inside, a thread holds only R values, and the out-of-line body fits its registers without spilling (the in-place
// form must hold all of a thread's butterflies across a barrier, and the call convention then saves the excess in
// local memory, which the many stages of a transform turn into DRAM traffic).
template <int R>
__device__ __forceinline__ void pstage_body(const float2* src, float2* dst, const float2* tw, int n, int L,
                                            unsigned magic, int jt, int T, bool ok)
{
    constexpr int B = (16 + R - 1) / R;
    const int nb = n / R;
#pragma unroll 1
    for (int b = 0; b < B; ++b)
    {
        const int j = jt + b * T;
        if (ok && j < nb)
        {
            float2 v[R];
#pragma unroll
            for (int r = 0; r < R; ++r)
                v[r] = src[spad(j + r * nb)];
            const int q = L == 1 ? j : static_cast<int>(__umulhi(static_cast<unsigned>(j), magic));
            const int k = j - q * L;
            if (L > 1)
            {
#pragma unroll
                for (int r = 1; r < R; ++r)
                    v[r] = cmul(v[r], __ldg(tw + (r - 1) * L + k));
            }
            Dft<R>::run(v);
            const int base = q * L * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r)
                dst[spad(base + r * L)] = v[r];
        }
    }
}

template <int R>
__device__ __noinline__ void pstage(const float2* src, float2* dst, const float2* tw, int n, int L, unsigned magic,
                                    int jt, int T, bool ok)
{
    pstage_body<R>(src, dst, tw, n, L, magic, jt, T, ok);
}

// One stage, out of line (its own register allocation) or, INL, inlined into a caller with registers to spare (a
// call site saves the caller's live registers in local memory at every call).
template <int R, bool INL>
__device__ __forceinline__ void pstage_at(const float2* src, float2* dst, const float2* tw, int n, int L,
                                          unsigned magic, int jt, int T, bool ok)
{
    if constexpr (INL)
        pstage_body<R>(src, dst, tw, n, L, magic, jt, T, ok);
    else
        pstage<R>(src, dst, tw, n, L, magic, jt, T, ok);
}

// All stages of a schedule, alternating between the line buffers a and b (a holds the input); returns the buffer
// with the result. Every thread of the CTA calls it (one barrier a stage).
// R25: the schedule may hold radix-25 stages (a caller whose schedules never do leaves their code out).
template <bool INL = false, bool R25 = true>
__device__ __forceinline__ float2* dyn_stages_pp(const int* radix, int nstages, const float2* tw, int n, float2* a,
                                                 float2* b, int jt, int T, bool ok)
{
    int L = 1;
    for (int st = 0; st < nstages; ++st)
    {
        const int R = radix[st];
        const unsigned magic = L == 1 ? 0u : (0xFFFFFFFFu / static_cast<unsigned>(L)) + 1u;
        switch (R)
        {
            case 2: pstage_at<2, INL>(a, b, tw, n, L, magic, jt, T, ok); break;
            case 3: pstage_at<3, INL>(a, b, tw, n, L, magic, jt, T, ok); break;
            case 4: pstage_at<4, INL>(a, b, tw, n, L, magic, jt, T, ok); break;
            case 5: pstage_at<5, INL>(a, b, tw, n, L, magic, jt, T, ok); break;
            case 7: pstage_at<7, INL>(a, b, tw, n, L, magic, jt, T, ok); break;
            case 9: pstage_at<9, INL>(a, b, tw, n, L, magic, jt, T, ok); break;
            case 25:
                if constexpr (R25)
                    pstage_at<25, INL>(a, b, tw, n, L, magic, jt, T, ok);
                break;
            case 8: pstage_at<8, INL>(a, b, tw, n, L, magic, jt, T, ok); break;
            case 32: pstage_at<32, INL>(a, b, tw, n, L, magic, jt, T, ok); break;
            default: pstage_at<16, INL>(a, b, tw, n, L, magic, jt, T, ok); break;
        }
        __syncthreads();
        float2* t = a;
        a = b;
        b = t;
        if (L > 1)
            tw += (R - 1) * L;
        L *= R;
    }
    return a;
}

} // namespace
} // namespace lfft
} // namespace crdfft
