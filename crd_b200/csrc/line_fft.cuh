#pragma once

// The line-FFT pass kernel: a CTA transforms `lines_per_cta` lines of length n held in shared memory with the
// self-sorting (Stockham) decimation-in-time schedule, one register-resident radix-R butterfly per thread per
// iteration. It stands in for the reference's Stockham / standalone-hier / in-place-3 / deep-split engines
// (engine/numerics/hesap-fft/kernels/fft_kernels.cpp:266-353, 520-585, 1603-1676, 359-515): where the reference runs
// log_R(n) passes over a cache-resident buffer, a pass here reads each element from HBM once and writes it once, and
// the intermediate stages exchange through shared memory.
//
// Stage s with radix R, after stages whose radices multiply to L:
//   for each butterfly j in [0, n/R):  k = j mod L
//     v_r = x[j + r n/R] * W_{LR}^{r k}   (r = 0 .. R-1)
//     v   = DFT_R(v)
//     y[(j - k) R + k + r L] = v_r
// so the first stage reads x[j + r n/R] and the last writes y[j + r n/R]: both coalesced when threads run along j.
// Those two stages go straight to and from global memory (direct_load / direct_store) when the thread map makes the
// access coalesced; otherwise the CTA stages the lines through shared memory cooperatively.

#include "codelets.cuh"
#include "kernels.hpp"
#include <initializer_list>
#include <type_traits>
#include "pass_desc.hpp"

#include <cuda_runtime.h>

namespace crdfft
{
namespace lfft
{

constexpr int kMaxLinesPerCta = 256;
constexpr int kMaxThreads = 512;

// Shared-memory slot of element e within a line: one pad slot every 16 complex (128 bytes) keeps the strided stage
// accesses (stride R or L between threads) spread over the banks.
__device__ __forceinline__ int spad(int e) { return e + (e >> 4); }
__host__ __device__ constexpr int line_pitch(int n) { return (n + (n >> 4)) | 1; }

template <int... Rs> struct Sched
{
    static constexpr int n = (Rs * ... * 1);
};
struct DynSched
{
};

struct Ctx
{
    const float2* in;  // this thread's line in global memory (element 0)
    float2* out;
    float2* sl;        // this thread's line in shared memory
    long long q;       // line index within its group (four-step twiddle row)
    int jt;            // thread index within the line
    int T;             // threads per line
    bool ok;           // the line exists (the last CTA may be partial)
};

__device__ __forceinline__ float2 load_in(const PassDesc& d, const float2* p)
{
    float2 x = __ldcs(p);
    if (d.conj_in)
        x.y = -x.y;
    return x;
}

// W_M^{(q e) mod M} = hi[m / base] * lo[m % base], the four-step twiddle.
__device__ __forceinline__ float2 four_step_twiddle(const PassDesc& d, long long q, int e)
{
    const long long m = (q * static_cast<long long>(e)) % d.ftw_M;
    const int hi = static_cast<int>(m / d.ftw_base);
    const int lo = static_cast<int>(m - static_cast<long long>(hi) * d.ftw_base);
    const float2* th = static_cast<const float2*>(d.ftw_hi);
    const float2* tl = static_cast<const float2*>(d.ftw_lo);
    return cmul(__ldg(th + hi), __ldg(tl + lo));
}

__device__ __forceinline__ float2 epilogue(const PassDesc& d, long long q, int e, float2 v)
{
    if (d.ftw_M != 0)
        v = cmul(v, four_step_twiddle(d, q, e));
    if (d.conj_out)
        v.y = -v.y;
    if (d.scale != 1.0f)
        v = cscale(v, d.scale);
    return v;
}

template <int R, int P, bool FROM_GLOBAL, bool TO_GLOBAL>
__device__ __forceinline__ void stage(const PassDesc& d, const Ctx& c, int n, int L)
{
    constexpr int B = (P + R - 1) / R;
    const int nb = n / R;
    float2 v[B][R];
#pragma unroll
    for (int b = 0; b < B; ++b)
    {
        const int j = c.jt + b * c.T;
        if (c.ok && j < nb)
        {
#pragma unroll
            for (int r = 0; r < R; ++r)
            {
                const int e = j + r * nb;
                if constexpr (FROM_GLOBAL)
                    v[b][r] = load_in(d, c.in + static_cast<long long>(e) * d.in.estride);
                else
                    v[b][r] = c.sl[spad(e)];
            }
        }
    }
    if constexpr (!FROM_GLOBAL && !TO_GLOBAL)
        __syncthreads(); // every thread has read the stage's input before any thread overwrites it in place
    const float2* tw = static_cast<const float2*>(d.tw);
#pragma unroll
    for (int b = 0; b < B; ++b)
    {
        const int j = c.jt + b * c.T;
        if (c.ok && j < nb)
        {
            const int k = j % L;
            if (L > 1)
            {
                const int m = n / (L * R);
#pragma unroll
                for (int r = 1; r < R; ++r)
                    v[b][r] = cmul(v[b][r], __ldg(tw + r * k * m));
            }
            Dft<R>::run(v[b]);
            const int base = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r)
            {
                const int e = base + r * L;
                if constexpr (TO_GLOBAL)
                    __stcs(c.out + static_cast<long long>(e) * d.out.estride, epilogue(d, c.q, e, v[b][r]));
                else
                    c.sl[spad(e)] = v[b][r];
            }
        }
    }
    if constexpr (!TO_GLOBAL)
        __syncthreads();
}

template <int P, bool DL, bool DS, int L, int R, int... Rest>
__device__ __forceinline__ void run_static(const PassDesc& d, const Ctx& c, int n)
{
    constexpr bool last = sizeof...(Rest) == 0;
    stage<R, P, (L == 1) && DL, last && DS>(d, c, n, L);
    if constexpr (!last)
        run_static<P, DL, DS, L * R, Rest...>(d, c, n);
}

template <int R, int P, bool DL, bool DS>
__device__ __forceinline__ void stage_dyn(const PassDesc& d, const Ctx& c, int n, int L, bool first, bool last)
{
    if constexpr (DL)
    {
        if (first)
        {
            if constexpr (DS)
            {
                if (last)
                {
                    stage<R, P, true, true>(d, c, n, L);
                    return;
                }
            }
            stage<R, P, true, false>(d, c, n, L);
            return;
        }
    }
    if constexpr (DS)
    {
        if (last)
        {
            stage<R, P, false, true>(d, c, n, L);
            return;
        }
    }
    stage<R, P, false, false>(d, c, n, L);
}

template <int P, bool DL, bool DS>
__device__ __forceinline__ void run_dynamic(const PassDesc& d, const Ctx& c, int n)
{
    int L = 1;
    for (int s = 0; s < d.nstages; ++s)
    {
        const int R = d.radix[s];
        const bool first = s == 0;
        const bool last = s == d.nstages - 1;
        switch (R)
        {
            case 2: stage_dyn<2, P, DL, DS>(d, c, n, L, first, last); break;
            case 3: stage_dyn<3, P, DL, DS>(d, c, n, L, first, last); break;
            case 4: stage_dyn<4, P, DL, DS>(d, c, n, L, first, last); break;
            case 5: stage_dyn<5, P, DL, DS>(d, c, n, L, first, last); break;
            case 7: stage_dyn<7, P, DL, DS>(d, c, n, L, first, last); break;
            case 8: stage_dyn<8, P, DL, DS>(d, c, n, L, first, last); break;
            default: stage_dyn<16, P, DL, DS>(d, c, n, L, first, last); break;
        }
        L *= R;
    }
}

template <class S> struct SchedRun
{
    template <int P, bool DL, bool DS> __device__ __forceinline__ static void go(const PassDesc& d, const Ctx& c, int n)
    {
        run_dyn_or_static<P, DL, DS>(d, c, n, static_cast<S*>(nullptr));
    }
    template <int P, bool DL, bool DS, int... Rs>
    __device__ __forceinline__ static void run_dyn_or_static(const PassDesc& d, const Ctx& c, int n, Sched<Rs...>*)
    {
        run_static<P, DL, DS, 1, Rs...>(d, c, n);
    }
};
template <> struct SchedRun<DynSched>
{
    template <int P, bool DL, bool DS> __device__ __forceinline__ static void go(const PassDesc& d, const Ctx& c, int n)
    {
        run_dynamic<P, DL, DS>(d, c, n);
    }
};

template <class S> __device__ __forceinline__ int sched_n(const PassDesc& d)
{
    if constexpr (std::is_same_v<S, DynSched>)
        return d.n;
    else
        return S::n;
}

// Global offset of line `line` under a line map.
__device__ __forceinline__ long long line_offset(const LineMap& m, long long line, long long lpg)
{
    const long long g = line / lpg;
    const long long q = line - g * lpg;
    return g * m.gdist + q * m.ldist;
}

template <class S, int P, PassMap MAP, bool DL, bool DS>
__global__ void __launch_bounds__(kMaxThreads) line_fft_kernel(const PassDesc d, const float2* __restrict__ gin,
                                                        float2* __restrict__ gout)
{
    extern __shared__ float2 sm[];
    __shared__ long long s_in_off[kMaxLinesPerCta];
    __shared__ long long s_out_off[kMaxLinesPerCta];

    const int n = sched_n<S>(d);
    const int T = (n + P - 1) / P;
    const int lpc = blockDim.x / T;
    const int tid = threadIdx.x;
    const int pitch = line_pitch(n);
    const long long line0 = static_cast<long long>(blockIdx.x) * lpc;

    int ll, jt;
    if constexpr (MAP == PassMap::Row)
    {
        ll = tid / T;
        jt = tid - ll * T;
    }
    else
    {
        jt = tid / lpc;
        ll = tid - jt * lpc;
    }

    if (!DL || !DS)
    {
        for (int i = tid; i < lpc; i += blockDim.x)
        {
            const long long line = line0 + i;
            s_in_off[i] = line_offset(d.in, line, d.lines_per_group);
            s_out_off[i] = line_offset(d.out, line, d.lines_per_group);
        }
        __syncthreads();
    }

    const long long line = line0 + ll;
    Ctx c;
    c.ok = line < d.lines;
    c.q = line % d.lines_per_group;
    c.in = gin + line_offset(d.in, line, d.lines_per_group);
    c.out = gout + line_offset(d.out, line, d.lines_per_group);
    c.sl = sm + ll * pitch;
    c.jt = jt;
    c.T = T;

    if constexpr (!DL)
    {
        // Cooperative coalesced load of the CTA's lines: threads run along whichever axis is unit-stride in memory.
        const int total = lpc * n;
        const bool along_e = d.in.estride == 1;
        for (int i = tid; i < total; i += blockDim.x)
        {
            int a, e;
            if (along_e)
            {
                a = i / n;
                e = i - a * n;
            }
            else
            {
                e = i / lpc;
                a = i - e * lpc;
            }
            if (line0 + a < d.lines)
                sm[a * pitch + spad(e)] = load_in(d, gin + s_in_off[a] + static_cast<long long>(e) * d.in.estride);
        }
        __syncthreads();
    }

    SchedRun<S>::template go<P, DL, DS>(d, c, n);

    if constexpr (!DS)
    {
        const int total = lpc * n;
        const bool along_e = d.out.estride == 1;
        for (int i = tid; i < total; i += blockDim.x)
        {
            int a, e;
            if (along_e)
            {
                a = i / n;
                e = i - a * n;
            }
            else
            {
                e = i / lpc;
                a = i - e * lpc;
            }
            const long long ln = line0 + a;
            if (ln < d.lines)
            {
                const long long q = ln % d.lines_per_group;
                __stcs(gout + s_out_off[a] + static_cast<long long>(e) * d.out.estride,
                       epilogue(d, q, e, sm[a * pitch + spad(e)]));
            }
        }
    }
}

using KernelFn = void (*)(const PassDesc, const float2*, float2*);

template <class S, int P> KernelFn pick(PassMap map, bool dl, bool ds)
{
    if (map == PassMap::Row)
    {
        if (dl && ds) return line_fft_kernel<S, P, PassMap::Row, true, true>;
        if (dl) return line_fft_kernel<S, P, PassMap::Row, true, false>;
        if (ds) return line_fft_kernel<S, P, PassMap::Row, false, true>;
        return line_fft_kernel<S, P, PassMap::Row, false, false>;
    }
    if (dl && ds) return line_fft_kernel<S, P, PassMap::Col, true, true>;
    if (dl) return line_fft_kernel<S, P, PassMap::Col, true, false>;
    if (ds) return line_fft_kernel<S, P, PassMap::Col, false, true>;
    return line_fft_kernel<S, P, PassMap::Col, false, false>;
}

// Instances live in line_fft_static.cu (compile-time schedules) and line_fft_dyn.cu (schedule read from the
// descriptor); each returns nullptr when it has no kernel for the pass.
KernelFn select_static(const PassDesc& d, const PassShape& sh);
KernelFn select_dynamic(const PassDesc& d, const PassShape& sh);

} // namespace lfft
} // namespace crdfft
