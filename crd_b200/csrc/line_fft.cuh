#pragma once

// The line-FFT pass kernels: a CTA transforms `lines_per_cta` lines of length n held in shared memory with the
// self-sorting (Stockham) decimation-in-time schedule, one register-resident radix-R butterfly per thread per
// iteration. They stand in for the reference's Stockham / standalone-hier / in-place-3 / deep-split engines
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
//
// Two kernels share the stage code:
//  * line_fft_kernel ("classic"): one CTA per group of lines; the first stage reads global memory itself when the
//    thread map makes that coalesced (direct_load), else the CTA stages the lines through shared memory; likewise the
//    last stage and the store.
//  * pipe_fft_kernel ("pipelined"): persistent CTAs; the CTA brings the next group of lines into the second of two
//    shared-memory buffers with bulk asynchronous copies (cp.async.bulk, completion on an mbarrier) while the CTA
//    transforms the current group, so HBM reads stay in flight through the compute. Every barrier wait is bounded.

#include "codelets.cuh"
#include "index.cuh"
#include "kernels.hpp"
#include "pass_desc.hpp"

#include <cuda_runtime.h>

#include <cstdint>
#include <initializer_list>
#include <type_traits>

namespace crdfft
{
namespace lfft
{

constexpr int kMaxLinesPerCta = 256;
constexpr int kMaxThreads = 512;
// The classic kernel's CTA size limit (both register budgets fit a 512-thread CTA).
__host__ __device__ constexpr int max_threads(int, int) { return kMaxThreads; }
// Register budgets of the classic kernel: each instance compiles twice (line_fft_kernel, line_fft_kernel_wide) and
// the launch takes the narrow build unless it spills, since a spill is a local-memory round trip inside the stages
// (measured: an 8-byte spill made the 4096-point kernel 35 % slower than the same code in 80 registers without one),
// while the extra registers cost resident warps (the 1024-point four-step row pass ran 3 % slower in 80, the 105-point
// lines 20 % slower under a plain 128-register cap than under the launch-bounds hint).
constexpr int kStaticThreads = 256; // the real-line and spectral kernels with a compile-time schedule
constexpr int kPipeThreads = 256;

// Classic layout: one pad slot every 16 complex (128 bytes) keeps the strided stage accesses spread over the banks.
__host__ __device__ constexpr int line_pitch(int n) { return (n + (n >> 4)) | 1; }
// The compile-time-schedule kernel's lines: with 2, 4 or 8 lines a CTA, line l starts 16 / lpc bank slots (8-byte
// slots, 16 to a 128-byte wavefront) after line l - 1 modulo 16, so that a warp reading the same elements of all its
// lines (the last stage of a transposed store, the coalesced loads across lines) touches 16 distinct slots in each
// half-warp: no bank conflict. Other line counts keep the odd pitch.
__host__ __device__ constexpr int cta_line_pitch(int n, int lpc)
{
    if (lpc != 2 && lpc != 4 && lpc != 8)
        return line_pitch(n);
    const int base = n + (n >> 4);
    const int want = 16 / lpc;
    return base + (((want - base) % 16) + 16) % 16;
}
// Pipelined row layout: two pad slots (16 bytes) every 16 complex, so each 128-byte chunk of a line lands on a
// 16-byte boundary for the bulk copy; the line pitch is 2 mod 4 slots to spread cross-line accesses.
__host__ __device__ constexpr int pipe_row_pitch(int n)
{
    return ((n + 2 * ((n + 15) >> 4)) & 3) == 0 ? n + 2 * ((n + 15) >> 4) + 2 : n + 2 * ((n + 15) >> 4);
}
// Pipelined column layout: element e of line ll at e * pitch + ll, pitch = lines + 2 (16-byte aligned rows).
__host__ __device__ constexpr int pipe_col_pitch(int lpc) { return lpc + 2; }

template <int PAD> struct LayRow
{
    float2* p;
    __device__ __forceinline__ float2& at(int e) const { return p[e + (e >> 4) * PAD]; }
};
struct LayCol
{
    float2* p;
    int pitch;
    __device__ __forceinline__ float2& at(int e) const { return p[e * pitch]; }
};

// Compile-time facts of a launch: the thread map (which fixes the unit-stride side of direct loads and stores) and
// whether any epilogue work exists (input conjugation, output conjugation or scale, four-step twiddle); a plain
// forward pass compiles all of it out.
template <PassMap M, bool E> struct Kind
{
    static constexpr PassMap map = M;
    static constexpr bool epi = E;
};

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
    long long q;       // line index within its group (four-step twiddle row)
    int jt;            // thread index within the line
    int T;             // threads per line
    bool ok;           // the line exists (the last CTA may be partial)
    float in_im;       // +1, or -1 to conjugate the input
    float out_re;      // output scale
    float out_im;      // output scale, negated to conjugate
};

template <bool EPI> __device__ __forceinline__ float2 load_in(const Ctx& c, const float2* p)
{
    float2 x = __ldcs(p);
    if constexpr (EPI)
        x.y *= c.in_im;
    return x;
}

// The four-step twiddle W_M^{q e} (line q < n2, element e < n1 = d.n) as W_M^{16 (q>>4) e} * W_M^{(q&15) e}: the
// first factor from hi[(q>>4) n1 + e], the same for the 16 lines of an aligned tile (a broadcast load), the second
// from lo[16 e + (q&15)], consecutive across those lines (a coalesced load).
__device__ __forceinline__ float2 four_step_twiddle(const PassDesc& d, long long q, int e)
{
    const int qi = static_cast<int>(q);
    const float2* th = static_cast<const float2*>(d.ftw_hi);
    const float2* tl = static_cast<const float2*>(d.ftw_lo);
    return cmul(__ldg(th + (qi >> 4) * d.n + e), __ldg(tl + e * 16 + (qi & 15)));
}

template <bool EPI>
__device__ __forceinline__ float2 epilogue(const PassDesc& d, const Ctx& c, long long q, int e, float2 v)
{
    if constexpr (EPI)
    {
        if (d.ftw_M != 0)
            v = cmul(v, four_step_twiddle(d, q, e));
        return make_float2(v.x * c.out_re, v.y * c.out_im);
    }
    else
        return v;
}

// APPLY_IN: this stage reads the pass input from shared memory and applies the input conjugation itself (the
// pipelined kernel's first stage; the classic kernel conjugates while loading). K is a Kind<map, epi>.
// Twiddles: the pass's stage-ordered table holds, for each stage after the first, W_{LR}^{r k} at
// tw_off + (r - 1) L + k (r = 1 .. R-1, k < L), so the threads of a warp (consecutive k, or equal k across lines)
// read consecutive or equal addresses: coalesced loads of exact, FP64-derived values (the reference's per-pass
// combine-twiddle table, include/crd/hesap/fft/fft.hpp:355-403).
template <int R, int P, bool FROM_GLOBAL, bool TO_GLOBAL, bool APPLY_IN, class K, class Lay>
__device__ __forceinline__ void stage(const PassDesc& d, const Ctx& c, const Lay& lay, int n, int L, int tw_off)
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
            if constexpr (FROM_GLOBAL)
            {
                // Row map: the input is unit-stride (a direct load is chosen only then); column map: runtime stride.
                const float2* src;
                long long step;
                if constexpr (K::map == PassMap::Row)
                {
                    src = c.in + j;
                    step = nb;
                }
                else
                {
                    src = c.in + static_cast<long long>(j) * d.in.estride;
                    step = static_cast<long long>(nb) * d.in.estride;
                }
#pragma unroll
                for (int r = 0; r < R; ++r)
                    v[b][r] = load_in<K::epi>(c, src + r * step);
            }
            else
            {
#pragma unroll
                for (int r = 0; r < R; ++r)
                {
                    const float2 x = lay.at(j + r * nb);
                    if constexpr (APPLY_IN && K::epi)
                        v[b][r] = make_float2(x.x, x.y * c.in_im);
                    else
                        v[b][r] = x;
                }
            }
        }
    }
    if constexpr (!FROM_GLOBAL && !TO_GLOBAL)
        __syncthreads(); // every thread has read the stage's input before any thread overwrites it in place
    const float2* tw = static_cast<const float2*>(d.tw) + tw_off;
#pragma unroll
    for (int b = 0; b < B; ++b)
    {
        const int j = c.jt + b * c.T;
        if (c.ok && j < nb)
        {
            const int k = j % L;
            if (L > 1)
            {
#pragma unroll
                for (int r = 1; r < R; ++r)
                    v[b][r] = cmul(v[b][r], __ldg(tw + (r - 1) * L + k));
            }
            Dft<R>::run(v[b]);
            const int base = (j - k) * R + k;
            if constexpr (TO_GLOBAL)
            {
                float2* dst;
                long long step;
                if constexpr (K::map == PassMap::Row)
                {
                    dst = c.out + base;
                    step = L;
                }
                else
                {
                    dst = c.out + static_cast<long long>(base) * d.out.estride;
                    step = static_cast<long long>(L) * d.out.estride;
                }
#pragma unroll
                for (int r = 0; r < R; ++r)
                    __stcs(dst + r * step, epilogue<K::epi>(d, c, c.q, base + r * L, v[b][r]));
            }
            else
            {
#pragma unroll
                for (int r = 0; r < R; ++r)
                    lay.at(base + r * L) = v[b][r];
            }
        }
    }
    if constexpr (!TO_GLOBAL)
        __syncthreads();
}

template <int P, bool DL, bool DS, bool PIPE, class K, int L, int OFF, int R, int... Rest, class Lay>
__device__ __forceinline__ void run_static(const PassDesc& d, const Ctx& c, const Lay& lay, int n)
{
    constexpr bool last = sizeof...(Rest) == 0;
    stage<R, P, (L == 1) && DL, last && DS, (L == 1) && PIPE, K>(d, c, lay, n, L, OFF);
    if constexpr (!last)
        run_static<P, DL, DS, PIPE, K, L * R, OFF + (L > 1 ? (R - 1) * L : 0), Rest...>(d, c, lay, n);
}

template <int R, int P, bool DL, bool DS, class K, class Lay>
__device__ __forceinline__ void stage_dyn(const PassDesc& d, const Ctx& c, const Lay& lay, int n, int L, int off,
                                          bool first, bool last)
{
    if constexpr (DL)
    {
        if (first)
        {
            if constexpr (DS)
            {
                if (last)
                {
                    stage<R, P, true, true, false, K>(d, c, lay, n, L, off);
                    return;
                }
            }
            stage<R, P, true, false, false, K>(d, c, lay, n, L, off);
            return;
        }
    }
    if constexpr (DS)
    {
        if (last)
        {
            stage<R, P, false, true, false, K>(d, c, lay, n, L, off);
            return;
        }
    }
    stage<R, P, false, false, false, K>(d, c, lay, n, L, off);
}

template <int P, bool DL, bool DS, class K, class Lay>
__device__ __forceinline__ void run_dynamic(const PassDesc& d, const Ctx& c, const Lay& lay, int n)
{
    int L = 1;
    int off = 0;
    for (int s = 0; s < d.nstages; ++s)
    {
        const int R = d.radix[s];
        const bool first = s == 0;
        const bool last = s == d.nstages - 1;
        switch (R)
        {
            case 2: stage_dyn<2, P, DL, DS, K>(d, c, lay, n, L, off, first, last); break;
            case 3: stage_dyn<3, P, DL, DS, K>(d, c, lay, n, L, off, first, last); break;
            case 4: stage_dyn<4, P, DL, DS, K>(d, c, lay, n, L, off, first, last); break;
            case 5: stage_dyn<5, P, DL, DS, K>(d, c, lay, n, L, off, first, last); break;
            case 7: stage_dyn<7, P, DL, DS, K>(d, c, lay, n, L, off, first, last); break;
            case 9: stage_dyn<9, P, DL, DS, K>(d, c, lay, n, L, off, first, last); break;
            case 25: stage_dyn<25, P, DL, DS, K>(d, c, lay, n, L, off, first, last); break;
            case 8: stage_dyn<8, P, DL, DS, K>(d, c, lay, n, L, off, first, last); break;
            case 32: stage_dyn<32, P, DL, DS, K>(d, c, lay, n, L, off, first, last); break;
            default: stage_dyn<16, P, DL, DS, K>(d, c, lay, n, L, off, first, last); break;
        }
        if (L > 1)
            off += (R - 1) * L;
        L *= R;
    }
}

template <class S> struct SchedRun
{
    template <int P, bool DL, bool DS, bool PIPE, class K, class Lay>
    __device__ __forceinline__ static void go(const PassDesc& d, const Ctx& c, const Lay& lay, int n)
    {
        run_s<P, DL, DS, PIPE, K>(d, c, lay, n, static_cast<S*>(nullptr));
    }
    template <int P, bool DL, bool DS, bool PIPE, class K, class Lay, int... Rs>
    __device__ __forceinline__ static void run_s(const PassDesc& d, const Ctx& c, const Lay& lay, int n, Sched<Rs...>*)
    {
        run_static<P, DL, DS, PIPE, K, 1, 0, Rs...>(d, c, lay, n);
    }
};
template <> struct SchedRun<DynSched>
{
    template <int P, bool DL, bool DS, bool PIPE, class K, class Lay>
    __device__ __forceinline__ static void go(const PassDesc& d, const Ctx& c, const Lay& lay, int n)
    {
        static_assert(!PIPE, "the pipelined kernel runs compile-time schedules only");
        run_dynamic<P, DL, DS, K>(d, c, lay, n);
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
    if (lpg == 1)
        return line * m.gdist;
    const long long g = idiv(line, lpg);
    const long long q = line - g * lpg;
    return g * m.gdist + q * m.ldist;
}

// The four-step twiddle row of a line: its index within its group divided by the pass's row divisor.
__device__ __forceinline__ long long line_row(const PassDesc& d, long long line)
{
    return idiv(imod(line, d.lines_per_group), d.ftw_div);
}

// Visits every (line a < lpc, element e < n) of the CTA's tile once across its threads, consecutive threads along
// e (along_e) or along the lines; blockDim is a multiple of lpc. No division inside the loop.
template <class F> __device__ __forceinline__ void for_tile(int n, int lpc, bool along_e, F&& f)
{
    const int tid = threadIdx.x;
    const int nt = blockDim.x;
    if (along_e)
    {
        int a = tid / n;
        int e = tid - a * n;
        const int da = nt / n;
        const int de = nt - da * n;
        while (a < lpc)
        {
            f(a, e);
            e += de;
            a += da;
            if (e >= n)
            {
                e -= n;
                ++a;
            }
        }
    }
    else
    {
        const int a = tid % lpc;
        const int step = nt / lpc;
        for (int e = tid / lpc; e < n; e += step)
            f(a, e);
    }
}

__device__ __forceinline__ void init_scales(const PassDesc& d, Ctx& c)
{
    c.in_im = d.conj_in ? -1.0f : 1.0f;
    c.out_re = d.scale;
    c.out_im = d.conj_out ? -d.scale : d.scale;
}

// ---- classic kernel ---------------------------------------------------------------------------------------------

// One tile of a pass inside a kernel that picks its tiles itself (chain_fft.cu): lines [blk * lpc, blk * lpc + lpc)
// of the `nlines` lines the maps address from gin / gout; `tid` is threadIdx.x. The CTA may be wider than the tile:
// threads from lpc * T on take part in the barriers only. The same steps as the classic kernel's body below, which
// keeps its own copy (its launch shape fixes the tile, and its register allocation stays as measured).
template <class S, int P, PassMap MAP, bool DL, bool DS, bool EPI>
__device__ __forceinline__ void line_fft_tile(const PassDesc& d, const float2* __restrict__ gin,
                                              float2* __restrict__ gout, long long blk, int lpc, long long nlines,
                                              int tid)
{
    extern __shared__ float2 sm[];
    __shared__ long long s_in_off[kMaxLinesPerCta];
    __shared__ long long s_out_off[kMaxLinesPerCta];
    __shared__ int s_q[kMaxLinesPerCta];

    const int n = sched_n<S>(d);
    const int T = (n + P - 1) / P;
    const int pitch = cta_line_pitch(n, lpc);
    const long long line0 = blk * lpc;

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
            s_q[i] = static_cast<int>(line_row(d, line));
        }
        __syncthreads();
    }

    const long long line = line0 + ll;
    Ctx c;
    c.ok = line < nlines && tid < lpc * T;
    c.q = line_row(d, line);
    c.in = gin + line_offset(d.in, line, d.lines_per_group);
    c.out = gout + line_offset(d.out, line, d.lines_per_group);
    c.jt = jt;
    c.T = T;
    init_scales(d, c);
    const LayRow<1> lay{sm + ll * pitch};

    if constexpr (!DL)
    {
        // Cooperative coalesced load of the CTA's lines: threads run along whichever axis is unit-stride in memory.
        const long long lines_here = nlines - line0;
        const long long es = d.in.estride;
        for_tile(n, lpc, es == 1, [&](int a, int e) {
            if (a < lines_here)
                LayRow<1>{sm + a * pitch}.at(e) = load_in<EPI>(c, gin + s_in_off[a] + static_cast<long long>(e) * es);
        });
        __syncthreads();
    }

    SchedRun<S>::template go<P, DL, DS, false, Kind<MAP, EPI>>(d, c, lay, n);

    if constexpr (!DS)
    {
        // (Storing the last stage straight from registers with the threads across the lines, which saves this
        // shared-memory round trip and its bank conflicts, measured 20 % slower on the four-step row pass.)
        const long long lines_here = nlines - line0;
        const long long es = d.out.estride;
        for_tile(n, lpc, es == 1, [&](int a, int e) {
            if (a < lines_here)
                __stcs(gout + s_out_off[a] + static_cast<long long>(e) * es,
                       epilogue<EPI>(d, c, s_q[a], e, LayRow<1>{sm + a * pitch}.at(e)));
        });
    }

    if constexpr (MAP == PassMap::Row && DL && !DS)
    {
        // A dead input (a four-step intermediate in L2, read by the first stage, which ends with a barrier: every
        // thread's loads of the CTA's lines are done): drop its 128-byte L2 lines, so that L2 does not write them
        // back to HBM. Unit-stride lines of whole 128-byte lines only; last, where the kernel holds the fewest values.
        if (d.discard_in && d.in.estride == 1 && (n & 15) == 0)
        {
            const int per = n / 16;
            const long long lines_here = nlines - line0;
            for (int i = tid; i < lpc * per; i += blockDim.x)
            {
                const int a = i / per;
                const float2* p = gin + s_in_off[a] + (i - a * per) * 16;
                if (a < lines_here && (reinterpret_cast<uintptr_t>(p) & 127) == 0)
                    asm volatile("discard.global.L2 [%0], 128;" ::"l"(p) : "memory");
            }
        }
    }
}

template <class S, int P, PassMap MAP, bool DL, bool DS, bool EPI>
__device__ __forceinline__ void line_fft_body(const PassDesc& d, const float2* __restrict__ gin,
                                              float2* __restrict__ gout)
{
    extern __shared__ float2 sm[];
    __shared__ long long s_in_off[kMaxLinesPerCta];
    __shared__ long long s_out_off[kMaxLinesPerCta];
    __shared__ int s_q[kMaxLinesPerCta];

    const int n = sched_n<S>(d);
    const int T = (n + P - 1) / P;
    const int lpc = blockDim.x / T;
    const int tid = threadIdx.x;
    const int pitch = cta_line_pitch(n, lpc);
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
            s_q[i] = static_cast<int>(line_row(d, line));
        }
        __syncthreads();
    }

    const long long line = line0 + ll;
    Ctx c;
    c.ok = line < d.lines;
    c.q = line_row(d, line);
    c.in = gin + line_offset(d.in, line, d.lines_per_group);
    c.out = gout + line_offset(d.out, line, d.lines_per_group);
    c.jt = jt;
    c.T = T;
    init_scales(d, c);
    const LayRow<1> lay{sm + ll * pitch};

    if constexpr (!DL)
    {
        // Cooperative coalesced load of the CTA's lines: threads run along whichever axis is unit-stride in memory.
        const long long lines_here = d.lines - line0;
        const long long es = d.in.estride;
        for_tile(n, lpc, es == 1, [&](int a, int e) {
            if (a < lines_here)
                LayRow<1>{sm + a * pitch}.at(e) = load_in<EPI>(c, gin + s_in_off[a] + static_cast<long long>(e) * es);
        });
        __syncthreads();
    }

    SchedRun<S>::template go<P, DL, DS, false, Kind<MAP, EPI>>(d, c, lay, n);

    if constexpr (!DS)
    {
        // (Storing the last stage straight from registers with the threads across the lines, which saves this
        // shared-memory round trip and its bank conflicts, measured 20 % slower on the four-step row pass.)
        const long long lines_here = d.lines - line0;
        const long long es = d.out.estride;
        for_tile(n, lpc, es == 1, [&](int a, int e) {
            if (a < lines_here)
                __stcs(gout + s_out_off[a] + static_cast<long long>(e) * es,
                       epilogue<EPI>(d, c, s_q[a], e, LayRow<1>{sm + a * pitch}.at(e)));
        });
    }

    if constexpr (MAP == PassMap::Row && DL && !DS)
    {
        // A dead input (a four-step intermediate in L2, read by the first stage, which ends with a barrier: every
        // thread's loads of the CTA's lines are done): drop its 128-byte L2 lines, so that L2 does not write them
        // back to HBM. Unit-stride lines of whole 128-byte lines only; last, where the kernel holds the fewest values.
        if (d.discard_in && d.in.estride == 1 && (n & 15) == 0)
        {
            const int per = n / 16;
            const long long lines_here = d.lines - line0;
            for (int i = tid; i < lpc * per; i += blockDim.x)
            {
                const int a = i / per;
                const float2* p = gin + s_in_off[a] + (i - a * per) * 16;
                if (a < lines_here && (reinterpret_cast<uintptr_t>(p) & 127) == 0)
                    asm volatile("discard.global.L2 [%0], 128;" ::"l"(p) : "memory");
            }
        }
    }
}

// The two register budgets of the classic kernel. The narrow build keeps the launch-bounds hint (two 512-thread CTAs
// an SM at 16 points a thread on lines of 256 points or more, 64 registers; the compiler's own choice within 128
// otherwise); the wide build caps the registers directly at 80 (16 points a thread; 32 points a thread keep 128,
// what a 512-thread CTA allows) and is what launches when the narrow build spills.
template <class S, int P, PassMap MAP, bool DL, bool DS, bool EPI>
__global__ void __launch_bounds__(kMaxThreads, (P <= 16 && S::n >= 256) ? 2 : 0)
    line_fft_kernel(const PassDesc d, const float2* __restrict__ gin, float2* __restrict__ gout)
{
    line_fft_body<S, P, MAP, DL, DS, EPI>(d, gin, gout);
}

template <class S, int P, PassMap MAP, bool DL, bool DS, bool EPI>
__global__ void __maxnreg__(P <= 16 ? 80 : 128)
    line_fft_kernel_wide(const PassDesc d, const float2* __restrict__ gin, float2* __restrict__ gout)
{
    line_fft_body<S, P, MAP, DL, DS, EPI>(d, gin, gout);
}

// ---- pipelined kernel -------------------------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_addr(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

// Bulk asynchronous copy global -> this CTA's shared memory; `bytes` a multiple of 16, both addresses 16-byte aligned.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Bounded wait on a phase of an mbarrier; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int limit)
{
    for (int i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity))
            return true;
    return false;
}

// Bytes of group `grp` (the last group may hold fewer lines).
template <int N, PassMap MAP>
__device__ __forceinline__ uint32_t pipe_group_bytes(const PassDesc& d, long long grp, int lpc)
{
    const long long left = d.lines - grp * lpc;
    const int nl = left < lpc ? static_cast<int>(left) : lpc;
    return static_cast<uint32_t>(nl) * N * 8u;
}

// 32-bit line offset (lines < 2^31, offsets < 2^31 elements per group stride product kept in 64 bits).
__device__ __forceinline__ long long line_offset32(const LineMap& m, int line, int lpg)
{
    const int g = lpg == 1 ? line : line / lpg;
    const int q = line - g * lpg;
    return static_cast<long long>(g) * m.gdist + static_cast<long long>(q) * m.ldist;
}

// All threads of the CTA issue the copies of group `grp` into `buf` (the barrier is armed separately).
template <int N, PassMap MAP>
__device__ __forceinline__ void pipe_issue(const PassDesc& d, const float2* gin, long long grp, int lpc, float2* buf,
                                           uint64_t* bar, int tid, int nthreads)
{
    const long long line0 = grp * lpc;
    if constexpr (MAP == PassMap::Row)
    {
        constexpr int chunks = (N + 15) / 16;
        const long long left = d.lines - line0;
        const int nl = left < lpc ? static_cast<int>(left) : lpc;
        constexpr int pitch = pipe_row_pitch(N);
        const int lpg = static_cast<int>(d.lines_per_group);
        for (int i = tid; i < nl * chunks; i += nthreads)
        {
            const int ll = i / chunks;
            const int ch = i - ll * chunks;
            const int cnt = (N - ch * 16) < 16 ? (N - ch * 16) : 16;
            const float2* src = gin + line_offset32(d.in, static_cast<int>(line0) + ll, lpg) + ch * 16;
            bulk_load(buf + ll * pitch + ch * 18, src, static_cast<uint32_t>(cnt) * 8u, bar);
        }
    }
    else
    {
        // lpc adjacent lines of one group: row e is lpc consecutive complex values
        const int pitch = pipe_col_pitch(lpc);
        const float2* base = gin + line_offset32(d.in, static_cast<int>(line0), static_cast<int>(d.lines_per_group));
        for (int e = tid; e < N; e += nthreads)
            bulk_load(buf + e * pitch, base + static_cast<long long>(e) * d.in.estride,
                      static_cast<uint32_t>(lpc) * 8u, bar);
    }
}

// REGS: 80 (three 256-thread CTAs an SM) or 128 (two); the launch takes the 80-register build unless it spills.
template <class S, int P, PassMap MAP, bool DS, bool EPI, int REGS>
__global__ void __maxnreg__(REGS) pipe_fft_kernel(const PassDesc d, const float2* __restrict__ gin,
                                                  float2* __restrict__ gout, int lpc, long long ngroups)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ long long s_out_off[kMaxLinesPerCta];
    __shared__ int s_q[kMaxLinesPerCta];
    constexpr int N = S::n;
    constexpr int T = (N + P - 1) / P;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);
    float2* buf0 = reinterpret_cast<float2*>(smem_raw + 128);
    const int buf_elems = MAP == PassMap::Row ? lpc * pipe_row_pitch(N) : N * pipe_col_pitch(lpc);
    const int tid = threadIdx.x;

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

    if (tid == 0)
    {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init(&bars[2], 1); // never armed: the test hook's wait on it can only run out
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    long long grp = blockIdx.x;
    if (grp < ngroups)
    {
        // An arming arrive and the copies it counts may land in either order: the phase cannot complete before the
        // arrive, and the transaction count may run below zero until it.
        if (tid == 0)
            mbar_expect_tx(&bars[0], pipe_group_bytes<N, MAP>(d, grp, lpc));
        pipe_issue<N, MAP>(d, gin, grp, lpc, buf0, &bars[0], tid, blockDim.x);
    }

    Ctx c;
    c.jt = jt;
    c.T = T;
    init_scales(d, c);

    for (int it = 0; grp < ngroups; grp += gridDim.x, ++it)
    {
        const int b = it & 1;
        const long long next = grp + gridDim.x;
        const bool issued_next = next < ngroups;
        if (issued_next)
        {
            if (tid == 0)
                mbar_expect_tx(&bars[b ^ 1], pipe_group_bytes<N, MAP>(d, next, lpc));
            pipe_issue<N, MAP>(d, gin, next, lpc, buf0 + (b ^ 1) * buf_elems, &bars[b ^ 1], tid, blockDim.x);
        }
        const bool stalled = d.debug_stall != 0 && it == 0;
        if (!mbar_wait_bounded(stalled ? &bars[2] : &bars[b], static_cast<uint32_t>((it >> 1) & 1), d.spin_limit))
        {
            // Give up on this group: record the error, let every copy this CTA issued land (bounded again), and
            // leave without touching shared memory further.
            if (tid == 0 && d.err != nullptr)
                atomicOr(d.err, 1);
            if (stalled)
                mbar_wait_bounded(&bars[b], static_cast<uint32_t>((it >> 1) & 1), d.spin_limit);
            if (issued_next)
                mbar_wait_bounded(&bars[b ^ 1], static_cast<uint32_t>(((it + 1) >> 1) & 1), d.spin_limit);
            return;
        }
        float2* buf = buf0 + b * buf_elems;
        if constexpr (!DS)
        {
            // per-line output offsets for the store below (visible after the stages' barriers)
            for (int i = tid; i < lpc; i += blockDim.x)
            {
                const long long ln = grp * lpc + i;
                s_out_off[i] = line_offset(d.out, ln, d.lines_per_group);
                s_q[i] = static_cast<int>(line_row(d, ln));
            }
        }
        const long long line = grp * lpc + ll;
        c.ok = line < d.lines;
        c.q = line_row(d, line);
        c.in = gin;
        c.out = gout + line_offset(d.out, line, d.lines_per_group);
        if constexpr (MAP == PassMap::Row)
        {
            const LayRow<2> lay{buf + ll * pipe_row_pitch(N)};
            SchedRun<S>::template go<P, false, DS, true, Kind<MAP, EPI>>(d, c, lay, N);
        }
        else
        {
            const LayCol lay{buf + ll, pipe_col_pitch(lpc)};
            SchedRun<S>::template go<P, false, DS, true, Kind<MAP, EPI>>(d, c, lay, N);
        }
        if constexpr (!DS)
        {
            // Store through shared memory: threads run along whichever axis is unit-stride in the output.
            const long long lines_here = d.lines - grp * lpc;
            const long long es = d.out.estride;
            for_tile(N, lpc, es == 1, [&](int a, int e) {
                if (a < lines_here)
                {
                    float2 v;
                    if constexpr (MAP == PassMap::Row)
                        v = LayRow<2>{buf + a * pipe_row_pitch(N)}.at(e);
                    else
                        v = buf[e * pipe_col_pitch(lpc) + a];
                    __stcs(gout + s_out_off[a] + static_cast<long long>(e) * es, epilogue<EPI>(d, c, s_q[a], e, v));
                }
            });
        }
        fence_proxy_async(); // this CTA's generic accesses to buf are ordered before the next bulk copy into it
        __syncthreads();
    }
}

using KernelFn = void (*)(const PassDesc, const float2*, float2*);
using PipeFn = void (*)(const PassDesc, const float2*, float2*, int, long long);

// The build of one classic instance that launches: the narrow register budget unless its build spills (local
// memory per thread above zero), decided once per instance.
KernelFn spill_free(KernelFn narrow, KernelFn wide);

// wide: the shape asks for the 80-register build; otherwise the narrow build, unless it spills.
template <class S, int P, PassMap MAP, bool DL, bool DS, bool EPI> KernelFn pick_regs(bool wide)
{
    if constexpr (P > 16) // 32 points a thread: 128 registers in both builds
        return line_fft_kernel<S, P, MAP, DL, DS, EPI>;
    else
    {
        if (wide)
            return line_fft_kernel_wide<S, P, MAP, DL, DS, EPI>;
        static const KernelFn k =
            spill_free(line_fft_kernel<S, P, MAP, DL, DS, EPI>, line_fft_kernel_wide<S, P, MAP, DL, DS, EPI>);
        return k;
    }
}

template <class S, int P, bool EPI> KernelFn pick_e(PassMap map, bool dl, bool ds, bool wide)
{
    if (map == PassMap::Row)
    {
        if (dl && ds) return pick_regs<S, P, PassMap::Row, true, true, EPI>(wide);
        if (dl) return pick_regs<S, P, PassMap::Row, true, false, EPI>(wide);
        if (ds) return pick_regs<S, P, PassMap::Row, false, true, EPI>(wide);
        return pick_regs<S, P, PassMap::Row, false, false, EPI>(wide);
    }
    if (dl && ds) return pick_regs<S, P, PassMap::Col, true, true, EPI>(wide);
    if (dl) return pick_regs<S, P, PassMap::Col, true, false, EPI>(wide);
    if (ds) return pick_regs<S, P, PassMap::Col, false, true, EPI>(wide);
    return pick_regs<S, P, PassMap::Col, false, false, EPI>(wide);
}

template <class S, int P> KernelFn pick(PassMap map, bool dl, bool ds, bool epi, bool wide)
{
    return epi ? pick_e<S, P, true>(map, dl, ds, wide) : pick_e<S, P, false>(map, dl, ds, wide);
}

PipeFn spill_free_pipe(PipeFn narrow, PipeFn wide);

template <class S, int P, PassMap MAP, bool DS, bool EPI> PipeFn pick_pipe_regs()
{
    static const PipeFn k = spill_free_pipe(pipe_fft_kernel<S, P, MAP, DS, EPI, 80>,
                                            pipe_fft_kernel<S, P, MAP, DS, EPI, 128>);
    return k;
}

template <class S, int P, bool EPI> PipeFn pick_pipe_e(PassMap map, bool ds)
{
    if (map == PassMap::Row)
        return ds ? pick_pipe_regs<S, P, PassMap::Row, true, EPI>() : pick_pipe_regs<S, P, PassMap::Row, false, EPI>();
    return ds ? pick_pipe_regs<S, P, PassMap::Col, true, EPI>() : pick_pipe_regs<S, P, PassMap::Col, false, EPI>();
}

template <class S, int P> PipeFn pick_pipe(PassMap map, bool ds, bool epi)
{
    return epi ? pick_pipe_e<S, P, true>(map, ds) : pick_pipe_e<S, P, false>(map, ds);
}

// Whether a pass has any epilogue work (the EPI instances).
inline bool pass_epi(const PassDesc& d)
{
    return d.conj_in != 0 || d.conj_out != 0 || d.scale != 1.0f || d.ftw_M != 0;
}

inline bool same_radices(const PassDesc& d, std::initializer_list<int> rs)
{
    if (static_cast<int>(rs.size()) != d.nstages)
        return false;
    int i = 0;
    for (int r : rs)
        if (d.radix[i++] != r)
            return false;
    return true;
}

// One translation unit per compile-time schedule defines its selectors with these (parallel compilation).
#define CRDFFT_DEFINE_SCHEDULE(NAME, P_, ...)                                                                         \
    KernelFn NAME##_classic(const PassDesc& d, const PassShape& sh)                                                   \
    {                                                                                                                  \
        if (sh.points_per_thread == P_ && same_radices(d, {__VA_ARGS__}))                                              \
            return pick<Sched<__VA_ARGS__>, P_>(sh.map, sh.direct_load, sh.direct_store, pass_epi(d), sh.wide_regs);    \
        return nullptr;                                                                                                \
    }
#define CRDFFT_DEFINE_PIPE(NAME, P_, ...)                                                                             \
    PipeFn NAME##_pipe(const PassDesc& d, const PassShape& sh)                                                        \
    {                                                                                                                  \
        if (sh.points_per_thread == P_ && same_radices(d, {__VA_ARGS__}))                                              \
            return pick_pipe<Sched<__VA_ARGS__>, P_>(sh.map, sh.direct_store, pass_epi(d));                           \
        return nullptr;                                                                                                \
    }

// Instances live in line_fft_static.cu (compile-time schedules, classic and pipelined) and line_fft_dyn.cu
// (schedule read from the descriptor); each returns nullptr when it has no kernel for the pass.
KernelFn select_static(const PassDesc& d, const PassShape& sh);
PipeFn select_pipe(const PassDesc& d, const PassShape& sh);
KernelFn select_dynamic(const PassDesc& d, const PassShape& sh);

} // namespace lfft
} // namespace crdfft
