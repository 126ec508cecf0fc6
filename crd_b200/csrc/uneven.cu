// Uneven batch: thousands of independent complex transforms of different 7-smooth lengths, each at its own offset
// in a packed buffer, in one persistent launch. The reference runs such a batch as a loop of per-size plans over
// crd-jobs ranges (include/crd/hesap/fft/detail/batch_arms.hpp:59-77, one plan per job); here one kernel walks a
// device work list:
//
//   SMALL  up to `lines` transforms of one length n <= 4096, one CTA, all stages in shared memory
//   COL    a tile of adjacent columns of one long transform (n = n1 n2 > 4096): length-n1 DFTs, four-step twiddle,
//          written to the transform's region of the workspace
//   ROW    a tile of rows of that transform's workspace region: length-n2 DFTs, transposed store to the output
//
// CTAs (as many as fit on the GPU at once, G of them) take items in list order, CTA c the items c, c + G, ...; each
// keeps two item slots in shared memory and issues the next item's loads before it transforms the current one. The
// list holds every COL item before any ROW item, so the COL items a ROW item waits for belong to CTAs that reach them
// without waiting on anything: the ROW item's wait on its transform's completion counter always ends. It is bounded
// anyway (spin_limit polls): a wait that runs out sets the plan's status word and skips the item.
//
// Each item runs its length's compile-time stages in place where the kernel has them (powers of two) and the planner
// chose them, else the stages of the length's run-time radix schedule out of place (dyn_stage.cuh).

#include "kernels.hpp"
#include "line_fft.cuh"
#include "uneven.hpp"
#include "dyn_stage.cuh"

namespace crdfft
{
namespace lfft
{
namespace
{

constexpr int kUnevenThreads = 256;

// Issues the loads of an item's lines into shared memory (row layout, one pad slot per 16), coalesced along
// whichever side of the global layout is unit-stride; line a starts at base[a]. Asynchronous 8-byte copies
// (cp.async) committed as one group: every copy of a thread is in flight at once without holding registers, and the
// CTA transforms the previous item while they land. The caller waits for the group (cp.async.wait_all) and
// synchronises; an inverse's conjugation is applied after that (uneven_conj).
__device__ __forceinline__ void uneven_issue(int n, int lines, long long estride, const long long* base,
                                             const float2* src, float2* sm, int pitch)
{
    for_tile(n, lines, estride == 1, [&](int a, int e) {
        const float2* p = src + base[a] + static_cast<long long>(e) * estride;
        float2* d = &LayRow<1>{sm + a * pitch}.at(e);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(d)), "l"(p) : "memory");
    });
    asm volatile("cp.async.commit_group;" ::: "memory");
}

__device__ __forceinline__ void uneven_conj(int n, int lines, float2* sm, int pitch)
{
    for_tile(n, lines, true, [&](int a, int e) {
        float2& x = LayRow<1>{sm + a * pitch}.at(e);
        x.y = -x.y;
    });
}

__device__ __forceinline__ void uneven_store(int n, int lines, long long estride, const long long* base, int q0,
                                             const float2* fh, const float2* fl, float2* dst, const float2* sm,
                                             int pitch, float out_re, float out_im)
{
    for_tile(n, lines, estride == 1, [&](int a, int e) {
        float2 v = LayRow<1>{const_cast<float2*>(sm) + a * pitch}.at(e);
        if (fh != nullptr)
        {
            const int q = q0 + a; // column index of the long transform
            v = cmul(v, cmul(__ldg(fh + (q >> 4) * n + e), __ldg(fl + e * 16 + (q & 15))));
        }
        __stcs(dst + base[a] + static_cast<long long>(e) * estride, make_float2(v.x * out_re, v.y * out_im));
    });
}

// A line length's compile-time schedule on the item's tile, in place: the Stockham stages of the line-FFT kernel
// (line_fft.cuh) with the radix, the stage's L and the line length known at compile time, 16 points a thread, the
// padded row layout (spad), one barrier between a stage's reads and its writes. Only the twiddle table, the line and
// the thread's place are run-time values, so the index arithmetic folds away. Out of line, so that its registers do
// not add to the persistent kernel's.
template <int R, int L, int N>
__device__ __forceinline__ void ustage(const float2* __restrict__ tw, float2* line, int jt, int T, bool ok)
{
    constexpr int nb = N / R;
    constexpr int B = (16 + R - 1) / R;
    float2 v[B][R];
#pragma unroll
    for (int b = 0; b < B; ++b)
    {
        const int j = jt + b * T;
        if (ok && j < nb)
        {
#pragma unroll
            for (int r = 0; r < R; ++r)
                v[b][r] = line[spad(j + r * nb)];
        }
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < B; ++b)
    {
        const int j = jt + b * T;
        if (ok && j < nb)
        {
            const int k = j % L;
            if constexpr (L > 1)
            {
#pragma unroll
                for (int r = 1; r < R; ++r)
                    v[b][r] = cmul(v[b][r], __ldg(tw + (r - 1) * L + k));
            }
            Dft<R>::run(v[b]);
            const int base = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r)
                line[spad(base + r * L)] = v[b][r];
        }
    }
    __syncthreads();
}

template <int N, int L, int OFF, int R, int... Rest>
__device__ __forceinline__ void ustages(const float2* tw, float2* line, int jt, int T, bool ok)
{
    ustage<R, L, N>(tw + OFF, line, jt, T, ok);
    if constexpr (sizeof...(Rest) > 0)
        ustages<N, L * R, OFF + (L > 1 ? (R - 1) * L : 0), Rest...>(tw, line, jt, T, ok);
}

template <int... Rs>
__device__ __noinline__ void static_item(const float2* tw, float2* line, int jt, int T, bool ok)
{
    ustages<(Rs * ... * 1), 1, 0, Rs...>(tw, line, jt, T, ok);
}

// The compile-time schedules by log2 n (16 .. 4096; the radix order of the planner's rule), reached through one
// indirect call site: a call site saves the caller's live registers, and one site keeps that to one save area.
using StaticFn = void (*)(const float2*, float2*, int, int, bool);
__device__ StaticFn const kStaticItems[13] = {nullptr,
                                              nullptr,
                                              nullptr,
                                              nullptr,
                                              static_item<16>,
                                              static_item<8, 4>,
                                              static_item<16, 4>,
                                              static_item<16, 8>,
                                              static_item<16, 16>,
                                              static_item<16, 8, 4>,
                                              static_item<16, 16, 4>,
                                              static_item<16, 16, 8>,
                                              static_item<16, 16, 16>};

// The persistent loop, software-pipelined over two item slots: CTA c takes items c, c + G, c + 2G, ... (G CTAs, all
// resident). While it transforms item i from one slot, the loads of item i + G land in the other. A ROW item is
// prefetched only once its transform's COL items are all done (checked without waiting); otherwise its loads are
// issued after the current item, behind a bounded wait. Every COL item precedes every ROW item in the list, and a CTA
// takes its items in list order, so the COL items a ROW item waits for are never behind a wait themselves.
struct SlotState
{
    int idx;  // item index, or -1
    int go;   // its dependencies were met and its loads issued
};

__global__ void __launch_bounds__(kUnevenThreads, 2)
    uneven_kernel(const UnevenDesc u, const float2* __restrict__ gin, float2* __restrict__ gout, float2* scratch)
{
    extern __shared__ float2 sm[];
    __shared__ UnevenItem s_it[2];
    __shared__ long long s_in[kMaxLinesPerCta];
    __shared__ long long s_out[2][kMaxLinesPerCta];
    __shared__ int s_flag;
    const int tid = threadIdx.x;
    const float in_im = u.conj ? -1.0f : 1.0f;
    const float out_im = u.conj ? -u.scale : u.scale;
    const int G = gridDim.x;
    float2* const tmp = sm + 2 * u.slot_elems; // the run-time stages' second buffer

    // Reads item idx into slot `slot` and issues its loads. wait: for a ROW item, wait (bounded) for its COL items;
    // else only check them, and return 0 without issuing when they are not all done. Every thread calls it.
    auto prepare = [&](int idx, int slot, bool wait) -> int {
        if (tid == 0)
        {
            s_it[slot] = u.items[idx];
            const UnevenItem& it = s_it[slot];
            int go = 1;
            if (it.kind == kUnevenRow)
            {
                const volatile int* done = u.done + it.transform;
                if (!wait)
                    go = *done >= it.need ? 1 : 0;
                else
                {
                    int i = 0;
                    while (*done < it.need)
                    {
                        if (++i > u.spin_limit)
                        {
                            go = -1; // gave up: the item is skipped
                            atomicOr(u.err, 1);
                            break;
                        }
                        __nanosleep(64);
                    }
                }
                __threadfence(); // acquire: the COL items' workspace writes are visible from here on
            }
            s_flag = go;
        }
        __syncthreads();
        const int go = s_flag;
        if (go != 1)
            return go;
        const UnevenItem& it = s_it[slot];
        for (int a = tid; a < it.lines; a += blockDim.x)
        {
            s_in[a] = it.line_table >= 0 ? u.line_off[it.line_table + a] : it.in_base + a * it.in_ldist;
            s_out[slot][a] = it.line_table >= 0 ? u.line_off[it.line_table + a] : it.out_base + a * it.out_ldist;
        }
        __syncthreads();
        const int n = u.scheds[it.sched].n;
        uneven_issue(n, it.lines, it.in_estride, s_in, it.kind == kUnevenRow ? scratch : gin, sm + slot * u.slot_elems,
                     line_pitch(n));
        return 1;
    };

    SlotState cur{static_cast<int>(blockIdx.x), 0};
    if (cur.idx >= u.nitems)
        return;
    cur.go = prepare(cur.idx, 0, true);
    for (int i = 0; cur.idx < u.nitems; ++i)
    {
        const int slot = i & 1;
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncthreads(); // this item's lines are in its slot; the other slot is free
        SlotState nxt{cur.idx + G, 0};
        if (nxt.idx < u.nitems)
            nxt.go = prepare(nxt.idx, slot ^ 1, false); // 0: a ROW item not ready yet, prepared after this one
        if (cur.go == 1)
        {
            const UnevenItem& it = s_it[slot];
            const UnevenSched& s = u.scheds[it.sched];
            float2* const buf = sm + slot * u.slot_elems;
            float2* dst = it.kind == kUnevenCol ? scratch : gout;
            const int n = s.n;
            const int pitch = line_pitch(n);
            // inverse: conjugate on the way into the first pass of each transform and out of the last
            const bool first_pass = it.kind != kUnevenRow;
            const bool last_pass = it.kind != kUnevenCol;
            if (first_pass && in_im < 0.0f)
            {
                uneven_conj(n, it.lines, buf, pitch); // each thread the elements it copied
                __syncthreads();
            }
            const int T = (n + 15) / 16;
            const int ll = tid / T;
            const bool ok = ll < it.lines;
            const int lrow = ok ? ll : 0;
            const float2* tile;
            if (s.variant == 1) // a power of two 16 .. 4096 (the planner sets the variant only then)
            {
                kStaticItems[31 - __clz(n)](static_cast<const float2*>(s.tw), buf + lrow * pitch, tid - ll * T, T,
                                            ok);
                tile = buf; // in place
            }
            else
            {
                const float2* res = dyn_stages_pp<true, false>(s.radix, s.nstages, static_cast<const float2*>(s.tw), s.n,
                                                  buf + lrow * pitch, tmp + lrow * pitch, tid - ll * T, T, ok);
                tile = res - lrow * pitch;
            }
            const float2* fh = it.ftw >= 0 ? static_cast<const float2*>(u.tables.ftw_hi[it.ftw]) : nullptr;
            const float2* fl = it.ftw >= 0 ? static_cast<const float2*>(u.tables.ftw_lo[it.ftw]) : nullptr;
            uneven_store(n, it.lines, it.out_estride, s_out[slot], it.q0, fh, fl, dst, tile, pitch,
                         last_pass ? u.scale : 1.0f, last_pass ? out_im : 1.0f);
            if (it.kind == kUnevenCol)
            {
                __threadfence(); // release: this item's workspace writes before its completion count
                __syncthreads();
                if (tid == 0)
                    atomicAdd(u.done + it.transform, 1);
            }
        }
        __syncthreads(); // this slot and the stage buffer are free again
        if (nxt.idx < u.nitems && nxt.go == 0)
            nxt.go = prepare(nxt.idx, slot ^ 1, true);
        cur = nxt;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
}

} // namespace
} // namespace lfft

int uneven_threads() { return lfft::kUnevenThreads; }

bool uneven_static_ok(int n) { return n >= 16 && n <= 4096 && (n & (n - 1)) == 0; }

cudaError_t launch_uneven(const UnevenDesc& u, int smem_bytes, const void* in, void* out, void* scratch,
                          cudaStream_t stream)
{
    auto fn = lfft::uneven_kernel;
    if (smem_bytes > 48 * 1024)
    {
        const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
        if (e != cudaSuccess)
            return e;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, lfft::kUnevenThreads, smem_bytes) != cudaSuccess ||
        per_sm < 1)
        return cudaErrorInvalidConfiguration;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // Every CTA of the grid is resident at once (a CTA waiting on a dependency never blocks one that would end it).
    long long grid = static_cast<long long>(sms) * per_sm;
    if (grid > u.nitems)
        grid = u.nitems;
    if (grid < 1)
        return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(u.counter, 0, sizeof(int) * (1 + u.ntransforms), stream);
    if (e != cudaSuccess)
        return e;
    fn<<<static_cast<unsigned>(grid), lfft::kUnevenThreads, smem_bytes, stream>>>(
        u, static_cast<const float2*>(in), static_cast<float2*>(out), static_cast<float2*>(scratch));
    return cudaGetLastError();
}

} // namespace crdfft
