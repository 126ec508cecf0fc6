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
// CTAs (as many as fit on the GPU at once) take items in list order from an atomic counter. The list holds every
// COL item before any ROW item, so a ROW item's transform has all of its COL items already taken by running CTAs,
// which finish without waiting on anything: the ROW item's wait on the transform's completion counter always ends.
// It is bounded anyway (spin_limit polls): a wait that runs out sets the plan's status word and skips the item.
//
// Each item runs the stages of its length's run-time radix schedule out of place (dyn_stage.cuh).

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

// Loads an item's lines into shared memory (row layout, one pad slot per 16), coalesced along whichever side of the
// global layout is unit-stride; line a starts at base[a]. Asynchronous 8-byte copies (cp.async): every copy of a
// thread is in flight at once without holding registers (a batch of loads in registers spilled in this 80-register
// kernel). The caller waits for them and synchronises; an inverse's conjugation is applied after that
// (uneven_conj).
__device__ __forceinline__ void uneven_load(int n, int lines, long long estride, const long long* base,
                                            const float2* src, float2* sm, int pitch)
{
    for_tile(n, lines, estride == 1, [&](int a, int e) {
        const float2* p = src + base[a] + static_cast<long long>(e) * estride;
        float2* d = &LayRow<1>{sm + a * pitch}.at(e);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(d)), "l"(p) : "memory");
    });
    asm volatile("cp.async.wait_all;" ::: "memory");
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

__global__ void __launch_bounds__(kUnevenThreads, 3)
    uneven_kernel(const UnevenDesc u, const float2* __restrict__ gin, float2* __restrict__ gout, float2* scratch)
{
    extern __shared__ float2 sm[];
    __shared__ int s_item;
    __shared__ int s_go;
    __shared__ long long s_in[kMaxLinesPerCta];
    __shared__ long long s_out[kMaxLinesPerCta];
    const int tid = threadIdx.x;
    const float in_im = u.conj ? -1.0f : 1.0f;
    const float out_im = u.conj ? -u.scale : u.scale;
    for (;;)
    {
        if (tid == 0)
            s_item = atomicAdd(u.counter, 1);
        __syncthreads();
        const int idx = s_item;
        if (idx >= u.nitems)
            break;
        const UnevenItem it = u.items[idx];
        const UnevenSched s = u.scheds[it.sched];
        if (it.kind == kUnevenRow)
        {
            if (tid == 0)
            {
                int go = 1;
                const volatile int* done = u.done + it.transform;
                int i = 0;
                while (*done < it.need)
                {
                    if (++i > u.spin_limit)
                    {
                        go = 0;
                        atomicOr(u.err, 1);
                        break;
                    }
                    __nanosleep(64);
                }
                __threadfence(); // acquire: the COL items' workspace writes are visible from here on
                s_go = go;
            }
            __syncthreads();
            if (!s_go)
                continue;
        }
        const float2* src = it.kind == kUnevenRow ? scratch : gin;
        float2* dst = it.kind == kUnevenCol ? scratch : gout;
        const int n = s.n;
        const int pitch = line_pitch(n);
        // per-line start offsets, once per item
        for (int a = tid; a < it.lines; a += blockDim.x)
        {
            s_in[a] = it.line_table >= 0 ? u.line_off[it.line_table + a] : it.in_base + a * it.in_ldist;
            s_out[a] = it.line_table >= 0 ? u.line_off[it.line_table + a] : it.out_base + a * it.out_ldist;
        }
        __syncthreads();
        // inverse: conjugate on the way into the first pass of each transform and out of the last
        const bool first_pass = it.kind != kUnevenRow;
        const bool last_pass = it.kind != kUnevenCol;
        uneven_load(n, it.lines, it.in_estride, s_in, src, sm, pitch);
        __syncthreads();
        if (first_pass && in_im < 0.0f)
        {
            uneven_conj(n, it.lines, sm, pitch); // each thread the elements it copied
            __syncthreads();
        }
        const int T = (n + 15) / 16;
        const int ll = tid / T;
        const bool ok = ll < it.lines;
        // out of place between two buffers of the item's lines (the second right after the first)
        const int lrow = ok ? ll : 0;
        const float2* tile;
        if (s.variant == 1) // a power of two 16 .. 4096 (the planner sets the variant only then)
        {
            kStaticItems[31 - __clz(n)](static_cast<const float2*>(s.tw), sm + lrow * pitch, tid - ll * T, T, ok);
            tile = sm; // in place
        }
        else
        {
            const float2* res = dyn_stages_pp(s.radix, s.nstages, static_cast<const float2*>(s.tw), s.n,
                                              sm + lrow * pitch, sm + (it.lines + lrow) * pitch, tid - ll * T, T, ok);
            tile = res - lrow * pitch;
        }
        const float2* fh = it.ftw >= 0 ? static_cast<const float2*>(u.tables.ftw_hi[it.ftw]) : nullptr;
        const float2* fl = it.ftw >= 0 ? static_cast<const float2*>(u.tables.ftw_lo[it.ftw]) : nullptr;
        uneven_store(n, it.lines, it.out_estride, s_out, it.q0, fh, fl, dst, tile, pitch,
                     last_pass ? u.scale : 1.0f, last_pass ? out_im : 1.0f);
        if (it.kind == kUnevenCol)
        {
            __threadfence(); // release: this item's workspace writes before its completion count
            __syncthreads();
            if (tid == 0)
                atomicAdd(u.done + it.transform, 1);
        }
        __syncthreads(); // shared memory and s_item are reused by the next item
    }
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
