// Uneven batch: thousands of independent complex transforms of different 7-smooth lengths, each at its own offset
// in a packed buffer, in one persistent launch. The reference runs such a batch as a loop of per-size plans over
// crd-jobs ranges (include/crd/hesap/fft/detail/batch_arms.hpp:59-77, one plan per job); here one kernel walks a
// device work list:
//
//   SMALL  up to `lines` transforms of one length n <= 8192, one CTA, all stages in shared memory
//   COL    a tile of adjacent columns of one long transform (n = n1 n2 > 8192): length-n1 DFTs, four-step twiddle,
//          written to the transform's region of the workspace
//   ROW    a tile of rows of that transform's workspace region: length-n2 DFTs, transposed store to the output
//
// CTAs (as many as fit on the GPU at once) take items in list order from an atomic counter. The list holds every
// COL item before any ROW item, so a ROW item's transform has all of its COL items already taken by running CTAs,
// which finish without waiting on anything: the ROW item's wait on the transform's completion counter always ends.
// It is bounded anyway (spin_limit polls): a wait that runs out sets the plan's status word and skips the item.
//
// Each item's stages are the line-FFT kernel's run-time radix schedule (line_fft.cuh).

#include "kernels.hpp"
#include "line_fft.cuh"
#include "uneven.hpp"

namespace crdfft
{
namespace lfft
{
namespace
{

constexpr int kUnevenThreads = 512;

// Loads an item's lines into shared memory (row layout, one pad slot per 16), coalesced along whichever side of the
// global layout is unit-stride.
__device__ __forceinline__ void uneven_load(const UnevenItem& it, const UnevenSched& s, const float2* src,
                                            const long long* line_off, float2* sm, int pitch, float in_im, bool l2_only)
{
    const int n = s.n;
    const bool along_e = it.in_estride == 1;
    for_tile(n, it.lines, along_e, [&](int a, int e) {
        const long long base = it.line_table >= 0 ? line_off[it.line_table + a] : it.in_base + a * it.in_ldist;
        const float2* p = src + base + static_cast<long long>(e) * it.in_estride;
        float2 x = l2_only ? __ldcg(p) : __ldcs(p);
        x.y *= in_im;
        LayRow<1>{sm + a * pitch}.at(e) = x;
    });
}

__device__ __forceinline__ void uneven_store(const UnevenItem& it, const UnevenSched& s, const UnevenTables& tb,
                                             float2* dst, const long long* line_off, const float2* sm, int pitch,
                                             float out_re, float out_im)
{
    const int n = s.n;
    const bool along_e = it.out_estride == 1;
    const float2* fh = it.ftw >= 0 ? static_cast<const float2*>(tb.ftw_hi[it.ftw]) : nullptr;
    const float2* fl = it.ftw >= 0 ? static_cast<const float2*>(tb.ftw_lo[it.ftw]) : nullptr;
    for_tile(n, it.lines, along_e, [&](int a, int e) {
        const long long base = it.line_table >= 0 ? line_off[it.line_table + a] : it.out_base + a * it.out_ldist;
        float2 v = LayRow<1>{const_cast<float2*>(sm) + a * pitch}.at(e);
        if (fh != nullptr)
        {
            const int q = it.q0 + a; // column index of the long transform
            v = cmul(v, cmul(__ldg(fh + (q >> 4) * n + e), __ldg(fl + e * 16 + (q & 15))));
        }
        __stcs(dst + base + static_cast<long long>(e) * it.out_estride, make_float2(v.x * out_re, v.y * out_im));
    });
}

__global__ void __launch_bounds__(kUnevenThreads, 1)
    uneven_kernel(const UnevenDesc u, const float2* __restrict__ gin, float2* __restrict__ gout, float2* scratch)
{
    extern __shared__ float2 sm[];
    __shared__ int s_item;
    __shared__ int s_go;
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
        const UnevenSched& s = u.scheds[it.sched];
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
        const int pitch = line_pitch(s.n);
        // inverse: conjugate on the way into the first pass of each transform and out of the last
        const bool first_pass = it.kind != kUnevenRow;
        const bool last_pass = it.kind != kUnevenCol;
        uneven_load(it, s, src, u.line_off, sm, pitch, first_pass ? in_im : 1.0f, it.kind == kUnevenRow);
        __syncthreads();
        const int T = (s.n + 15) / 16;
        const int ll = tid / T;
        Ctx c;
        c.jt = tid - ll * T;
        c.T = T;
        c.ok = ll < it.lines;
        c.q = 0;
        c.in = nullptr;
        c.out = nullptr;
        c.in_im = 1.0f;
        c.out_re = 1.0f;
        c.out_im = 1.0f;
        PassDesc d{};
        d.n = s.n;
        d.nstages = s.nstages;
        for (int i = 0; i < kMaxStages; ++i)
            d.radix[i] = s.radix[i];
        d.tw = s.tw;
        const LayRow<1> lay{sm + (ll < it.lines ? ll : 0) * pitch};
        run_dynamic<16, false, false, Kind<PassMap::Row, false>>(d, c, lay, s.n);
        uneven_store(it, s, u.tables, dst, u.line_off, sm, pitch, last_pass ? u.scale : 1.0f,
                     last_pass ? out_im : 1.0f);
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
