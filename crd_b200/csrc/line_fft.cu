// Launchers of the line-FFT pass kernels (line_fft.cuh): the pipelined persistent kernel where the planner chose it,
// else the compile-time schedule when one exists for the pass, else the run-time schedule.

#include "kernels.hpp"
#include "line_fft.cuh"

#include <mutex>
#include <unordered_map>

namespace crdfft
{
namespace lfft
{
// The compile-time schedules (one translation unit each, sched_*.cu).
KernelFn s_1024_classic(const PassDesc&, const PassShape&);
KernelFn s_1024w_classic(const PassDesc&, const PassShape&);
KernelFn s_1024x_classic(const PassDesc&, const PassShape&);
KernelFn s_8192x_classic(const PassDesc&, const PassShape&);
KernelFn s_16_classic(const PassDesc&, const PassShape&);
KernelFn s_32_classic(const PassDesc&, const PassShape&);
KernelFn s_64_classic(const PassDesc&, const PassShape&);
KernelFn s_128_classic(const PassDesc&, const PassShape&);
KernelFn s_2048_classic(const PassDesc&, const PassShape&);
KernelFn s_8192_classic(const PassDesc&, const PassShape&);
KernelFn s_8192w_classic(const PassDesc&, const PassShape&);
KernelFn s_256_classic(const PassDesc&, const PassShape&);
KernelFn s_512_classic(const PassDesc&, const PassShape&);
KernelFn s_4096_classic(const PassDesc&, const PassShape&);
KernelFn s_4096c_classic(const PassDesc&, const PassShape&);
KernelFn s_16384_classic(const PassDesc&, const PassShape&);
KernelFn s_105_classic(const PassDesc&, const PassShape&);
PipeFn s_1024_pipe(const PassDesc&, const PassShape&);
PipeFn s_256_pipe(const PassDesc&, const PassShape&);
PipeFn s_512_pipe(const PassDesc&, const PassShape&);
PipeFn s_4096_pipe(const PassDesc&, const PassShape&);
PipeFn s_105_pipe(const PassDesc&, const PassShape&);

KernelFn spill_free(KernelFn narrow, KernelFn wide)
{
    cudaFuncAttributes a{};
    if (cudaFuncGetAttributes(&a, reinterpret_cast<const void*>(narrow)) != cudaSuccess)
    {
        cudaGetLastError();
        return narrow;
    }
    return a.localSizeBytes > 0 ? wide : narrow;
}

PipeFn spill_free_pipe(PipeFn narrow, PipeFn wide)
{
    cudaFuncAttributes a{};
    if (cudaFuncGetAttributes(&a, reinterpret_cast<const void*>(narrow)) != cudaSuccess)
    {
        cudaGetLastError();
        return narrow;
    }
    return a.localSizeBytes > 0 ? wide : narrow;
}

KernelFn select_static(const PassDesc& d, const PassShape& sh)
{
    for (auto f : {s_1024_classic, s_1024w_classic, s_256_classic, s_512_classic, s_4096_classic, s_4096c_classic,
                   s_16384_classic, s_105_classic, s_16_classic, s_32_classic, s_64_classic, s_128_classic,
                   s_2048_classic, s_8192_classic, s_8192w_classic, s_1024x_classic, s_8192x_classic})
        if (KernelFn k = f(d, sh))
            return k;
    return nullptr;
}

PipeFn select_pipe(const PassDesc& d, const PassShape& sh)
{
    for (auto f : {s_1024_pipe, s_256_pipe, s_512_pipe, s_4096_pipe, s_105_pipe})
        if (PipeFn k = f(d, sh))
            return k;
    return nullptr;
}
} // namespace lfft

bool pass_has_static(const PassDesc& d, int points_per_thread)
{
    PassShape sh{};
    sh.points_per_thread = points_per_thread;
    return lfft::select_static(d, sh) != nullptr;
}

int pass_lines_per_cta_limit() { return lfft::kMaxLinesPerCta; }
int pass_threads_limit(int points_per_thread, long long n)
{
    return lfft::max_threads(points_per_thread, static_cast<int>(n));
}
int pass_pipe_threads() { return lfft::kPipeThreads; }
int pass_line_pitch(int n) { return lfft::line_pitch(n); }
int pass_cta_line_pitch(int n, int lpc) { return lfft::cta_line_pitch(n, lpc); }

int pass_pipe_smem(int n, PassMap map, int lpc)
{
    const int elems = map == PassMap::Row ? lpc * lfft::pipe_row_pitch(n) : n * lfft::pipe_col_pitch(lpc);
    return 128 + 2 * elems * 8;
}

bool pass_has_kernel(const PassDesc& d, const PassShape& sh)
{
    if (sh.tma_store)
        return row_tstore_supported(d, sh);
    if (sh.pipelined)
        return lfft::select_pipe(d, sh) != nullptr;
    return lfft::select_static(d, sh) != nullptr || lfft::select_dynamic(d, sh) != nullptr;
}

namespace
{

// CTAs of a pipelined kernel resident per SM (queried once per kernel and shape).
int resident_ctas(const void* fn, int threads, int smem)
{
    static std::mutex mu;
    static std::unordered_map<const void*, std::unordered_map<long long, int>> cache;
    std::lock_guard<std::mutex> lk(mu);
    const long long key = (static_cast<long long>(threads) << 32) | static_cast<unsigned>(smem);
    auto& m = cache[fn];
    auto it = m.find(key);
    if (it != m.end())
        return it->second;
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fn, threads, smem) != cudaSuccess || blocks < 1)
        blocks = 1;
    m[key] = blocks;
    return blocks;
}

int sm_count()
{
    static int count = 0;
    if (count == 0)
    {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
        if (count < 1)
            count = 1;
    }
    return count;
}

} // namespace

cudaError_t launch_line_pass(const PassDesc& d, const PassShape& sh, const void* in, void* out, cudaStream_t stream)
{
    const int T = (d.n + sh.points_per_thread - 1) / sh.points_per_thread;
    const int threads = T * sh.lines_per_cta;
    if (sh.lines_per_cta > lfft::kMaxLinesPerCta || sh.lines_per_cta < 1)
        return cudaErrorInvalidConfiguration;
    const long long groups = (d.lines + sh.lines_per_cta - 1) / sh.lines_per_cta;
    if (groups <= 0)
        return cudaSuccess;
    if (sh.tma_store && (reinterpret_cast<uintptr_t>(out) & 15u) == 0)
        return launch_row_tstore(d, sh, in, out, stream);
    if (sh.tma_store)
    {
        // an output off a 16-byte boundary (the tensor map needs one): the thread-stored kernel, same lines a CTA
        PassShape cs = sh;
        cs.tma_store = false;
        cs.smem_bytes = sh.lines_per_cta * lfft::cta_line_pitch(d.n, sh.lines_per_cta) * 8;
        return launch_line_pass(d, cs, in, out, stream);
    }
    if (sh.pipelined && (reinterpret_cast<uintptr_t>(in) & 15u) == 0)
    {
        lfft::PipeFn fn = lfft::select_pipe(d, sh);
        if (fn == nullptr || threads > lfft::kPipeThreads)
            return cudaErrorInvalidConfiguration;
        if (sh.smem_bytes > 48 * 1024)
        {
            const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, sh.smem_bytes);
            if (e != cudaSuccess)
                return e;
        }
        const long long cap = static_cast<long long>(sm_count()) *
                              resident_ctas(reinterpret_cast<const void*>(fn), threads, sh.smem_bytes);
        const long long grid = groups < cap ? groups : cap;
        fn<<<static_cast<unsigned>(grid), threads, sh.smem_bytes, stream>>>(
            d, static_cast<const float2*>(in), static_cast<float2*>(out), sh.lines_per_cta, groups);
        return cudaGetLastError();
    }
    PassShape cs = sh;
    if (sh.pipelined)
    {
        // an input pointer off a 16-byte boundary: the classic kernel with the same thread map
        cs.pipelined = false;
        cs.direct_load = sh.map == PassMap::Row ? d.in.estride == 1 : d.in.ldist == 1;
        cs.smem_bytes = sh.lines_per_cta * lfft::cta_line_pitch(d.n, sh.lines_per_cta) * 8;
    }
    lfft::KernelFn fn = lfft::select_static(d, cs);
    if (fn == nullptr)
    {
        // the run-time schedule kernel always stages its lines through shared memory, in two buffers (even for a
        // one-stage pass that a compile-time kernel runs register to register)
        fn = lfft::select_dynamic(d, cs);
        cs.smem_bytes = 2 * sh.lines_per_cta * lfft::line_pitch(d.n) * 8; // two line buffers: out-of-place stages
        if (cs.smem_bytes > 227 * 1024)
            return cudaErrorInvalidConfiguration;
    }
    if (fn == nullptr || threads > lfft::max_threads(sh.points_per_thread, d.n))
        return cudaErrorInvalidConfiguration;
    if (groups > 0x7fffffffLL)
        return cudaErrorInvalidConfiguration;
    if (cs.smem_bytes > 48 * 1024)
    {
        const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, cs.smem_bytes);
        if (e != cudaSuccess)
            return e;
    }
    fn<<<static_cast<unsigned>(groups), threads, cs.smem_bytes, stream>>>(d, static_cast<const float2*>(in),
                                                                           static_cast<float2*>(out));
    return cudaGetLastError();
}

} // namespace crdfft
