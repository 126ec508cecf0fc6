// Launcher of the line-FFT pass kernel (line_fft.cuh): picks the compile-time schedule when one exists for the pass,
// else the run-time schedule, and launches one CTA per `lines_per_cta` lines.

#include "kernels.hpp"
#include "line_fft.cuh"

namespace crdfft
{

int pass_lines_per_cta_limit() { return lfft::kMaxLinesPerCta; }
int pass_threads_limit() { return lfft::kMaxThreads; }
int pass_line_pitch(int n) { return lfft::line_pitch(n); }

bool pass_has_kernel(const PassDesc& d, const PassShape& sh)
{
    return lfft::select_static(d, sh) != nullptr || lfft::select_dynamic(d, sh) != nullptr;
}

cudaError_t launch_line_pass(const PassDesc& d, const PassShape& sh, const void* in, void* out, cudaStream_t stream)
{
    lfft::KernelFn fn = lfft::select_static(d, sh);
    if (fn == nullptr)
        fn = lfft::select_dynamic(d, sh);
    if (fn == nullptr)
        return cudaErrorInvalidConfiguration;
    const int T = (d.n + sh.points_per_thread - 1) / sh.points_per_thread;
    const int threads = T * sh.lines_per_cta;
    if (threads > lfft::kMaxThreads || sh.lines_per_cta > lfft::kMaxLinesPerCta || sh.lines_per_cta < 1)
        return cudaErrorInvalidConfiguration;
    const long long grid = (d.lines + sh.lines_per_cta - 1) / sh.lines_per_cta;
    if (grid <= 0)
        return cudaSuccess;
    if (grid > 0x7fffffffLL)
        return cudaErrorInvalidConfiguration;
    if (sh.smem_bytes > 48 * 1024)
    {
        const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, sh.smem_bytes);
        if (e != cudaSuccess)
            return e;
    }
    fn<<<static_cast<unsigned>(grid), threads, sh.smem_bytes, stream>>>(d, static_cast<const float2*>(in),
                                                                         static_cast<float2*>(out));
    return cudaGetLastError();
}

} // namespace crdfft
