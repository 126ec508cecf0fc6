// The line-FFT kernel with its radix schedule read from the descriptor at run time: every 7-smooth line length up to
// 8192 that has no compile-time schedule (2048, 8192, 1000, 6144, ..., the uneven batches' lengths, Bluestein's inner
// lengths, odd N-D axes).
//
// The CTA stages its lines through shared memory with coalesced cooperative loads (every load of a thread in flight
// at once) and stores (along whichever side is unit-stride, with the epilogue on the way out), and runs the stages
// per radix, out of place between two halves of shared memory (dyn_stage.cuh), inlined into the kernel at 128
// registers (out-of-line calls on request).

#include "dyn_stage.cuh"
#include "line_fft.cuh"

#include <cstdlib>

namespace crdfft
{
namespace lfft
{
namespace
{

template <PassMap MAP, bool EPI, bool INL>
__global__ void __launch_bounds__(kMaxThreads) dyn_fft_kernel(const PassDesc d, const float2* __restrict__ gin,
                                                              float2* __restrict__ gout)
{
    extern __shared__ float2 sm[];
    __shared__ long long s_in_off[kMaxLinesPerCta];
    __shared__ long long s_out_off[kMaxLinesPerCta];
    __shared__ int s_q[kMaxLinesPerCta];
    __shared__ int s_radix[kMaxStages];

    const int n = d.n;
    const int T = (n + 15) / 16;
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
    for (int i = tid; i < lpc; i += blockDim.x)
    {
        const long long line = line0 + i;
        s_in_off[i] = line_offset(d.in, line, d.lines_per_group);
        s_out_off[i] = line_offset(d.out, line, d.lines_per_group);
        s_q[i] = static_cast<int>(line_row(d, line));
    }
    if (tid < kMaxStages)
        s_radix[tid] = d.radix[tid];
    __syncthreads();

    Ctx c;
    init_scales(d, c);
    const long long lines_here = d.lines - line0;
    const long long ies = d.in.estride;
    tile_load<16>(
        n, lpc, ies == 1,
        [&](int a, int e) {
            return a < lines_here ? load_in<EPI>(c, gin + s_in_off[a] + static_cast<long long>(e) * ies)
                                  : make_float2(0.f, 0.f);
        },
        [&](int a, int e, float2 x) { LayRow<1>{sm + a * pitch}.at(e) = x; });
    __syncthreads();

    // out of place between the two halves of shared memory (lpc lines each)
    const float2* res = dyn_stages_pp<INL>(s_radix, d.nstages, static_cast<const float2*>(d.tw), n, sm + ll * pitch,
                                      sm + (lpc + ll) * pitch, jt, T, ll < lines_here);
    float2* tile = const_cast<float2*>(res) - ll * pitch; // the half that holds the result

    const long long oes = d.out.estride;
    for_tile(n, lpc, oes == 1, [&](int a, int e) {
        if (a < lines_here)
            __stcs(gout + s_out_off[a] + static_cast<long long>(e) * oes,
                   epilogue<EPI>(d, c, s_q[a], e, LayRow<1>{tile + a * pitch}.at(e)));
    });
}

} // namespace

KernelFn select_dynamic(const PassDesc& d, const PassShape& sh)
{
    if (sh.points_per_thread != 16)
        return nullptr;
    const bool epi = pass_epi(d);
    // The stages inlined into the kernel (the default: 240 0.339 -> 0.310 ms, 1000 0.377 -> 0.352, 3000 0.458 ->
    // 0.434 per 256 MiB; a few bytes of spills in its radix-25 path), or out-of-line calls (CRDFFT_DYN_INLINE=0)
    static const bool inl = std::getenv("CRDFFT_DYN_INLINE") == nullptr || std::atoi(std::getenv("CRDFFT_DYN_INLINE"));
    if (inl)
    {
        if (sh.map == PassMap::Row)
            return epi ? dyn_fft_kernel<PassMap::Row, true, true> : dyn_fft_kernel<PassMap::Row, false, true>;
        return epi ? dyn_fft_kernel<PassMap::Col, true, true> : dyn_fft_kernel<PassMap::Col, false, true>;
    }
    if (sh.map == PassMap::Row)
        return epi ? dyn_fft_kernel<PassMap::Row, true, false> : dyn_fft_kernel<PassMap::Row, false, false>;
    return epi ? dyn_fft_kernel<PassMap::Col, true, false> : dyn_fft_kernel<PassMap::Col, false, false>;
}

} // namespace lfft
} // namespace crdfft
