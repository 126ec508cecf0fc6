// Fused FFT convolution: forward FFT -> multiply by a filter spectrum -> inverse FFT, one HBM read and one write per
// point. The vendor route is three global passes (forward FFT, an elementwise multiply kernel, inverse FFT:
// bench/gpu-fft/cufft_conv_bench.cu:3-5); the reference's own GPU kernel fuses them on chip
// (engine/gpu/kir/include/crd/kir/ckir_fft.hpp:279-296): y = IFFT(FFT(x) * H) * scale, scale 1/N by default, one
// filter spectrum shared by the batch or one per transform.
//
// Each CTA holds whole lines in shared memory: the forward stages leave the spectrum there in natural order (the
// Stockham stages sort as they go); each thread multiplies its elements by H and conjugates them; the same forward
// stages then run again and the last one stores conj(.) * scale, since IFFT(Z) = conj(FFT(conj(Z))). The line
// stages are the line-FFT kernel's (line_fft.cuh). A row map serves 1-D batches; a column map serves the column
// pass of a 2-D convolution (rows FFT, fused column convolution, inverse rows FFT).

#include "dyn_stage.cuh"
#include "kernels.hpp"
#include "line_fft.cuh"

namespace crdfft
{
namespace lfft
{
namespace
{

template <class S, int P, PassMap MAP>
__global__ void __launch_bounds__(kMaxThreads)
    conv_kernel(const PassDesc d, const float2* __restrict__ gin, const float2* __restrict__ spec,
                const LineMap smap, float2* __restrict__ gout)
{
    extern __shared__ float2 sm[];
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
    const long long line = line0 + ll;
    Ctx c;
    c.ok = line < d.lines;
    c.q = line_row(d, line);
    c.in = gin + line_offset(d.in, line, d.lines_per_group);
    c.out = gout + line_offset(d.out, line, d.lines_per_group);
    c.jt = jt;
    c.T = T;
    init_scales(d, c); // conj_out and the scale: the inverse's epilogue
    c.in_im = 1.0f;
    const LayRow<1> lay{sm + ll * pitch};

    // forward FFT of the lines, read straight from global memory, result in shared memory
    SchedRun<S>::template go<P, true, false, false, Kind<MAP, false>>(d, c, lay, n);
    // Z = conj(X H), each thread on its own elements of its line
    if (c.ok)
    {
        const float2* h = spec + line_offset(smap, line, d.lines_per_group);
        for (int e = jt; e < n; e += T)
        {
            const float2 v = cmul(lay.at(e), __ldg(h + static_cast<long long>(e) * smap.estride));
            lay.at(e) = make_float2(v.x, -v.y);
        }
    }
    __syncthreads();
    // conj(FFT(Z)) * scale = IFFT(X H) * scale, stored straight to global memory
    SchedRun<S>::template go<P, false, true, false, Kind<MAP, true>>(d, c, lay, n);
}

// The same convolution for lengths without a compile-time schedule: lines staged through shared memory with
// coalesced loads and stores, both FFTs as out-of-place run-time stages between two line buffers (dyn_stage.cuh).
template <PassMap MAP>
__global__ void __launch_bounds__(kMaxThreads)
    conv_dyn_kernel(const PassDesc d, const float2* __restrict__ gin, const float2* __restrict__ spec,
                    const LineMap smap, float2* __restrict__ gout)
{
    extern __shared__ float2 sm[];
    __shared__ long long s_in_off[kMaxLinesPerCta];
    __shared__ long long s_out_off[kMaxLinesPerCta];
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
        s_in_off[i] = line_offset(d.in, line0 + i, d.lines_per_group);
        s_out_off[i] = line_offset(d.out, line0 + i, d.lines_per_group);
    }
    if (tid < kMaxStages)
        s_radix[tid] = d.radix[tid];
    __syncthreads();
    const long long lines_here = d.lines - line0;
    const bool ok = ll < lines_here;
    const long long ies = d.in.estride;
    tile_load<16>(
        n, lpc, ies == 1,
        [&](int a, int e) {
            return a < lines_here ? __ldcs(gin + s_in_off[a] + static_cast<long long>(e) * ies) : make_float2(0.f, 0.f);
        },
        [&](int a, int e, float2 x) { LayRow<1>{sm + a * pitch}.at(e) = x; });
    __syncthreads();
    const float2* tw = static_cast<const float2*>(d.tw);
    float2* bufa = sm + ll * pitch;
    float2* bufb = sm + (lpc + ll) * pitch;
    // forward FFT
    float2* x = dyn_stages_pp(s_radix, d.nstages, tw, n, bufa, bufb, jt, T, ok);
    // Z = conj(X H)
    if (ok)
    {
        const float2* h = spec + line_offset(smap, line0 + ll, d.lines_per_group);
        for (int e = jt; e < n; e += T)
        {
            const float2 v = cmul(LayRow<1>{x}.at(e), __ldg(h + static_cast<long long>(e) * smap.estride));
            LayRow<1>{x}.at(e) = make_float2(v.x, -v.y);
        }
    }
    __syncthreads();
    // conj(FFT(Z)) * scale
    float2* y = dyn_stages_pp(s_radix, d.nstages, tw, n, x, x == bufa ? bufb : bufa, jt, T, ok);
    float2* tile = y - ll * pitch;
    const float re = d.scale;
    const float im = d.conj_out ? -d.scale : d.scale;
    const long long oes = d.out.estride;
    for_tile(n, lpc, oes == 1, [&](int a, int e) {
        if (a < lines_here)
        {
            const float2 v = LayRow<1>{tile + a * pitch}.at(e);
            __stcs(gout + s_out_off[a] + static_cast<long long>(e) * oes, make_float2(v.x * re, v.y * im));
        }
    });
}

// The continuous wavelet transform's lines (crd-hesap-wavelet cwt.hpp:583-596) in one kernel: line l is signal
// l / nscales at scale l mod nscales. Z = conj(X K) goes to shared memory, the forward stages leave FFT(Z) there in
// natural order, and w = IFFT(X K) = conj(FFT(Z)) (unnormalised) is differenced on the way out:
// out[l][i] = amp (w[off + i + 1] - w[off + i]) / lfft, or 0 for a scale with fewer than two taps. Only the n
// coefficients of a line reach HBM; the spectra X (one line a signal) and K (one a scale) are read once a line.
template <class S, int P>
__global__ void __launch_bounds__(kMaxThreads)
    cwt_line_kernel(const PassDesc d, const float2* __restrict__ X, const float2* __restrict__ K,
                    const CwtScale* __restrict__ scales, long long nscales, long long nsamples, float inv_n,
                    float2* __restrict__ gout)
{
    extern __shared__ float2 sm[];
    constexpr int n = S::n;
    constexpr int T = n / P;
    const int lpc = blockDim.x / T;
    const int tid = threadIdx.x;
    const int ll = tid / T;
    const int jt = tid - ll * T;
    const long long line = static_cast<long long>(blockIdx.x) * lpc + ll;
    Ctx c;
    c.ok = line < d.lines;
    c.q = 0;
    c.in = X;
    c.out = gout;
    c.jt = jt;
    c.T = T;
    init_scales(d, c);
    c.in_im = 1.0f;
    const LayRow<1> lay{sm + ll * line_pitch(n)};
    const long long sig = idiv(line, nscales), s = line - sig * nscales;
    if (c.ok)
    {
        const float2* x = X + sig * n;
        const float2* k = K + s * n;
        for (int e = jt; e < n; e += T)
        {
            const float2 v = cmul(__ldg(x + e), __ldg(k + e));
            lay.at(e) = make_float2(v.x, -v.y);
        }
    }
    __syncthreads();
    SchedRun<S>::template go<P, false, false, false, Kind<PassMap::Row, false>>(d, c, lay, n);
    __syncthreads();
    if (c.ok)
    {
        const CwtScale p = scales[s];
        float2* o = gout + line * nsamples;
        for (long long i = jt; i < nsamples; i += T)
        {
            float2 v = make_float2(0.0f, 0.0f);
            if (p.taps_ok)
            {
                const float2 a = lay.at(static_cast<int>(p.off + i)), b = lay.at(static_cast<int>(p.off + i + 1));
                v = make_float2(p.amp * (b.x - a.x) * inv_n, p.amp * (a.y - b.y) * inv_n);
            }
            __stcs(o + i, v);
        }
    }
}

using CwtFn = void (*)(const PassDesc, const float2*, const float2*, const CwtScale*, long long, long long, float,
                       float2*);

// Compile-time schedules only (the lengths conv_select runs statically on a row map).
CwtFn cwt_select(const PassDesc& d, int P)
{
    if (P == 32)
    {
        if (same_radices(d, {16, 16, 16}))
            return cwt_line_kernel<Sched<16, 16, 16>, 32>;
        if (same_radices(d, {32, 32}))
            return cwt_line_kernel<Sched<32, 32>, 32>;
        if (same_radices(d, {32, 16, 16}))
            return cwt_line_kernel<Sched<32, 16, 16>, 32>;
        return nullptr;
    }
    if (same_radices(d, {16, 16}))
        return cwt_line_kernel<Sched<16, 16>, 16>;
    if (same_radices(d, {16, 8, 4}))
        return cwt_line_kernel<Sched<16, 8, 4>, 16>;
    if (same_radices(d, {16, 16, 4}))
        return cwt_line_kernel<Sched<16, 16, 4>, 16>;
    return nullptr;
}

using ConvFn = void (*)(const PassDesc, const float2*, const float2*, const LineMap, float2*);

template <class S, int P> ConvFn conv_pick(PassMap map)
{
    return map == PassMap::Row ? conv_kernel<S, P, PassMap::Row> : conv_kernel<S, P, PassMap::Col>;
}

// The kernel for the pass at `P` points a thread: compile-time schedules for the common lengths, else the run-time
// schedule (16 points a thread).
ConvFn conv_select(const PassDesc& d, PassMap map, int P)
{
    if (P == 32)
    {
        if (map != PassMap::Row)
            return nullptr;
        if (same_radices(d, {16, 16, 16}))
            return conv_kernel<Sched<16, 16, 16>, 32, PassMap::Row>;
        if (same_radices(d, {32, 32}))
            return conv_kernel<Sched<32, 32>, 32, PassMap::Row>;
        if (same_radices(d, {32, 16, 16}))
            return conv_kernel<Sched<32, 16, 16>, 32, PassMap::Row>;
        return nullptr;
    }
    if (same_radices(d, {16, 16}))
        return conv_pick<Sched<16, 16>, 16>(map);
    if (same_radices(d, {16, 8, 4}))
        return conv_pick<Sched<16, 8, 4>, 16>(map);
    if (same_radices(d, {16, 16, 4}))
        return conv_pick<Sched<16, 16, 4>, 16>(map);
    return map == PassMap::Row ? conv_dyn_kernel<PassMap::Row> : conv_dyn_kernel<PassMap::Col>;
}

bool conv_is_dynamic(const PassDesc& d, PassMap map, int P)
{
    return P == 16 && !same_radices(d, {16, 16}) && !same_radices(d, {16, 8, 4}) && !same_radices(d, {16, 16, 4});
}

} // namespace
} // namespace lfft

bool conv_supported(const PassDesc& d)
{
    return d.nstages > 0 && (d.n + 15) / 16 <= lfft::kMaxThreads;
}

// Lines a CTA and points a thread: about 256 threads a CTA (32 points a thread for the n = 4096 lines and the
// radix-32 schedules).
void conv_shape(const PassDesc& d, PassMap map, int* P, int* lpc, int* smem)
{
    *P = (map == PassMap::Row && (lfft::same_radices(d, {16, 16, 16}) || d.radix[0] == 32)) ? 32 : 16;
    const int T = (d.n + *P - 1) / *P;
    int l = std::max(1, 256 / T);
    if (map == PassMap::Col)
        l = std::max(1, std::min(l, 16));
    while (l > 1 && l * lfft::line_pitch(d.n) * 8 > 100 * 1024)
        --l;
    *lpc = l;
    *smem = l * lfft::line_pitch(d.n) * 8;
}

cudaError_t launch_conv(const PassDesc& d, PassMap map, const LineMap& smap, const void* in, const void* spec,
                        void* out, cudaStream_t stream)
{
    int P = 16, lpc = 1, smem = 0;
    conv_shape(d, map, &P, &lpc, &smem);
    lfft::ConvFn fn = lfft::conv_select(d, map, P);
    if (fn == nullptr)
        return cudaErrorInvalidConfiguration;
    if (lfft::conv_is_dynamic(d, map, P))
    {
        smem *= 2; // two line buffers
        if (smem > 227 * 1024)
            return cudaErrorInvalidConfiguration;
    }
    const int T = (d.n + P - 1) / P;
    const long long groups = (d.lines + lpc - 1) / lpc;
    if (groups <= 0)
        return cudaSuccess;
    if (groups > 0x7fffffffLL)
        return cudaErrorInvalidConfiguration;
    if (smem > 48 * 1024)
    {
        const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess)
            return e;
    }
    fn<<<static_cast<unsigned>(groups), T * lpc, smem, stream>>>(d, static_cast<const float2*>(in),
                                                                 static_cast<const float2*>(spec), smap,
                                                                 static_cast<float2*>(out));
    return cudaGetLastError();
}

bool cwt_lines_supported(const PassDesc& d)
{
    int P = 16, lpc = 1, smem = 0;
    conv_shape(d, PassMap::Row, &P, &lpc, &smem);
    return conv_supported(d) && lfft::cwt_select(d, P) != nullptr;
}

cudaError_t launch_cwt_lines(const PassDesc& d, const void* X, const void* K, const CwtScale* scales, long long nscales,
                             long long n, void* out, cudaStream_t stream)
{
    int P = 16, lpc = 1, smem = 0;
    conv_shape(d, PassMap::Row, &P, &lpc, &smem);
    lfft::CwtFn fn = lfft::cwt_select(d, P);
    if (fn == nullptr || n < 1 || n >= d.n)
        return cudaErrorInvalidConfiguration;
    const int T = d.n / P;
    const long long groups = (d.lines + lpc - 1) / lpc;
    if (groups <= 0)
        return cudaSuccess;
    if (groups > 0x7fffffffLL)
        return cudaErrorInvalidConfiguration;
    if (smem > 48 * 1024)
    {
        const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess)
            return e;
    }
    fn<<<static_cast<unsigned>(groups), T * lpc, smem, stream>>>(
        d, static_cast<const float2*>(X), static_cast<const float2*>(K), scales, nscales, n,
        static_cast<float>(1.0 / static_cast<double>(d.n)), static_cast<float2*>(out));
    return cudaGetLastError();
}

} // namespace crdfft
