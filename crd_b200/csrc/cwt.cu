// The element-wise kernels around the FFTs of the continuous wavelet transform (cwt_plan.cpp): the zero-padded complex
// copy of the signals, the product of the data spectrum with the per-scale kernel spectra (lengths the fused
// convolution does not take), and the epilogue that turns each scale's filtered sequence into coefficients
// (crd-hesap-wavelet cwt.hpp:509-516, 583-596). All three are HBM-bound: one read and one write per element,
// 64-bit indices, grid-stride loops over a grid of a few CTAs per SM.
#include "kernels.hpp"

#include <algorithm>

namespace crdfft
{
namespace
{

constexpr int kThreads = 256;

int grid_for(long long elements)
{
    const long long blocks = (elements + kThreads - 1) / kThreads;
    return static_cast<int>(std::max<long long>(1, std::min<long long>(blocks, 148LL * 8)));
}

// X[c][i] = (x[c][i], 0) for i < n, 0 up to lfft (cwt.hpp:509-516)
__global__ void __launch_bounds__(kThreads) cwt_pad_kernel(const float* __restrict__ x, float2* __restrict__ X,
                                                           long long n, long long lfft, long long total)
{
    for (long long e = blockIdx.x * static_cast<long long>(kThreads) + threadIdx.x; e < total;
         e += static_cast<long long>(gridDim.x) * kThreads)
    {
        const long long c = e / lfft, i = e - c * lfft;
        X[e] = i < n ? make_float2(__ldg(x + c * n + i), 0.0f) : make_float2(0.0f, 0.0f);
    }
}

// W[s][i] = X[i] * K[s][i] (cwt.hpp:583-587: the data spectrum times the kernel spectrum)
__global__ void __launch_bounds__(kThreads) cwt_product_kernel(const float2* __restrict__ X,
                                                               const float2* __restrict__ K, float2* __restrict__ W,
                                                               long long lfft, long long total)
{
    for (long long e = blockIdx.x * static_cast<long long>(kThreads) + threadIdx.x; e < total;
         e += static_cast<long long>(gridDim.x) * kThreads)
    {
        const float2 d = __ldg(X + e % lfft);
        const float2 k = K[e];
        W[e] = make_float2(d.x * k.x - d.y * k.y, d.x * k.y + d.y * k.x);
    }
}

// out[s][i] = amp_s (W[s][off_s + i + 1] - W[s][off_s + i]) / lfft, or 0 for a scale with fewer than two taps
// (cwt.hpp:561-567, 589-596). One CTA row per scale; consecutive threads read consecutive W elements.
__global__ void __launch_bounds__(kThreads) cwt_diff_kernel(const float2* __restrict__ W,
                                                            const CwtScale* __restrict__ sc, float2* __restrict__ out,
                                                            long long n, long long lfft, float inv_lfft)
{
    const long long s = blockIdx.y;
    const CwtScale p = sc[s];
    const float2* w = W + s * lfft + p.off;
    float2* o = out + s * n;
    for (long long i = blockIdx.x * static_cast<long long>(kThreads) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * kThreads)
    {
        float2 v = make_float2(0.0f, 0.0f);
        if (p.taps_ok)
        {
            const float2 a = w[i], b = w[i + 1];
            v = make_float2(p.amp * (b.x - a.x) * inv_lfft, p.amp * (b.y - a.y) * inv_lfft);
        }
        o[i] = v;
    }
}

} // namespace

cudaError_t launch_cwt_pad(const float* x, void* X, long long n, long long lfft, long long count, cudaStream_t stream)
{
    const long long total = lfft * count;
    cwt_pad_kernel<<<grid_for(total), kThreads, 0, stream>>>(x, static_cast<float2*>(X), n, lfft, total);
    return cudaGetLastError();
}

cudaError_t launch_cwt_product(const void* X, const void* K, void* W, long long lfft, long long nscales,
                               cudaStream_t stream)
{
    const long long total = lfft * nscales;
    cwt_product_kernel<<<grid_for(total), kThreads, 0, stream>>>(
        static_cast<const float2*>(X), static_cast<const float2*>(K), static_cast<float2*>(W), lfft, total);
    return cudaGetLastError();
}

cudaError_t launch_cwt_diff(const void* W, const CwtScale* scales, void* out, long long n, long long lfft,
                            long long nscales, cudaStream_t stream)
{
    const long long bx = std::max<long long>(1, std::min<long long>((n + kThreads - 1) / kThreads, 64));
    const dim3 grid(static_cast<unsigned>(bx), static_cast<unsigned>(nscales));
    cwt_diff_kernel<<<grid, kThreads, 0, stream>>>(static_cast<const float2*>(W), scales, static_cast<float2*>(out),
                                                   n, lfft, static_cast<float>(1.0 / static_cast<double>(lfft)));
    return cudaGetLastError();
}

} // namespace crdfft
