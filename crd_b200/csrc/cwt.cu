// The element-wise kernels around the FFTs of the continuous wavelet transform (cwt_plan.cpp): the zero-padded complex
// copy of the signals, the product of each signal's spectrum with every scale's kernel spectrum, and the epilogue
// that turns each filtered sequence into coefficients (crd-hesap-wavelet cwt.hpp:509-516, 583-596). All three are
// HBM-bound: one read and one write per element, 64-bit indices, grid-stride loops.
#include "index.cuh"
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
        const long long c = idiv(e, lfft), i = e - c * lfft;
        X[e] = i < n ? make_float2(__ldg(x + c * n + i), 0.0f) : make_float2(0.0f, 0.0f);
    }
}

// W[c][s][i] = X[c][i] * K[s][i] (cwt.hpp:583-587: the data spectrum times the kernel spectrum). One grid row
// (blockIdx.y) per (signal, scale) line; consecutive threads take consecutive elements of it.
__global__ void __launch_bounds__(kThreads) cwt_product_kernel(const float2* __restrict__ X,
                                                               const float2* __restrict__ K, float2* __restrict__ W,
                                                               long long lfft, long long nscales)
{
    const long long line = blockIdx.y;
    const long long c = idiv(line, nscales), s = line - c * nscales;
    const float2* x = X + c * lfft;
    const float2* k = K + s * lfft;
    float2* w = W + line * lfft;
    for (long long i = blockIdx.x * static_cast<long long>(kThreads) + threadIdx.x; i < lfft;
         i += static_cast<long long>(gridDim.x) * kThreads)
    {
        const float2 d = __ldg(x + i), v = __ldg(k + i);
        w[i] = make_float2(d.x * v.x - d.y * v.y, d.x * v.y + d.y * v.x);
    }
}

// out[c][s][i] = amp_s (W[c][s][off_s + i + 1] - W[c][s][off_s + i]) / lfft, or 0 for a scale with fewer than two
// taps (cwt.hpp:561-567, 589-596). One grid row per (signal, scale) line.
__global__ void __launch_bounds__(kThreads) cwt_diff_kernel(const float2* __restrict__ W,
                                                            const CwtScale* __restrict__ sc, float2* __restrict__ out,
                                                            long long n, long long lfft, long long nscales,
                                                            float inv_lfft)
{
    const long long line = blockIdx.y;
    const CwtScale p = sc[imod(line, nscales)];
    const float2* w = W + line * lfft + p.off;
    float2* o = out + line * n;
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
                               long long signals, cudaStream_t stream)
{
    const long long bx = std::max<long long>(1, std::min<long long>(lfft / (kThreads * 4), 64));
    const dim3 grid(static_cast<unsigned>(bx), static_cast<unsigned>(signals * nscales));
    cwt_product_kernel<<<grid, kThreads, 0, stream>>>(static_cast<const float2*>(X), static_cast<const float2*>(K),
                                                      static_cast<float2*>(W), lfft, nscales);
    return cudaGetLastError();
}

cudaError_t launch_cwt_diff(const void* W, const CwtScale* scales, void* out, long long n, long long lfft,
                            long long nscales, long long signals, cudaStream_t stream)
{
    const long long bx = std::max<long long>(1, std::min<long long>(n / (kThreads * 4), 64));
    const dim3 grid(static_cast<unsigned>(bx), static_cast<unsigned>(signals * nscales));
    cwt_diff_kernel<<<grid, kThreads, 0, stream>>>(static_cast<const float2*>(W), scales, static_cast<float2*>(out),
                                                   n, lfft, nscales,
                                                   static_cast<float>(1.0 / static_cast<double>(lfft)));
    return cudaGetLastError();
}

} // namespace crdfft
