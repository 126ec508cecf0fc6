// Elementwise passes around the line-FFT kernel: the real <-> half-length complex recombination of R2C/C2R and the
// three chirp passes of Bluestein. All are streaming, HBM-bound grid-stride kernels.

#include "codelets.cuh"
#include "index.cuh"
#include "kernels.hpp"

#include <cuda_runtime.h>

namespace crdfft
{
namespace
{

int grid_for(long long work, int threads)
{
    long long g = (work + threads - 1) / threads;
    const long long cap = 148LL * 16;
    if (g > cap)
        g = cap;
    return static_cast<int>(g < 1 ? 1 : g);
}

// Forward recombine, in place allowed (z and out may alias): one thread owns the mirror pair (k, h-k), reads both
// half-spectrum values before writing either output. With Z = FFT_h(z), z_j = x_{2j} + i x_{2j+1}:
//   E_k = (Z_k + conj Z_{h-k}) / 2,  O_k = (Z_k - conj Z_{h-k}) / (2i),  X_k = E_k + W_n^k O_k,  k = 0 .. h
// (include/crd/hesap/fft/real_fft.hpp:54-63).
__device__ __forceinline__ float2 r2c_one(float2 zk, float2 znk, float2 w)
{
    const float er = (zk.x + znk.x) * 0.5f;
    const float ei = (zk.y - znk.y) * 0.5f;
    const float orr = (zk.y + znk.y) * 0.5f;
    const float oii = (znk.x - zk.x) * 0.5f;
    return make_float2(er + (w.x * orr - w.y * oii), ei + (w.x * oii + w.y * orr));
}

__global__ void r2c_post_kernel(const RealRecombine p, const float2* z, float2* out)
{
    const long long half = p.h / 2 + 1; // k = 0 .. h/2 owns pairs
    const long long total = half * p.batch;
    const float2* wn = static_cast<const float2*>(p.wn);
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
    {
        const long long t = i / half;
        const long long k = i - t * half;
        const float2* zt = z + t * p.zdist;
        float2* ot = out + t * p.xdist;
        if (k == 0)
        {
            const float2 z0 = zt[0];
            const float2 a = r2c_one(z0, z0, wn[0]);
            const float2 b = r2c_one(z0, z0, wn[p.h]);
            ot[0] = cscale(a, p.scale);
            ot[p.h] = cscale(b, p.scale);
        }
        else
        {
            const float2 zk = zt[k];
            const float2 znk = zt[p.h - k];
            const float2 a = r2c_one(zk, znk, wn[k]);
            const float2 b = r2c_one(znk, zk, wn[p.h - k]);
            ot[k] = cscale(a, p.scale);
            if (p.h - k != k)
                ot[p.h - k] = cscale(b, p.scale);
        }
    }
}

// Inverse recombine (include/crd/hesap/fft/real_fft.hpp:72-84): E_k = (X_k + conj X_{h-k})/2,
// D_k = (X_k - conj X_{h-k})/2, O_k = W_n^{-k} D_k, Z_k = E_k + i O_k, k = 0 .. h-1. One thread per mirror pair.
__device__ __forceinline__ float2 c2r_one(float2 xk, float2 xhk, float2 w)
{
    const float er = (xk.x + xhk.x) * 0.5f;
    const float ei = (xk.y - xhk.y) * 0.5f;
    const float dr = (xk.x - xhk.x) * 0.5f;
    const float di = (xk.y + xhk.y) * 0.5f;
    const float orr = w.x * dr + w.y * di;
    const float oii = w.x * di - w.y * dr;
    return make_float2(er - oii, ei + orr);
}

__global__ void c2r_pre_kernel(const RealRecombine p, const float2* in, float2* z)
{
    const long long half = p.h / 2 + 1;
    const long long total = half * p.batch;
    const float2* wn = static_cast<const float2*>(p.wn);
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
    {
        const long long t = i / half;
        const long long k = i - t * half;
        const float2* xt = in + t * p.xdist;
        float2* zt = z + t * p.zdist;
        if (k == 0)
        {
            const float2 x0 = xt[0];
            const float2 xh = xt[p.h];
            zt[0] = cscale(c2r_one(x0, xh, wn[0]), p.scale);
        }
        else
        {
            const float2 xk = xt[k];
            const float2 xhk = xt[p.h - k];
            const float2 a = c2r_one(xk, xhk, wn[k]);
            const float2 b = c2r_one(xhk, xk, wn[p.h - k]);
            zt[k] = cscale(a, p.scale);
            if (p.h - k != k)
                zt[p.h - k] = cscale(b, p.scale);
        }
    }
}

// a_k = x_k conj(chirp_k) (x conjugated first for the inverse), zero-padded to m (bluestein.hpp:95-106).
__global__ void chirp_pre_kernel(const ChirpDesc p, const float2* x, float2* w)
{
    const long long total = p.m * p.batch;
    const float2* ch = static_cast<const float2*>(p.chirp);
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
    {
        const long long t = idiv(i, p.m);
        const long long k = i - t * p.m;
        float2 r = make_float2(0.f, 0.f);
        if (k < p.n)
        {
            float2 v = x[t * p.xdist + k];
            if (p.conj)
                v.y = -v.y;
            const float2 c = ch[k];
            r = make_float2(v.x * c.x + v.y * c.y, v.y * c.x - v.x * c.y);
        }
        w[t * p.wdist + k] = r;
    }
}

// C = A * FFT_m(b) (bluestein.hpp:109-116).
__global__ void spectrum_mul_kernel(const ChirpDesc p, float2* w)
{
    const long long total = p.m * p.batch;
    const float2* bf = static_cast<const float2*>(p.bfft);
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
    {
        const long long t = idiv(i, p.m);
        const long long k = i - t * p.m;
        float2* wt = w + t * p.wdist;
        wt[k] = cmul(wt[k], bf[k]);
    }
}

// X_k = conj(chirp_k) c_k scale, conjugated for the inverse (bluestein.hpp:121-134).
__global__ void chirp_post_kernel(const ChirpDesc p, const float2* w, float2* x)
{
    const long long total = p.n * p.batch;
    const float2* ch = static_cast<const float2*>(p.chirp);
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
    {
        const long long t = idiv(i, p.n);
        const long long k = i - t * p.n;
        const float2 v = w[t * p.wdist + k];
        const float2 c = ch[k];
        float yr = (v.x * c.x + v.y * c.y) * p.scale;
        float yi = (v.y * c.x - v.x * c.y) * p.scale;
        if (p.conj)
            yi = -yi;
        x[t * p.xdist + k] = make_float2(yr, yi);
    }
}

__global__ void scale_kernel(float2* data, long long count, float s)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        data[i] = cscale(data[i], s);
}

} // namespace

cudaError_t launch_r2c_post(const RealRecombine& p, const void* z, void* out, cudaStream_t stream)
{
    const long long work = (p.h / 2 + 1) * p.batch;
    r2c_post_kernel<<<grid_for(work, 256), 256, 0, stream>>>(p, static_cast<const float2*>(z),
                                                               static_cast<float2*>(out));
    return cudaGetLastError();
}

cudaError_t launch_c2r_pre(const RealRecombine& p, const void* in, void* z, cudaStream_t stream)
{
    const long long work = (p.h / 2 + 1) * p.batch;
    c2r_pre_kernel<<<grid_for(work, 256), 256, 0, stream>>>(p, static_cast<const float2*>(in),
                                                              static_cast<float2*>(z));
    return cudaGetLastError();
}

cudaError_t launch_chirp_pre(const ChirpDesc& p, const void* x, void* w, cudaStream_t stream)
{
    chirp_pre_kernel<<<grid_for(p.m * p.batch, 256), 256, 0, stream>>>(p, static_cast<const float2*>(x),
                                                                         static_cast<float2*>(w));
    return cudaGetLastError();
}

cudaError_t launch_spectrum_mul(const ChirpDesc& p, void* w, cudaStream_t stream)
{
    spectrum_mul_kernel<<<grid_for(p.m * p.batch, 256), 256, 0, stream>>>(p, static_cast<float2*>(w));
    return cudaGetLastError();
}

cudaError_t launch_chirp_post(const ChirpDesc& p, const void* w, void* x, cudaStream_t stream)
{
    chirp_post_kernel<<<grid_for(p.n * p.batch, 256), 256, 0, stream>>>(p, static_cast<const float2*>(w),
                                                                          static_cast<float2*>(x));
    return cudaGetLastError();
}

// Split-complex (planar) operands: the re and im planes of `count` complex values to interleaved pairs, and back.
// Streaming, one element a thread per iteration, both sides coalesced.
__global__ void planar_gather_kernel(const float* __restrict__ re, const float* __restrict__ im, float2* out,
                                     long long count)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        __stcs(out + i, make_float2(__ldcs(re + i), __ldcs(im + i)));
}

__global__ void planar_scatter_kernel(const float2* __restrict__ in, float* re, float* im, long long count)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
    {
        const float2 v = __ldcs(in + i);
        __stcs(re + i, v.x);
        __stcs(im + i, v.y);
    }
}

cudaError_t launch_planar_gather(const void* re, const void* im, void* out, long long count, cudaStream_t stream)
{
    planar_gather_kernel<<<grid_for(count, 256), 256, 0, stream>>>(static_cast<const float*>(re),
                                                                    static_cast<const float*>(im),
                                                                    static_cast<float2*>(out), count);
    return cudaGetLastError();
}

cudaError_t launch_planar_scatter(const void* in, void* re, void* im, long long count, cudaStream_t stream)
{
    planar_scatter_kernel<<<grid_for(count, 256), 256, 0, stream>>>(static_cast<const float2*>(in),
                                                                     static_cast<float*>(re),
                                                                     static_cast<float*>(im), count);
    return cudaGetLastError();
}

cudaError_t launch_scale(void* data, long long count, float s, cudaStream_t stream)
{
    scale_kernel<<<grid_for(count, 256), 256, 0, stream>>>(static_cast<float2*>(data), count, s);
    return cudaGetLastError();
}

} // namespace crdfft
