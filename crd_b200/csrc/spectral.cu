// Spectral estimators on the device: the segment periodograms of hesap-dsp (the reference's Welch PSD and
// spectrogram, engine/numerics/hesap-dsp/include/crd/hesap/dsp/spectral.hpp:44-183, and its periodogram, :188-220)
// as one launch over every segment of every signal, the window, detrend and |X|^2 epilogue fused around the real
// FFT of each segment:
//
//   segment s of signal g: x[g nsamples + s hop + i], i < nperseg = 2M
//   -> minus the segment mean (detrend 'constant'), times the window
//   -> M-point complex FFT of the real pairs in shared memory, recombined into X[k], k = 0 .. M (real_pair.cuh)
//   -> P[k] = scale |X[k]|^2, doubled except at k = 0 and k = M; scale = 1 / (fs sum w^2)
//
// A CTA takes lpc consecutive segments of one signal, so the overlapping samples of neighbouring segments are read
// from HBM once and from L1/L2 after. The spectrogram writes each segment's row; Welch sums its segments' rows in
// segment order into one row a CTA, and a second kernel adds those rows in CTA order and divides by the segment count
// (a fixed order: the PSD is bit-identical from run to run, as the reference's serial average is, :158-171).

#include "dyn_stage.cuh"
#include "kernels.hpp"
#include "line_fft.cuh"
#include "real_pair.cuh"

namespace crdfft
{
namespace lfft
{
namespace
{

// At most 256 threads with a compile-time schedule (four CTAs an SM at 16 points a thread), 512 with the run-time one.
template <class S, int P, bool DYN>
__global__ void __launch_bounds__(DYN ? kMaxThreads : kStaticThreads, DYN ? 1 : (P == 16 ? 4 : 2))
    spectral_kernel(const PassDesc d, const SpectralDesc sd, const float* __restrict__ x, float* __restrict__ out)
{
    extern __shared__ float2 sm[];
    __shared__ float s_mean[kMaxLinesPerCta];
    __shared__ int s_radix[kMaxStages];
    const int M = DYN ? d.n : sched_n<S>(d);
    const int T = (M + P - 1) / P;
    const int lpc = sd.lpc;
    const int tid = threadIdx.x;
    const int ll = tid / T;
    const int jt = tid - ll * T;
    const int pitch = line_pitch(M);
    const int nfreq = M + 1;
    const long long g = idiv(blockIdx.x, sd.ntiles);
    const int tile = static_cast<int>(blockIdx.x - g * sd.ntiles);
    const long long seg0 = static_cast<long long>(tile) * lpc;
    const int nl = static_cast<int>(sd.nseg - seg0 < lpc ? sd.nseg - seg0 : lpc);
    const bool ok = ll < nl;
    float2* line = sm + ll * pitch;
    float* red = reinterpret_cast<float*>(sm + (DYN ? 2 : 1) * lpc * pitch);
    if (DYN && tid < kMaxStages)
        s_radix[tid] = d.radix[tid];

    if constexpr (!DYN)
    {
        // 1-2 (compile-time schedule). Every pair of the thread in registers at once (all loads in flight), the
        // segment's sum by warp shuffles (a line's T threads are consecutive lanes, or whole warps), then detrend
        // and window applied in registers and one store to shared memory.
        constexpr int TS = (S::n + P - 1) / P;
        constexpr int ROUND = P < 16 ? P : 16;
        static_assert(TS <= 32 ? (32 % TS == 0) : (TS % 32 == 0),
                      "a line is a power-of-two part of a warp or whole warps");
        const float* src = x + g * sd.nsamples + (seg0 + (ok ? ll : 0)) * sd.hop;
        const bool al = (reinterpret_cast<uintptr_t>(src) & 7) == 0;
        float2 v[P];
        float sum = 0.0f;
#pragma unroll
        for (int r0 = 0; r0 < P; r0 += ROUND)
        {
#pragma unroll
            for (int r = r0; r < r0 + ROUND; ++r)
            {
                const int m = jt + r * TS;
                v[r] = make_float2(0.0f, 0.0f);
                if (ok && m < M)
                    v[r] = al ? __ldg(reinterpret_cast<const float2*>(src) + m)
                              : make_float2(__ldg(src + 2 * m), __ldg(src + 2 * m + 1));
            }
        }
#pragma unroll
        for (int r = 0; r < P; ++r)
            sum += v[r].x + v[r].y;
        if constexpr (TS <= 32)
        {
#pragma unroll
            for (int o = TS / 2; o > 0; o >>= 1)
                sum += __shfl_xor_sync(0xffffffffu, sum, o);
        }
        else
        {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
                sum += __shfl_xor_sync(0xffffffffu, sum, o);
            if ((tid & 31) == 0)
                red[tid >> 5] = sum;
            __syncthreads();
            sum = 0.0f;
#pragma unroll
            for (int i = 0; i < TS / 32; ++i)
                sum += red[ll * (TS / 32) + i];
        }
        const float mean = sd.detrend ? sum / static_cast<float>(2 * M) : 0.0f;
        const float2* w2 = reinterpret_cast<const float2*>(sd.win);
        const LayRow<1> lay{line};
        if (ok)
        {
#pragma unroll
            for (int r = 0; r < P; ++r)
            {
                const int m = jt + r * TS;
                if (m < M)
                {
                    const float2 w = __ldg(w2 + m);
                    lay.at(m) = make_float2((v[r].x - mean) * w.x, (v[r].y - mean) * w.y);
                }
            }
        }
    }
    else
    {
        // 1. the segment as real pairs, and its sum
        float sum = 0.0f;
        if (ok)
        {
            const float* src = x + g * sd.nsamples + (seg0 + ll) * sd.hop;
            const LayRow<1> lay{line};
            if ((reinterpret_cast<uintptr_t>(src) & 7) == 0)
            {
                const float2* s2 = reinterpret_cast<const float2*>(src);
#pragma unroll 4
                for (int m = jt; m < M; m += T)
                {
                    const float2 v = __ldg(s2 + m);
                    lay.at(m) = v;
                    sum += v.x + v.y;
                }
            }
            else
            {
#pragma unroll 4
                for (int m = jt; m < M; m += T)
                {
                    const float2 v = make_float2(__ldg(src + 2 * m), __ldg(src + 2 * m + 1));
                    lay.at(m) = v;
                    sum += v.x + v.y;
                }
            }
        }
        red[tid] = sum;
        __syncthreads();
        if (ok && jt == 0)
        {
            float s = 0.0f;
            for (int t = 0; t < T; ++t)
                s += red[ll * T + t];
            s_mean[ll] = sd.detrend ? s / static_cast<float>(2 * M) : 0.0f;
        }
        __syncthreads();
        // 2. detrend and window, each thread on the pairs it loaded
        if (ok)
        {
            const float mean = s_mean[ll];
            const float2* w2 = reinterpret_cast<const float2*>(sd.win);
            const LayRow<1> lay{line};
            for (int m = jt; m < M; m += T)
            {
                const float2 v = lay.at(m);
                const float2 w = __ldg(w2 + m);
                lay.at(m) = make_float2((v.x - mean) * w.x, (v.y - mean) * w.y);
            }
        }
    }
    // 3. the M-point FFT of the pairs
    float2* res = line;
    if constexpr (DYN)
    {
        __syncthreads();
        res = dyn_stages_pp(s_radix, d.nstages, static_cast<const float2*>(d.tw), M, line, sm + (lpc + ll) * pitch,
                            jt, T, ok);
    }
    else
    {
        Ctx c;
        c.ok = ok;
        c.q = 0;
        c.in = nullptr;
        c.out = nullptr;
        c.jt = jt;
        c.T = T;
        c.in_im = 1.0f;
        c.out_re = 1.0f;
        c.out_im = 1.0f;
        SchedRun<S>::template go<P, false, false, false, Kind<PassMap::Row, false>>(d, c, LayRow<1>{line}, M);
    }
    // 4. the one-sided density periodogram of the segment
    const float scale = sd.scale;
    const float2* wn = static_cast<const float2*>(sd.wn);
    float* row = sd.welch ? red + ll * nfreq : out + ((g * sd.nseg) + seg0 + ll) * nfreq;
    if (ok)
    {
        const LayRow<1> lr{res};
        for (int k = jt; k <= M / 2; k += T)
        {
            if (k == 0)
            {
                const float2 z0 = lr.at(0);
                const float a = z0.x + z0.y, b = z0.x - z0.y;
                row[0] = scale * (a * a);
                row[M] = scale * (b * b);
                continue;
            }
            float2 xk, xm;
            r2c_pair(lr.at(k), lr.at(M - k), __ldg(wn + k), xk, xm);
            row[k] = 2.0f * scale * (xk.x * xk.x + xk.y * xk.y);
            if (M - k != k)
                row[M - k] = 2.0f * scale * (xm.x * xm.x + xm.y * xm.y);
        }
    }
    if (!sd.welch)
        return;
    // 5. Welch: this CTA's segments summed in segment order
    __syncthreads();
    float* dst = out + static_cast<long long>(blockIdx.x) * nfreq;
    for (int k = tid; k < nfreq; k += blockDim.x)
    {
        float acc = 0.0f;
        for (int a = 0; a < nl; ++a)
            acc += red[a * nfreq + k];
        dst[k] = acc;
    }
}

// The per-CTA sums of each signal added in CTA order, divided by the segment count (spectral.hpp:158-171).
__global__ void welch_finish_kernel(const float* __restrict__ part, float* __restrict__ psd, long long count,
                                    int ntiles, int nfreq, float nseg)
{
    const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= count * nfreq)
        return;
    const long long g = idx / nfreq;
    const int k = static_cast<int>(idx - g * nfreq);
    const float* p = part + g * ntiles * static_cast<long long>(nfreq) + k;
    float acc = 0.0f;
    for (int t = 0; t < ntiles; ++t)
        acc += p[static_cast<long long>(t) * nfreq];
    psd[idx] = acc / nseg;
}

using SpecFn = void (*)(const PassDesc, const SpectralDesc, const float*, float*);

SpecFn spectral_select(const PassDesc& d, int P, bool* dyn)
{
    *dyn = false;
    if (P == 32)
    {
        if (same_radices(d, {16, 16, 16}))
            return spectral_kernel<Sched<16, 16, 16>, 32, false>;
        if (same_radices(d, {32, 32}))
            return spectral_kernel<Sched<32, 32>, 32, false>;
        if (same_radices(d, {32, 16, 16}))
            return spectral_kernel<Sched<32, 16, 16>, 32, false>;
        return nullptr;
    }
    if (same_radices(d, {16, 4}))
        return spectral_kernel<Sched<16, 4>, 16, false>;
    if (same_radices(d, {16, 8}))
        return spectral_kernel<Sched<16, 8>, 16, false>;
    if (same_radices(d, {16, 16}))
        return spectral_kernel<Sched<16, 16>, 16, false>;
    if (same_radices(d, {16, 8, 4}))
        return spectral_kernel<Sched<16, 8, 4>, 16, false>;
    if (same_radices(d, {16, 16, 8}))
        return spectral_kernel<Sched<16, 16, 8>, 16, false>;
    if (same_radices(d, {16, 16, 4}))
        return spectral_kernel<Sched<16, 16, 4>, 16, false>;
    *dyn = true;
    return spectral_kernel<DynSched, 16, true>;
}

} // namespace
} // namespace lfft

bool spectral_shape(const PassDesc& d, int* P, int* lpc, int* threads, int* smem)
{
    int p = 16, l = 1, s = 0;
    conv_shape(d, PassMap::Row, &p, &l, &s);
    bool dyn = false;
    if (lfft::spectral_select(d, p, &dyn) == nullptr)
        return false;
    const int T = (d.n + p - 1) / p;
    const int pitch = lfft::line_pitch(d.n);
    const int line_bytes = (dyn ? 2 : 1) * pitch * 8;
    while (l > 1 && l * line_bytes + std::max(T * l, l * (d.n + 1)) * 4 > 200 * 1024)
        --l;
    // whole warps (the compile-time path reduces a line's sum with warp shuffles)
    if (!dyn && T < 32)
        l = std::max(32 / T, l - l % (32 / T));
    const long long bytes = static_cast<long long>(l) * line_bytes + std::max(T * l, l * (d.n + 1)) * 4LL;
    if (bytes > 227 * 1024 || T * l > (dyn ? lfft::kMaxThreads : lfft::kStaticThreads))
        return false;
    *P = p;
    *lpc = l;
    *threads = T * l;
    *smem = static_cast<int>(bytes);
    return true;
}

cudaError_t launch_spectral(const PassDesc& d, const SpectralDesc& sd, int threads, int smem, const void* x,
                            void* out, cudaStream_t stream)
{
    int P = 16, lpc = 1, smem0 = 0;
    conv_shape(d, PassMap::Row, &P, &lpc, &smem0);
    bool dyn = false;
    lfft::SpecFn fn = lfft::spectral_select(d, P, &dyn);
    if (fn == nullptr)
        return cudaErrorInvalidConfiguration;
    const long long blocks = sd.count * sd.ntiles;
    if (blocks <= 0)
        return cudaSuccess;
    if (blocks > 0x7fffffffLL)
        return cudaErrorInvalidConfiguration;
    if (smem > 48 * 1024)
    {
        const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess)
            return e;
    }
    fn<<<static_cast<unsigned>(blocks), threads, smem, stream>>>(d, sd, static_cast<const float*>(x),
                                                                 static_cast<float*>(out));
    return cudaGetLastError();
}

cudaError_t launch_welch_finish(const SpectralDesc& sd, const void* part, void* psd, cudaStream_t stream)
{
    const int nfreq = sd.nperseg / 2 + 1;
    const long long total = sd.count * nfreq;
    if (total <= 0)
        return cudaSuccess;
    const long long blocks = (total + 255) / 256;
    if (blocks > 0x7fffffffLL)
        return cudaErrorInvalidConfiguration;
    lfft::welch_finish_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(
        static_cast<const float*>(part), static_cast<float*>(psd), sd.count, sd.ntiles, nfreq,
        static_cast<float>(sd.nseg));
    return cudaGetLastError();
}

} // namespace crdfft
