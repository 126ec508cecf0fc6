// Real-data line kernels: a real transform of n = 2M points as one M-point complex FFT of z[m] = x[2m] + i x[2m+1]
// plus the recombination of the pairs (k, M-k), fused into one launch with the line in shared memory.
//
//   R2C rows   x (n reals) -> Z = FFT_M(z) -> X[k], k = 0 .. M                  (the reference's RealFftPlan::rfft,
//                                                                               include/crd/hesap/fft/real_fft.hpp:41-63)
//   C2R rows   Y (M + 1 values) -> Q (pairs) -> y = conj(FFT_M(conj Q)) * scale (RealFftPlan::irfft, real_fft.hpp:65-92)
//   real conv  x -> Z -> X -> Y = X H -> Q -> y, one HBM read and one write per point, the real edition of the
//              fused convolution (engine/gpu/kir/include/crd/kir/ckir_fft.hpp:2300-2308 runs the real 2-D case as R2C
//              rows, a half-width column convolution and C2R rows)
//
// With W = exp(-2 pi i / n), E = (Z[k] + conj Z[M-k]) / 2 and O = (Z[k] - conj Z[M-k]) / 2i:
//   X[k] = E + W^k O,   X[M-k] = conj(E - W^k O),   X[0] = Re Z[0] + Im Z[0],   X[M] = Re Z[0] - Im Z[0];
// and for the inverse, with a = Y[k] + conj Y[M-k], b = Y[k] - conj Y[M-k]:
//   Q[k] = a + i b W^-k,   Q[M-k] = conj(a) + i conj(b W^-k),
// so that IFFT_M(Q) (unnormalised) = y[2m] + i y[2m+1] with y the unnormalised inverse real transform. Q[0] pairs
// Y[0] with Y[M] by the same formula (W^0 = 1), imaginary parts included, as the reference's irfft does
// (real_fft.hpp:72-84). IFFT(Q) is computed as conj(FFT(conj Q)), which runs the forward stages again.

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

// The pairs of one line, handled by the line's T threads (thread jt takes k = jt, jt + T, ...). `get(i)` reads Z or
// Y at i <= M; `put(i, v)` writes the result at i <= M.
template <int MODE, class Get, class Put>
__device__ __forceinline__ void pair_pass(int M, int jt, int T, const float2* __restrict__ wn,
                                          const float2* __restrict__ h, long long hes, Get&& get, Put&& put)
{
    const int half = M / 2;
    for (int k = jt; k <= half; k += T)
    {
        if (k == 0)
        {
            const float2 z0 = get(0);
            if constexpr (MODE == kRealR2C)
            {
                put(0, make_float2(z0.x + z0.y, 0.0f));
                put(M, make_float2(z0.x - z0.y, 0.0f));
            }
            else if constexpr (MODE == kRealC2R)
            {
                // the pair (0, M) with W^0 = 1, imaginary parts included, as the reference's irfft forms it
                float2 q0, unused;
                c2r_pair(z0, get(M), make_float2(1.0f, 0.0f), q0, unused);
                put(0, q0);
            }
            else
            {
                const float2 y0 = cmul(make_float2(z0.x + z0.y, 0.0f), __ldg(h));
                const float2 ym = cmul(make_float2(z0.x - z0.y, 0.0f), __ldg(h + static_cast<long long>(M) * hes));
                float2 q0, unused;
                c2r_pair(y0, ym, make_float2(1.0f, 0.0f), q0, unused);
                put(0, q0);
            }
            continue;
        }
        const float2 w = __ldg(wn + k);
        const float2 vk = get(k);
        const float2 vm = get(M - k);
        float2 a, b;
        if constexpr (MODE == kRealR2C)
            r2c_pair(vk, vm, w, a, b);
        else if constexpr (MODE == kRealC2R)
            c2r_pair(vk, vm, w, a, b);
        else
        {
            float2 xk, xm;
            r2c_pair(vk, vm, w, xk, xm);
            xk = cmul(xk, __ldg(h + static_cast<long long>(k) * hes));
            xm = cmul(xm, __ldg(h + static_cast<long long>(M - k) * hes));
            c2r_pair(xk, xm, w, a, b);
        }
        put(k, a);
        if (M - k != k)
            put(M - k, b);
    }
}

// Compile-time schedule of the M-point line. One CTA holds lpc whole lines (row map, unit stride on both sides).
// At most 256 threads (the launch shapes of conv_shape for these schedules); 16 points a thread leave registers for
// four CTAs an SM.
template <class S, int P, int MODE>
__global__ void __launch_bounds__(kStaticThreads, P == 16 ? 4 : 2)
    real_line_kernel(const PassDesc d, const float2* __restrict__ gin, const float2* __restrict__ spec,
                     const RealLineAux r, float2* __restrict__ gout)
{
    extern __shared__ float2 sm[];
    const int M = sched_n<S>(d);
    const int T = (M + P - 1) / P;
    const int lpc = blockDim.x / T;
    const int tid = threadIdx.x;
    const int pitch = line_pitch(M);
    const int ll = tid / T;
    const int jt = tid - ll * T;
    const long long line = static_cast<long long>(blockIdx.x) * lpc + ll;
    const float2* wn = static_cast<const float2*>(r.wn);
    Ctx c;
    c.ok = line < d.lines;
    c.q = 0;
    c.in = gin + line_offset(d.in, line, d.lines_per_group);
    c.out = gout + line_offset(d.out, line, d.lines_per_group);
    c.jt = jt;
    c.T = T;
    init_scales(d, c);
    c.in_im = 1.0f;
    const LayRow<1> lay{sm + ll * pitch};
    const float2* h = spec != nullptr ? spec + line_offset(r.smap, line, d.lines_per_group) : nullptr;
    auto put_lay = [&](int i, float2 v) { lay.at(i) = conjf2(v); };
    if constexpr (MODE == kRealC2R)
    {
        if (c.ok)
            pair_pass<MODE>(M, jt, T, wn, nullptr, 0, [&](int i) { return __ldcs(c.in + i); }, put_lay);
        __syncthreads();
        SchedRun<S>::template go<P, false, true, false, Kind<PassMap::Row, true>>(d, c, lay, M);
    }
    else
    {
        SchedRun<S>::template go<P, true, false, false, Kind<PassMap::Row, false>>(d, c, lay, M);
        if constexpr (MODE == kRealR2C)
        {
            if (c.ok)
                pair_pass<MODE>(
                    M, jt, T, wn, nullptr, 0, [&](int i) { return lay.at(i == M ? 0 : i); },
                    [&](int i, float2 v) { __stcs(c.out + i, make_float2(v.x * c.out_re, v.y * c.out_re)); });
        }
        else
        {
            if (c.ok)
                pair_pass<MODE>(M, jt, T, wn, h, r.smap.estride, [&](int i) { return lay.at(i); }, put_lay);
            __syncthreads();
            SchedRun<S>::template go<P, false, true, false, Kind<PassMap::Row, true>>(d, c, lay, M);
        }
    }
}

// Lengths without a compile-time schedule: staged loads, run-time stages out of place between two line buffers.
template <int MODE>
__global__ void __launch_bounds__(kMaxThreads)
    real_line_dyn_kernel(const PassDesc d, const float2* __restrict__ gin, const float2* __restrict__ spec,
                         const RealLineAux r, float2* __restrict__ gout)
{
    extern __shared__ float2 sm[];
    __shared__ long long s_in_off[kMaxLinesPerCta];
    __shared__ long long s_out_off[kMaxLinesPerCta];
    __shared__ int s_radix[kMaxStages];
    const int M = d.n;
    const int T = (M + 15) / 16;
    const int lpc = blockDim.x / T;
    const int tid = threadIdx.x;
    const int pitch = line_pitch(M);
    const int ll = tid / T;
    const int jt = tid - ll * T;
    const long long line0 = static_cast<long long>(blockIdx.x) * lpc;
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
    const float2* wn = static_cast<const float2*>(r.wn);
    const float2* tw = static_cast<const float2*>(d.tw);
    float2* bufa = sm + ll * pitch;
    float2* bufb = sm + (lpc + ll) * pitch;
    const LayRow<1> la{bufa};
    auto put_a = [&](int i, float2 v) { la.at(i) = conjf2(v); };
    if constexpr (MODE == kRealC2R)
    {
        if (ok)
        {
            const float2* src = gin + s_in_off[ll];
            pair_pass<MODE>(M, jt, T, wn, nullptr, 0, [&](int i) { return __ldcs(src + i); }, put_a);
        }
    }
    else
    {
        tile_load<16>(
            M, lpc, true,
            [&](int a, int e) { return a < lines_here ? __ldcs(gin + s_in_off[a] + e) : make_float2(0.f, 0.f); },
            [&](int a, int e, float2 x) { LayRow<1>{sm + a * pitch}.at(e) = x; });
    }
    __syncthreads();
    float2* x = dyn_stages_pp(s_radix, d.nstages, tw, M, bufa, bufb, jt, T, ok);
    if constexpr (MODE == kRealR2C)
    {
        if (ok)
        {
            const LayRow<1> lx{x};
            float2* dst = gout + s_out_off[ll];
            const float s = d.scale;
            pair_pass<MODE>(
                M, jt, T, wn, nullptr, 0, [&](int i) { return lx.at(i == M ? 0 : i); },
                [&](int i, float2 v) { __stcs(dst + i, make_float2(v.x * s, v.y * s)); });
        }
        return;
    }
    if constexpr (MODE == kRealConv)
    {
        if (ok)
        {
            const LayRow<1> lx{x};
            const float2* h = spec + line_offset(r.smap, line0 + ll, d.lines_per_group);
            pair_pass<MODE>(M, jt, T, wn, h, r.smap.estride, [&](int i) { return lx.at(i); },
                            [&](int i, float2 v) { lx.at(i) = conjf2(v); });
        }
        __syncthreads();
        x = dyn_stages_pp(s_radix, d.nstages, tw, M, x, x == bufa ? bufb : bufa, jt, T, ok);
    }
    // conj(FFT(conj Q)) * scale: the real pairs y[2m], y[2m + 1]
    const float2* tile = x - ll * pitch;
    const float re = d.scale;
    for_tile(M, lpc, true, [&](int a, int e) {
        if (a < lines_here)
        {
            const float2 v = LayRow<1>{const_cast<float2*>(tile) + a * pitch}.at(e);
            __stcs(gout + s_out_off[a] + e, make_float2(v.x * re, -v.y * re));
        }
    });
}

// Row pass + R2C recombination. LP pair slots a CTA: slot j takes rows p = p0 + j (low) and (n1 - p) mod n1
// (high); p runs over 0 .. n1/2 (p = 0 and p = n1/2 pair with themselves). For k = p + n1 k2 the partner is
// M - k = (n1 - p) + n1 (n2 - 1 - k2) for 0 < p < n1/2; within row 0 it is n1 (n2 - k2), within row n1/2 it is
// n1/2 + n1 (n2 - 1 - k2). Consecutive threads take consecutive p, so each store is a run of LP elements.
template <class S, int P, int LP>
__global__ void __launch_bounds__(kStaticThreads, 2)
    row_r2c_kernel(const PassDesc d, const RowR2CDesc r, const float2* __restrict__ ws, float2* __restrict__ out)
{
    extern __shared__ float2 sm[];
    constexpr int N2 = S::n;
    constexpr int T = (N2 + P - 1) / P;
    const int tid = threadIdx.x;
    const int pitch = line_pitch(N2);
    const int half1 = r.n1 / 2;
    const long long blocks_per_t = (half1 + LP) / LP;
    const long long t = blockIdx.x / blocks_per_t;
    const int p0 = static_cast<int>(blockIdx.x - t * blocks_per_t) * LP;
    const int ll = tid / T;
    const int jt = tid - ll * T;
    const int j = ll < LP ? ll : ll - LP;
    const int pj = p0 + j;
    const int row = ll < LP ? pj : (r.n1 - pj) % r.n1;
    Ctx c;
    c.ok = pj <= half1;
    c.q = 0;
    c.in = ws + t * r.M + static_cast<long long>(c.ok ? row : 0) * N2;
    c.out = nullptr;
    c.jt = jt;
    c.T = T;
    init_scales(d, c);
    c.in_im = 1.0f;
    SchedRun<S>::template go<P, true, false, false, Kind<PassMap::Row, false>>(d, c, LayRow<1>{sm + ll * pitch}, N2);
    // the recombination (every line of the CTA is in shared memory)
    float2* ot = out + t * r.odist;
    const float2* wn = static_cast<const float2*>(r.wn);
    const long long M = r.M;
    const float s = r.scale;
    for (int idx = tid; idx < LP * N2; idx += blockDim.x)
    {
        const int jj = idx % LP;
        const int k2 = idx / LP;
        const int p = p0 + jj;
        if (p > half1)
            continue;
        const LayRow<1> lo{sm + jj * pitch};
        const LayRow<1> hi{sm + (LP + jj) * pitch};
        float2 zk, zm;
        long long k;
        if (p == 0)
        {
            if (2 * k2 > N2)
                continue;
            if (k2 == 0)
            {
                const float2 z0 = lo.at(0);
                __stcs(ot, make_float2((z0.x + z0.y) * s, 0.0f));
                __stcs(ot + M, make_float2((z0.x - z0.y) * s, 0.0f));
                continue;
            }
            k = static_cast<long long>(r.n1) * k2;
            zk = lo.at(k2);
            zm = lo.at(N2 - k2);
        }
        else if (2 * p == r.n1)
        {
            if (2 * k2 > N2 - 1)
                continue;
            k = p + static_cast<long long>(r.n1) * k2;
            zk = lo.at(k2);
            zm = lo.at(N2 - 1 - k2);
        }
        else
        {
            k = p + static_cast<long long>(r.n1) * k2;
            zk = lo.at(k2);
            zm = hi.at(N2 - 1 - k2);
        }
        float2 xk, xm;
        r2c_pair(zk, zm, __ldg(wn + k), xk, xm);
        __stcs(ot + k, make_float2(xk.x * s, xk.y * s));
        if (M - k != k)
            __stcs(ot + (M - k), make_float2(xm.x * s, xm.y * s));
    }
}

using RowR2CFn = void (*)(const PassDesc, const RowR2CDesc, const float2*, float2*);

// The row schedules it has: 512-point rows (2^19 = 1024 x 512, R2C of 2^20) and 1024-point rows.
RowR2CFn row_r2c_select(const PassDesc& d, int* P, int* LP)
{
    if (same_radices(d, {16, 8, 4}))
    {
        *P = 32;
        *LP = 8;
        return row_r2c_kernel<Sched<16, 8, 4>, 32, 8>;
    }
    if (same_radices(d, {16, 16, 4}))
    {
        *P = 32;
        *LP = 4;
        return row_r2c_kernel<Sched<16, 16, 4>, 32, 4>;
    }
    return nullptr;
}

using RealFn = void (*)(const PassDesc, const float2*, const float2*, const RealLineAux, float2*);

template <int MODE> RealFn real_select(const PassDesc& d, int P)
{
    if (P == 32)
    {
        if (same_radices(d, {16, 16, 16}))
            return real_line_kernel<Sched<16, 16, 16>, 32, MODE>;
        if (same_radices(d, {32, 32}))
            return real_line_kernel<Sched<32, 32>, 32, MODE>;
        if (same_radices(d, {32, 16, 16}))
            return real_line_kernel<Sched<32, 16, 16>, 32, MODE>;
        return nullptr;
    }
    if (same_radices(d, {16, 4}))
        return real_line_kernel<Sched<16, 4>, 16, MODE>;
    if (same_radices(d, {16, 8}))
        return real_line_kernel<Sched<16, 8>, 16, MODE>;
    if (same_radices(d, {16, 16}))
        return real_line_kernel<Sched<16, 16>, 16, MODE>;
    if (same_radices(d, {16, 8, 4}))
        return real_line_kernel<Sched<16, 8, 4>, 16, MODE>;
    if (same_radices(d, {16, 16, 8}))
        return real_line_kernel<Sched<16, 16, 8>, 16, MODE>;
    if (same_radices(d, {16, 16, 4}))
        return real_line_kernel<Sched<16, 16, 4>, 16, MODE>;
    return real_line_dyn_kernel<MODE>;
}

bool real_is_dynamic(const PassDesc& d, int P)
{
    return P == 16 && !same_radices(d, {16, 4}) && !same_radices(d, {16, 8}) && !same_radices(d, {16, 16}) &&
           !same_radices(d, {16, 8, 4}) && !same_radices(d, {16, 16, 8}) && !same_radices(d, {16, 16, 4});
}

} // namespace
} // namespace lfft

bool real_line_supported(const PassDesc& d)
{
    return d.nstages > 0 && d.n >= 2 && (d.n + 15) / 16 <= lfft::kMaxThreads && d.in.estride == 1 &&
           d.out.estride == 1;
}

bool row_r2c_supported(const PassDesc& row)
{
    int P = 0, LP = 0;
    return lfft::row_r2c_select(row, &P, &LP) != nullptr;
}

cudaError_t launch_row_r2c(const PassDesc& row, const RowR2CDesc& r, const void* ws, void* out,
                           cudaStream_t stream)
{
    int P = 0, LP = 0;
    lfft::RowR2CFn fn = lfft::row_r2c_select(row, &P, &LP);
    if (fn == nullptr || r.n2 != row.n || r.n1 < 2 || (r.n1 & 1) != 0 || r.M != static_cast<long long>(r.n1) * r.n2)
        return cudaErrorInvalidConfiguration;
    const int T = (row.n + P - 1) / P;
    const int threads = T * 2 * LP;
    if (threads > lfft::kStaticThreads)
        return cudaErrorInvalidConfiguration;
    const int smem = 2 * LP * lfft::line_pitch(row.n) * 8;
    const long long blocks = r.batch * ((r.n1 / 2 + LP) / LP);
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
    fn<<<static_cast<unsigned>(blocks), threads, smem, stream>>>(row, r, static_cast<const float2*>(ws),
                                                                 static_cast<float2*>(out));
    return cudaGetLastError();
}

cudaError_t launch_real_line(const PassDesc& d, int mode, const RealLineAux& r, const void* in, const void* spec,
                             void* out, cudaStream_t stream)
{
    int P = 16, lpc = 1, smem = 0;
    conv_shape(d, PassMap::Row, &P, &lpc, &smem);
    lfft::RealFn fn = mode == kRealR2C   ? lfft::real_select<kRealR2C>(d, P)
                      : mode == kRealC2R ? lfft::real_select<kRealC2R>(d, P)
                                         : lfft::real_select<kRealConv>(d, P);
    if (fn == nullptr)
        return cudaErrorInvalidConfiguration;
    if (lfft::real_is_dynamic(d, P))
    {
        smem *= 2; // two line buffers
        if (smem > 227 * 1024)
            return cudaErrorInvalidConfiguration;
    }
    const int T = (d.n + P - 1) / P;
    if (!lfft::real_is_dynamic(d, P) && T * lpc > lfft::kStaticThreads)
        return cudaErrorInvalidConfiguration;
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
                                                                 static_cast<const float2*>(spec), r,
                                                                 static_cast<float2*>(out));
    return cudaGetLastError();
}

} // namespace crdfft
