// Tensor-core line FFT: the first radix-16 stage of each line as a dense GEMM on the 5th-generation tensor cores
// (tcgen05.mma, accumulator in tensor memory), the remaining stages on the FP32 pipes (line_fft.cuh).
//
// A line of n = 16 m points, viewed as X (16 rows x m columns, X[s][j] = x[j + s m]), has its first Stockham stage
// Y = F16 X (y[16 j + r] = Y[r][j]). Real-ified, [Yr; Yi] = [[Fr, -Fi], [Fi, Fr]] [Xr; Xi]: a 32 x 32 real matrix
// times a 32 x (m * lines) real matrix, K = 32. Precision forms:
//
//  * split-BF16: X = X1 + X2 + X3 and F = F1 + F2 + F3 with each term the bf16 rounding of what the previous terms
//    leave, so the three terms carry 24 significant bits. The six products that matter at FP32 accuracy (F1X1, F1X2,
//    F2X1, F1X3, F2X2, F3X1) accumulate in FP32 in one TMEM accumulator: 6 MMAs of K = 32 (12 instructions).
//  * FP16 with a per-line scale: X scaled by a power of two that puts its largest component near 2^14, one term
//    each of F and X in fp16, one MMA (2 instructions); the result is scaled back. About 11 bits: reported, not a
//    1e-6 form.
//  * split-BF16 hi+lo, three products (the two-term form): X = X1 + X2, F = F1 + F2 in bf16, products F1X1, F1X2,
//    F2X1 (3 MMAs of K = 32). About 16 significant bits of the data: reported, not a 1e-6 form.
//  * split-FP16 hi+lo with a per-line scale, three products: X scaled as in the FP16 form, X = X1 + X2 and
//    F = F1 + F2 in fp16 (each second term the fp16 rounding of what the first leaves, about 22 bits together),
//    products F1X1, F1X2, F2X1 in one accumulator. Values more than 2^17 below the line's largest lose bits of their
//    second term to fp16's subnormal range; relative to the line's norm that is below 1e-7.
//
// A (M = 128) holds the same 32 rows four times, so every 32-lane slice of the accumulator holds the whole result and
// each warp drains its own slice (tcgen05.ld): no cross-warp reduction. Operands are K-major, no swizzle: 8 x 16-byte
// core matrices, the two K-halves of a K = 16 slice 128 bytes apart (LBO), 8-row groups 256 bytes apart (SBO).
//
// The kernel waits on one mbarrier (MMA completion) with a bounded poll; a wait that runs out sets the plan's status
// word, and every path frees the tensor memory the CTA allocated.

#include "kernels.hpp"
#include "line_fft.cuh"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cmath>
#include <cstdint>
#include <vector>

namespace crdfft
{
namespace lfft
{
namespace
{

constexpr int kTcThreads = 256;
constexpr int kTcCols = 256; // GEMM N per CTA = m * lines

__device__ __forceinline__ uint64_t umma_desc(uint32_t smem_byte_addr)
{
    // start address >> 4 (bits 0-13), LBO = 128 B (bits 16-29), SBO = 256 B (bits 32-45), version 1 (bits 46-47),
    // base offset 0, layout SWIZZLE_NONE (bits 61-63 = 0)
    uint64_t d = 0;
    d |= static_cast<uint64_t>((smem_byte_addr >> 4) & 0x3FFFu);
    d |= static_cast<uint64_t>(128u >> 4) << 16;
    d |= static_cast<uint64_t>(256u >> 4) << 32;
    d |= static_cast<uint64_t>(1u) << 46;
    return d;
}

// kind::f16 instruction descriptor: F32 accumulate, A/B format (0 f16, 1 bf16), K-major A and B, N, M = 128.
__host__ __device__ constexpr uint32_t umma_idesc(uint32_t ab_format, uint32_t n)
{
    return (1u << 4) | (ab_format << 7) | (ab_format << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

// Byte offset of element (row, k) of a K-major operand with K = 32 stored as two K = 16 slices of rows*32 bytes.
__device__ __forceinline__ uint32_t kmajor_offset(int row, int k, int rows)
{
    const int slice = k >> 4;
    const int kk = k & 15;
    return static_cast<uint32_t>(slice * rows * 32 + (row >> 3) * 256 + (kk >> 3) * 128 + (row & 7) * 16 + (kk & 7) * 2);
}

__device__ __forceinline__ void mma_f16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, bool accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                 "l"(a), "l"(b), "r"(idesc), "r"(accumulate ? 1u : 0u)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float* v)
{
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 8; ++i)
        v[i] = __uint_as_float(r[i]);
}

template <int R0, int... Rest> struct Peel
{
    static constexpr int first = R0;
    template <int P, class K, class Lay>
    __device__ __forceinline__ static void rest(const PassDesc& d, const Ctx& c, const Lay& lay, int n)
    {
        run_static<P, false, true, false, K, R0, 0, Rest...>(d, c, lay, n);
    }
};
template <class S> struct PeelOf;
template <int... Rs> struct PeelOf<Sched<Rs...>>
{
    using type = Peel<Rs...>;
};

// Terms of each operand and the products of a precision form (CRDFFT_PREC_*: 1 split-BF16 three terms, 2 FP16
// scaled, 3 split-BF16 two terms, 4 split-FP16 two terms scaled).
__host__ __device__ constexpr int tc_terms(int prec) { return prec == 1 ? 3 : prec == 2 ? 1 : 2; }
__host__ __device__ constexpr int tc_products(int prec) { return prec == 1 ? 6 : prec == 2 ? 1 : 3; }
__host__ __device__ constexpr bool tc_fp16(int prec) { return prec == 2 || prec == 4; }

template <class S, int PREC, bool EPI>
__global__ void __launch_bounds__(kTcThreads, 2)
    tc_line_kernel(const PassDesc d, const float2* __restrict__ gin, float2* __restrict__ gout,
                   const uint4* __restrict__ amat)
{
    using PS = typename PeelOf<S>::type;
    static_assert(PS::first == 16, "the tensor-core stage is a radix-16 first stage");
    constexpr int N = S::n;
    constexpr int M = N / 16;           // columns per line
    constexpr int LPC = kTcCols / M;    // lines per CTA
    constexpr int T = N / 16;           // FP32 stages: 16 points a thread
    static_assert(T * LPC == kTcThreads, "one GEMM column per thread, one line tile per CTA");
    constexpr int NTERMS = tc_terms(PREC);
    constexpr int A_BYTES = 128 * 32 * 2; // one A operand
    constexpr int B_BYTES = kTcCols * 32 * 2;

    extern __shared__ __align__(1024) unsigned char smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + 16);
    unsigned char* a_s = smem + 1024;
    unsigned char* b_s = a_s + NTERMS * A_BYTES;
    float2* line_s = reinterpret_cast<float2*>(b_s + NTERMS * B_BYTES);
    constexpr int pitch = line_pitch(N);

    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const long long line0 = static_cast<long long>(blockIdx.x) * LPC;

    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(kTcCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    }
    if (tid == 0)
    {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // A operands (precomputed on the host in their shared-memory image)
    for (int i = tid; i < NTERMS * A_BYTES / 16; i += kTcThreads)
        reinterpret_cast<uint4*>(a_s)[i] = __ldg(amat + i);

    // One GEMM column per thread: column c = (line ll, j), K = 32 values Re/Im of x[j + s M], s < 16.
    const int ll = tid / M;
    const int j = tid - ll * M;
    const long long line = line0 + ll;
    const bool ok = line < d.lines;
    const float2* src = gin + line_offset(d.in, ok ? line : line0, d.lines_per_group);
    const float in_im = d.conj_in ? -1.0f : 1.0f;
    float2 x[16];
#pragma unroll
    for (int s = 0; s < 16; ++s)
    {
        float2 v = ok ? __ldcs(src + j + s * M) : make_float2(0.f, 0.f);
        if constexpr (EPI)
            v.y *= in_im;
        x[s] = v;
    }
    __shared__ float s_back[kTcCols];
    float scale_back = 1.0f;
    if constexpr (tc_fp16(PREC))
    {
        // per-line power-of-two scale: the line's largest component near 2^14 (fp16 max 65504)
        float mx = 0.f;
#pragma unroll
        for (int s = 0; s < 16; ++s)
            mx = fmaxf(mx, fmaxf(fabsf(x[s].x), fabsf(x[s].y)));
        for (int o = 16; o > 0; o >>= 1)
            mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        __shared__ float s_max[kTcThreads / 32];
        if (lane == 0)
            s_max[warp] = mx;
        __syncthreads();
        mx = 0.f;
        for (int w = (ll * M) / 32; w < ((ll + 1) * M + 31) / 32 && w < kTcThreads / 32; ++w)
            mx = fmaxf(mx, s_max[w]);
        const int e = mx > 0.f ? 14 - ilogbf(mx) : 0;
        const float sc = ldexpf(1.0f, e);
        scale_back = ldexpf(1.0f, -e);
#pragma unroll
        for (int s = 0; s < 16; ++s)
            x[s] = make_float2(x[s].x * sc, x[s].y * sc);
    }
    s_back[tid] = scale_back; // column tid's scale; every column of a line shares its line's
    // write the B terms (K-major)
#pragma unroll
    for (int t = 0; t < NTERMS; ++t)
    {
        unsigned char* bt = b_s + t * B_BYTES;
#pragma unroll
        for (int k8 = 0; k8 < 4; ++k8)
        {
            uint4 pk;
            uint32_t w[4];
#pragma unroll
            for (int h = 0; h < 4; ++h)
            {
                const int k0 = k8 * 8 + 2 * h; // two K values, k0 and k0 + 1
                float v0 = k0 < 16 ? x[k0].x : x[k0 - 16].y;
                float v1 = (k0 + 1) < 16 ? x[k0 + 1].x : x[k0 + 1 - 16].y;
                uint32_t lo, hi;
                if constexpr (!tc_fp16(PREC))
                {
                    const __nv_bfloat16 b0 = __float2bfloat16_rn(v0);
                    const __nv_bfloat16 b1 = __float2bfloat16_rn(v1);
                    lo = static_cast<uint32_t>(__bfloat16_as_ushort(b0));
                    hi = static_cast<uint32_t>(__bfloat16_as_ushort(b1));
                    // what this term leaves goes to the next term
                    v0 -= __bfloat162float(b0);
                    v1 -= __bfloat162float(b1);
                }
                else
                {
                    const __half h0 = __float2half_rn(v0);
                    const __half h1 = __float2half_rn(v1);
                    lo = static_cast<uint32_t>(__half_as_ushort(h0));
                    hi = static_cast<uint32_t>(__half_as_ushort(h1));
                    v0 -= __half2float(h0);
                    v1 -= __half2float(h1);
                }
                w[h] = lo | (hi << 16);
                // store the remainders back for the next term
                if (k0 < 16)
                    x[k0].x = v0;
                else
                    x[k0 - 16].y = v0;
                if ((k0 + 1) < 16)
                    x[k0 + 1].x = v1;
                else
                    x[k0 + 1 - 16].y = v1;
            }
            pk = make_uint4(w[0], w[1], w[2], w[3]);
            *reinterpret_cast<uint4*>(bt + kmajor_offset(tid, k8 * 8, kTcCols)) = pk;
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (tid == 0)
    {
        const uint32_t a0 = smem_addr(a_s);
        const uint32_t b0 = smem_addr(b_s);
        const uint32_t idesc = umma_idesc(tc_fp16(PREC) ? 0u : 1u, kTcCols);
        // (A term, B term) products: three terms the six that matter at FP32 accuracy, two terms the three, one the one
        constexpr int np = tc_products(PREC);
        const int pa[6] = {0, 0, 1, 0, 1, 2};
        const int pb[6] = {0, 1, 0, 2, 1, 0};
        bool acc = false;
        for (int p = 0; p < np; ++p)
            for (int ks = 0; ks < 2; ++ks)
            {
                const uint64_t da = umma_desc(a0 + pa[p] * A_BYTES + ks * 128 * 32);
                const uint64_t db = umma_desc(b0 + pb[p] * B_BYTES + ks * kTcCols * 32);
                mma_f16(tmem, da, db, idesc, acc);
                acc = true;
            }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(bar))
                     : "memory");
    }
    const bool done = mbar_wait_bounded(bar, 0, d.spin_limit);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!done)
    {
        if (tid == 0 && d.err != nullptr)
            atomicOr(d.err, 1);
        mbar_wait_bounded(bar, 0, d.spin_limit); // let the MMAs finish before the tensor memory is freed
    }
    else
    {
        // Drain: every 32-lane slice holds the whole result (rows: 0-15 Re Y[r], 16-31 Im Y[r]); warp w reads its
        // own slice (lanes 32 (w % 4) ..) for columns [32 w, 32 w + 32). y[16 j + r] of line ll goes to the tile.
        const uint32_t lane_base = static_cast<uint32_t>((warp & 3) * 32) << 16;
        const int c0 = warp * (kTcCols / 8);
        const int r = lane & 15;
        const bool im = lane >= 16;
        for (int cc = 0; cc < kTcCols / 8; cc += 8)
        {
            float v[8];
            tmem_ld8(tmem + lane_base + static_cast<uint32_t>(c0 + cc), v);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int i = 0; i < 8; ++i)
            {
                const int c = c0 + cc + i;
                const int l2 = c / M;
                const int j2 = c - l2 * M;
                float* dst = reinterpret_cast<float*>(&LayRow<1>{line_s + l2 * pitch}.at(16 * j2 + r));
                dst[im ? 1 : 0] = v[i] * s_back[c];
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols));
    if (!done)
        return;

    // Remaining stages on the FP32 pipes, the last one storing to global memory.
    Ctx c;
    c.ok = ok;
    c.q = line_row(d, line);
    c.in = nullptr;
    c.out = gout + line_offset(d.out, ok ? line : line0, d.lines_per_group);
    c.jt = tid - ll * T;
    c.T = T;
    init_scales(d, c);
    c.in_im = 1.0f;
    const LayRow<1> lay{line_s + ll * pitch};
    PS::template rest<16, Kind<PassMap::Row, EPI>>(d, c, lay, N);
}

} // namespace

// Shared memory of a tensor-core pass: barrier/slot page, A and B operand images, the line tile.
int tc_smem_bytes(int n, int prec)
{
    const int terms = tc_terms(prec);
    const int lpc = kTcCols / (n / 16);
    return 1024 + terms * (128 * 32 * 2) + terms * (kTcCols * 32 * 2) + lpc * line_pitch(n) * 8;
}

using TcFn = void (*)(const PassDesc, const float2*, float2*, const uint4*);

template <class S> TcFn tc_pick(int prec, bool epi)
{
    switch (prec)
    {
        case 1: return epi ? tc_line_kernel<S, 1, true> : tc_line_kernel<S, 1, false>;
        case 3: return epi ? tc_line_kernel<S, 3, true> : tc_line_kernel<S, 3, false>;
        case 4: return epi ? tc_line_kernel<S, 4, true> : tc_line_kernel<S, 4, false>;
        default: return epi ? tc_line_kernel<S, 2, true> : tc_line_kernel<S, 2, false>;
    }
}

TcFn tc_select(const PassDesc& d, int prec)
{
    if (same_radices(d, {16, 16, 16}))
        return tc_pick<Sched<16, 16, 16>>(prec, pass_epi(d));
    if (same_radices(d, {16, 8, 4}))
        return tc_pick<Sched<16, 8, 4>>(prec, pass_epi(d));
    if (same_radices(d, {16, 16, 4}))
        return tc_pick<Sched<16, 16, 4>>(prec, pass_epi(d));
    return nullptr;
}

} // namespace lfft

bool tc_pass_supported(const PassDesc& d, int prec)
{
    return prec >= 1 && prec <= 4 && d.in.estride == 1 && d.out.estride == 1 && lfft::tc_select(d, prec) != nullptr;
}

// The A operand images of the real-ified DFT-16 matrix, in the K-major shared-memory layout the kernel copies as is:
// term t of A at bytes [t*8192, (t+1)*8192), rows r (0..127) holding real row r % 32 of [[Fr, -Fi], [Fi, Fr]].
void tc_build_a(int prec, std::vector<uint16_t>* out)
{
    const int terms = lfft::tc_terms(prec);
    out->assign(static_cast<size_t>(terms) * 128 * 32, 0);
    for (int row = 0; row < 128; ++row)
        for (int k = 0; k < 32; ++k)
        {
            const int r32 = row % 32;
            const int rr = r32 & 15, kk = k & 15;
            // F16[rr][kk] = exp(-2πi rr kk / 16)
            const double ang = -6.283185307179586476925286766559 * static_cast<double>((rr * kk) % 16) / 16.0;
            const double fr = std::cos(ang), fi = std::sin(ang);
            double v;
            if (r32 < 16)
                v = k < 16 ? fr : -fi; // Yr = Fr Xr - Fi Xi
            else
                v = k < 16 ? fi : fr;  // Yi = Fi Xr + Fr Xi
            double rem = v;
            for (int t = 0; t < terms; ++t)
            {
                uint16_t bits;
                double q;
                if (!lfft::tc_fp16(prec))
                {
                    const __nv_bfloat16 b = __float2bfloat16_rn(static_cast<float>(rem));
                    bits = __bfloat16_as_ushort(b);
                    q = static_cast<double>(__bfloat162float(b));
                }
                else
                {
                    const __half h = __float2half_rn(static_cast<float>(rem));
                    bits = __half_as_ushort(h);
                    q = static_cast<double>(__half2float(h));
                }
                rem -= q;
                const int slice = k >> 4, kq = k & 15;
                const size_t byte = static_cast<size_t>(t) * 8192 + static_cast<size_t>(slice) * 128 * 32 +
                                    static_cast<size_t>((row >> 3) * 256 + (kq >> 3) * 128 + (row & 7) * 16 + (kq & 7) * 2);
                (*out)[byte / 2] = bits;
            }
        }
}

cudaError_t launch_tc_pass(const PassDesc& d, int prec, const void* amat, const void* in, void* out,
                           cudaStream_t stream)
{
    lfft::TcFn fn = lfft::tc_select(d, prec);
    if (fn == nullptr)
        return cudaErrorInvalidConfiguration;
    const int smem = lfft::tc_smem_bytes(d.n, prec);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess)
        return e;
    const int lpc = lfft::kTcCols / (d.n / 16);
    const long long grid = (d.lines + lpc - 1) / lpc;
    if (grid <= 0)
        return cudaSuccess;
    fn<<<static_cast<unsigned>(grid), lfft::kTcThreads, smem, stream>>>(
        d, static_cast<const float2*>(in), static_cast<float2*>(out), static_cast<const uint4*>(amat));
    return cudaGetLastError();
}

} // namespace crdfft
