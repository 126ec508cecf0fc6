// The column pass of the four-step (n = n1 n2: n1-point DFTs down the columns of each transform's n1 x n2 matrix,
// times the four-step twiddle) as a persistent kernel fed by the Tensor Memory Accelerator.
//
// A tile is 8 adjacent columns of one transform: an n1 x 8 box of the input seen as a [transforms * n1] x n2 matrix
// of 8-byte elements, brought into shared memory by 2-D bulk tensor copies (cp.async.bulk.tensor, boxes of at most
// 256 rows, completion counted in bytes on an mbarrier). Each CTA (one an SM) keeps `nbuf` tiles in flight: while it
// transforms tile i from its buffer, tiles i+1 .. i+nbuf-1 are landing in the others, so the loads of the next
// tiles overlap the arithmetic and the strided 64-byte runs of the column reads are always in flight. The stages are
// the line kernels' (line_fft.cuh) on a column layout of pitch 8; the last stage writes the output straight to global
// memory with the four-step twiddle. No cluster multicast: each CTA loads its own tiles.
//
// Every wait is bounded (the pass's spin limit): a wait that runs out sets the plan's status word, waits (bounded)
// for the copies the CTA still has in flight and returns.
//
// The file also holds the four-step's row pass whose transposed tile leaves by 2-D tensor stores
// (row_tstore_kernel, below): the other half of the four-step, with the Tensor Memory Accelerator on its strided side.

#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdlib>


#include "kernels.hpp"
#include "line_fft.cuh"

namespace crdfft
{
namespace lfft
{
namespace
{

constexpr int kTmaMaxRows = 256; // rows of one copy box
constexpr int kTmaMaxBufs = 8;
constexpr int kSmPerSm = 228 * 1024; // shared memory of an SM; each CTA also takes 1 KiB of it

// Bytes a CTA may give to tile buffers when `ctas` CTAs share an SM (1 KiB reserved a CTA, 1 KiB of alignment slack,
// the barriers).
__host__ __device__ constexpr int tma_buffer_budget(int ctas) { return kSmPerSm / ctas - 2 * 1024 - 64; }

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
                 "[%4];" ::"r"(smem_addr(dst)),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
                 : "memory");
}

// Tile geometry. G = 0: columns a tile 8 (64-byte rows) for 512- and 1024-point columns, so that three tiles fit in
// shared memory, one CTA an SM; 32 columns (256-byte rows) for short columns, whose tiles are small, four CTAs an SM
// so that short columns, with few threads a tile, still keep enough warps resident. G = 1 (CRDFFT_TMA_GEOM=1, long
// columns only): 4 columns a tile (32-byte rows), two CTAs an SM with three tiles each, so that a CTA's barriers stall
// only half the SM's warps.
__host__ __device__ constexpr int tma_cols(int n, int g = 0) { return n <= 256 ? 32 : (g == 1 ? 4 : 8); }
__host__ __device__ constexpr int tma_ctas(int n, int g = 0) { return n <= 256 ? 4 : (g == 1 ? 2 : 1); }

// Bytes between tile buffers: a tile rounded up to 1 KiB (copy destinations 128-byte aligned).
__host__ __device__ constexpr int tma_tile_stride(int n, int g = 0)
{
    return (n * tma_cols(n, g) * 8 + 1023) / 1024 * 1024;
}

int tma_geom()
{
    static const int g = [] {
        const char* e = std::getenv("CRDFFT_TMA_GEOM");
        return e != nullptr && std::atoi(e) == 1 ? 1 : 0;
    }();
    return g;
}

template <class S, int P, int GEOM>
__global__ void __launch_bounds__(((S::n + P - 1) / P) * tma_cols(S::n, GEOM), tma_ctas(S::n, GEOM))
    tma_col_kernel(const __grid_constant__ CUtensorMap map, const PassDesc d, float2* __restrict__ gout, int nbuf,
                   int box_rows, long long tiles)
{
    constexpr int N = S::n;
    constexpr int kTmaCols = tma_cols(N, GEOM);
    constexpr int T = (N + P - 1) / P;
    constexpr int STRIDE = tma_tile_stride(N, GEOM) / 8; // float2 elements between buffers
    extern __shared__ unsigned char smraw[];
    // the buffers from the first 1 KiB boundary of the dynamic shared memory, then the mbarriers and a flag
    const uint32_t base = smem_addr(smraw);
    unsigned char* aligned = smraw + ((1024u - (base & 1023u)) & 1023u);
    float2* bufs = reinterpret_cast<float2*>(aligned);
    uint64_t* bars = reinterpret_cast<uint64_t*>(aligned + static_cast<size_t>(nbuf) * STRIDE * 8);
    int& s_fail = *reinterpret_cast<int*>(bars + nbuf);
    const int tid = threadIdx.x;
    const int jt = tid / kTmaCols; // element group within the column
    const int ll = tid - jt * kTmaCols;
    const long long n2 = d.lines_per_group;
    const long long tiles_per_group = n2 / kTmaCols;
    const long long G = gridDim.x;
    const uint32_t tile_bytes = static_cast<uint32_t>(N) * kTmaCols * 8u;

    auto issue = [&](long long k, int b) {
        const long long grp = idiv(k, tiles_per_group);
        const int q0 = static_cast<int>(k - grp * tiles_per_group) * kTmaCols;
        uint64_t* bar = bars + b;
        mbar_expect_tx(bar, tile_bytes);
        float2* dst = bufs + static_cast<size_t>(b) * STRIDE;
        for (int r0 = 0; r0 < N; r0 += box_rows)
            tma_load_2d(dst + static_cast<size_t>(r0) * kTmaCols, &map, q0, static_cast<int>(grp * N + r0), bar);
    };

    if (tid == 0)
    {
        s_fail = 0;
        for (int b = 0; b < nbuf; ++b)
            mbar_init(bars + b, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fence_proxy_async();
        for (int b = 0; b < nbuf; ++b)
        {
            const long long k = blockIdx.x + b * G;
            if (k < tiles)
                issue(k, b);
        }
    }
    __syncthreads();

    int it = 0;
    for (long long k = blockIdx.x; k < tiles; k += G, ++it)
    {
        const int b = it % nbuf;
        const uint32_t parity = static_cast<uint32_t>(it / nbuf) & 1u;
        const bool ready = mbar_wait_bounded(bars + b, parity, d.spin_limit);
        if (!ready)
            atomicExch(&s_fail, 1);
        __syncthreads();
        if (s_fail)
        {
            // the copies this CTA still has in flight: tiles k .. k + (nbuf-1) G, in buffers b, b+1, ...
            if (tid == 0)
            {
                atomicOr(d.err, 1);
                for (int j = 0; j < nbuf; ++j)
                {
                    const long long kk = k + j * G;
                    if (kk >= tiles)
                        break;
                    const int itj = it + j;
                    mbar_wait_bounded(bars + itj % nbuf, static_cast<uint32_t>(itj / nbuf) & 1u, d.spin_limit);
                }
            }
            __syncthreads();
            return;
        }
        const long long grp = idiv(k, tiles_per_group);
        const long long q0 = (k - grp * tiles_per_group) * kTmaCols;
        const long long line = grp * n2 + q0 + ll;
        Ctx c;
        c.ok = true;
        c.q = idiv(q0 + ll, d.ftw_div);
        c.in = nullptr;
        c.out = gout + line_offset(d.out, line, n2);
        c.jt = jt;
        c.T = T;
        init_scales(d, c);
        const LayCol lay{bufs + static_cast<size_t>(b) * STRIDE + ll, kTmaCols};
        // stages in shared memory (the first applies the input conjugation), the last one stores to global memory
        SchedRun<S>::template go<P, false, true, true, Kind<PassMap::Col, true>>(d, c, lay, N);
        __syncthreads(); // every thread has read buffer b
        if (tid == 0)
        {
            const long long kn = k + nbuf * G;
            if (kn < tiles)
            {
                fence_proxy_async(); // the stages' shared-memory accesses before the copy engine's writes
                issue(kn, b);
            }
        }
    }
}

using TmaFn = void (*)(const CUtensorMap, const PassDesc, float2*, int, int, long long);

TmaFn tma_select(const PassDesc& d, int* P)
{
    // 1024- and 512-point columns at 16 points a thread (512 and 256 threads). Measured slower here, and left to the
    // line kernel: radix-32 stages on this column layout (bank conflicts), 32 points a thread (half the warps).
    const bool narrow = tma_geom() == 1;
    if (same_radices(d, {16, 16, 4}))
    {
        *P = 16;
        return narrow ? tma_col_kernel<Sched<16, 16, 4>, 16, 1> : tma_col_kernel<Sched<16, 16, 4>, 16, 0>;
    }
    if (same_radices(d, {16, 8, 4}))
    {
        *P = 16;
        return narrow ? tma_col_kernel<Sched<16, 8, 4>, 16, 1> : tma_col_kernel<Sched<16, 8, 4>, 16, 0>;
    }
    // 105-point columns (32-column tiles, four CTAs an SM): faster for 3*5*7*4096 (2.86 -> 2.71 ms per 2 GiB),
    // slower for 107520 (2.23 -> 2.36 ms), so only on request (CRDFFT_TMA_SHORT=1)
    if (std::getenv("CRDFFT_TMA_SHORT") != nullptr && same_radices(d, {7, 5, 3}))
    {
        *P = 16;
        return tma_col_kernel<Sched<7, 5, 3>, 16, 0>;
    }
    return nullptr;
}

// ---- row pass with a tensor store --------------------------------------------------------------------------------
//
// The four-step's row pass writes its lines transposed: element e of line q of a group goes to (t n + e) lpg + q, so
// a CTA of lpc lines writes runs of lpc elements, 32 bytes for four lines. Issued by the threads, those stores take
// a quarter of the L1 data pipe's wavefronts and, with the transposed tile read back from shared memory, 40 % of
// the pass's time (measured by leaving the global store out of a copy of the kernel: 0.527 -> 0.319 ms per GiB).
// Here the threads only put the tile into shared memory in the output's order, a dense [n][lpc] block, and one
// thread hands it to the Tensor Memory Accelerator as 2-D stores of at most 256 rows: the copy engine does the
// scattered writes, not the load/store unit.
//
// The stages are the line kernel's (row map, first stage reading HBM directly); every tile is whole (the launch
// checks lines % lpc == 0 and lines_per_group % lpc == 0), so a tile's lines are consecutive lines of one group.

// policy: an L2 eviction policy (evict-first for a pass's output, as the thread-stored kernel's streaming stores):
// the output is not read again soon, and left at normal priority its dirty lines stay in L2 until the next
// operation's traffic pushes them out.
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, int x, int y, const void* src, uint64_t policy)
{
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group.L2::cache_hint [%0, {%1, %2}], [%3], %4;" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(smem_addr(src)), "l"(policy)
                 : "memory");
}

__device__ __forceinline__ uint64_t l2_evict_first_policy()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

template <class S, int P, bool EPI>
__global__ void __launch_bounds__(kMaxThreads, 2)
    row_tstore_kernel(const __grid_constant__ CUtensorMap map, const PassDesc d, const float2* __restrict__ gin)
{
    constexpr int N = S::n;
    constexpr int T = N / P;
    constexpr int BOX = N < 256 ? N : 256; // rows of one store box
    static_assert(N % P == 0 && N % BOX == 0, "whole threads and whole boxes");
    extern __shared__ unsigned char smraw[];
    // the tile from the first 1 KiB boundary of the dynamic shared memory (tensor-copy sources 128-byte aligned)
    float2* sm = reinterpret_cast<float2*>(smraw + ((1024u - (smem_addr(smraw) & 1023u)) & 1023u));
    const int lpc = blockDim.x / T;
    const int tid = threadIdx.x;
    const int pitch = cta_line_pitch(N, lpc);
    const long long line0 = static_cast<long long>(blockIdx.x) * lpc;

    const int ll = tid / T;
    Ctx c;
    c.ok = true;
    c.q = 0;
    c.in = gin + line_offset(d.in, line0 + ll, d.lines_per_group);
    c.out = nullptr;
    c.jt = tid - ll * T;
    c.T = T;
    init_scales(d, c);
    SchedRun<S>::template go<P, true, false, false, Kind<PassMap::Row, EPI>>(d, c, LayRow<1>{sm + ll * pitch}, N);

    // The tile in output order, in place: every thread first reads its P elements (lines fastest across the
    // threads, so a warp reads the same elements of every line: no bank conflict with the staggered line starts),
    // then writes them at e * lpc + a (a warp writes 32 consecutive slots).
    const int a = tid % lpc;
    const int e0 = tid / lpc; // T threads a line: e = e0 + k T covers the line once
    float2 v[P];
#pragma unroll
    for (int k = 0; k < P; ++k)
    {
        const int e = e0 + k * T;
        v[k] = epilogue<EPI>(d, c, 0, e, LayRow<1>{sm + a * pitch}.at(e));
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < P; ++k)
        sm[(e0 + k * T) * lpc + a] = v[k];
    fence_proxy_async(); // these generic writes before the copy engine's reads
    __syncthreads();
    if (tid == 0)
    {
        const long long g = idiv(line0, d.lines_per_group);
        const int x = static_cast<int>(line0 - g * d.lines_per_group);
        const uint64_t policy = l2_evict_first_policy();
#pragma unroll 1
        for (int b = 0; b < N / BOX; ++b)
            tma_store_2d(&map, x, static_cast<int>(g * N + b * BOX), sm + b * BOX * lpc, policy);
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        // the shared memory must outlive the copy engine's reads of it
        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
    }
}

using RowTstoreFn = void (*)(const CUtensorMap, const PassDesc, const float2*);

RowTstoreFn row_tstore_select(const PassDesc& d, bool epi)
{
    if (d.n == 1024 && same_radices(d, {16, 16, 4}))
        return epi ? row_tstore_kernel<Sched<16, 16, 4>, 16, true> : row_tstore_kernel<Sched<16, 16, 4>, 16, false>;
    if (d.n == 512 && same_radices(d, {16, 8, 4}))
        return epi ? row_tstore_kernel<Sched<16, 8, 4>, 16, true> : row_tstore_kernel<Sched<16, 8, 4>, 16, false>;
    return nullptr;
}

PFN_cuTensorMapEncodeTiled_v12000 encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return static_cast<PFN_cuTensorMapEncodeTiled_v12000>(nullptr);
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

} // namespace
} // namespace lfft

// The pass shapes this kernel takes: a column pass (elements n2 apart, adjacent lines adjacent) over packed groups
// of n2 lines (n2 a multiple of 8, the input row of n2 elements a multiple of 16 bytes), a schedule it has, n1 a
// multiple of its box rows.
bool tma_col_supported(const PassDesc& d)
{
    int P = 0;
    if (lfft::tma_select(d, &P) == nullptr)
        return false;
    const long long n2 = d.lines_per_group;
    const int g = lfft::tma_geom();
    if (n2 % lfft::tma_cols(d.n, g) != 0 || d.in.ldist != 1 || d.in.estride != n2 || d.in.gdist != n2 * d.n)
        return false;
    if (d.n > lfft::kTmaMaxRows && d.n % lfft::kTmaMaxRows != 0)
        return false;
    if (d.lines % n2 != 0 || d.lines / n2 * d.n > 0x7fffffffLL)
        return false;
    if (2 * lfft::tma_tile_stride(d.n, g) > lfft::tma_buffer_budget(lfft::tma_ctas(d.n, g))) // two tiles in flight
        return false;
    return lfft::encoder() != nullptr;
}

cudaError_t launch_tma_col(const PassDesc& d, const void* in, void* out, cudaStream_t stream)
{
    int P = 0;
    lfft::TmaFn fn = lfft::tma_select(d, &P);
    if (fn == nullptr || lfft::encoder() == nullptr)
        return cudaErrorInvalidConfiguration;
    const long long n2 = d.lines_per_group;
    const long long groups = d.lines / n2;
    const int box_rows = d.n <= lfft::kTmaMaxRows ? d.n : lfft::kTmaMaxRows;
    if ((reinterpret_cast<uintptr_t>(in) & 15) != 0)
        return cudaErrorInvalidConfiguration;
    CUtensorMap map;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(n2), static_cast<cuuint64_t>(groups * d.n)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(n2) * 8};
    const int g = lfft::tma_geom();
    const int cols = lfft::tma_cols(d.n, g);
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(cols), static_cast<cuuint32_t>(box_rows)};
    const cuuint32_t estr[2] = {1, 1};
    if (lfft::encoder()(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void*>(in), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return cudaErrorInvalidValue; // the tensor map was refused
    const int tile_stride = lfft::tma_tile_stride(d.n, g);
    int nbuf = lfft::tma_buffer_budget(lfft::tma_ctas(d.n, g)) / tile_stride;
    if (nbuf > lfft::kTmaMaxBufs)
        nbuf = lfft::kTmaMaxBufs;
    if (nbuf < 2)
        return cudaErrorInvalidConfiguration;
    const int smem = 1024 + nbuf * tile_stride + nbuf * 8 + 16;
    const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess)
        return e;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long tiles = groups * (n2 / cols);
    long long grid = static_cast<long long>(sms) * lfft::tma_ctas(d.n, g);
    if (grid > tiles)
        grid = tiles;
    if (grid < 1)
        return cudaSuccess;
    const int threads = ((d.n + P - 1) / P) * cols;
    fn<<<static_cast<unsigned>(grid), threads, smem, stream>>>(map, d, static_cast<float2*>(out), nbuf, box_rows,
                                                               tiles);
    return cudaGetLastError();
}

// The row pass with a tensor store: rows read unit-stride (the first stage loads them directly), each group of
// lines_per_group lines written transposed as a [groups * n] x lines_per_group matrix (element e of line q of group
// t at (t n + e) lines_per_group + q), whole tiles of an even number of lines, no four-step twiddle, a schedule the
// kernel has (512 or 1024 points, 16 points a thread).
bool row_tstore_supported(const PassDesc& d, const PassShape& sh)
{
    const int lpc = sh.lines_per_cta;
    const long long lpg = d.lines_per_group;
    if (sh.pipelined || sh.map != PassMap::Row || !sh.direct_load || sh.direct_store || sh.points_per_thread != 16)
        return false;
    if (lpc < 2 || lpc % 2 != 0 || lpc * (d.n / 16) > lfft::kMaxThreads)
        return false;
    if (d.in.estride != 1 || d.out.ldist != 1 || d.out.estride != lpg || d.out.gdist != d.n * lpg || d.ftw_M != 0)
        return false;
    if (lpg % lpc != 0 || d.lines % lpg != 0 || (lpg * 8) % 16 != 0 || d.lines / lpg * d.n > 0x7fffffffLL)
        return false;
    return lfft::row_tstore_select(d, false) != nullptr && lfft::encoder() != nullptr;
}

cudaError_t launch_row_tstore(const PassDesc& d, const PassShape& sh, const void* in, void* out, cudaStream_t stream)
{
    if (!row_tstore_supported(d, sh) || (reinterpret_cast<uintptr_t>(out) & 15) != 0)
        return cudaErrorInvalidConfiguration;
    const bool epi = d.conj_in != 0 || d.conj_out != 0 || d.scale != 1.0f;
    lfft::RowTstoreFn fn = lfft::row_tstore_select(d, epi);
    const int lpc = sh.lines_per_cta;
    const long long lpg = d.lines_per_group;
    const long long groups = d.lines / lpg;
    const int box_rows = d.n < 256 ? d.n : 256;
    CUtensorMap map;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(lpg), static_cast<cuuint64_t>(groups * d.n)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(lpg) * 8};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(lpc), static_cast<cuuint32_t>(box_rows)};
    const cuuint32_t estr[2] = {1, 1};
    if (lfft::encoder()(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, out, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return cudaErrorInvalidValue; // the tensor map was refused
    const int smem = 1024 + lpc * lfft::cta_line_pitch(d.n, lpc) * 8;
    if (smem > 48 * 1024)
    {
        const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess)
            return e;
    }
    const long long grid = d.lines / lpc;
    if (grid > 0x7fffffffLL)
        return cudaErrorInvalidConfiguration;
    fn<<<static_cast<unsigned>(grid), (d.n / 16) * lpc, smem, stream>>>(map, d, static_cast<const float2*>(in));
    return cudaGetLastError();
}

} // namespace crdfft
