// The two-pass four-step as one launch over the whole batch: the column pass and the row pass of every L2-sized wave
// are tiles of one work list, one CTA a tile, each CTA claiming its tile in list order from a device counter when it
// starts (whatever order the hardware starts CTAs in).
//
// The work list (chain_list.hpp), for waves w = 0 .. W-1 of wave_t transforms each (C column tiles and R row tiles
// a wave):
//     col(0) .. col(lag-1) | col(lag) row(0) | col(lag+1) row(1) | ... | [no-op col tiles] row(W-1)
// A row tile of wave w waits until the C column tiles of wave w have signalled; a column tile of wave w >= slots
// waits until the R row tiles of wave w - slots have signalled (the wave's intermediate slot is free again). Both
// waits are on tiles earlier in the list, which were claimed by CTAs already running, so the earliest unfinished
// tile never waits and the list drains whatever the number of resident CTAs. (A persistent loop over tiles, one CTA
// an SM slot, spilled the stages' registers to local memory at every register budget up to 128; one tile a CTA
// compiles like the standalone pass kernels.) Each wait is bounded: when it runs out the CTA ORs 1 into the plan's
// status word, skips the tile's work, and still signals it, so every CTA returns.
//
// The intermediate of wave w lives in workspace slot w mod slots; `slots` waves of it (a few tens of MB) stay in
// L2 between the two passes, and the row pass drops its lines there after reading them (discard_in), so the batch
// moves its algorithmic 16 B a point through HBM in one launch instead of two launches per wave, whose ramps and
// tails (launches of about 20 us each) bounded the wave-by-wave form. The reference's four-step runs the same
// column / twiddle / row steps over its own cache-sized blocks (engine/numerics/hesap-fft/kernels/fft_kernels.cpp:
// 2363-2658).

#include "chain_list.hpp"
#include "kernels.hpp"
#include "line_fft.cuh"

#include <mutex>

namespace crdfft
{
namespace
{

using lfft::Sched;

__device__ __forceinline__ int load_acquire(const int* p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Thread 0 only: wait until *p >= target, at most `limit` polls.
__device__ __forceinline__ bool wait_at_least(const int* p, int target, int limit)
{
    for (int i = 0; i < limit; ++i)
    {
        if (load_acquire(p) >= target)
            return true;
        __nanosleep(128);
    }
    return false;
}

template <class SC, int PC, class SR, int PR, bool REPI>
__global__ void __maxnreg__(80) chain_fft_kernel(const ChainDesc cd, const float2* __restrict__ src,
                                                 float2* __restrict__ dst, float2* ws)
{
    __shared__ int s_item, s_ok;
    const int tid = threadIdx.x;
    if (tid == 0)
        s_item = atomicAdd(cd.ctr, 1);
    __syncthreads();
    const int t = s_item;
    const int C = static_cast<int>(cd.col_items);
    const int R = static_cast<int>(cd.row_items);
    const int W = static_cast<int>(cd.waves);
    const ChainTile tile = chain_tile_at(t, C, R, cd.lag);
    const bool is_col = tile.col;
    const int w = tile.wave;
    const int idx = tile.idx;
    if (w >= W)
        return; // a no-op column tile past the last wave (the list's tail holds row tiles only)
    int* const col_done = cd.ctr + 1;
    int* const row_done = cd.ctr + 1 + W;
    if (tid == 0)
    {
        bool ok = true;
        // (test hook: with the plan's debug stall set, a row tile waits for one column tile more than exist, so that
        // the wait runs out without any fault)
        if (!is_col)
            ok = wait_at_least(col_done + w, C + (cd.col.debug_stall ? 1 : 0), cd.spin_limit);
        else if (w >= cd.slots)
            ok = wait_at_least(row_done + (w - cd.slots), R, cd.spin_limit);
        if (!ok && cd.col.err != nullptr)
            atomicOr(cd.col.err, 1);
        s_ok = ok ? 1 : 0;
    }
    __syncthreads();
    if (s_ok)
    {
        const long long t0 = static_cast<long long>(w) * cd.wave_t;
        const long long wt = cd.batch - t0 < cd.wave_t ? cd.batch - t0 : cd.wave_t;
        float2* slot = ws + static_cast<long long>(w % cd.slots) * cd.slot_elems;
        if (is_col)
            lfft::line_fft_tile<SC, PC, PassMap::Col, true, true, true>(cd.col, src + t0 * cd.idist, slot, idx,
                                                                        cd.col_lpc, wt * cd.row.n, tid);
        else
            lfft::line_fft_tile<SR, PR, PassMap::Row, true, false, REPI>(cd.row, slot, dst + t0 * cd.odist, idx,
                                                                         cd.row_lpc, wt * cd.col.n, tid);
    }
    // Every thread's stores of the tile are issued; one release makes them visible before the tile's signal.
    __syncthreads();
    if (tid == 0)
    {
        __threadfence();
        atomicAdd(is_col ? col_done + w : row_done + w, 1);
    }
}

using ChainFn = void (*)(const ChainDesc, const float2*, float2*, float2*);

template <class SC, int PC, class SR, int PR> ChainFn pick(bool repi)
{
    return repi ? chain_fft_kernel<SC, PC, SR, PR, true> : chain_fft_kernel<SC, PC, SR, PR, false>;
}

bool radices_are(const PassDesc& d, std::initializer_list<int> rs)
{
    return lfft::same_radices(d, rs);
}

// The column / row schedule pairs with a chained instance (points a thread 16 on both sides).
ChainFn select(const PassDesc& col, const PassDesc& row)
{
    const bool repi = lfft::pass_epi(row);
    if (radices_are(row, {16, 16, 4}))
    {
        if (radices_are(col, {7, 5, 3}))
            return pick<Sched<7, 5, 3>, 16, Sched<16, 16, 4>, 16>(repi); // 107520 = 105 x 1024
        if (radices_are(col, {16, 16, 4}))
            return pick<Sched<16, 16, 4>, 16, Sched<16, 16, 4>, 16>(repi); // 2^20 = 1024 x 1024
        if (radices_are(col, {16, 8, 4}))
            return pick<Sched<16, 8, 4>, 16, Sched<16, 16, 4>, 16>(repi); // 2^19 = 512 x 1024
        if (radices_are(col, {16, 4}))
            return pick<Sched<16, 4>, 16, Sched<16, 16, 4>, 16>(repi); // 65536 = 64 x 1024
    }
    if (radices_are(row, {16, 8, 4}) && radices_are(col, {16, 16, 4}))
        return pick<Sched<16, 16, 4>, 16, Sched<16, 8, 4>, 16>(repi); // 2^19 = 1024 x 512
    return nullptr;
}

} // namespace

bool chain_supported(const PassDesc& col, const PassDesc& row)
{
    if (select(col, row) == nullptr)
        return false;
    // the column tile reads and writes across adjacent lines; the row tile reads unit-stride rows
    return col.in.ldist == 1 && col.out.ldist == 1 && row.in.estride == 1 && row.ftw_M == 0 && col.ftw_M != 0;
}

int chain_smem_bytes(int n1, int n2)
{
    const int l1 = chain_lines_per_tile(n1);
    const int l2 = chain_lines_per_tile(n2);
    const int a = l1 * lfft::cta_line_pitch(n1, l1) * 8;
    const int b = l2 * lfft::cta_line_pitch(n2, l2) * 8;
    return a > b ? a : b;
}

cudaError_t launch_chain(const ChainDesc& cd, const void* in, void* out, void* ws, cudaStream_t stream)
{
    const ChainFn fn = select(cd.col, cd.row);
    if (fn == nullptr || cd.waves < 1 || cd.col_items < 1 || cd.row_items < 1 || cd.lag < 1 || cd.slots <= cd.lag)
        return cudaErrorInvalidConfiguration;
    const int smem = chain_smem_bytes(cd.col.n, cd.row.n);
    static std::mutex mu;
    {
        std::lock_guard<std::mutex> lk(mu);
        const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess)
            return e;
    }
    const long long total = chain_list_length(cd.waves, cd.col_items, cd.row_items, cd.lag);
    if (total >= 0x7fffffffLL)
        return cudaErrorInvalidConfiguration;
    const long long grid = total;
    fn<<<static_cast<unsigned>(grid), kChainThreads, smem, stream>>>(cd, static_cast<const float2*>(in),
                                                                      static_cast<float2*>(out),
                                                                      static_cast<float2*>(ws));
    return cudaGetLastError();
}

} // namespace crdfft
