// The planner and the C ABI (include/crdfft.h). A plan is a list of steps per direction, each a kernel launch with
// its buffers named symbolically (the caller's input, the caller's output, the plan's workspace). The planner is the
// deterministic plan-from-size rule of the reference (include/crd/hesap/fft/fft.hpp:3-8, 112-210): no runtime
// measurement here; the same descriptor always builds the same steps, and execution uses no atomics, so a plan is
// bit-identical run to run.
//
//   n <= 16384 (a line fits one CTA's shared memory)  one pass, one HBM read and one write per element
//   larger 7-smooth n                                 four-step n = n1 * n2: pass 1 column FFTs of length n1 with
//                                                     the W_n^{n2 k1} twiddle fused into the store, pass 2 row FFTs
//                                                     of length n2 with the transposed store; the batch runs in
//                                                     waves whose intermediate fits in L2 (the reference's Bailey
//                                                     four-step, kernels/fft_kernels.cpp:2363-2658)
//   n with a prime factor above 7                     Bluestein chirp-z over a power-of-two plan (bluestein.hpp)
//   R2C / C2R                                         half-length complex plan + recombine pass (real_fft.hpp)
//   rank 2 / 3                                        one pass per axis, inverse by the conjugation trick
//                                                     (nd_fft.hpp:105-147)

#include "../../include/crdfft.h"
#include "kernels.hpp"
#include "pass_desc.hpp"
#include "tuner.hpp"
#include "learned.hpp"
#include "uneven.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

namespace crdfft
{
namespace
{

constexpr int kMaxSmemBytes = 200 * 1024;

std::atomic<int> g_fail_alloc_after{0};
thread_local Arena* t_arena = nullptr; // plan memory comes from this arena instead of cudaMalloc when set
std::atomic<int> g_debug_stall{0};
constexpr int kSpinLimit = 1 << 22; // bounded waits: about a second of try_wait polling
constexpr int kMaxLanes = 4;       // internal streams a plan may run L2-sized four-step waves on

cudaError_t dev_alloc(void** p, size_t bytes)
{
    if (t_arena != nullptr)
    {
        const size_t need = (bytes == 0 ? 256 : bytes + 255) / 256 * 256;
        if (t_arena->used + need > t_arena->size)
        {
            *p = nullptr;
            return cudaErrorMemoryAllocation;
        }
        *p = t_arena->base + t_arena->used;
        t_arena->used += need;
        return cudaSuccess;
    }
    int k = g_fail_alloc_after.load();
    if (k > 0)
    {
        if (k == 1)
        {
            g_fail_alloc_after.store(0);
            *p = nullptr;
            return cudaErrorMemoryAllocation;
        }
        g_fail_alloc_after.store(k - 1);
    }
    return cudaMalloc(p, bytes == 0 ? 256 : bytes);
}

enum class Buf : int
{
    In,
    Out,
    Ws
};

struct BufRef
{
    Buf b = Buf::In;
    long long off = 0; // in complex (8-byte) elements
};

enum class StepKind : int
{
    Line,
    Cluster,
    TcLine,
    Conv,
    RealLine,
    RowR2C,
    Spectral,
    WelchFinish,
    TmaCol,
    Zero,
    R2CPost,
    C2RPre,
    ChirpPre,
    SpecMul,
    ChirpPost,
    Scale,
    Chain
};

struct Step
{
    StepKind kind = StepKind::Line;
    PassDesc pass{};
    PassDesc pass2{}; // Cluster: the row phase
    int prec = 0;     // TcLine: 1 split-BF16, 2 FP16 scaled
    const void* amat = nullptr;
    PassShape shape{};
    LineMap smap{};   // Conv: where each line's filter spectrum sits
    int rmode = 0;    // RealLine: kRealR2C, kRealC2R or kRealConv
    RealLineAux raux{};
    SpectralDesc sdesc{}; // Spectral, WelchFinish
    RowR2CDesc rr{};      // RowR2C
    int sthreads = 0, ssmem = 0;
    int lane = 0;     // 0: the caller's stream; 1 .. kMaxLanes: the plan's internal streams (L2-sized four-step waves)
    RealRecombine real{};
    ChirpDesc chirp{};
    ChainDesc chain{};  // Chain: the persistent four-step; aux is its first workspace slot, counters after the slots
    BufRef aux{};
    BufRef src, dst;
    long long count = 0;
    float scale = 1.0f;
};

// 7-smooth test and the radix schedule: powers of two as 16s with an 8, 4 or 2 for the remainder, then 7s, 5s, 3s.
// With use32, the lengths where a radix-32 schedule measured faster as a unit-stride single pass take it (one
// exchange through shared memory fewer): 1024 = 32 32 (66 -> 94 % of HBM), 8192 = 32 16 16. (512, 16384 and 32 were
// slower with radix-32 stages, and so were the strided passes of the four-step.)
// group25: pairs of 5s as radix-25 stages (off for the uneven kernel, whose inlined stages run out of registers with
// a 25-point butterfly: 3.57 -> 3.72 ms for its 20,000-transform batch, where the line kernels gain 7-18 %).
bool radices_for(long long n, std::vector<int>& out, bool use32 = false, bool group25 = true)
{
    out.clear();
    if (n < 1)
        return false;
    if (use32)
    {
        switch (n)
        {
            case 1024: out = {32, 32}; return true;
            case 8192: out = {32, 16, 16}; return true;
            default: break;
        }
    }
    long long m = n;
    int twos = 0;
    while (m % 2 == 0)
    {
        m /= 2;
        ++twos;
    }
    std::vector<int> odd;
    for (int p : {7, 5, 3})
        while (m % p == 0)
        {
            m /= p;
            odd.push_back(p);
        }
    if (m != 1)
        return false;
    // pairs of 5s as radix-25 stages and pairs of 3s as radix-9 stages (one exchange through shared memory fewer
    // each), each before the odd one left over
    if (group25 && std::getenv("CRDFFT_NO_RADIX25") == nullptr)
    {
        std::vector<int> grouped;
        size_t i = 0;
        while (i < odd.size() && odd[i] == 7)
            grouped.push_back(odd[i++]);
        int fives = 0;
        while (i < odd.size() && odd[i] == 5)
        {
            ++fives;
            ++i;
        }
        for (int k = 0; k < fives / 2; ++k)
            grouped.push_back(25);
        if (fives % 2)
            grouped.push_back(5);
        while (i < odd.size())
            grouped.push_back(odd[i++]);
        odd.swap(grouped);
    }
    int threes = 0;
    while (!odd.empty() && odd.back() == 3)
    {
        odd.pop_back();
        ++threes;
    }
    for (int i = 0; i < threes / 2; ++i)
        odd.push_back(9);
    if (threes % 2)
        odd.push_back(3);
    const int a = twos / 4, b = twos % 4;
    if (b == 1 && a >= 1)
    {
        for (int i = 0; i < a - 1; ++i)
            out.push_back(16);
        out.push_back(8);
        out.push_back(4);
    }
    else
    {
        for (int i = 0; i < a; ++i)
            out.push_back(16);
        if (b == 1)
            out.push_back(2);
        else if (b == 2)
            out.push_back(4);
        else if (b == 3)
            out.push_back(8);
    }
    for (int p : odd)
        out.push_back(p);
    return true;
}

bool is_smooth(long long n)
{
    std::vector<int> r;
    return radices_for(n, r);
}

// Line lengths one pass transforms: every 7-smooth n up to 8192, and 16384.
bool single_pass_ok(long long n) { return n >= 1 && (n <= 8192 || n == 16384) && is_smooth(n); }

bool has_static_schedule(long long n, bool use32 = false)
{
    std::vector<int> rad;
    if (!radices_for(n, rad, use32) || static_cast<int>(rad.size()) > kMaxStages)
        return false;
    PassDesc d{};
    d.n = static_cast<int>(n);
    d.nstages = static_cast<int>(rad.size());
    for (size_t i = 0; i < rad.size(); ++i)
        d.radix[i] = rad[i];
    return pass_has_static(d, 16) || pass_has_static(d, 32);
}

// The four-step split n = n1 * n2 (pass 1 transforms the n2 columns of length n1, pass 2 the n1 rows of length n2),
// both halves within one CTA. Preference, in order: both halves have compile-time schedules (e.g. 107520 = 105 x
// 1024); n2 a multiple of 16, so pass 1's column tiles stay whole; closest to square.
bool four_step_split(long long n, long long* n1, long long* n2)
{
    long long best1 = 0, best2 = 0;
    double best_score = 1e300;
    for (long long d = 1; d * d <= n; ++d)
    {
        if (n % d != 0)
            continue;
        const long long other = n / d;
        if (!single_pass_ok(d) || !single_pass_ok(other))
            continue;
        const bool stat = has_static_schedule(d) && has_static_schedule(other);
        for (int o = 0; o < 2; ++o)
        {
            const long long a = o ? d : other; // n1
            const long long b = o ? other : d; // n2
            const double score = (stat ? 0.0 : 1e6) + (b % 16 != 0 ? 10.0 : 0.0) +
                                 std::fabs(std::log(static_cast<double>(a) / static_cast<double>(b)));
            if (score < best_score)
            {
                best_score = score;
                best1 = a;
                best2 = b;
            }
        }
    }
    if (best1 == 0)
        return false;
    *n1 = best1;
    *n2 = best2;
    return true;
}

struct Plan
{
    crdfft_desc desc{};
    int device = 0;
    std::vector<Step> steps[2];
    std::vector<void*> tables;
    std::map<long long, void*> tw_by_n;
    long long table_bytes = 0;
    size_t ws_bytes = 0;
    void* ws = nullptr;
    bool ws_owned = false;
    std::string algorithm;
    std::vector<long long> factors;
    long long split_n1 = 0; // the column length of the last two-pass four-step planned for this plan
    int split_kind = 0;     // the last 1-D decomposition planned: 1 one pass, 2 cluster, 3 two-pass four-step
    int* err = nullptr; // device word the pipelined kernels flag a given-up wait in
    const void* tc_amat = nullptr; // tensor-core DFT-16 operand image for the plan's precision
    int tc_steps = 0;
    // FftPlan::execute_batched sub-plans, one per batch value used (element-major layout).
    std::map<long long, Plan*> batched;
    std::mutex batched_mu;
    int api_kind = 0; // 0 general, 1 FftPlan, 2 RealFftPlan, 3 BluesteinPlan, 4 NdFftPlan
    bool arena_backed = t_arena != nullptr; // device memory belongs to an arena: nothing to free
    // Uneven batch: the work list descriptor, its shared memory, and one instantiated graph per (in, out, direction)
    bool uneven = false;
    UnevenDesc udesc{};
    int usmem = 0;
    std::map<std::tuple<const void*, void*, int>, cudaGraphExec_t> graphs;
    std::mutex graphs_mu;
    // Host-buffer execute (crdfft_execute_host): chunk plans, staging buffers and streams, made by the first call.
    // Host-memory execute: a three-stage pipeline over chunks of the batch, each stage on its own stream (copy in,
    // transform, copy out) and kHostSlots buffer slots, so that both copy engines stay busy while the transforms run.
    static constexpr int kHostSlots = 3;
    struct HostPipe
    {
        long long chunk = 0;             // transforms a chunk
        Plan* full = nullptr;            // plan of `chunk` transforms
        Plan* tail = nullptr;            // plan of the last, shorter chunk (or null)
        void* din[kHostSlots] = {};
        void* dout[kHostSlots] = {};
        cudaStream_t st[3] = {nullptr, nullptr, nullptr}; // copy in, transform, copy out
        cudaEvent_t loaded[kHostSlots] = {};   // a slot's input is on the device
        cudaEvent_t computed[kHostSlots] = {}; // a slot's transform is done (its input is free, its output ready)
        cudaEvent_t drained[kHostSlots] = {};  // a slot's output is back on the host (its output buffer is free)
        cudaEvent_t start = nullptr;           // the caller's stream at the call
    };
    HostPipe* host = nullptr;
    std::mutex host_mu;
    // Split-complex execute (crdfft_execute_planar): the interleaved staging buffer, made by the first call.
    void* planar = nullptr;
    std::mutex planar_mu;
    bool conv = false; // fused convolution plan (crdfft_conv_plan_create): executes with a filter spectrum
    bool spectral = false; // spectral estimator plan (crdfft_spectral_plan_create)
    // Radix-32 schedules for the lengths that have them (FP32 unit-stride passes); off for the tensor-core precision
    // forms and the uneven batch, whose kernels take the radix-16 schedules.
    bool use32 = true;
    // Internal streams for steps with lane 1 .. kMaxLanes, forked from and joined back to the caller's stream.
    cudaStream_t lanes[kMaxLanes] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[kMaxLanes] = {};

    ~Plan()
    {
        if (host != nullptr)
        {
            for (cudaStream_t st : host->st)
                if (st != nullptr)
                {
                    cudaStreamSynchronize(st);
                    cudaStreamDestroy(st);
                }
            for (int i = 0; i < kHostSlots; ++i)
            {
                cudaFree(host->din[i]);
                cudaFree(host->dout[i]);
                for (cudaEvent_t e : {host->loaded[i], host->computed[i], host->drained[i]})
                    if (e != nullptr)
                        cudaEventDestroy(e);
            }
            if (host->start != nullptr)
                cudaEventDestroy(host->start);
            delete host->full;
            delete host->tail;
            delete host;
        }
        for (auto& kv : graphs)
            cudaGraphExecDestroy(kv.second);
        for (int i = 0; i < kMaxLanes; ++i)
        {
            if (lanes[i] != nullptr)
                cudaStreamDestroy(lanes[i]);
            if (join[i] != nullptr)
                cudaEventDestroy(join[i]);
        }
        if (fork != nullptr)
            cudaEventDestroy(fork);
        if (planar != nullptr)
            cudaFree(planar);
        for (auto& kv : batched)
            delete kv.second;
        if (arena_backed)
            return;
        for (void* p : tables)
            cudaFree(p);
        if (ws_owned && ws != nullptr)
            cudaFree(ws);
    }
};

// The tables are uploaded with cudaMemcpy and the status word cleared with cudaMemset, both on the legacy default
// stream: a pageable-memory cudaMemcpy may return before its DMA lands and cudaMemset does not wait at all, and a
// caller's non-blocking stream is not ordered after the legacy stream. So plan creation waits for the legacy stream
// before it hands out a plan; an execute on any stream then reads finished tables.
bool uploads_landed() { return cudaStreamSynchronize(cudaStreamLegacy) == cudaSuccess; }

crdfft_status upload_table(Plan& p, const std::vector<float>& host, void** dev)
{
    const size_t bytes = host.size() * sizeof(float);
    void* d = nullptr;
    if (dev_alloc(&d, bytes) != cudaSuccess)
        return CRDFFT_OOM;
    p.tables.push_back(d);
    p.table_bytes += static_cast<long long>(bytes);
    if (cudaMemcpy(d, host.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        return CRDFFT_LAUNCH;
    *dev = d;
    return CRDFFT_OK;
}

// W_n^k = exp(-2πik/n), computed in extended precision and rounded to FP64; the callers narrow it to FP32 (the
// reference's convention, fft.hpp:253-260). The angle is reduced to at most π/4 with exact integer arithmetic
// (k mod n, octant of 8k/n), and the quarter turns are applied by exact swaps and negations, so the table is exact at
// the quarter points and symmetric.
void root(long long k, long long n, double* re, double* im)
{
    k %= n;
    if (k < 0)
        k += n;
    const long double quarter_pi = 0.78539816339744830961566084581987572L;
    const unsigned __int128 num = static_cast<unsigned __int128>(k) * 8u;
    const long long oct = static_cast<long long>(num / static_cast<unsigned __int128>(n));
    const long long rem = static_cast<long long>(num - static_cast<unsigned __int128>(oct) * n);
    long double c, s;
    long long quarters;
    if ((oct & 1) == 0)
    {
        const long double th = quarter_pi * static_cast<long double>(rem) / static_cast<long double>(n);
        c = std::cos(th);
        s = std::sin(th);
        quarters = oct / 2;
    }
    else
    {
        const long double th = quarter_pi * static_cast<long double>(n - rem) / static_cast<long double>(n);
        c = std::cos(th);
        s = -std::sin(th);
        quarters = (oct + 1) / 2;
    }
    long double cr = c, sr = s;
    switch (quarters & 3)
    {
        case 0: cr = c; sr = s; break;
        case 1: cr = -s; sr = c; break;
        case 2: cr = -c; sr = -s; break;
        default: cr = s; sr = -c; break;
    }
    *re = static_cast<double>(cr);
    *im = static_cast<double>(-sr);
}

// The stage-ordered twiddle table of a line length n with the planner's radix schedule: for each stage after the
// first (radix R, after radices multiplying to L), W_{LR}^{r k} = W_n^{r k n/(L R)} at (r-1) L + k. Each entry is
// computed in FP64 and narrowed once (fft.hpp:251-260).
crdfft_status twiddle_table(Plan& p, long long n, const void** out, bool r32 = false, bool group25 = true)
{
    // one table per (length, schedule family)
    const long long key = n | (r32 ? (1LL << 48) : 0) | (group25 ? 0 : (1LL << 49));
    auto it = p.tw_by_n.find(key);
    if (it != p.tw_by_n.end())
    {
        *out = it->second;
        return CRDFFT_OK;
    }
    std::vector<int> rad;
    if (!radices_for(n, rad, r32, group25))
        return CRDFFT_UNSUPPORTED_SIZE;
    std::vector<float> h;
    long long L = 1;
    for (int R : rad)
    {
        if (L > 1)
            for (int r = 1; r < R; ++r)
                for (long long k = 0; k < L; ++k)
                {
                    double re, im;
                    root(static_cast<long long>(r) * k * (n / (L * R)), n, &re, &im);
                    h.push_back(static_cast<float>(re));
                    h.push_back(static_cast<float>(im));
                }
        L *= R;
    }
    if (h.empty())
        h.assign(2, 0.0f);
    void* d = nullptr;
    const crdfft_status st = upload_table(p, h, &d);
    if (st != CRDFFT_OK)
        return st;
    p.tw_by_n[key] = d;
    *out = d;
    return CRDFFT_OK;
}

// A classic launch shape with P points a thread and `lpc` lines a CTA (0: the default for the map).
PassShape shape_with(long long n, int nstages, PassMap map, bool dl, bool ds, int P, int lpc = 0)
{
    PassShape sh{};
    sh.map = map;
    sh.direct_load = dl;
    sh.direct_store = ds;
    sh.points_per_thread = P;
    const int T = static_cast<int>((n + P - 1) / P);
    sh.threads_per_line = T;
    // the compile-time-schedule kernel's pitch (at least the run-time kernel's, which sizes its own two buffers)
    auto tile_bytes = [&](int l) { return l * pass_cta_line_pitch(static_cast<int>(n), l) * 8; };
    if (lpc <= 0)
        lpc = map == PassMap::Row ? std::max(1, 256 / T) : std::max(1, 512 / T);
    lpc = std::min(lpc, pass_lines_per_cta_limit());
    while (lpc > 1 && lpc * T > pass_threads_limit(P, n))
        --lpc;
    const bool needs_smem = !(dl && ds && nstages == 1);
    while (needs_smem && lpc > 1 && tile_bytes(lpc) > kMaxSmemBytes)
        --lpc;
    sh.lines_per_cta = lpc;
    sh.smem_bytes = needs_smem ? tile_bytes(lpc) : 0;
    return sh;
}

// The pipelined (persistent, bulk-copy) shape when the pass qualifies: a compile-time schedule with a pipelined
// instance, 16 points a thread, and 16-byte aligned, 16-byte multiple copies: rows of even length with even line
// offsets (row map), or tiles of an even number of adjacent columns inside one group with even strides (column map).
bool pipe_shape(const PassDesc& d, PassMap map, PassShape* out, int want_lpc = 0)
{
    const int P = 16;
    const int T = (d.n + P - 1) / P;
    if (T > pass_pipe_threads())
        return false;
    PassShape sh{};
    sh.pipelined = true;
    sh.map = map;
    sh.points_per_thread = P;
    sh.threads_per_line = T;
    sh.direct_load = false;
    int lpc = want_lpc > 0 ? want_lpc : pass_pipe_threads() / T;
    if (lpc * T > pass_pipe_threads())
        return false;
    if (map == PassMap::Row)
    {
        if (d.in.estride != 1 || (d.n & 1) != 0 || (d.in.gdist & 1) != 0)
            return false;
        if (d.lines_per_group > 1 && (d.in.ldist & 1) != 0)
            return false;
        lpc = std::max(1, std::min<int>(lpc, static_cast<int>(std::min<long long>(d.lines, 256))));
        sh.direct_store = d.out.estride == 1;
    }
    else
    {
        if (d.in.ldist != 1 || d.lines_per_group < 2 || (d.in.estride & 1) != 0 || (d.in.gdist & 1) != 0)
            return false;
        lpc &= ~1;
        while (lpc >= 2 && (d.lines_per_group % lpc != 0 || d.lines % lpc != 0))
            lpc -= 2;
        if (lpc < 4)
            return false;
        sh.direct_store = d.out.ldist == 1;
    }
    sh.lines_per_cta = lpc;
    sh.smem_bytes = pass_pipe_smem(d.n, map, lpc);
    if (sh.smem_bytes > 110 * 1024 || !pass_has_kernel(d, sh))
        return false;
    *out = sh;
    return true;
}

// The heuristic launch shape of a pass (the planner's estimate when no measurement decides): the classic kernel,
// 16 points a thread, or 32 where a compile-time schedule exists for it (lines longer than 8192, and long columns,
// which then keep 4+ adjacent lines a CTA for 32-byte coalesced segments).
bool heuristic_shape(const PassDesc& d, PassMap map, bool dl, bool ds, PassShape* out)
{
    if (std::getenv("CRDFFT_PIPELINE") != nullptr && pipe_shape(d, map, out))
        return true;
    const bool want32 = d.n > 8192 || (map == PassMap::Col && d.n >= 2048);
    if (want32)
    {
        const PassShape sh = shape_with(d.n, d.nstages, map, dl, ds, 32);
        if (sh.threads_per_line * sh.lines_per_cta <= pass_threads_limit(sh.points_per_thread, d.n) && pass_has_kernel(d, sh))
        {
            *out = sh;
            return true;
        }
    }
    // A compile-time schedule first, at either thread width (the radix-32 schedules exist at 32 points a thread
    // only: without this order 1024 and 8192 took the run-time kernel at 16 points a thread, 4x slower for 1024),
    // then the run-time schedule. A four-step row pass the tensor-store kernel takes goes to it (its transposed
    // store is 40 % of the thread-stored pass's time).
    for (int pass = 0; pass < 2; ++pass)
        for (int P : {16, 32})
        {
            PassShape sh = shape_with(d.n, d.nstages, map, dl, ds, P);
            if (sh.threads_per_line * sh.lines_per_cta > pass_threads_limit(P, d.n))
                continue;
            if (pass == 0 ? pass_has_static(d, P) : pass_has_kernel(d, sh))
            {
                PassShape t = sh;
                t.tma_store = true;
                if (pass == 0 && row_tstore_supported(d, t))
                {
                    t.smem_bytes = 1024 + t.lines_per_cta * pass_cta_line_pitch(d.n, t.lines_per_cta) * 8;
                    sh = t;
                }
                *out = sh;
                return true;
            }
        }
    return false;
}

// Every launch shape the planner can measure for a pass: classic at 16 and 32 points a thread with one, two or
// four times the default lines a CTA, and the pipelined kernel at its default and half lines a CTA.
std::vector<PassShape> candidate_shapes(const PassDesc& d, PassMap map, bool dl, bool ds)
{
    std::vector<PassShape> out;
    auto add = [&](const PassShape& sh) {
        if (sh.threads_per_line * sh.lines_per_cta >
            (sh.pipelined ? pass_pipe_threads() : pass_threads_limit(sh.points_per_thread, d.n)))
            return;
        if (!pass_has_kernel(d, sh))
            return;
        for (const PassShape& o : out)
            if (o.pipelined == sh.pipelined && o.points_per_thread == sh.points_per_thread &&
                o.lines_per_cta == sh.lines_per_cta && o.wide_regs == sh.wide_regs && o.tma_store == sh.tma_store)
                return;
        out.push_back(sh);
        if (!sh.pipelined && sh.points_per_thread == 16 && pass_has_static(d, 16))
        {
            PassShape w = sh;
            w.wide_regs = true; // the same shape on the 80-register build
            out.push_back(w);
        }
        PassShape t = sh;
        t.tma_store = true; // a four-step row pass whose transposed tile leaves by tensor stores
        if (!sh.pipelined && row_tstore_supported(d, t))
        {
            t.smem_bytes = 1024 + t.lines_per_cta * pass_cta_line_pitch(d.n, t.lines_per_cta) * 8;
            out.push_back(t);
        }
    };
    for (int P : {16, 32})
    {
        const int T = (d.n + P - 1) / P;
        const int base = map == PassMap::Row ? std::max(1, 256 / T) : std::max(1, 512 / T);
        for (int mul : {1, 2, 4})
        {
            const int lpc = std::max(1, base * mul / 2);
            add(shape_with(d.n, d.nstages, map, dl, ds, P, lpc));
        }
    }
    PassShape ps;
    if (pipe_shape(d, map, &ps))
        add(ps);
    if (pipe_shape(d, map, &ps, std::max(1, (pass_pipe_threads() / ((d.n + 15) / 16)) / 2)))
        add(ps);
    return out;
}

int learned_top_k();
int learned_top_k_shapes();
bool tma_col_enabled();

// The planner's choice of launch shape for a pass: remembered wisdom for its geometry class if any; else, in
// measure mode, the fastest of the timed candidates (remembered); else the heuristic.
bool choose_shape(const PassDesc& d, PassMap map, bool dl, bool ds, PassShape* out)
{
    const std::string key = pass_key(d, map, dl, ds);
    WisdomEntry w;
    if (wisdom_lookup(key, &w))
    {
        PassShape sh;
        if (w.pipelined ? pipe_shape(d, map, &sh, w.lines_per_cta)
                        : (sh = shape_with(d.n, d.nstages, map, dl, ds, w.points_per_thread, w.lines_per_cta),
                           sh.wide_regs = w.wide_regs, sh.tma_store = w.tma_store,
                           sh.threads_per_line * sh.lines_per_cta <= pass_threads_limit(sh.points_per_thread, d.n) &&
                               pass_has_kernel(d, sh)))
        {
            *out = sh;
            return true;
        }
    }
    const int mode = planner_mode();
    if (mode == kPlannerLearned && learned_ready())
    {
        // The model ranks the candidates; its top proposals (learned_top_k) are then timed and the fastest is kept
        // and remembered: the measuring planner judges what the model proposes. From an arena (nothing may be
        // allocated) or with a top-k of 1, the model's first choice stands untimed.
        const std::vector<PassShape> cands = candidate_shapes(d, map, dl, ds);
        std::vector<std::pair<float, int>> ranked;
        for (size_t i = 0; i < cands.size(); ++i)
        {
            float f[kPassFeatures];
            pass_features(d, cands[i], f);
            ranked.emplace_back(learned_predict(f), static_cast<int>(i));
        }
        std::sort(ranked.begin(), ranked.end());
        const int k = std::min<int>(learned_top_k_shapes(), static_cast<int>(ranked.size()));
        if (k >= 2 && t_arena == nullptr)
        {
            std::vector<PassShape> top;
            for (int i = 0; i < k; ++i)
                top.push_back(cands[ranked[i].second]);
            std::vector<float> ms;
            const int best = measure_shapes(d, key, top, &ms, 0);
            if (best >= 0)
            {
                WisdomEntry e;
                e.pipelined = top[best].pipelined;
                e.points_per_thread = top[best].points_per_thread;
                e.lines_per_cta = top[best].lines_per_cta;
                e.wide_regs = top[best].wide_regs;
                e.tma_store = top[best].tma_store;
                e.ms = ms[best];
                wisdom_store(key, e);
                *out = top[best];
                return true;
            }
        }
        if (!ranked.empty())
        {
            *out = cands[ranked[0].second];
            return true;
        }
    }
    if (mode == kPlannerMeasure && t_arena == nullptr) // measuring allocates scratch: never from an arena
    {
        const std::vector<PassShape> cands = candidate_shapes(d, map, dl, ds);
        std::vector<float> ms;
        int heur = -1;
        PassShape hs;
        if (heuristic_shape(d, map, dl, ds, &hs))
            for (size_t i = 0; i < cands.size(); ++i)
                if (cands[i].pipelined == hs.pipelined && cands[i].points_per_thread == hs.points_per_thread &&
                    cands[i].lines_per_cta == hs.lines_per_cta)
                    heur = static_cast<int>(i);
        const int best = measure_shapes(d, key, cands, &ms, heur);
        if (best >= 0)
        {
            WisdomEntry e;
            e.pipelined = cands[best].pipelined;
            e.points_per_thread = cands[best].points_per_thread;
            e.lines_per_cta = cands[best].lines_per_cta;
            e.wide_regs = cands[best].wide_regs;
            e.tma_store = cands[best].tma_store;
            e.ms = ms[best];
            wisdom_store(key, e);
            *out = cands[best];
            return true;
        }
    }
    return heuristic_shape(d, map, dl, ds, out);
}

// How many of the learned models' top proposals the measuring planner times: decompositions (whole executes,
// CRDFFT_LEARNED_TOP_K, default 2) and launch shapes (single passes, CRDFFT_LEARNED_TOP_K_SHAPES, default 1: the
// shape model's first choice is taken untimed, its error is small and a pass timing costs as much as the ranking
// saves).
int env_top_k(const char* name, int dflt)
{
    const char* e = std::getenv(name);
    const int v = e != nullptr ? std::atoi(e) : dflt;
    return v < 1 ? 1 : v;
}
int learned_top_k()
{
    static const int k = env_top_k("CRDFFT_LEARNED_TOP_K", 2);
    return k;
}
int learned_top_k_shapes()
{
    static const int k = env_top_k("CRDFFT_LEARNED_TOP_K_SHAPES", 1);
    return k;
}

// ---- Decomposition of a 1-D transform --------------------------------------------------------------------------
//
// kind 1: one pass (n <= 8192, or 16384); 2: the cluster four-step (one launch, DSMEM transpose); 3: the two-pass
// four-step with columns of n1 and rows of n / n1. The rule (estimate mode) is the size rule of the plan's header;
// measure mode times every candidate on the device (a plan of a sample of the batch with that decomposition forced,
// executed cold); learned mode ranks the candidates with the decomposition model and times only its top proposals.
// The choice is remembered as decomposition wisdom.
struct Decomp
{
    int kind = 0;
    long long n1 = 0;
};

thread_local const Decomp* t_forced = nullptr; // the decomposition a timing plan is built with
thread_local long long t_forced_n = 0;
std::mutex g_hint_mu;
std::map<long long, Decomp> g_hints; // crdfft_set_decomposition: per-length overrides

bool cluster_ok(const Plan& p, long long n, long long istride, long long idist, long long ostride, long long odist)
{
    long long a = 0, b = 0;
    return istride == 1 && ostride == 1 && idist == n && odist == n && std::getenv("CRDFFT_NO_CLUSTER") == nullptr &&
           p.desc.precision == CRDFFT_PREC_FP32 && cluster_split(n, &a, &b);
}

Decomp rule_decomp(const Plan& p, long long n, long long istride, long long idist, long long ostride, long long odist)
{
    if (single_pass_ok(n))
        return Decomp{1, 0};
    if (cluster_ok(p, n, istride, idist, ostride, odist))
        return Decomp{2, 0};
    long long n1 = 0, n2 = 0;
    if (four_step_split(n, &n1, &n2))
        return Decomp{3, n1};
    return Decomp{0, 0};
}

bool decomp_valid(const std::vector<Decomp>& cands, const Decomp& d)
{
    for (const Decomp& c : cands)
        if (c.kind == d.kind && (c.kind != 3 || c.n1 == d.n1))
            return true;
    return false;
}

std::vector<Decomp> decomp_candidates(const Plan& p, long long n, long long istride, long long idist,
                                      long long ostride, long long odist)
{
    std::vector<Decomp> out;
    if (single_pass_ok(n))
        out.push_back(Decomp{1, 0});
    if (cluster_ok(p, n, istride, idist, ostride, odist))
        out.push_back(Decomp{2, 0});
    // Four-step splits: those whose two line lengths both have compile-time schedules, and the four splits closest
    // to square among the others (run on the run-time schedule); the rule's own split is always among them.
    if (n >= 2048 && n < (1LL << 31))
    {
        std::vector<std::pair<double, long long>> other;
        for (long long a = 16; a * 16 <= n; ++a)
        {
            if (n % a != 0 || !single_pass_ok(a) || !single_pass_ok(n / a))
                continue;
            if (has_static_schedule(a) && has_static_schedule(n / a))
                out.push_back(Decomp{3, a});
            else
                other.emplace_back(std::fabs(std::log(static_cast<double>(a) * a / static_cast<double>(n))), a);
        }
        std::sort(other.begin(), other.end());
        for (size_t i = 0; i < other.size() && i < 4; ++i)
            out.push_back(Decomp{3, other[i].second});
        long long r1 = 0, r2 = 0;
        if (four_step_split(n, &r1, &r2) && !decomp_valid(out, Decomp{3, r1}))
            out.push_back(Decomp{3, r1});
    }
    return out;
}

void radix_list(long long n, std::vector<int>& r)
{
    r.clear();
    radices_for(n, r);
}

void decomp_feature_vector(const Plan& p, long long n, const Decomp& c, long long batch, bool packed_unit,
                           bool padded, float* f)
{
    std::vector<int> r1, r2;
    const long long a = c.kind == 3 ? c.n1 : n;
    const long long b = c.kind == 3 ? n / c.n1 : 1;
    radix_list(a, r1);
    if (b > 1)
        radix_list(b, r2);
    const bool tma = c.kind == 3 && tma_col_enabled() && b % 8 == 0 && (a == 1024 || a == 512);
    decomp_features(n, c.kind, c.n1, batch, packed_unit, padded, p.desc.precision, r1.data(),
                    static_cast<int>(r1.size()), r2.data(), static_cast<int>(r2.size()), has_static_schedule(a),
                    b > 1 && has_static_schedule(b), tma, f);
}

struct ConvReq;
crdfft_status create(const crdfft_desc* desc, Plan** out, const ConvReq* conv, const crdfft_spectral_desc* spec);
void destroy_plan(Plan* p) { delete p; }
crdfft_status run(Plan& p, const void* in, void* out, int dir, cudaStream_t stream, const void* spec);

// Times one decomposition: a plan of `sample` transforms of the same layout with `c` forced, executed cold; the
// time is scaled to the whole batch. Negative when the plan could not be built or run.
float time_decomp(const Plan& p, long long n, const Decomp& c, long long batch, long long sample, long long istride,
                  long long idist, long long ostride, long long odist)
{
    crdfft_desc d{};
    d.rank = 1;
    d.kind = CRDFFT_C2C;
    d.precision = p.desc.precision;
    d.norm = CRDFFT_NORM_NONE;
    d.dims[0] = n;
    d.batch = sample;
    d.istride = istride;
    d.idist = idist;
    d.ostride = ostride;
    d.odist = odist;
    const Decomp* prev = t_forced;
    const long long prev_n = t_forced_n;
    t_forced = &c;
    t_forced_n = n;
    Plan* tp = nullptr;
    const crdfft_status st = create(&d, &tp, nullptr, nullptr);
    t_forced = prev;
    t_forced_n = prev_n;
    if (st != CRDFFT_OK)
        return -1.0f;
    const long long in_ext = (sample - 1) * idist + (n - 1) * istride + 1;
    const long long out_ext = (sample - 1) * odist + (n - 1) * ostride + 1;
    void* in = nullptr;
    void* outb = nullptr;
    float ms = -1.0f;
    if (cudaMalloc(&in, static_cast<size_t>(in_ext) * 8) == cudaSuccess &&
        cudaMalloc(&outb, static_cast<size_t>(out_ext) * 8) == cudaSuccess &&
        cudaMemset(in, 0, static_cast<size_t>(in_ext) * 8) == cudaSuccess)
    {
        auto go = [&](cudaStream_t s) {
            return run(*tp, in, outb, CRDFFT_FORWARD, s, nullptr) == CRDFFT_OK ? cudaSuccess : cudaErrorLaunchFailure;
        };
        ms = time_cold(go);
        if (ms > 0.0f)
            ms *= static_cast<float>(static_cast<double>(batch) / static_cast<double>(sample));
    }
    cudaGetLastError();
    cudaFree(in);
    cudaFree(outb);
    destroy_plan(tp);
    return ms;
}

Decomp choose_decomp(const Plan& p, long long n, long long batch, long long istride, long long idist,
                     long long ostride, long long odist, bool fused_r2c)
{
    if (t_forced != nullptr && t_forced_n == n)
        return *t_forced;
    const Decomp rule = rule_decomp(p, n, istride, idist, ostride, odist);
    const std::vector<Decomp> cands = decomp_candidates(p, n, istride, idist, ostride, odist);
    {
        std::lock_guard<std::mutex> lk(g_hint_mu);
        auto it = g_hints.find(n);
        if (it != g_hints.end())
        {
            const Decomp& h = it->second;
            const bool ok = (h.kind == 1 && single_pass_ok(n)) ||
                            (h.kind == 2 && cluster_ok(p, n, istride, idist, ostride, odist)) ||
                            (h.kind == 3 && h.n1 >= 2 && n % h.n1 == 0 && single_pass_ok(h.n1) &&
                             single_pass_ok(n / h.n1));
            if (ok)
                return h;
        }
    }
    if (fused_r2c || p.desc.precision != CRDFFT_PREC_FP32 || cands.size() <= 1 || t_forced != nullptr)
        return rule;
    const bool packed_unit = istride == 1 && ostride == 1 && idist == n && odist == n;
    const bool padded = (idist != n && idist % 16 != 0) || (odist != n && odist % 16 != 0);
    const std::string key = decomp_key(n, batch, packed_unit, padded, p.desc.precision);
    DecompEntry w;
    if (decomp_lookup(key, &w) && decomp_valid(cands, Decomp{w.kind, w.n1}))
        return Decomp{w.kind, w.n1};
    const int mode = planner_mode();
    if (mode == kPlannerEstimate || t_arena != nullptr)
        return rule;
    // the candidates to time: all of them (measure, or learned without a decomposition model), or the model's top k
    std::vector<std::pair<float, Decomp>> order;
    for (const Decomp& c : cands)
    {
        float f[kPassFeatures];
        decomp_feature_vector(p, n, c, batch, packed_unit, padded, f);
        order.emplace_back(mode == kPlannerLearned && learned_decomp_ready() ? learned_decomp_predict(f) : 0.0f, c);
    }
    size_t k = order.size();
    if (mode == kPlannerLearned && learned_decomp_ready())
    {
        std::stable_sort(order.begin(), order.end(),
                         [](const std::pair<float, Decomp>& a, const std::pair<float, Decomp>& b) {
                             return a.first < b.first;
                         });
        k = std::min<size_t>(k, static_cast<size_t>(learned_top_k()));
        if (k == 1)
            return order[0].second;
    }
    // a sample of kPlannerSampleBytes of input (two buffers of it must fit beside the device's current use)
    size_t free_b = 0, total_b = 0;
    const bool roomy = cudaMemGetInfo(&free_b, &total_b) == cudaSuccess &&
                       free_b > static_cast<size_t>(4 * kPlannerSampleBytes);
    cudaGetLastError();
    const long long sample_bytes = roomy ? kPlannerSampleBytes : kPlannerSmallSampleBytes;
    const long long sample = std::max(1LL, std::min(batch, sample_bytes / (8 * n)));
    int best = -1;
    std::vector<float> ms(k, -1.0f);
    for (size_t i = 0; i < k; ++i)
    {
        ms[i] = time_decomp(p, n, order[i].second, batch, sample, istride, idist, ostride, odist);
        if (ms[i] > 0.0f && (best < 0 || ms[i] < ms[best]))
            best = static_cast<int>(i);
    }
    for (size_t i = 0; i < k; ++i)
    {
        const Decomp& c = order[i].second;
        float f[kPassFeatures];
        decomp_feature_vector(p, n, c, batch, packed_unit, padded, f);
        char buf[256];
        std::snprintf(buf, sizeof(buf), "%s decomp kind=%d n1=%lld batch=%lld ms=%.6f", key.c_str(), c.kind, c.n1,
                      batch, static_cast<double>(ms[i]));
        std::string line = buf;
        line += " feat=";
        for (int j = 0; j < kPassFeatures; ++j)
        {
            std::snprintf(buf, sizeof(buf), j ? ",%.6g" : "%.6g", static_cast<double>(f[j]));
            line += buf;
        }
        if (static_cast<int>(i) == best)
            line += " best";
        if (c.kind == rule.kind && c.n1 == (rule.kind == 3 ? rule.n1 : c.n1))
            line += " heur";
        planner_log_append(line);
    }
    if (best < 0)
        return rule;
    decomp_store(key, DecompEntry{order[best].second.kind, order[best].second.n1, ms[best]});
    return order[best].second;
}

// Four-step twiddle of a pass (pass 1 of the four-step), or none.
struct FourStepTw
{
    long long M = 0;
    int div = 1; // twiddle row = (line index within its group) / div
    const void* hi = nullptr;
    const void* lo = nullptr;
};

// The descriptor of a line pass (no launch shape yet).
crdfft_status make_pass_desc(Plan& p, long long n, long long lines, long long lpg, LineMap in, LineMap out,
                             bool conj_in, bool conj_out, float scale, const FourStepTw& ftw, PassDesc* out_desc)
{
    std::vector<int> rad;
    // radix-32 schedules for unit-stride passes only (the single passes); CRDFFT_R32_ROWS=1 also for passes that
    // read unit-stride rows and store with a stride (the four-step's row pass)
    static const bool r32_rows = std::getenv("CRDFFT_R32_ROWS") != nullptr && std::atoi(std::getenv("CRDFFT_R32_ROWS")) != 0;
    const bool r32 = p.use32 && in.estride == 1 && (out.estride == 1 || r32_rows);
    if (!single_pass_ok(n) || !radices_for(n, rad, r32) || static_cast<int>(rad.size()) > kMaxStages)
        return CRDFFT_UNSUPPORTED_SIZE;
    PassDesc d{};
    d.n = static_cast<int>(n);
    d.nstages = static_cast<int>(rad.size());
    for (size_t i = 0; i < rad.size(); ++i)
        d.radix[i] = rad[i];
    d.lines = lines;
    d.lines_per_group = lpg;
    d.in = in;
    d.out = out;
    const crdfft_status st = twiddle_table(p, n, &d.tw, r32);
    if (st != CRDFFT_OK)
        return st;
    d.ftw_M = ftw.M;
    d.ftw_div = ftw.div > 0 ? ftw.div : 1;
    d.discard_in = 0;
    d.ftw_hi = ftw.hi;
    d.ftw_lo = ftw.lo;
    d.err = p.err;
    d.debug_stall = g_debug_stall.load();
    d.spin_limit = d.debug_stall ? (1 << 14) : kSpinLimit;
    d.conj_in = conj_in ? 1 : 0;
    d.conj_out = conj_out ? 1 : 0;
    d.scale = scale;
    *out_desc = d;
    return CRDFFT_OK;
}

crdfft_status make_line_step(Plan& p, long long n, long long lines, long long lpg, LineMap in, LineMap out,
                             BufRef src, BufRef dst, bool conj_in, bool conj_out, float scale, Step* step,
                             const FourStepTw& ftw = FourStepTw{})
{
    Step s;
    s.kind = StepKind::Line;
    PassDesc& d = s.pass;
    const crdfft_status st = make_pass_desc(p, n, lines, lpg, in, out, conj_in, conj_out, scale, ftw, &d);
    if (st != CRDFFT_OK)
        return st;
    // Thread map: along the elements when the loading side is unit-stride, across lines when adjacent lines are
    // adjacent in memory (columns); the store side decides for the rest.
    PassMap map;
    if (in.estride == 1)
        map = PassMap::Row;
    else if (in.ldist == 1 && lpg > 1)
        map = PassMap::Col;
    else if (out.ldist == 1 && lpg > 1 && out.estride != 1)
        map = PassMap::Col;
    else
        map = PassMap::Row;
    bool dl, ds;
    if (map == PassMap::Row)
    {
        dl = in.estride == 1;
        ds = out.estride == 1;
    }
    else
    {
        dl = in.ldist == 1 && lpg > 1;
        ds = out.ldist == 1 && lpg > 1;
    }
    if (d.nstages == 0) // n == 1: no butterflies; the pass is a copy with the epilogue, staged through smem
        dl = ds = false;
    // Row lines of 32 points or fewer: one or two threads a line, so a direct load or store would touch a separate
    // 128-byte line per thread; staged through shared memory the CTA's accesses are contiguous.
    if (map == PassMap::Row && n <= 32)
        dl = ds = false;
    const int prec = p.desc.precision;
    if (prec != CRDFFT_PREC_FP32 && tc_pass_supported(d, prec))
    {
        // the first radix-16 stage on the tensor cores (tc_fft.cu); other passes of the plan stay FP32
        if (p.tc_amat == nullptr)
        {
            std::vector<uint16_t> img;
            tc_build_a(prec, &img);
            std::vector<float> as_float(img.size() / 2);
            std::memcpy(as_float.data(), img.data(), img.size() * sizeof(uint16_t));
            void* dev = nullptr;
            const crdfft_status st2 = upload_table(p, as_float, &dev);
            if (st2 != CRDFFT_OK)
                return st2;
            p.tc_amat = dev;
        }
        s.kind = StepKind::TcLine;
        s.prec = prec;
        s.amat = p.tc_amat;
        s.src = src;
        s.dst = dst;
        ++p.tc_steps;
        *step = s;
        return CRDFFT_OK;
    }
    if (!choose_shape(d, map, dl, ds, &s.shape))
        return CRDFFT_UNSUPPORTED_SIZE;
    s.src = src;
    s.dst = dst;
    *step = s;
    return CRDFFT_OK;
}

// Four-step twiddle tables for pass 1 (columns of length n1, n2 of them): hi[a n1 + e] = W_M^{16 a e} for
// a < ceil(n2/16), lo[16 e + b] = W_M^{b e} for b < 16, e < n1 (exact FP64 roots, narrowed).
crdfft_status four_step_tables(Plan& p, long long M, long long n1, long long n2, const void** hi, const void** lo)
{
    const long long na = (n2 + 15) / 16;
    std::vector<float> th(static_cast<size_t>(2 * na * n1)), tl(static_cast<size_t>(2 * 16 * n1));
    for (long long a = 0; a < na; ++a)
        for (long long e = 0; e < n1; ++e)
        {
            double re, im;
            root(16 * a * e, M, &re, &im);
            th[static_cast<size_t>(2 * (a * n1 + e))] = static_cast<float>(re);
            th[static_cast<size_t>(2 * (a * n1 + e) + 1)] = static_cast<float>(im);
        }
    for (long long e = 0; e < n1; ++e)
        for (long long b = 0; b < 16; ++b)
        {
            double re, im;
            root(b * e, M, &re, &im);
            tl[static_cast<size_t>(2 * (16 * e + b))] = static_cast<float>(re);
            tl[static_cast<size_t>(2 * (16 * e + b) + 1)] = static_cast<float>(im);
        }
    void* dh = nullptr;
    void* dl = nullptr;
    crdfft_status st = upload_table(p, th, &dh);
    if (st != CRDFFT_OK)
        return st;
    st = upload_table(p, tl, &dl);
    if (st != CRDFFT_OK)
        return st;
    *hi = dh;
    *lo = dl;
    return CRDFFT_OK;
}

long long wave_bytes()
{
    if (t_arena != nullptr) // half of an arena holds the intermediate; tables and the status word use the rest
        return static_cast<long long>(t_arena->size / 2);
    const char* e = std::getenv("CRDFFT_WAVE_BYTES");
    if (e != nullptr)
    {
        const long long v = std::atoll(e);
        if (v > 0)
            return v;
    }
    return 512LL << 20;
}

// The four-step column pass on the tensor-copy kernel (tma_col.cu) where it applies (1024- and 512-point columns:
// 2^20 2.68 -> 2.39 ms, 2^19 2.54 -> 2.19 ms per 2 GiB); CRDFFT_TMA_COL=0 keeps the line kernel.
bool tma_col_enabled()
{
    const char* e = std::getenv("CRDFFT_TMA_COL");
    return e == nullptr || std::atoi(e) != 0;
}

// L2 waves run round-robin over this many internal streams and workspace slots (CRDFFT_L2_LANES, 2 .. kMaxLanes).
// Two measured best for 107520 (2.170 ms per 2 GiB; three lanes 2.286 with 24 MiB waves, 2.172 with 16 MiB, four
// 2.422): more than about 48 MiB of waves in flight pushes the intermediates out of L2.
int l2_lanes()
{
    const char* e = std::getenv("CRDFFT_L2_LANES");
    const int v = e != nullptr ? std::atoi(e) : 2;
    return v < 2 ? 2 : (v > kMaxLanes ? kMaxLanes : v);
}

// The L2 wave's row pass drops the intermediate's L2 lines once it has read them (CRDFFT_L2_DISCARD=0: kept, and
// written back to HBM when L2 evicts them). Read at plan creation.
bool l2_discard()
{
    const char* e = std::getenv("CRDFFT_L2_DISCARD");
    return e == nullptr || std::atoi(e) != 0;
}

// Four-step waves sized for L2 on two internal streams (CRDFFT_L2_WAVES=1) or one large wave at a time (=0).
bool l2_waves()
{
    static const bool on = [] {
        const char* e = std::getenv("CRDFFT_L2_WAVES");
        return e == nullptr || std::atoi(e) != 0;
    }();
    return on;
}

// The L2 wave size and the largest transform (bytes) that takes L2 waves; CRDFFT_L2_WAVE_BYTES and
// CRDFFT_L2_WAVE_MAX_TRANSFORM override them.
long long env_bytes(const char* name, long long dflt)
{
    const char* e = std::getenv(name);
    if (e != nullptr)
    {
        const long long v = std::atoll(e);
        if (v > 0)
            return v;
    }
    return dflt;
}
long long l2_wave_bytes()
{
    static const long long v = env_bytes("CRDFFT_L2_WAVE_BYTES", 24LL << 20);
    return v;
}
long long l2_wave_max_transform()
{
    static const long long v = env_bytes("CRDFFT_L2_WAVE_MAX_TRANSFORM", 2LL << 20);
    return v;
}

// The four-step as one persistent launch over L2-sized waves (chain_fft.cu) where an instance exists for its two
// line lengths (CRDFFT_CHAIN=1 on, 0 off); its wave size (CRDFFT_CHAIN_WAVE_BYTES) and number of intermediate slots
// in flight (CRDFFT_CHAIN_SLOTS, 3 .. 8; a wave's row tiles trail its column tiles by slots / 2 waves).
bool chain_enabled()
{
    const char* e = std::getenv("CRDFFT_CHAIN");
    return e != nullptr && std::atoi(e) != 0;
}
long long chain_wave_bytes() { return env_bytes("CRDFFT_CHAIN_WAVE_BYTES", 16LL << 20); }
int chain_slots()
{
    const char* e = std::getenv("CRDFFT_CHAIN_SLOTS");
    const int v = e != nullptr ? std::atoi(e) : 4;
    return v < 3 ? 3 : (v > 8 ? 8 : v);
}

// A batch of 1-D complex transforms of length n: element j of transform t at base + t*dist + j*stride on each side.
// Appends the steps of one direction; `ws_off` is where in the workspace this transform's scratch may start; the
// scratch it needs is returned in *ws_need (complex elements).
// r2c_wn: the half-length transform of an R2C plan (wn = W_{2n}^k, k = 0 .. n): where the four-step's row pass has a
// fused form, it also recombines the pairs and writes the n + 1 values of each real transform's spectrum (odist
// apart); *r2c_fused tells the caller whether it did.
crdfft_status plan_c2c_1d(Plan& p, long long n, long long batch, long long istride, long long idist,
                          long long ostride, long long odist, BufRef src, BufRef dst, bool conj_in, bool conj_out,
                          float scale, long long ws_off, std::vector<Step>& steps, long long* ws_need,
                          const void* r2c_wn = nullptr, bool* r2c_fused = nullptr)
{
    if (r2c_fused != nullptr)
        *r2c_fused = false;
    *ws_need = 0;
    const Decomp dc = choose_decomp(p, n, batch, istride, idist, ostride, odist, r2c_wn != nullptr);
    if (dc.kind == 0)
        return CRDFFT_UNSUPPORTED_SIZE;
    p.split_kind = dc.kind;
    if (dc.kind == 1)
    {
        LineMap in{idist, 0, istride};
        LineMap out{odist, 0, ostride};
        long long lpg = 1;
        if (idist == 1 && odist == 1 && batch > 1)
        {
            // element-major batch: lines are adjacent in memory
            in = LineMap{0, 1, istride};
            out = LineMap{0, 1, ostride};
            lpg = batch;
        }
        Step s;
        const crdfft_status st =
            make_line_step(p, n, batch, lpg, in, out, src, dst, conj_in, conj_out, scale, &s);
        if (st != CRDFFT_OK)
            return st;
        steps.push_back(s);
        return CRDFFT_OK;
    }
    long long n1 = 0, n2 = 0;
    if (dc.kind == 2 && cluster_split(n, &n1, &n2))
    {
        // One cluster per transform: columns of n1, DSMEM transpose with the four-step twiddle, rows of n2. The
        // twiddle W_n^{j k1} (column j, row k1) is factored like the two-pass four-step's, hi[(j>>4) n1 + k1] times
        // lo[16 k1 + (j&15)]: two tables of 32 KiB that stay in L1, where one full 512 KiB table was read from L2
        // between the cluster barriers.
        Step s;
        s.kind = StepKind::Cluster;
        const void* hi = nullptr;
        const void* lo = nullptr;
        crdfft_status st = four_step_tables(p, n, n1, n2, &hi, &lo);
        if (st != CRDFFT_OK)
            return st;
        FourStepTw ftw;
        ftw.M = n;
        ftw.hi = hi;
        ftw.lo = lo;
        st = make_pass_desc(p, n1, batch * n2, n2, LineMap{n, 1, n2}, LineMap{n, 1, n2}, conj_in, false, 1.0f, ftw,
                            &s.pass);
        if (st != CRDFFT_OK)
            return st;
        st = make_pass_desc(p, n2, batch * n1, n1, LineMap{n, n2, 1}, LineMap{n, 1, n1}, false, conj_out, scale,
                            FourStepTw{}, &s.pass2);
        if (st != CRDFFT_OK)
            return st;
        s.count = batch;
        s.src = src;
        s.dst = dst;
        steps.push_back(s);
        return CRDFFT_OK;
    }
    if (dc.kind != 3 || dc.n1 < 2 || n % dc.n1 != 0)
        return CRDFFT_UNSUPPORTED_SIZE;
    n1 = dc.n1;
    n2 = n / n1;
    p.split_n1 = n1;
    const void* hi = nullptr;
    const void* lo = nullptr;
    if (n >= (1LL << 31))
        return CRDFFT_UNSUPPORTED_SIZE;
    crdfft_status st = four_step_tables(p, n, n1, n2, &hi, &lo);
    if (st != CRDFFT_OK)
        return st;
    // The chained form: every wave's two passes as tiles of one persistent launch (forward and inverse alike).
    if (chain_enabled() && r2c_wn == nullptr && t_arena == nullptr && istride == 1 &&
        n * 8 <= chain_wave_bytes() && batch * n * 8 > 2 * chain_wave_bytes())
    {
        ChainDesc cd{};
        cd.wave_t = std::min(batch, std::max(1LL, chain_wave_bytes() / (n * 8)));
        const int l1 = chain_lines_per_tile(static_cast<int>(n1));
        const int l2 = chain_lines_per_tile(static_cast<int>(n2));
        FourStepTw ftw;
        ftw.M = n;
        ftw.hi = hi;
        ftw.lo = lo;
        st = make_pass_desc(p, n1, cd.wave_t * n2, n2, LineMap{idist, 1, n2}, LineMap{n, 1, n2}, conj_in, false,
                            1.0f, ftw, &cd.col);
        if (st != CRDFFT_OK)
            return st;
        st = make_pass_desc(p, n2, cd.wave_t * n1, n1, LineMap{n, n2, 1}, LineMap{odist, ostride, n1 * ostride}, false,
                            conj_out, scale, FourStepTw{}, &cd.row);
        if (st != CRDFFT_OK)
            return st;
        cd.row.discard_in = l2_discard() ? 1 : 0;
        if (l1 >= 1 && l2 >= 1 && l1 <= pass_lines_per_cta_limit() && l2 <= pass_lines_per_cta_limit() &&
            chain_supported(cd.col, cd.row))
        {
            cd.batch = batch;
            cd.waves = (batch + cd.wave_t - 1) / cd.wave_t;
            cd.idist = idist;
            cd.odist = odist;
            cd.slot_elems = cd.wave_t * n;
            cd.slots = chain_slots();
            cd.lag = chain_lag(cd.slots);
            cd.col_lpc = l1;
            cd.row_lpc = l2;
            cd.col_items = (cd.wave_t * n2 + l1 - 1) / l1;
            cd.row_items = (cd.wave_t * n1 + l2 - 1) / l2;
            cd.spin_limit = g_debug_stall.load() ? (1 << 10) : (1 << 20);
            const long long ctr_bytes = (1 + 2 * cd.waves) * 4;
            const long long ctr_off = ws_off + cd.slots * cd.slot_elems;
            *ws_need = cd.slots * cd.slot_elems + (ctr_bytes + 7) / 8;
            Step z;
            z.kind = StepKind::Zero;
            z.count = ctr_bytes;
            z.src = z.dst = BufRef{Buf::Ws, ctr_off};
            steps.push_back(z);
            Step c;
            c.kind = StepKind::Chain;
            c.chain = cd;
            c.src = src;
            c.dst = dst;
            c.aux = BufRef{Buf::Ws, ws_off};
            steps.push_back(c);
            return CRDFFT_OK;
        }
    }
    // L2 waves: a wave small enough that pass 1's output is still in L2 when pass 2 reads it, one workspace slot a
    // lane, consecutive waves round-robin on the plan's internal streams so that one wave's pass 2 overlaps the next
    // one's pass 1 (and fills its tail). Otherwise one large wave at a time on the caller's stream.
    // (Transforms above 2 MiB are left to large waves: a 24 MiB wave of them is too few tiles to fill the GPU.)
    const bool l2w = l2_waves() && t_arena == nullptr && n * 8 <= l2_wave_max_transform() &&
                     batch * n * 8 > 2 * l2_wave_bytes();
    long long wave = std::max(1LL, (l2w ? l2_wave_bytes() : wave_bytes()) / (n * 8));
    wave = std::min(wave, batch);
    const int nl = l2_lanes();
    *ws_need = (l2w ? nl : 1) * wave * n;
    int wi = 0;
    for (long long t0 = 0; t0 < batch; t0 += wave, ++wi)
    {
        const long long w = std::min(wave, batch - t0);
        const long long slot_off = l2w ? (wi % nl) * wave * n : 0;
        const int lane = l2w ? 1 + wi % nl : 0;
        // pass 1: columns n2' in [0, n2), elements n1' along stride n2 -> scratch Y[t][k1][n2']
        Step s1;
        FourStepTw ftw;
        ftw.M = n;
        ftw.hi = hi;
        ftw.lo = lo;
        st = make_line_step(p, n1, w * n2, n2, LineMap{idist, istride, n2 * istride}, LineMap{n, 1, n2},
                            BufRef{src.b, src.off + t0 * idist}, BufRef{Buf::Ws, ws_off + slot_off}, conj_in, false,
                            1.0f, &s1, ftw);
        if (st != CRDFFT_OK)
            return st;
        if (tma_col_enabled() && s1.kind == StepKind::Line && tma_col_supported(s1.pass))
            s1.kind = StepKind::TmaCol;
        s1.lane = lane;
        steps.push_back(s1);
        // pass 2: rows k1 of length n2 -> X[t][k1 + n1 k2]
        Step s2;
        st = make_line_step(p, n2, w * n1, n1, LineMap{n, n2, 1}, LineMap{odist, ostride, n1 * ostride},
                            BufRef{Buf::Ws, ws_off + slot_off}, BufRef{dst.b, dst.off + t0 * odist}, false, conj_out,
                            scale, &s2);
        if (st != CRDFFT_OK)
            return st;
        // the fused row pass pairs rows p and n1 - p in one CTA: even n1 only
        if (r2c_wn != nullptr && ostride == 1 && !conj_out && n1 % 2 == 0 &&
            std::getenv("CRDFFT_NO_FUSED_REAL") == nullptr && row_r2c_supported(s2.pass))
        {
            s2.kind = StepKind::RowR2C;
            s2.rr = RowR2CDesc{n, odist, w, static_cast<int>(n1), static_cast<int>(n2), r2c_wn, scale};
            if (r2c_fused != nullptr && t0 == 0)
                *r2c_fused = true;
        }
        else if (r2c_fused != nullptr && *r2c_fused)
            return CRDFFT_UNSUPPORTED_SIZE; // every wave takes the same form
        // an L2 wave's intermediate is read once, from L2, by this row pass: its lines are dropped there instead of
        // being written back to HBM (1 GB of the 3.1 GB 107520 moved a GiB)
        if (l2w && l2_discard())
            s2.pass.discard_in = 1;
        s2.lane = lane;
        steps.push_back(s2);
    }
    return CRDFFT_OK;
}

crdfft_status build_c2c_rank1(Plan& p)
{
    const crdfft_desc& d = p.desc;
    const long long n = d.dims[0];
    const long long istride = d.istride ? d.istride : 1;
    const long long ostride = d.ostride ? d.ostride : 1;
    const long long idist = d.idist ? d.idist : n;
    const long long odist = d.odist ? d.odist : n;
    const float inv_scale = d.norm == CRDFFT_NORM_INVERSE ? static_cast<float>(1.0 / static_cast<double>(n)) : 1.0f;
    if (is_smooth(n))
    {
        long long ws_f = 0, ws_i = 0;
        crdfft_status st = plan_c2c_1d(p, n, d.batch, istride, idist, ostride, odist, BufRef{Buf::In, 0},
                                       BufRef{Buf::Out, 0}, false, false, 1.0f, 0, p.steps[0], &ws_f);
        if (st != CRDFFT_OK)
            return st;
        st = plan_c2c_1d(p, n, d.batch, istride, idist, ostride, odist, BufRef{Buf::In, 0}, BufRef{Buf::Out, 0},
                         true, true, inv_scale, 0, p.steps[1], &ws_i);
        if (st != CRDFFT_OK)
            return st;
        p.ws_bytes = static_cast<size_t>(std::max(ws_f, ws_i)) * 8;
        if (p.split_kind == 1)
        {
            p.algorithm = "single-pass";
            p.factors = {n};
        }
        else if (p.split_kind == 2)
        {
            p.algorithm = "cluster-four-step";
            p.factors = {p.steps[0][0].pass.n, p.steps[0][0].pass2.n};
        }
        else
        {
            p.algorithm = "four-step";
            p.factors = {p.split_n1, n / p.split_n1};
        }
        return CRDFFT_OK;
    }
    // Bluestein: m = smallest power of two >= 2n - 1 (bluestein.hpp:36-41).
    long long m = 1;
    while (m < 2 * n - 1)
        m <<= 1;
    // chirp_k = exp(+iπ k²/n), k² reduced mod 2n (bluestein.hpp:47-53)
    std::vector<float> chirp(static_cast<size_t>(2 * n));
    std::vector<std::complex<double>> bcirc(static_cast<size_t>(m), {0.0, 0.0});
    for (long long k = 0; k < n; ++k)
    {
        const long long kk = static_cast<long long>((static_cast<unsigned __int128>(k) * k) % (2 * n));
        // exp(+iπ kk/n) = conj(W_{2n}^{kk})
        double re, im;
        root(kk, 2 * n, &re, &im);
        chirp[2 * k] = static_cast<float>(re);
        chirp[2 * k + 1] = static_cast<float>(-im);
        const std::complex<double> c(re, -im);
        bcirc[static_cast<size_t>(k)] = c;
        if (k > 0)
            bcirc[static_cast<size_t>(m - k)] = c;
    }
    // FFT_m(b_circ) in FP64 on the host (the reference runs its f32 plan on the narrowed chirp; an FP64 spectrum
    // narrowed once is at least as accurate).
    std::vector<std::complex<double>> bf(static_cast<size_t>(m));
    {
        // iterative radix-2 DIT in FP64
        std::vector<std::complex<double>> a = bcirc;
        int lg = 0;
        while ((1LL << lg) < m)
            ++lg;
        for (long long i = 0; i < m; ++i)
        {
            long long r = 0;
            for (int b = 0; b < lg; ++b)
                if (i & (1LL << b))
                    r |= 1LL << (lg - 1 - b);
            if (i < r)
                std::swap(a[static_cast<size_t>(i)], a[static_cast<size_t>(r)]);
        }
        for (long long len = 2; len <= m; len <<= 1)
        {
            for (long long k = 0; k < len / 2; ++k)
            {
                double wr, wi;
                root(k * (m / len), m, &wr, &wi);
                const std::complex<double> w(wr, wi);
                for (long long s = 0; s < m; s += len)
                {
                    const std::complex<double> u = a[static_cast<size_t>(s + k)];
                    const std::complex<double> v = a[static_cast<size_t>(s + k + len / 2)] * w;
                    a[static_cast<size_t>(s + k)] = u + v;
                    a[static_cast<size_t>(s + k + len / 2)] = u - v;
                }
            }
        }
        bf = a;
    }
    std::vector<float> bff(static_cast<size_t>(2 * m));
    for (long long k = 0; k < m; ++k)
    {
        bff[static_cast<size_t>(2 * k)] = static_cast<float>(bf[static_cast<size_t>(k)].real());
        bff[static_cast<size_t>(2 * k + 1)] = static_cast<float>(bf[static_cast<size_t>(k)].imag());
    }
    void* dchirp = nullptr;
    void* dbf = nullptr;
    crdfft_status st = upload_table(p, chirp, &dchirp);
    if (st != CRDFFT_OK)
        return st;
    st = upload_table(p, bff, &dbf);
    if (st != CRDFFT_OK)
        return st;
    const long long B = d.batch;
    const long long conv = B * m; // the padded sequences live at the start of the workspace
    long long inner_f = 0, inner_i = 0;
    for (int dir = 0; dir < 2; ++dir)
    {
        std::vector<Step>& steps = p.steps[dir];
        ChirpDesc c{};
        c.n = n;
        c.m = m;
        c.batch = B;
        c.wdist = m;
        c.chirp = dchirp;
        c.bfft = dbf;
        c.conj = dir;
        Step pre;
        pre.kind = StepKind::ChirpPre;
        pre.chirp = c;
        pre.chirp.xdist = idist;
        pre.src = BufRef{Buf::In, 0};
        pre.dst = BufRef{Buf::Ws, 0};
        if (istride != 1 || ostride != 1)
            return CRDFFT_UNSUPPORTED_SIZE;
        steps.push_back(pre);
        long long need = 0;
        st = plan_c2c_1d(p, m, B, 1, m, 1, m, BufRef{Buf::Ws, 0}, BufRef{Buf::Ws, 0}, false, false, 1.0f, conv,
                         steps, &need);
        if (st != CRDFFT_OK)
            return st;
        inner_f = std::max(inner_f, need);
        Step mul;
        mul.kind = StepKind::SpecMul;
        mul.chirp = c;
        mul.dst = BufRef{Buf::Ws, 0};
        steps.push_back(mul);
        st = plan_c2c_1d(p, m, B, 1, m, 1, m, BufRef{Buf::Ws, 0}, BufRef{Buf::Ws, 0}, true, true, 1.0f, conv,
                         steps, &need);
        if (st != CRDFFT_OK)
            return st;
        inner_i = std::max(inner_i, need);
        Step post;
        post.kind = StepKind::ChirpPost;
        post.chirp = c;
        post.chirp.xdist = odist;
        double sc = 1.0 / static_cast<double>(m);
        if (dir == 1 && d.norm == CRDFFT_NORM_INVERSE)
            sc /= static_cast<double>(n);
        post.chirp.scale = static_cast<float>(sc);
        post.src = BufRef{Buf::Ws, 0};
        post.dst = BufRef{Buf::Out, 0};
        steps.push_back(post);
    }
    p.ws_bytes = static_cast<size_t>(conv + std::max(inner_f, inner_i)) * 8;
    p.algorithm = "bluestein";
    p.factors = {n, m};
    return CRDFFT_OK;
}

crdfft_status build_real(Plan& p)
{
    const crdfft_desc& d = p.desc;
    const long long n = d.dims[0];
    if (n < 2 || (n & 1) != 0)
        return CRDFFT_UNSUPPORTED_SIZE;
    const long long h = n / 2;
    if (!is_smooth(h))
        return CRDFFT_UNSUPPORTED_SIZE;
    if ((d.istride != 0 && d.istride != 1) || (d.ostride != 0 && d.ostride != 1))
        return CRDFFT_UNSUPPORTED_SIZE;
    // W_n^k, k = 0 .. h (real_fft.hpp:25-35)
    std::vector<float> wn(static_cast<size_t>(2 * (h + 1)));
    for (long long k = 0; k <= h; ++k)
    {
        double re, im;
        root(k, n, &re, &im);
        wn[static_cast<size_t>(2 * k)] = static_cast<float>(re);
        wn[static_cast<size_t>(2 * k + 1)] = static_cast<float>(im);
    }
    void* dwn = nullptr;
    crdfft_status st = upload_table(p, wn, &dwn);
    if (st != CRDFFT_OK)
        return st;
    // A half length that runs as a single pass: one launch, the recombination fused with the line FFT in shared
    // memory (real_line.cu); the real data crosses HBM once each way.
    if (single_pass_ok(h) && std::getenv("CRDFFT_NO_FUSED_REAL") == nullptr)
    {
        const bool r2c = d.kind == CRDFFT_R2C;
        const long long idist = d.idist ? d.idist : (r2c ? n : h + 1);
        const long long odist = d.odist ? d.odist : (r2c ? h + 1 : n);
        if ((r2c ? idist : odist) % 2 != 0)
            return CRDFFT_UNSUPPORTED_SIZE;
        Step s;
        s.kind = StepKind::RealLine;
        s.rmode = r2c ? kRealR2C : kRealC2R;
        s.raux = RealLineAux{dwn, LineMap{0, 0, 1}};
        const LineMap in = r2c ? LineMap{idist / 2, 0, 1} : LineMap{idist, 0, 1};
        const LineMap out = r2c ? LineMap{odist, 0, 1} : LineMap{odist / 2, 0, 1};
        const float sc = (!r2c && d.norm == CRDFFT_NORM_INVERSE) ? static_cast<float>(1.0 / static_cast<double>(n))
                                                                 : 1.0f;
        st = make_pass_desc(p, h, d.batch, 1, in, out, false, !r2c, sc, FourStepTw{}, &s.pass);
        if (st == CRDFFT_OK && real_line_supported(s.pass))
        {
            s.src = BufRef{Buf::In, 0};
            s.dst = BufRef{Buf::Out, 0};
            p.steps[r2c ? 0 : 1].push_back(s);
            p.algorithm = "real-fused";
            p.factors = {h};
            return CRDFFT_OK;
        }
    }
    long long need = 0;
    if (d.kind == CRDFFT_R2C)
    {
        const long long idist = d.idist ? d.idist : n;       // floats
        const long long odist = d.odist ? d.odist : h + 1;   // complex
        if (idist % 2 != 0)
            return CRDFFT_UNSUPPORTED_SIZE;
        bool fused = false;
        st = plan_c2c_1d(p, h, d.batch, 1, idist / 2, 1, odist, BufRef{Buf::In, 0}, BufRef{Buf::Out, 0}, false,
                         false, 1.0f, 0, p.steps[0], &need, dwn, &fused);
        if (st != CRDFFT_OK)
            return st;
        if (fused)
        {
            p.ws_bytes = static_cast<size_t>(need) * 8;
            p.algorithm = "real+four-step-fused";
            p.factors = {h};
            return CRDFFT_OK;
        }
        Step post;
        post.kind = StepKind::R2CPost;
        post.real = RealRecombine{h, d.batch, odist, odist, dwn, 1.0f};
        post.src = BufRef{Buf::Out, 0};
        post.dst = BufRef{Buf::Out, 0};
        p.steps[0].push_back(post);
    }
    else
    {
        const long long idist = d.idist ? d.idist : h + 1;   // complex
        const long long odist = d.odist ? d.odist : n;       // floats
        if (odist % 2 != 0)
            return CRDFFT_UNSUPPORTED_SIZE;
        // (A column pass that formed the pairs itself, reading Y directly, measured no faster than this separate
        // pass followed by the tensor-copy column pass: Y's odd transform distance rules the tensor copies out.)
        Step pre;
        pre.kind = StepKind::C2RPre;
        pre.real = RealRecombine{h, d.batch, odist / 2, idist, dwn, 1.0f};
        pre.src = BufRef{Buf::In, 0};
        pre.dst = BufRef{Buf::Out, 0};
        p.steps[1].push_back(pre);
        // IFFT_h unnormalised gives h z; the reference scales by 1/h (normalised irfft); unnormalised C2R is
        // n times that.
        const float sc = d.norm == CRDFFT_NORM_INVERSE ? static_cast<float>(1.0 / static_cast<double>(h)) : 2.0f;
        st = plan_c2c_1d(p, h, d.batch, 1, odist / 2, 1, odist / 2, BufRef{Buf::Out, 0}, BufRef{Buf::Out, 0}, true,
                         true, sc, 0, p.steps[1], &need);
        if (st != CRDFFT_OK)
            return st;
    }
    p.ws_bytes = static_cast<size_t>(need) * 8;
    p.algorithm = single_pass_ok(h) ? "real+single-pass" : "real+four-step";
    p.factors = {h};
    return CRDFFT_OK;
}

// 2-D and 3-D real transforms (the reference's NdFftPlan is complex only, nd_fft.hpp:28-194; the real plan is 1-D,
// real_fft.hpp:18-101): the Hermitian half along the last axis, dims[0..rank-2] x (n/2 + 1) complex values a batch
// member. R2C: fused R2C rows (real_line.cu) from the input into the output, then one in-place complex pass per
// remaining axis. C2R: the complex axes inverse from the input into the workspace (the input stays untouched), then
// fused C2R rows into the output. Unnormalised both ways unless norm = CRDFFT_NORM_INVERSE (1 / the real size on
// C2R). Packed batches only.
crdfft_status build_nd_real(Plan& p)
{
    const crdfft_desc& d = p.desc;
    const int rank = d.rank;
    const long long n = d.dims[rank - 1];
    if (n < 2 || (n & 1) != 0 || !single_pass_ok(n / 2))
        return CRDFFT_UNSUPPORTED_SIZE;
    const long long h = n / 2, hw = h + 1;
    long long outer = 1; // rows of the real axis in one batch member
    for (int i = 0; i < rank - 1; ++i)
        outer *= d.dims[i];
    const long long rtotal = outer * n, ctotal = outer * hw;
    const bool r2c = d.kind == CRDFFT_R2C;
    if ((d.idist != 0 && d.idist != (r2c ? rtotal : ctotal)) || (d.odist != 0 && d.odist != (r2c ? ctotal : rtotal)))
        return CRDFFT_UNSUPPORTED_SIZE;
    if ((d.istride != 0 && d.istride != 1) || (d.ostride != 0 && d.ostride != 1))
        return CRDFFT_UNSUPPORTED_SIZE;
    std::vector<float> wn(static_cast<size_t>(2 * (h + 1)));
    for (long long k = 0; k <= h; ++k)
    {
        double re, im;
        root(k, n, &re, &im);
        wn[static_cast<size_t>(2 * k)] = static_cast<float>(re);
        wn[static_cast<size_t>(2 * k + 1)] = static_cast<float>(im);
    }
    void* dwn = nullptr;
    crdfft_status st = upload_table(p, wn, &dwn);
    if (st != CRDFFT_OK)
        return st;
    Step row;
    row.kind = StepKind::RealLine;
    row.rmode = r2c ? kRealR2C : kRealC2R;
    row.raux = RealLineAux{dwn, LineMap{0, 0, 1}};
    const float scale = (!r2c && d.norm == CRDFFT_NORM_INVERSE)
                            ? static_cast<float>(1.0 / static_cast<double>(rtotal))
                            : 1.0f;
    st = make_pass_desc(p, h, d.batch * outer, 1, r2c ? LineMap{h, 0, 1} : LineMap{hw, 0, 1},
                        r2c ? LineMap{hw, 0, 1} : LineMap{h, 0, 1}, false, !r2c, scale, FourStepTw{}, &row.pass);
    if (st != CRDFFT_OK)
        return st;
    if (!real_line_supported(row.pass))
        return CRDFFT_UNSUPPORTED_SIZE;
    // the complex axes of the half array, last to first
    std::vector<int> axes;
    for (int ax = rank - 2; ax >= 0; --ax)
        if (d.dims[ax] > 1)
            axes.push_back(ax);
    std::vector<Step> cplx;
    for (size_t i = 0; i < axes.size(); ++i)
    {
        const int ax = axes[i];
        const long long m = d.dims[ax];
        if (!single_pass_ok(m))
            return CRDFFT_UNSUPPORTED_SIZE;
        long long st_ax = hw;
        for (int j = ax + 1; j < rank - 1; ++j)
            st_ax *= d.dims[j];
        const LineMap map{m * st_ax, 1, st_ax};
        const bool first = i == 0, last = i + 1 == axes.size();
        BufRef src, dst;
        if (r2c)
            src = dst = BufRef{Buf::Out, 0};
        else
        {
            src = first ? BufRef{Buf::In, 0} : BufRef{Buf::Ws, 0};
            dst = BufRef{Buf::Ws, 0};
        }
        Step s;
        st = make_line_step(p, m, d.batch * (ctotal / m), st_ax, map, map, src, dst, !r2c && first, !r2c && last,
                            1.0f, &s);
        if (st != CRDFFT_OK)
            return st;
        cplx.push_back(s);
    }
    if (r2c)
    {
        row.src = BufRef{Buf::In, 0};
        row.dst = BufRef{Buf::Out, 0};
        p.steps[0].push_back(row);
        for (const Step& s : cplx)
            p.steps[0].push_back(s);
    }
    else
    {
        for (const Step& s : cplx)
            p.steps[1].push_back(s);
        row.src = cplx.empty() ? BufRef{Buf::In, 0} : BufRef{Buf::Ws, 0};
        row.dst = BufRef{Buf::Out, 0};
        p.steps[1].push_back(row);
        if (!cplx.empty())
            p.ws_bytes = static_cast<size_t>(d.batch * ctotal) * 8;
    }
    p.algorithm = "nd-real";
    for (int i = 0; i < rank; ++i)
        p.factors.push_back(d.dims[i]);
    return CRDFFT_OK;
}

crdfft_status build_nd(Plan& p)
{
    const crdfft_desc& d = p.desc;
    const int rank = d.rank;
    long long total = 1;
    for (int i = 0; i < rank; ++i)
        total *= d.dims[i];
    const long long idist = d.idist ? d.idist : total;
    const long long odist = d.odist ? d.odist : total;
    if (idist < total || odist < total || d.istride > 1 || d.ostride > 1)
        return CRDFFT_UNSUPPORTED_SIZE;
    // The lines of one axis as groups of lpg lines. Packed batches: the classic maps. Padded batches (a distance
    // above the transform's size) need each group inside one batch member: the last axis (groups = batch members,
    // lines n apart) and the first (groups = batch members, lines adjacent); a middle axis of a padded 3-D batch has
    // no such map.
    auto axis_map = [&](int ax, long long n, long long st_ax, long long dist, LineMap* m, long long* lpg) {
        if (dist == total)
        {
            *m = st_ax == 1 ? LineMap{n, 0, 1} : LineMap{n * st_ax, 1, st_ax};
            *lpg = st_ax == 1 ? 1 : st_ax;
            return true;
        }
        if (st_ax == 1)
        {
            *m = LineMap{dist, n, 1};
            *lpg = total / n;
            return true;
        }
        if (ax == 0)
        {
            *m = LineMap{dist, 1, st_ax};
            *lpg = st_ax;
            return true;
        }
        return false;
    };
    const float inv_scale =
        d.norm == CRDFFT_NORM_INVERSE ? static_cast<float>(1.0 / static_cast<double>(total)) : 1.0f;
    // Long columns of a packed 2-D batch (rows x cols, rows >= 2048): one column pass would hold only a few columns
    // a CTA (32-byte runs). Instead the column FFT of length rows = n1 n2 runs as two strided passes of short lines,
    // each CTA holding 64 or more adjacent columns (512-byte runs): C1 transforms the n1-point sub-columns j1 n2 + q
    // in place with the four-step twiddle W_rows^{q k1}, C2 the n2-point sub-columns k1 n2 + q into rows
    // k1 + n1 k2. The row pass writes the workspace, C1 works on it, C2 writes the output (one step per batch
    // member, up to 8).
    long long cn1 = 0, cn2 = 0;
    const bool split_cols = rank == 2 && d.dims[0] >= 2048 && d.dims[1] >= 16 && idist == total && odist == total &&
                            d.batch <= 8 && std::getenv("CRDFFT_NO_SPLIT_COLUMNS") == nullptr &&
                            four_step_split(d.dims[0], &cn1, &cn2) && single_pass_ok(d.dims[1]);
    if (split_cols)
    {
        const long long rows = d.dims[0], cols = d.dims[1];
        const void* hi = nullptr;
        const void* lo = nullptr;
        crdfft_status st = four_step_tables(p, rows, cn1, cn2, &hi, &lo);
        if (st != CRDFFT_OK)
            return st;
        for (int dir = 0; dir < 2; ++dir)
        {
            Step r;
            st = make_line_step(p, cols, d.batch * rows, 1, LineMap{cols, 0, 1}, LineMap{cols, 0, 1},
                                BufRef{Buf::In, 0}, BufRef{Buf::Ws, 0}, dir == 1, false, 1.0f, &r);
            if (st != CRDFFT_OK)
                return st;
            p.steps[dir].push_back(r);
            FourStepTw ftw;
            ftw.M = rows;
            ftw.hi = hi;
            ftw.lo = lo;
            ftw.div = static_cast<int>(cols);
            Step c1;
            st = make_line_step(p, cn1, d.batch * cn2 * cols, cn2 * cols, LineMap{total, 1, cn2 * cols},
                                LineMap{total, 1, cn2 * cols}, BufRef{Buf::Ws, 0}, BufRef{Buf::Ws, 0}, false, false,
                                1.0f, &c1, ftw);
            if (st != CRDFFT_OK)
                return st;
            p.steps[dir].push_back(c1);
            for (long long b = 0; b < d.batch; ++b)
            {
                Step c2;
                st = make_line_step(p, cn2, cn1 * cols, cols, LineMap{cn2 * cols, 1, cols},
                                    LineMap{cols, 1, cn1 * cols}, BufRef{Buf::Ws, b * total},
                                    BufRef{Buf::Out, b * total}, false, dir == 1, dir == 1 ? inv_scale : 1.0f, &c2);
                if (st != CRDFFT_OK)
                    return st;
                p.steps[dir].push_back(c2);
            }
        }
        p.ws_bytes = static_cast<size_t>(d.batch * total) * 8;
        p.algorithm = "nd-axes-split-columns"; // (+tc-... appended by create() when the row pass is a TC pass)
        p.factors = {rows, cols, cn1, cn2};
        return CRDFFT_OK;
    }
    for (int dir = 0; dir < 2; ++dir)
    {
        // Axes from the last (unit stride) to the first; the first pass reads the input, later ones work in place
        // on the output. The inverse conjugates on the way in and out (nd_fft.hpp:116-146).
        bool first = true;
        int last_axis = -1;
        for (int ax = rank - 1; ax >= 0; --ax)
            if (d.dims[ax] > 1)
                last_axis = ax;
        for (int ax = rank - 1; ax >= 0; --ax)
        {
            const long long n = d.dims[ax];
            if (n == 1)
                continue;
            if (!single_pass_ok(n))
                return CRDFFT_UNSUPPORTED_SIZE;
            long long st_ax = 1;
            for (int j = ax + 1; j < rank; ++j)
                st_ax *= d.dims[j];
            const long long lines = d.batch * (total / n);
            LineMap mi, mo;
            long long lpg = 1, lpg_o = 1;
            if (!axis_map(ax, n, st_ax, first ? idist : odist, &mi, &lpg) ||
                !axis_map(ax, n, st_ax, odist, &mo, &lpg_o) || lpg != lpg_o)
                return CRDFFT_UNSUPPORTED_SIZE;
            const bool is_last = ax == last_axis;
            Step s;
            const crdfft_status st =
                make_line_step(p, n, lines, lpg, mi, mo, first ? BufRef{Buf::In, 0} : BufRef{Buf::Out, 0},
                               BufRef{Buf::Out, 0}, dir == 1 && first, dir == 1 && is_last,
                               (dir == 1 && is_last) ? inv_scale : 1.0f, &s);
            if (st != CRDFFT_OK)
                return st;
            p.steps[dir].push_back(s);
            first = false;
        }
        if (first)
        {
            // every axis has length 1: a copy with the inverse's scale
            Step s;
            if (idist != total || odist != total)
                return CRDFFT_UNSUPPORTED_SIZE;
            const crdfft_status st = make_line_step(p, 1, d.batch * total, 1, LineMap{1, 0, 1}, LineMap{1, 0, 1},
                                                    BufRef{Buf::In, 0}, BufRef{Buf::Out, 0}, false, false,
                                                    dir == 1 ? inv_scale : 1.0f, &s);
            if (st != CRDFFT_OK)
                return st;
            p.steps[dir].push_back(s);
        }
    }
    p.algorithm = "nd-axes";
    for (int i = 0; i < rank; ++i)
        p.factors.push_back(d.dims[i]);
    return CRDFFT_OK;
}

// A fused-convolution request: one filter spectrum for the batch or one per transform, and the output scale
// (negative: 1 / the transform size).
struct ConvReq
{
    bool per_transform = false;
    double scale = -1.0;
};

// The fused convolution (conv.cu): y = IFFT(FFT(x) * H) * scale. Rank 1: one launch, lines of the batch in shared
// memory. Rank 2 (rows x cols): forward row FFTs, the fused convolution along the columns, inverse row FFTs with the
// scale, as the reference's 2-D GPU convolution orders them (engine/gpu/kir/include/crd/kir/ckir_fft.hpp:2075-2090).
crdfft_status build_real_conv(Plan& p, const ConvReq& req);

crdfft_status build_conv(Plan& p, const ConvReq& req)
{
    const crdfft_desc& d = p.desc;
    if (d.kind == CRDFFT_R2C)
        return build_real_conv(p, req);
    if (d.kind != CRDFFT_C2C || d.rank > 2 || d.istride > 1 || d.ostride > 1)
        return CRDFFT_UNSUPPORTED_SIZE;
    long long total = 1;
    for (int i = 0; i < d.rank; ++i)
        total *= d.dims[i];
    if ((d.idist != 0 && d.idist != total) || (d.odist != 0 && d.odist != total))
        return CRDFFT_UNSUPPORTED_SIZE;
    const float scale = static_cast<float>(req.scale < 0.0 ? 1.0 / static_cast<double>(total) : req.scale);
    p.conv = true;
    if (d.rank == 1)
    {
        const long long n = d.dims[0];
        if (n < 2 || !single_pass_ok(n))
            return CRDFFT_UNSUPPORTED_SIZE;
        Step s;
        s.kind = StepKind::Conv;
        crdfft_status st = make_pass_desc(p, n, d.batch, 1, LineMap{n, 0, 1}, LineMap{n, 0, 1}, false, true, scale,
                                          FourStepTw{}, &s.pass);
        if (st != CRDFFT_OK)
            return st;
        if (!conv_supported(s.pass))
            return CRDFFT_UNSUPPORTED_SIZE;
        s.shape.map = PassMap::Row;
        s.smap = LineMap{req.per_transform ? n : 0, 0, 1};
        s.src = BufRef{Buf::In, 0};
        s.dst = BufRef{Buf::Out, 0};
        p.steps[0].push_back(s);
        p.algorithm = "fused-conv";
        p.factors = {n};
        return CRDFFT_OK;
    }
    const long long rows = d.dims[0], cols = d.dims[1];
    if (rows < 2 || cols < 2 || !single_pass_ok(rows) || !single_pass_ok(cols))
        return CRDFFT_UNSUPPORTED_SIZE;
    const long long lines = d.batch * rows;
    Step r1;
    crdfft_status st = make_line_step(p, cols, lines, 1, LineMap{cols, 0, 1}, LineMap{cols, 0, 1},
                                      BufRef{Buf::In, 0}, BufRef{Buf::Out, 0}, false, false, 1.0f, &r1);
    if (st != CRDFFT_OK)
        return st;
    Step cv;
    cv.kind = StepKind::Conv;
    st = make_pass_desc(p, rows, d.batch * cols, cols, LineMap{total, 1, cols}, LineMap{total, 1, cols}, false, true,
                        1.0f, FourStepTw{}, &cv.pass);
    if (st != CRDFFT_OK)
        return st;
    if (!conv_supported(cv.pass))
        return CRDFFT_UNSUPPORTED_SIZE;
    cv.shape.map = PassMap::Col;
    cv.smap = LineMap{req.per_transform ? total : 0, 1, cols};
    cv.src = BufRef{Buf::Out, 0};
    cv.dst = BufRef{Buf::Out, 0};
    Step r2;
    st = make_line_step(p, cols, lines, 1, LineMap{cols, 0, 1}, LineMap{cols, 0, 1}, BufRef{Buf::Out, 0},
                        BufRef{Buf::Out, 0}, true, true, scale, &r2);
    if (st != CRDFFT_OK)
        return st;
    p.steps[0] = {r1, cv, r2};
    p.algorithm = "fused-conv-2d";
    p.factors = {rows, cols};
    return CRDFFT_OK;
}

// The fused convolution of real signals (kind R2C): real input and output, the filter as the half spectrum
// (n/2 + 1 values a row). Rank 1: one launch (real_line.cu, kRealConv). Rank 2 (rows x cols): R2C rows into the
// workspace (rows x (cols/2 + 1)), the fused convolution along those half-width columns, C2R rows with the scale:
// the three dispatches of the reference's real 2-D convolution (engine/gpu/kir/include/crd/kir/ckir_fft.hpp:
// 2300-2308), here without its padding of the half width.
crdfft_status build_real_conv(Plan& p, const ConvReq& req)
{
    const crdfft_desc& d = p.desc;
    if (d.rank > 2 || d.istride > 1 || d.ostride > 1)
        return CRDFFT_UNSUPPORTED_SIZE;
    long long total = 1;
    for (int i = 0; i < d.rank; ++i)
        total *= d.dims[i];
    if ((d.idist != 0 && d.idist != total) || (d.odist != 0 && d.odist != total))
        return CRDFFT_UNSUPPORTED_SIZE;
    const long long n = d.dims[d.rank - 1]; // the real (last) axis
    const long long h = n / 2;
    if (n < 2 || (n & 1) != 0 || !single_pass_ok(h))
        return CRDFFT_UNSUPPORTED_SIZE;
    const float scale = static_cast<float>(req.scale < 0.0 ? 1.0 / static_cast<double>(total) : req.scale);
    std::vector<float> wn(static_cast<size_t>(2 * (h + 1)));
    for (long long k = 0; k <= h; ++k)
    {
        double re, im;
        root(k, n, &re, &im);
        wn[static_cast<size_t>(2 * k)] = static_cast<float>(re);
        wn[static_cast<size_t>(2 * k + 1)] = static_cast<float>(im);
    }
    void* dwn = nullptr;
    crdfft_status st = upload_table(p, wn, &dwn);
    if (st != CRDFFT_OK)
        return st;
    p.conv = true;
    const long long hw = h + 1;
    if (d.rank == 1)
    {
        Step s;
        s.kind = StepKind::RealLine;
        s.rmode = kRealConv;
        s.raux = RealLineAux{dwn, LineMap{req.per_transform ? hw : 0, 0, 1}};
        st = make_pass_desc(p, h, d.batch, 1, LineMap{h, 0, 1}, LineMap{h, 0, 1}, false, true, scale, FourStepTw{},
                            &s.pass);
        if (st != CRDFFT_OK)
            return st;
        if (!real_line_supported(s.pass))
            return CRDFFT_UNSUPPORTED_SIZE;
        s.src = BufRef{Buf::In, 0};
        s.dst = BufRef{Buf::Out, 0};
        p.steps[0].push_back(s);
        p.algorithm = "fused-real-conv";
        p.factors = {n};
        return CRDFFT_OK;
    }
    const long long rows = d.dims[0];
    if (rows < 2 || !single_pass_ok(rows))
        return CRDFFT_UNSUPPORTED_SIZE;
    const long long lines = d.batch * rows;
    const long long half_total = rows * hw;
    Step r1;
    r1.kind = StepKind::RealLine;
    r1.rmode = kRealR2C;
    r1.raux = RealLineAux{dwn, LineMap{0, 0, 1}};
    st = make_pass_desc(p, h, lines, 1, LineMap{h, 0, 1}, LineMap{hw, 0, 1}, false, false, 1.0f, FourStepTw{},
                        &r1.pass);
    if (st != CRDFFT_OK)
        return st;
    Step cv;
    cv.kind = StepKind::Conv;
    st = make_pass_desc(p, rows, d.batch * hw, hw, LineMap{half_total, 1, hw}, LineMap{half_total, 1, hw}, false,
                        true, 1.0f, FourStepTw{}, &cv.pass);
    if (st != CRDFFT_OK)
        return st;
    Step r2;
    r2.kind = StepKind::RealLine;
    r2.rmode = kRealC2R;
    r2.raux = RealLineAux{dwn, LineMap{0, 0, 1}};
    st = make_pass_desc(p, h, lines, 1, LineMap{hw, 0, 1}, LineMap{h, 0, 1}, false, true, scale, FourStepTw{},
                        &r2.pass);
    if (st != CRDFFT_OK)
        return st;
    if (!real_line_supported(r1.pass) || !real_line_supported(r2.pass) || !conv_supported(cv.pass))
        return CRDFFT_UNSUPPORTED_SIZE;
    cv.shape.map = PassMap::Col;
    cv.smap = LineMap{req.per_transform ? half_total : 0, 1, hw};
    r1.src = BufRef{Buf::In, 0};
    r1.dst = BufRef{Buf::Ws, 0};
    cv.src = BufRef{Buf::Ws, 0};
    cv.dst = BufRef{Buf::Ws, 0};
    r2.src = BufRef{Buf::Ws, 0};
    r2.dst = BufRef{Buf::Out, 0};
    p.steps[0] = {r1, cv, r2};
    p.ws_bytes = static_cast<size_t>(d.batch * half_total) * 8;
    p.algorithm = "fused-real-conv-2d";
    p.factors = {rows, n};
    return CRDFFT_OK;
}

// The split of a long uneven-batch transform: n = n1 * n2 with both halves at most `cap`, closest to square, n2
// preferring a multiple of 16 (whole column tiles).
bool uneven_split(long long n, long long cap, long long* n1, long long* n2)
{
    double best = 1e300;
    for (long long d = 2; d * d <= n; ++d)
    {
        if (n % d != 0 || d > cap || n / d > cap || !is_smooth(d) || !is_smooth(n / d))
            continue;
        for (int o = 0; o < 2; ++o)
        {
            const long long a = o ? d : n / d, b = o ? n / d : d;
            // halves the kernel has as compile-time stages first, then whole 16-column tiles, then near square
            const double stat = (uneven_static_ok(static_cast<int>(a)) ? 1.0 : 0.0) +
                                (uneven_static_ok(static_cast<int>(b)) ? 1.0 : 0.0);
            const double score = -3.0 * stat + (b % 16 != 0 ? 10.0 : 0.0) +
                                 std::fabs(std::log(static_cast<double>(a) / b));
            if (score < best)
            {
                best = score;
                *n1 = a;
                *n2 = b;
            }
        }
    }
    return best < 1e299;
}

// The uneven kernel's variant for items of line length n: its compile-time stages (1) or the run-time stages (0).
// CRDFFT_UNEVEN_STATIC=0/1 forces it; otherwise wisdom, else in measure and learned mode a timed choice (an uneven
// plan of that length alone, each variant executed cold) that is remembered, else the compile-time stages.
thread_local int t_uneven_force = -1;
std::atomic<int> g_uneven_force{-1}; // crdfft_debug_uneven_variant

crdfft_status create_uneven(const int64_t* sizes, int64_t count, const int64_t* offsets, Plan** out);

int uneven_variant(long long n)
{
    if (!uneven_static_ok(static_cast<int>(n)))
        return 0;
    if (t_uneven_force >= 0)
        return t_uneven_force;
    if (g_uneven_force.load() >= 0)
        return g_uneven_force.load();
    static const int env = [] {
        const char* e = std::getenv("CRDFFT_UNEVEN_STATIC");
        return e != nullptr ? (std::atoi(e) != 0 ? 1 : 0) : -1;
    }();
    if (env >= 0)
        return env;
    std::ostringstream k;
    k << "D|uneven|n" << n;
    const std::string key = k.str();
    DecompEntry w;
    if (decomp_lookup(key, &w))
        return w.kind == 2 ? 1 : 0;
    const int mode = planner_mode();
    if (mode == kPlannerEstimate || t_arena != nullptr)
        return 1;
    const long long count = std::max(1LL, std::min(8192LL, (64LL << 20) / (8 * n)));
    std::vector<int64_t> sz(static_cast<size_t>(count), n);
    float ms[2] = {-1.0f, -1.0f};
    for (int v = 0; v < 2; ++v)
    {
        t_uneven_force = v;
        Plan* tp = nullptr;
        const crdfft_status st = create_uneven(sz.data(), count, nullptr, &tp);
        t_uneven_force = -1;
        if (st != CRDFFT_OK)
            continue;
        void* in = nullptr;
        void* outb = nullptr;
        if (cudaMalloc(&in, static_cast<size_t>(count * n) * 8) == cudaSuccess &&
            cudaMalloc(&outb, static_cast<size_t>(count * n) * 8) == cudaSuccess &&
            cudaMemset(in, 0, static_cast<size_t>(count * n) * 8) == cudaSuccess)
        {
            auto go = [&](cudaStream_t s) {
                return run(*tp, in, outb, CRDFFT_FORWARD, s, nullptr) == CRDFFT_OK ? cudaSuccess
                                                                                     : cudaErrorLaunchFailure;
            };
            ms[v] = time_cold(go);
        }
        cudaGetLastError();
        cudaFree(in);
        cudaFree(outb);
        destroy_plan(tp);
    }
    if (ms[0] < 0.0f && ms[1] < 0.0f)
        return 1;
    const int pick = (ms[1] > 0.0f && (ms[0] < 0.0f || ms[1] <= ms[0])) ? 1 : 0;
    char buf[160];
    std::snprintf(buf, sizeof(buf), "%s uneven-variant run-time=%.6f compile-time=%.6f pick=%d", key.c_str(),
                  static_cast<double>(ms[0]), static_cast<double>(ms[1]), pick);
    planner_log_append(buf);
    decomp_store(key, DecompEntry{pick ? 2 : 1, 0, ms[pick]});
    return pick;
}

template <typename T> crdfft_status upload_vec(Plan& p, const std::vector<T>& v, const T** out)
{
    void* d = nullptr;
    const size_t bytes = std::max<size_t>(sizeof(T), v.size() * sizeof(T));
    if (dev_alloc(&d, bytes) != cudaSuccess)
        return CRDFFT_OOM;
    p.tables.push_back(d);
    p.table_bytes += static_cast<long long>(bytes);
    if (!v.empty() && cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
        return CRDFFT_LAUNCH;
    *out = static_cast<const T*>(d);
    return CRDFFT_OK;
}

// The uneven batch's work list (uneven.cu): transforms up to kUnevenSingle points grouped by length into CTA-sized
// items; longer ones (7-smooth, up to kUnevenSingle^2) as four-step column and row tiles through a workspace region
// of their own.
// List order: every COL item (longest transforms first), then SMALL items (longest first), then ROW items.
crdfft_status build_uneven(Plan& p, const int64_t* sizes, int64_t count, const int64_t* offsets)
{
    p.use32 = false; // the uneven kernel's stages run 16 points a thread
    const int threads = uneven_threads();
    const long long kUnevenSingle = 16LL * threads; // the longest line one item transforms (16 points a thread)
    std::map<long long, int> sched_of;
    std::vector<UnevenSched> scheds;
    auto sched_index = [&](long long n, int* idx) -> crdfft_status {
        auto it = sched_of.find(n);
        if (it != sched_of.end())
        {
            *idx = it->second;
            return CRDFFT_OK;
        }
        std::vector<int> rad;
        if (!radices_for(n, rad, false, false) || n > kUnevenSingle || static_cast<int>(rad.size()) > kMaxStages)
            return CRDFFT_UNSUPPORTED_SIZE;
        UnevenSched sc{};
        sc.n = static_cast<int>(n);
        sc.variant = uneven_variant(n);
        sc.nstages = static_cast<int>(rad.size());
        for (size_t i = 0; i < rad.size(); ++i)
            sc.radix[i] = rad[i];
        const crdfft_status st = twiddle_table(p, n, &sc.tw, false, false);
        if (st != CRDFFT_OK)
            return st;
        *idx = static_cast<int>(scheds.size());
        sched_of[n] = *idx;
        scheds.push_back(sc);
        return CRDFFT_OK;
    };
    std::map<long long, std::vector<long long>, std::greater<long long>> small; // n -> transforms
    std::vector<long long> large;                                            // transforms, longest first
    for (int64_t t = 0; t < count; ++t)
    {
        const long long n = sizes[t];
        if (n < 2 || !is_smooth(n))
            return CRDFFT_UNSUPPORTED_SIZE;
        if (offsets[t] < 0)
            return CRDFFT_INVALID_ARG;
        if (n <= kUnevenSingle)
            small[n].push_back(t);
        else
            large.push_back(t);
    }
    std::stable_sort(large.begin(), large.end(), [&](long long a, long long b) { return sizes[a] > sizes[b]; });
    std::vector<UnevenItem> col, mid, row;
    std::vector<long long> line_off;
    std::vector<const void*> fh, fl;
    std::map<long long, int> ftw_of;
    long long scratch = 0;
    int maxsmem = 0;
    for (size_t li = 0; li < large.size(); ++li)
    {
        const long long t = large[li];
        const long long n = sizes[t];
        long long n1 = 0, n2 = 0;
        if (!uneven_split(n, kUnevenSingle, &n1, &n2))
            return CRDFFT_UNSUPPORTED_SIZE;
        int s1 = 0, s2 = 0;
        crdfft_status st = sched_index(n1, &s1);
        if (st == CRDFFT_OK)
            st = sched_index(n2, &s2);
        if (st != CRDFFT_OK)
            return st;
        int fidx;
        auto fit = ftw_of.find(n);
        if (fit == ftw_of.end())
        {
            const void* hi = nullptr;
            const void* lo = nullptr;
            st = four_step_tables(p, n, n1, n2, &hi, &lo);
            if (st != CRDFFT_OK)
                return st;
            fidx = static_cast<int>(fh.size());
            fh.push_back(hi);
            fl.push_back(lo);
            ftw_of[n] = fidx;
        }
        else
            fidx = fit->second;
        const long long base = offsets[t];
        const long long reg = scratch;
        scratch += (n + 1) / 2 * 2;
        const int lc = std::max(1, std::min(threads / static_cast<int>((n1 + 15) / 16),
                                            kMaxSmemBytes / (pass_line_pitch(static_cast<int>(n1)) * 8)));
        int ncol = 0;
        for (long long q0 = 0; q0 < n2; q0 += lc, ++ncol)
        {
            UnevenItem it{};
            it.kind = kUnevenCol;
            it.sched = s1;
            it.lines = static_cast<int>(std::min<long long>(lc, n2 - q0));
            it.line_table = -1;
            it.in_base = base + q0;
            it.in_ldist = 1;
            it.in_estride = n2;
            it.out_base = reg + q0;
            it.out_ldist = 1;
            it.out_estride = n2;
            it.transform = static_cast<int>(li);
            it.q0 = static_cast<int>(q0);
            it.ftw = fidx;
            col.push_back(it);
            maxsmem = std::max(maxsmem, it.lines * pass_line_pitch(static_cast<int>(n1)) * 8);
        }
        const int lr = std::max(1, std::min(threads / static_cast<int>((n2 + 15) / 16),
                                            kMaxSmemBytes / (pass_line_pitch(static_cast<int>(n2)) * 8)));
        for (long long k0 = 0; k0 < n1; k0 += lr)
        {
            UnevenItem it{};
            it.kind = kUnevenRow;
            it.sched = s2;
            it.lines = static_cast<int>(std::min<long long>(lr, n1 - k0));
            it.line_table = -1;
            it.in_base = reg + k0 * n2;
            it.in_ldist = n2;
            it.in_estride = 1;
            it.out_base = base + k0;
            it.out_ldist = 1;
            it.out_estride = n1;
            it.transform = static_cast<int>(li);
            it.need = ncol + (g_debug_stall.load() ? 1 : 0); // the test hook asks for a COL item that never comes
            it.ftw = -1;
            row.push_back(it);
            maxsmem = std::max(maxsmem, it.lines * pass_line_pitch(static_cast<int>(n2)) * 8);
        }
    }
    for (auto& kv : small)
    {
        const long long n = kv.first;
        int sidx = 0;
        const crdfft_status st = sched_index(n, &sidx);
        if (st != CRDFFT_OK)
            return st;
        const int lpi = std::max(1, std::min(threads / static_cast<int>((n + 15) / 16),
                                             kMaxSmemBytes / (pass_line_pitch(static_cast<int>(n)) * 8)));
        const std::vector<long long>& ts = kv.second;
        for (size_t i = 0; i < ts.size(); i += lpi)
        {
            UnevenItem it{};
            it.kind = kUnevenSmall;
            it.sched = sidx;
            it.lines = static_cast<int>(std::min<size_t>(lpi, ts.size() - i));
            it.line_table = static_cast<int>(line_off.size());
            for (int a = 0; a < it.lines; ++a)
                line_off.push_back(offsets[ts[i + a]]);
            it.in_estride = 1;
            it.out_estride = 1;
            it.transform = -1;
            it.ftw = -1;
            mid.push_back(it);
            maxsmem = std::max(maxsmem, it.lines * pass_line_pitch(static_cast<int>(n)) * 8);
        }
    }
    std::vector<UnevenItem> items;
    items.insert(items.end(), col.begin(), col.end());
    items.insert(items.end(), mid.begin(), mid.end());
    items.insert(items.end(), row.begin(), row.end());
    UnevenDesc& u = p.udesc;
    crdfft_status st = upload_vec(p, items, &u.items);
    if (st == CRDFFT_OK)
        st = upload_vec(p, scheds, &u.scheds);
    if (st == CRDFFT_OK)
        st = upload_vec(p, line_off, &u.line_off);
    if (st == CRDFFT_OK)
        st = upload_vec(p, fh, &u.tables.ftw_hi);
    if (st == CRDFFT_OK)
        st = upload_vec(p, fl, &u.tables.ftw_lo);
    std::vector<int> counters(1 + large.size(), 0);
    const int* cdev = nullptr;
    if (st == CRDFFT_OK)
        st = upload_vec(p, counters, &cdev);
    if (st != CRDFFT_OK)
        return st;
    u.counter = const_cast<int*>(cdev);
    u.done = u.counter + 1;
    u.err = p.err;
    u.nitems = static_cast<int>(items.size());
    u.ntransforms = static_cast<int>(large.size());
    u.spin_limit = g_debug_stall.load() ? (1 << 10) : (1 << 24);
    u.conj = 0;
    u.scale = 1.0f;
    // two item slots (one transformed while the next one's loads land) and the run-time stages' second buffer
    u.slot_elems = (std::max(maxsmem, 1024) + 127) / 128 * 128 / 8;
    p.usmem = 3 * u.slot_elems * 8;
    p.ws_bytes = static_cast<size_t>(scratch) * 8;
    p.uneven = true;
    p.algorithm = "uneven-batch";
    p.factors = {count, static_cast<long long>(items.size()), static_cast<long long>(large.size())};
    // one launch per execute (counter reset + the persistent kernel)
    p.steps[0].assign(1, Step{});
    p.steps[1].assign(1, Step{});
    return CRDFFT_OK;
}

// The uneven-batch plan (crdfft_plan_create_uneven); also the timing plans of uneven_variant.
crdfft_status create_uneven(const int64_t* sizes, int64_t count, const int64_t* offsets, Plan** out)
{
    *out = nullptr;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return CRDFFT_NO_DEVICE;
    const crdfft_status chk = first_use_self_check(dev);
    if (chk != CRDFFT_OK)
        return chk;
    std::vector<int64_t> packed;
    if (offsets == nullptr)
    {
        packed.resize(static_cast<size_t>(count));
        long long off = 0;
        for (int64_t t = 0; t < count; ++t) // packed, each transform 16-byte aligned (crdfft_uneven_offsets)
        {
            packed[static_cast<size_t>(t)] = off;
            off += (sizes[t] + 1) / 2 * 2;
        }
        offsets = packed.data();
    }
    std::unique_ptr<Plan> p(new Plan());
    p->desc = crdfft_desc{};
    p->desc.rank = 1;
    p->desc.kind = CRDFFT_C2C;
    p->desc.batch = count;
    p->device = dev;
    {
        void* e = nullptr;
        if (dev_alloc(&e, 256) != cudaSuccess)
            return CRDFFT_OOM;
        p->tables.push_back(e);
        if (cudaMemset(e, 0, 256) != cudaSuccess)
            return CRDFFT_LAUNCH;
        p->err = static_cast<int*>(e);
    }
    crdfft_status st = build_uneven(*p, sizes, count, offsets);
    if (st != CRDFFT_OK)
        return st;
    if (p->ws_bytes > 0)
    {
        if (dev_alloc(&p->ws, p->ws_bytes) != cudaSuccess)
        {
            p->ws = nullptr;
            return CRDFFT_OOM;
        }
        p->ws_owned = true;
    }
    if (!uploads_landed())
        return CRDFFT_LAUNCH;
    *out = p.release();
    return CRDFFT_OK;
}

crdfft_status validate(const crdfft_desc& d)
{
    if (d.rank < 1 || d.rank > 3 || d.batch < 1)
        return CRDFFT_INVALID_DESC;
    if (d.kind < CRDFFT_C2C || d.kind > CRDFFT_C2R || d.norm < 0 || d.norm > 1)
        return CRDFFT_INVALID_DESC;
    if (d.precision < 0 || d.precision > 4)
        return CRDFFT_INVALID_DESC;
    for (int i = 0; i < d.rank; ++i)
        if (d.dims[i] < 1)
            return CRDFFT_INVALID_DESC;
    if (d.istride < 0 || d.ostride < 0 || d.idist < 0 || d.odist < 0)
        return CRDFFT_INVALID_DESC;
    if (d.rank > 1 && (d.istride > 1 || d.ostride > 1))
        return CRDFFT_INVALID_DESC;
    return CRDFFT_OK;
}

// The segment geometry of a spectral descriptor (spectral.hpp:50-54, 146-149): the periodogram is one segment of
// the whole signal; Welch reads noverlap 0 as nperseg / 2.
struct SpecGeom
{
    long long nperseg = 0, noverlap = 0, hop = 0, nseg = 0;
};

bool spectral_geometry(const crdfft_spectral_desc& s, SpecGeom* g)
{
    if (s.nsamples < 1 || s.count < 1 || !(s.fs > 0.0) || s.mode < CRDFFT_SPECTRAL_WELCH ||
        s.mode > CRDFFT_SPECTRAL_PERIODOGRAM)
        return false;
    if (s.mode == CRDFFT_SPECTRAL_PERIODOGRAM)
    {
        g->nperseg = s.nsamples;
        g->noverlap = 0;
    }
    else
    {
        g->nperseg = s.nperseg;
        g->noverlap = (s.mode == CRDFFT_SPECTRAL_WELCH && s.noverlap == 0) ? s.nperseg / 2 : s.noverlap;
    }
    if (g->nperseg < 4 || (g->nperseg & 1) != 0 || !single_pass_ok(g->nperseg / 2) || g->noverlap < 0 ||
        g->noverlap >= g->nperseg)
        return false;
    g->hop = g->nperseg - g->noverlap;
    g->nseg = s.nsamples < g->nperseg ? 0 : (s.nsamples - g->noverlap) / g->hop;
    return true;
}

// The spectral estimators (spectral.cu): one launch over every segment of every signal, plus the fixed-order
// average for Welch.
crdfft_status build_spectral(Plan& p, const crdfft_spectral_desc& s)
{
    SpecGeom g;
    if (!spectral_geometry(s, &g))
        return CRDFFT_UNSUPPORTED_SIZE;
    const long long n = g.nperseg, M = n / 2, nfreq = M + 1;
    // the window in FP64, narrowed (windows.hpp:56-124: the periodic Hann window, fac = -pi + 2 pi i / n); the
    // density scale 1 / (fs sum w^2) over the narrowed values
    std::vector<float> win(static_cast<size_t>(n));
    double ss = 0.0;
    for (long long i = 0; i < n; ++i)
    {
        double w;
        if (s.mode == CRDFFT_SPECTRAL_PERIODOGRAM)
            w = 1.0;
        else if (s.window != nullptr)
            w = s.window[i];
        else
            w = 0.5 + 0.5 * std::cos(-M_PI + 2.0 * M_PI * static_cast<double>(i) / static_cast<double>(n));
        win[static_cast<size_t>(i)] = static_cast<float>(w);
        ss += static_cast<double>(win[static_cast<size_t>(i)]) * win[static_cast<size_t>(i)];
    }
    if (!(ss > 0.0))
        return CRDFFT_INVALID_ARG;
    void* dwin = nullptr;
    crdfft_status st = upload_table(p, win, &dwin);
    if (st != CRDFFT_OK)
        return st;
    std::vector<float> wn(static_cast<size_t>(2 * (M + 1)));
    for (long long k = 0; k <= M; ++k)
    {
        double re, im;
        root(k, n, &re, &im);
        wn[static_cast<size_t>(2 * k)] = static_cast<float>(re);
        wn[static_cast<size_t>(2 * k + 1)] = static_cast<float>(im);
    }
    void* dwn = nullptr;
    st = upload_table(p, wn, &dwn);
    if (st != CRDFFT_OK)
        return st;
    p.spectral = true;
    p.factors = {n, g.nseg};
    const bool welch = s.mode == CRDFFT_SPECTRAL_WELCH;
    p.algorithm = welch ? "spectral-welch" : s.mode == CRDFFT_SPECTRAL_SPECTROGRAM ? "spectral-spectrogram"
                                                                                    : "spectral-periodogram";
    if (g.nseg == 0)
    {
        if (welch)
        {
            Step z;
            z.kind = StepKind::Zero;
            z.count = s.count * nfreq * 4;
            z.src = z.dst = BufRef{Buf::Out, 0};
            p.steps[0].push_back(z);
        }
        return CRDFFT_OK;
    }
    Step sp;
    sp.kind = StepKind::Spectral;
    st = make_pass_desc(p, M, s.count * g.nseg, 1, LineMap{M, 0, 1}, LineMap{M, 0, 1}, false, false, 1.0f,
                        FourStepTw{}, &sp.pass);
    if (st != CRDFFT_OK)
        return st;
    int P = 16, lpc = 1, threads = 0, smem = 0;
    if (!spectral_shape(sp.pass, &P, &lpc, &threads, &smem))
        return CRDFFT_UNSUPPORTED_SIZE;
    SpectralDesc sd{};
    sd.nsamples = s.nsamples;
    sd.count = s.count;
    sd.nseg = g.nseg;
    sd.hop = g.hop;
    sd.nperseg = static_cast<int>(n);
    sd.lpc = lpc;
    sd.ntiles = static_cast<int>((g.nseg + lpc - 1) / lpc);
    sd.detrend = s.detrend ? 1 : 0;
    sd.welch = welch ? 1 : 0;
    sd.scale = static_cast<float>(1.0 / (s.fs * ss));
    sd.win = static_cast<const float*>(dwin);
    sd.wn = dwn;
    sp.sdesc = sd;
    sp.sthreads = threads;
    sp.ssmem = smem;
    sp.src = BufRef{Buf::In, 0};
    if (!welch)
    {
        sp.dst = BufRef{Buf::Out, 0};
        p.steps[0].push_back(sp);
        return CRDFFT_OK;
    }
    sp.dst = BufRef{Buf::Ws, 0};
    Step fin;
    fin.kind = StepKind::WelchFinish;
    fin.sdesc = sd;
    fin.src = BufRef{Buf::Ws, 0};
    fin.dst = BufRef{Buf::Out, 0};
    p.steps[0] = {sp, fin};
    p.ws_bytes = static_cast<size_t>(s.count * sd.ntiles * nfreq) * 4 + 8;
    return CRDFFT_OK;
}

crdfft_status create(const crdfft_desc* desc, Plan** out, const ConvReq* conv = nullptr,
                     const crdfft_spectral_desc* spec = nullptr)
{
    if (desc == nullptr || out == nullptr)
        return CRDFFT_INVALID_ARG;
    *out = nullptr;
    crdfft_status st = validate(*desc);
    if (st != CRDFFT_OK)
        return st;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return CRDFFT_NO_DEVICE;
    if (t_arena == nullptr) // the static-scratch entry point allocates nothing, so it cannot run the check
    {
        st = first_use_self_check(dev);
        if (st != CRDFFT_OK)
            return st;
    }
    std::unique_ptr<Plan> p(new Plan());
    p->desc = *desc;
    p->device = dev;
    p->use32 = desc->precision == CRDFFT_PREC_FP32;
    {
        void* e = nullptr;
        if (dev_alloc(&e, 256) != cudaSuccess)
            return CRDFFT_OOM;
        p->tables.push_back(e);
        if (cudaMemset(e, 0, 256) != cudaSuccess)
            return CRDFFT_LAUNCH;
        p->err = static_cast<int*>(e);
    }
    if (spec != nullptr)
        st = build_spectral(*p, *spec);
    else if (conv != nullptr)
        st = build_conv(*p, *conv);
    else if (desc->kind != CRDFFT_C2C)
        st = desc->rank == 1 ? build_real(*p) : build_nd_real(*p);
    else if (desc->rank == 1)
        st = build_c2c_rank1(*p);
    else
        st = build_nd(*p);
    if (st != CRDFFT_OK)
        return st;
    if (p->ws_bytes > 0)
    {
        if (dev_alloc(&p->ws, p->ws_bytes) != cudaSuccess)
        {
            p->ws = nullptr;
            return CRDFFT_OOM;
        }
        p->ws_owned = true;
    }
    if (p->tc_steps > 0)
    {
        static const char* const kForm[5] = {"", "+tc-bf16x3", "+tc-fp16", "+tc-bf16x2", "+tc-fp16x2"};
        p->algorithm += kForm[desc->precision];
    }
    if (!uploads_landed())
        return CRDFFT_LAUNCH;
    *out = p.release();
    return CRDFFT_OK;
}

void* resolve(const BufRef& r, const void* in, void* out, void* ws)
{
    char* base = r.b == Buf::In ? static_cast<char*>(const_cast<void*>(in))
               : r.b == Buf::Out ? static_cast<char*>(out)
                                 : static_cast<char*>(ws);
    return base + r.off * 8;
}

// The uneven batch's execute: the counter reset and the persistent kernel, captured once per (in, out, direction)
// into a CUDA graph and launched as one graph on the caller's stream.
crdfft_status run_uneven(Plan& p, const void* in, void* out, int dir, cudaStream_t stream)
{
    UnevenDesc u = p.udesc;
    u.conj = dir;
    const std::tuple<const void*, void*, int> key{in, out, dir};
    cudaGraphExec_t exec = nullptr;
    {
        std::lock_guard<std::mutex> lk(p.graphs_mu);
        auto it = p.graphs.find(key);
        if (it != p.graphs.end())
            exec = it->second;
    }
    if (exec == nullptr)
    {
        cudaStream_t cap = nullptr;
        if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess)
            return CRDFFT_LAUNCH;
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess)
        {
            const cudaError_t le = launch_uneven(u, p.usmem, in, out, p.ws, cap);
            e = cudaStreamEndCapture(cap, &g);
            if (le != cudaSuccess)
                e = le;
        }
        if (e == cudaSuccess)
            e = cudaGraphInstantiate(&exec, g, 0);
        if (g != nullptr)
            cudaGraphDestroy(g);
        cudaStreamDestroy(cap);
        if (e != cudaSuccess)
            return CRDFFT_LAUNCH;
        std::lock_guard<std::mutex> lk(p.graphs_mu);
        p.graphs[key] = exec;
    }
    return cudaGraphLaunch(exec, stream) == cudaSuccess ? CRDFFT_OK : CRDFFT_LAUNCH;
}

crdfft_status run(Plan& p, const void* in, void* out, int dir, cudaStream_t stream, const void* spec = nullptr)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev != p.device)
        return CRDFFT_NO_DEVICE;
    if (p.ws_bytes > 0 && p.ws == nullptr)
        return CRDFFT_INVALID_ARG;
    if (p.uneven)
        return run_uneven(p, in, out, dir, stream);
    // Steps on the plan's internal streams (lanes 1 .. kMaxLanes) fork from the caller's stream and join back before
    // the next step on the caller's stream, and at the end.
    const cudaStream_t user = stream;
    bool forked = false;          // the current segment's fork event is recorded
    bool on[kMaxLanes] = {};      // lanes forked in the current segment
    auto join = [&]() {
        for (int i = 0; i < kMaxLanes; ++i)
            if (on[i])
            {
                if (cudaEventRecord(p.join[i], p.lanes[i]) != cudaSuccess ||
                    cudaStreamWaitEvent(user, p.join[i], 0) != cudaSuccess)
                    return false;
                on[i] = false;
            }
        forked = false;
        return true;
    };
    for (const Step& s : p.steps[dir])
    {
        if (s.lane != 0)
        {
            const int li = s.lane - 1;
            if (p.lanes[li] == nullptr &&
                (cudaStreamCreateWithFlags(&p.lanes[li], cudaStreamNonBlocking) != cudaSuccess ||
                 cudaEventCreateWithFlags(&p.join[li], cudaEventDisableTiming) != cudaSuccess))
                return CRDFFT_LAUNCH;
            if (p.fork == nullptr && cudaEventCreateWithFlags(&p.fork, cudaEventDisableTiming) != cudaSuccess)
                return CRDFFT_LAUNCH;
            if (!forked)
            {
                if (cudaEventRecord(p.fork, user) != cudaSuccess)
                    return CRDFFT_LAUNCH;
                forked = true;
            }
            if (!on[li])
            {
                if (cudaStreamWaitEvent(p.lanes[li], p.fork, 0) != cudaSuccess)
                    return CRDFFT_LAUNCH;
                on[li] = true;
            }
        }
        else if (forked && !join())
            return CRDFFT_LAUNCH;
        stream = s.lane == 0 ? user : p.lanes[s.lane - 1];
        void* src = resolve(s.src, in, out, p.ws);
        void* dst = resolve(s.dst, in, out, p.ws);
        cudaError_t e = cudaSuccess;
        switch (s.kind)
        {
            case StepKind::Line: e = launch_line_pass(s.pass, s.shape, src, dst, stream); break;
            case StepKind::Cluster: e = launch_cluster_fft(s.pass, s.pass2, s.count, src, dst, stream); break;
            case StepKind::TcLine: e = launch_tc_pass(s.pass, s.prec, s.amat, src, dst, stream); break;
            case StepKind::Conv:
                if (spec == nullptr)
                    return CRDFFT_INVALID_ARG;
                e = launch_conv(s.pass, s.shape.map, s.smap, src, spec, dst, stream);
                break;
            case StepKind::Spectral:
                e = launch_spectral(s.pass, s.sdesc, s.sthreads, s.ssmem, src, dst, stream);
                break;
            case StepKind::WelchFinish: e = launch_welch_finish(s.sdesc, src, dst, stream); break;
            case StepKind::TmaCol: e = launch_tma_col(s.pass, src, dst, stream); break;
            case StepKind::Zero: e = cudaMemsetAsync(dst, 0, static_cast<size_t>(s.count), stream); break;
            case StepKind::RowR2C: e = launch_row_r2c(s.pass, s.rr, src, dst, stream); break;
            case StepKind::RealLine:
                if (s.rmode == kRealConv && spec == nullptr)
                    return CRDFFT_INVALID_ARG;
                e = launch_real_line(s.pass, s.rmode, s.raux, src, spec, dst, stream);
                break;
            case StepKind::R2CPost: e = launch_r2c_post(s.real, src, dst, stream); break;
            case StepKind::C2RPre: e = launch_c2r_pre(s.real, src, dst, stream); break;
            case StepKind::ChirpPre: e = launch_chirp_pre(s.chirp, src, dst, stream); break;
            case StepKind::SpecMul: e = launch_spectrum_mul(s.chirp, dst, stream); break;
            case StepKind::ChirpPost: e = launch_chirp_post(s.chirp, src, dst, stream); break;
            case StepKind::Scale: e = launch_scale(dst, s.count, s.scale, stream); break;
            case StepKind::Chain:
            {
                ChainDesc cd = s.chain;
                void* wsb = resolve(s.aux, in, out, p.ws);
                cd.ctr = reinterpret_cast<int*>(static_cast<char*>(wsb) + cd.slots * cd.slot_elems * 8);
                e = launch_chain(cd, src, dst, wsb, stream);
                break;
            }
        }
        if (e != cudaSuccess)
        {
            // CRDFFT_LOG_ERRORS=1: name the failing step and the CUDA error on stderr
            static const bool log = std::getenv("CRDFFT_LOG_ERRORS") != nullptr;
            if (log)
                std::fprintf(stderr, "crdfft: step kind %d (n %d, lines %lld) failed: %s\n", static_cast<int>(s.kind),
                             s.pass.n, s.pass.lines, cudaGetErrorString(e));
            return CRDFFT_LAUNCH;
        }
    }
    if (forked && !join())
        return CRDFFT_LAUNCH;
    return CRDFFT_OK;
}

crdfft_status simple_plan(int api_kind, const crdfft_desc& d, crdfft_plan** plan)
{
    if (plan == nullptr)
        return CRDFFT_INVALID_ARG;
    Plan* p = nullptr;
    const crdfft_status st = create(&d, &p);
    if (st != CRDFFT_OK)
    {
        *plan = nullptr;
        return st;
    }
    p->api_kind = api_kind;
    *plan = reinterpret_cast<crdfft_plan*>(p);
    return CRDFFT_OK;
}

crdfft_desc desc_1d(long long n, int kind, int norm)
{
    crdfft_desc d{};
    d.rank = 1;
    d.kind = kind;
    d.precision = CRDFFT_PREC_FP32;
    d.norm = norm;
    d.dims[0] = n;
    d.batch = 1;
    return d;
}

Plan* as_plan(crdfft_plan* p) { return reinterpret_cast<Plan*>(p); }

} // namespace

// The line pass of a 1-D fused-convolution plan (its stages and forward twiddles), for kernels that run the same line
// FFT with their own load and store (the CWT's (signal, scale) lines, cwt_plan.cpp).
bool conv_line_pass(crdfft_plan* plan, PassDesc* out)
{
    if (plan == nullptr || out == nullptr)
        return false;
    const Plan& p = *as_plan(plan);
    if (!p.conv || p.algorithm != "fused-conv" || p.steps[0].size() != 1)
        return false;
    *out = p.steps[0][0].pass;
    return true;
}

} // namespace crdfft

namespace crdfft
{
void arena_bind(Arena* a) { t_arena = a; }
} // namespace crdfft

using namespace crdfft;

extern "C" {

crdfft_status crdfft_plan_create(const crdfft_desc* desc, crdfft_plan** plan)
{
    if (plan == nullptr)
        return CRDFFT_INVALID_ARG;
    Plan* p = nullptr;
    const crdfft_status st = create(desc, &p);
    *plan = reinterpret_cast<crdfft_plan*>(p);
    return st;
}

crdfft_status crdfft_plan_destroy(crdfft_plan* plan)
{
    delete as_plan(plan);
    return CRDFFT_OK;
}

crdfft_status crdfft_conv_plan_create(const crdfft_desc* desc, int32_t filter_per_transform, double scale,
                                      crdfft_plan** plan)
{
    if (plan == nullptr)
        return CRDFFT_INVALID_ARG;
    *plan = nullptr;
    ConvReq req;
    req.per_transform = filter_per_transform != 0;
    req.scale = scale;
    Plan* p = nullptr;
    const crdfft_status st = create(desc, &p, &req);
    if (st != CRDFFT_OK)
        return st;
    *plan = reinterpret_cast<crdfft_plan*>(p);
    return CRDFFT_OK;
}

crdfft_status crdfft_spectral_plan_create(const crdfft_spectral_desc* desc, crdfft_plan** plan)
{
    if (plan == nullptr || desc == nullptr)
        return CRDFFT_INVALID_ARG;
    *plan = nullptr;
    SpecGeom g;
    if (!spectral_geometry(*desc, &g))
        return CRDFFT_INVALID_DESC;
    // the descriptor of the segment transforms, for the plan's bookkeeping (info, validation)
    crdfft_desc d{};
    d.rank = 1;
    d.kind = CRDFFT_R2C;
    d.precision = CRDFFT_PREC_FP32;
    d.norm = CRDFFT_NORM_NONE;
    d.dims[0] = g.nperseg;
    d.batch = std::max<long long>(1, desc->count * g.nseg);
    Plan* p = nullptr;
    const crdfft_status st = create(&d, &p, nullptr, desc);
    if (st != CRDFFT_OK)
        return st;
    *plan = reinterpret_cast<crdfft_plan*>(p);
    return CRDFFT_OK;
}

int64_t crdfft_spectral_segments(const crdfft_spectral_desc* desc)
{
    SpecGeom g;
    if (desc == nullptr || !spectral_geometry(*desc, &g))
        return -1;
    return g.nseg;
}

crdfft_status crdfft_spectral_execute(crdfft_plan* plan, const float* x, float* out, void* stream)
{
    if (plan == nullptr || x == nullptr || out == nullptr)
        return CRDFFT_INVALID_ARG;
    Plan& p = *as_plan(plan);
    if (!p.spectral)
        return CRDFFT_INVALID_ARG;
    return run(p, x, out, 0, static_cast<cudaStream_t>(stream));
}

crdfft_status crdfft_conv_execute(crdfft_plan* plan, const void* in, const void* spectrum, void* out, void* stream)
{
    if (plan == nullptr || in == nullptr || spectrum == nullptr || out == nullptr)
        return CRDFFT_INVALID_ARG;
    Plan& p = *as_plan(plan);
    if (!p.conv)
        return CRDFFT_INVALID_ARG;
    return run(p, in, out, 0, static_cast<cudaStream_t>(stream), spectrum);
}

crdfft_status crdfft_execute(crdfft_plan* plan, const void* in, void* out, int32_t direction, void* stream)
{
    if (plan == nullptr || in == nullptr || out == nullptr)
        return CRDFFT_INVALID_ARG;
    Plan& p = *as_plan(plan);
    if (p.conv || p.spectral)
        return CRDFFT_INVALID_ARG;
    if (direction != CRDFFT_FORWARD && direction != CRDFFT_INVERSE)
        return CRDFFT_INVALID_ARG;
    if ((p.desc.kind == CRDFFT_R2C && direction != CRDFFT_FORWARD) ||
        (p.desc.kind == CRDFFT_C2R && direction != CRDFFT_INVERSE))
        return CRDFFT_INVALID_ARG;
    return run(p, in, out, direction, static_cast<cudaStream_t>(stream));
}

crdfft_status crdfft_execute_planar(crdfft_plan* plan, const float* re_in, const float* im_in, float* re_out,
                                    float* im_out, int32_t direction, void* stream)
{
    if (plan == nullptr || re_in == nullptr || im_in == nullptr || re_out == nullptr || im_out == nullptr)
        return CRDFFT_INVALID_ARG;
    Plan& p = *as_plan(plan);
    const crdfft_desc& d = p.desc;
    if (p.conv || p.spectral || p.uneven || d.kind != CRDFFT_C2C)
        return CRDFFT_INVALID_ARG;
    if (direction != CRDFFT_FORWARD && direction != CRDFFT_INVERSE)
        return CRDFFT_INVALID_ARG;
    long long total = 1;
    for (int i = 0; i < d.rank; ++i)
        total *= d.dims[i];
    // The planes are gathered and scattered whole, so the transforms must tile them exactly: packed batches
    // (stride 1, distance prod(dims)) or, for rank 1, the element-major batch (stride batch, distance 1).
    const bool packed = (d.istride == 0 || d.istride == 1) && (d.ostride == 0 || d.ostride == 1) &&
                        (d.idist == 0 || d.idist == total) && (d.odist == 0 || d.odist == total);
    const bool element_major = d.rank == 1 && d.istride == d.batch && d.ostride == d.batch && d.idist == 1 &&
                               d.odist == 1;
    if (!packed && !element_major)
        return CRDFFT_INVALID_ARG;
    const long long count = total * d.batch;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    {
        std::lock_guard<std::mutex> lk(p.planar_mu);
        if (p.planar == nullptr)
        {
            int dev = -1;
            if (cudaGetDevice(&dev) != cudaSuccess || dev != p.device)
                return CRDFFT_NO_DEVICE;
            if (dev_alloc(&p.planar, static_cast<size_t>(count) * 8) != cudaSuccess)
            {
                p.planar = nullptr;
                return CRDFFT_OOM;
            }
        }
    }
    if (launch_planar_gather(re_in, im_in, p.planar, count, s) != cudaSuccess)
        return CRDFFT_LAUNCH;
    const crdfft_status st = run(p, p.planar, p.planar, direction, s);
    if (st != CRDFFT_OK)
        return st;
    return launch_planar_scatter(p.planar, re_out, im_out, count, s) == cudaSuccess ? CRDFFT_OK : CRDFFT_LAUNCH;
}

namespace
{

// Element sizes and per-transform extents (elements) of a plan's input and output, and its transform distances.
struct HostLayout
{
    size_t in_elem, out_elem;
    long long in_ext, out_ext, idist, odist;
};

bool host_layout(const crdfft_desc& d, HostLayout* L)
{
    if ((d.istride != 0 && d.istride != 1) || (d.ostride != 0 && d.ostride != 1))
        return false;
    long long total = 1;
    for (int i = 0; i < d.rank; ++i)
        total *= d.dims[i];
    const long long last = d.rank > 0 ? d.dims[d.rank - 1] : 1;
    const long long half = (total / last) * (last / 2 + 1); // the Hermitian half along the last axis
    L->in_elem = d.kind == CRDFFT_R2C ? 4 : 8;
    L->out_elem = d.kind == CRDFFT_C2R ? 4 : 8;
    L->in_ext = d.kind == CRDFFT_C2R ? half : total;
    L->out_ext = d.kind == CRDFFT_R2C ? half : total;
    L->idist = d.idist ? d.idist : L->in_ext;
    L->odist = d.odist ? d.odist : L->out_ext;
    return true;
}

crdfft_status host_pipe_setup(Plan& p, const HostLayout& L)
{
    std::unique_ptr<Plan::HostPipe> h(new Plan::HostPipe());
    // Chunks of an eighth of the batch, between 4 and 64 MiB of input: enough chunks for the copies in both
    // directions to overlap, each large enough to run the copy engines at full rate.
    const long long per = std::max<long long>(1, static_cast<long long>(L.in_elem) * L.idist);
    const long long target = std::min<long long>(64LL << 20, std::max<long long>(4LL << 20, per * p.desc.batch / 8));
    h->chunk = std::max<long long>(1, std::min<long long>(p.desc.batch, target / per));
    crdfft_desc cd = p.desc;
    cd.batch = h->chunk;
    crdfft_status st = create(&cd, &h->full);
    if (st != CRDFFT_OK)
        return st;
    const long long rest = p.desc.batch % h->chunk;
    if (rest != 0 && p.desc.batch > h->chunk)
    {
        cd.batch = rest;
        st = create(&cd, &h->tail);
        if (st != CRDFFT_OK)
        {
            delete h->full;
            return st;
        }
    }
    const size_t in_bytes = static_cast<size_t>((h->chunk - 1) * L.idist + L.in_ext) * L.in_elem;
    const size_t out_bytes = static_cast<size_t>((h->chunk - 1) * L.odist + L.out_ext) * L.out_elem;
    bool ok = true;
    for (int i = 0; i < Plan::kHostSlots && ok; ++i)
        ok = dev_alloc(&h->din[i], in_bytes) == cudaSuccess && dev_alloc(&h->dout[i], out_bytes) == cudaSuccess &&
             cudaEventCreateWithFlags(&h->loaded[i], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&h->computed[i], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&h->drained[i], cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; i < 3 && ok; ++i)
        ok = cudaStreamCreateWithFlags(&h->st[i], cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&h->start, cudaEventDisableTiming) == cudaSuccess;
    p.host = h.release();
    return ok ? CRDFFT_OK : CRDFFT_OOM;
}

} // namespace

crdfft_status crdfft_execute_host(crdfft_plan* plan, const void* in, void* out, int32_t direction, void* stream)
{
    if (plan == nullptr || in == nullptr || out == nullptr)
        return CRDFFT_INVALID_ARG;
    Plan& p = *as_plan(plan);
    if (direction != CRDFFT_FORWARD && direction != CRDFFT_INVERSE)
        return CRDFFT_INVALID_ARG;
    if ((p.desc.kind == CRDFFT_R2C && direction != CRDFFT_FORWARD) ||
        (p.desc.kind == CRDFFT_C2R && direction != CRDFFT_INVERSE))
        return CRDFFT_INVALID_ARG;
    HostLayout L{};
    if (p.uneven || p.conv || p.spectral || !host_layout(p.desc, &L))
        return CRDFFT_INVALID_ARG;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev != p.device)
        return CRDFFT_NO_DEVICE;
    std::lock_guard<std::mutex> lk(p.host_mu);
    if (p.host == nullptr)
    {
        const crdfft_status st = host_pipe_setup(p, L);
        if (st != CRDFFT_OK)
            return st;
    }
    Plan::HostPipe& h = *p.host;
    if (h.st[2] == nullptr || h.start == nullptr)
        return CRDFFT_OOM;
    const cudaStream_t user = static_cast<cudaStream_t>(stream);
    const cudaStream_t s_in = h.st[0], s_run = h.st[1], s_out = h.st[2];
    // the three stages start after the work already on the caller's stream
    if (cudaEventRecord(h.start, user) != cudaSuccess)
        return CRDFFT_LAUNCH;
    for (cudaStream_t st : h.st)
        if (cudaStreamWaitEvent(st, h.start, 0) != cudaSuccess)
            return CRDFFT_LAUNCH;
    const char* hin = static_cast<const char*>(in);
    char* hout = static_cast<char*>(out);
    long long k = 0;
    for (long long t0 = 0; t0 < p.desc.batch; t0 += h.chunk, ++k)
    {
        const int s = static_cast<int>(k % Plan::kHostSlots);
        const bool reused = k >= Plan::kHostSlots; // the slot served chunk k - kHostSlots
        const long long c = std::min(h.chunk, p.desc.batch - t0);
        Plan* cp = c == h.chunk ? h.full : h.tail;
        const size_t ib = static_cast<size_t>((c - 1) * L.idist + L.in_ext) * L.in_elem;
        const size_t ob = static_cast<size_t>((c - 1) * L.odist + L.out_ext) * L.out_elem;
        // copy in once the slot's previous transform has read its input
        if ((reused && cudaStreamWaitEvent(s_in, h.computed[s], 0) != cudaSuccess) ||
            cudaMemcpyAsync(h.din[s], hin + static_cast<size_t>(t0 * L.idist) * L.in_elem, ib,
                            cudaMemcpyHostToDevice, s_in) != cudaSuccess ||
            cudaEventRecord(h.loaded[s], s_in) != cudaSuccess)
            return CRDFFT_LAUNCH;
        // transform once the input is in and the slot's previous output has been copied out
        if (cudaStreamWaitEvent(s_run, h.loaded[s], 0) != cudaSuccess ||
            (reused && cudaStreamWaitEvent(s_run, h.drained[s], 0) != cudaSuccess))
            return CRDFFT_LAUNCH;
        const crdfft_status st = run(*cp, h.din[s], h.dout[s], direction, s_run);
        if (st != CRDFFT_OK)
            return st;
        if (cudaEventRecord(h.computed[s], s_run) != cudaSuccess)
            return CRDFFT_LAUNCH;
        // copy out once the transform is done
        if (cudaStreamWaitEvent(s_out, h.computed[s], 0) != cudaSuccess ||
            cudaMemcpyAsync(hout + static_cast<size_t>(t0 * L.odist) * L.out_elem, h.dout[s], ob,
                            cudaMemcpyDeviceToHost, s_out) != cudaSuccess ||
            cudaEventRecord(h.drained[s], s_out) != cudaSuccess)
            return CRDFFT_LAUNCH;
    }
    // the caller's stream waits for the last copy out (which follows every transform and every copy in)
    const int last = static_cast<int>((k - 1) % Plan::kHostSlots);
    if (cudaStreamWaitEvent(user, h.drained[last], 0) != cudaSuccess)
        return CRDFFT_LAUNCH;
    return CRDFFT_OK;
}

crdfft_status crdfft_plan_info_get(const crdfft_plan* plan, crdfft_plan_info* info)
{
    if (plan == nullptr || info == nullptr)
        return CRDFFT_INVALID_ARG;
    const Plan& p = *reinterpret_cast<const Plan*>(plan);
    std::memset(info, 0, sizeof(*info));
    std::strncpy(info->algorithm, p.algorithm.c_str(), sizeof(info->algorithm) - 1);
    info->passes = static_cast<int32_t>(p.steps[p.desc.kind == CRDFFT_C2R ? 1 : 0].size());
    info->device = p.device;
    info->workspace_bytes = static_cast<int64_t>(p.ws_bytes);
    info->table_bytes = p.table_bytes;
    for (size_t i = 0; i < p.factors.size() && i < 7; ++i)
        info->factors[i] = p.factors[i];
    return CRDFFT_OK;
}

size_t crdfft_workspace_size(const crdfft_plan* plan)
{
    return plan == nullptr ? 0 : reinterpret_cast<const Plan*>(plan)->ws_bytes;
}

crdfft_status crdfft_set_workspace(crdfft_plan* plan, void* workspace, size_t bytes)
{
    if (plan == nullptr)
        return CRDFFT_INVALID_ARG;
    Plan& p = *as_plan(plan);
    if (workspace == nullptr)
    {
        if (p.ws_owned || p.ws_bytes == 0)
            return CRDFFT_OK;
        void* w = nullptr;
        if (dev_alloc(&w, p.ws_bytes) != cudaSuccess)
            return CRDFFT_OOM;
        p.ws = w;
        p.ws_owned = true;
        return CRDFFT_OK;
    }
    if (bytes < p.ws_bytes || (reinterpret_cast<uintptr_t>(workspace) & 255u) != 0)
        return CRDFFT_INVALID_ARG;
    if (p.ws_owned && p.ws != nullptr)
        cudaFree(p.ws);
    p.ws = workspace;
    p.ws_owned = false;
    return CRDFFT_OK;
}

const char* crdfft_status_string(crdfft_status status)
{
    switch (status)
    {
        case CRDFFT_OK: return "ok";
        case CRDFFT_INVALID_DESC: return "invalid descriptor";
        case CRDFFT_UNSUPPORTED_SIZE: return "unsupported size or layout";
        case CRDFFT_OOM: return "device out of memory";
        case CRDFFT_LAUNCH: return "kernel launch failed";
        case CRDFFT_DEVICE_TIMEOUT: return "device-side wait timed out";
        case CRDFFT_NUMERIC_SELFCHECK: return "device self-check failed";
        case CRDFFT_INVALID_ARG: return "invalid argument";
        case CRDFFT_NO_DEVICE: return "no CUDA device / wrong device";
    }
    return "unknown status";
}

crdfft_status crdfft_fft_plan_create(int64_t n, crdfft_plan** plan)
{
    return simple_plan(1, desc_1d(n, CRDFFT_C2C, CRDFFT_NORM_NONE), plan);
}

crdfft_status crdfft_fft_execute(crdfft_plan* plan, void* data, int32_t direction, void* stream)
{
    return crdfft_execute(plan, data, data, direction, stream);
}

crdfft_status crdfft_fft_execute_batched(crdfft_plan* plan, void* data, int64_t batch, int32_t direction,
                                         void* stream)
{
    if (plan == nullptr || data == nullptr || batch < 1)
        return CRDFFT_INVALID_ARG;
    Plan& p = *as_plan(plan);
    if (p.desc.rank != 1 || p.desc.kind != CRDFFT_C2C)
        return CRDFFT_INVALID_ARG;
    Plan* sub = nullptr;
    {
        std::lock_guard<std::mutex> lk(p.batched_mu);
        auto it = p.batched.find(batch);
        if (it != p.batched.end())
            sub = it->second;
        else
        {
            crdfft_desc d = p.desc;
            d.batch = batch;
            d.istride = batch;
            d.ostride = batch;
            d.idist = 1;
            d.odist = 1;
            const crdfft_status st = create(&d, &sub);
            if (st != CRDFFT_OK)
                return st;
            p.batched[batch] = sub;
        }
    }
    return crdfft_execute(reinterpret_cast<crdfft_plan*>(sub), data, data, direction, stream);
}

crdfft_status crdfft_real_plan_create(int64_t n, crdfft_plan** plan)
{
    // One plan answers both verbs: the forward steps are R2C, the inverse steps C2R.
    if (plan == nullptr)
        return CRDFFT_INVALID_ARG;
    Plan* f = nullptr;
    crdfft_desc d = desc_1d(n, CRDFFT_R2C, CRDFFT_NORM_INVERSE);
    crdfft_status st = create(&d, &f);
    if (st != CRDFFT_OK)
    {
        *plan = nullptr;
        return st;
    }
    Plan* inv = nullptr;
    d.kind = CRDFFT_C2R;
    st = create(&d, &inv);
    if (st != CRDFFT_OK)
    {
        delete f;
        *plan = nullptr;
        return st;
    }
    // Fold the C2R steps, tables and workspace into the R2C plan.
    f->steps[1] = inv->steps[1];
    for (void* t : inv->tables)
        f->tables.push_back(t);
    inv->tables.clear();
    f->table_bytes += inv->table_bytes;
    if (inv->ws_bytes > f->ws_bytes)
    {
        if (f->ws_owned && f->ws)
            cudaFree(f->ws);
        f->ws = inv->ws;
        f->ws_owned = inv->ws_owned;
        f->ws_bytes = inv->ws_bytes;
        inv->ws = nullptr;
        inv->ws_owned = false;
    }
    delete inv;
    f->api_kind = 2;
    f->desc.kind = CRDFFT_C2C; // both directions allowed through the verbs below
    *plan = reinterpret_cast<crdfft_plan*>(f);
    return CRDFFT_OK;
}

crdfft_status crdfft_rfft(crdfft_plan* plan, const float* real_in, void* out, void* stream)
{
    if (plan == nullptr || as_plan(plan)->api_kind != 2 || real_in == nullptr || out == nullptr)
        return CRDFFT_INVALID_ARG;
    return run(*as_plan(plan), real_in, out, 0, static_cast<cudaStream_t>(stream));
}

crdfft_status crdfft_irfft(crdfft_plan* plan, const void* in, float* real_out, void* stream)
{
    if (plan == nullptr || as_plan(plan)->api_kind != 2 || in == nullptr || real_out == nullptr)
        return CRDFFT_INVALID_ARG;
    return run(*as_plan(plan), in, real_out, 1, static_cast<cudaStream_t>(stream));
}

crdfft_status crdfft_bluestein_plan_create(int64_t n, crdfft_plan** plan)
{
    return simple_plan(3, desc_1d(n, CRDFFT_C2C, CRDFFT_NORM_INVERSE), plan);
}

crdfft_status crdfft_bluestein_execute(crdfft_plan* plan, void* data, int32_t direction, void* stream)
{
    return crdfft_execute(plan, data, data, direction, stream);
}

crdfft_status crdfft_nd_plan_create(int32_t ndim, const int64_t* dims, crdfft_plan** plan)
{
    if (dims == nullptr || ndim < 1 || ndim > 3)
        return CRDFFT_INVALID_DESC;
    crdfft_desc d{};
    d.rank = ndim;
    d.kind = CRDFFT_C2C;
    d.precision = CRDFFT_PREC_FP32;
    d.norm = CRDFFT_NORM_INVERSE;
    for (int i = 0; i < ndim; ++i)
        d.dims[i] = dims[i];
    d.batch = 1;
    return simple_plan(4, d, plan);
}

crdfft_status crdfft_nd_execute(crdfft_plan* plan, void* data, int32_t direction, void* stream)
{
    return crdfft_execute(plan, data, data, direction, stream);
}

crdfft_status crdfft_fft(void* data, int64_t n, int32_t direction, void* stream)
{
    crdfft_plan* p = nullptr;
    crdfft_status st = crdfft_fft_plan_create(n, &p);
    if (st != CRDFFT_OK)
        return st;
    st = crdfft_fft_execute(p, data, direction, stream);
    cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    crdfft_plan_destroy(p);
    return st;
}

crdfft_status crdfft_ifft_normalized(void* data, int64_t n, void* stream)
{
    crdfft_plan* p = nullptr;
    crdfft_desc d = desc_1d(n, CRDFFT_C2C, CRDFFT_NORM_INVERSE);
    crdfft_status st = simple_plan(1, d, &p);
    if (st != CRDFFT_OK)
        return st;
    st = crdfft_execute(p, data, data, CRDFFT_INVERSE, stream);
    cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    crdfft_plan_destroy(p);
    return st;
}

void crdfft_debug_fail_alloc_after(int32_t k) { g_fail_alloc_after.store(k < 0 ? 0 : k); }

void crdfft_debug_stall_waits(int32_t on) { g_debug_stall.store(on ? 1 : 0); }

void crdfft_set_planner_mode(int32_t mode) { set_planner_mode(mode); }

void crdfft_debug_uneven_variant(int32_t variant) { g_uneven_force.store(variant < 0 ? -1 : (variant ? 1 : 0)); }

crdfft_status crdfft_set_decomposition(int64_t n, int32_t kind, int64_t n1)
{
    if (kind < 0 || kind > 3 || n < 1 || (kind == 3 && (n1 < 2 || n % n1 != 0)))
        return CRDFFT_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_hint_mu);
    if (kind == 0)
        g_hints.erase(n);
    else
        g_hints[n] = Decomp{kind, kind == 3 ? n1 : 0};
    return CRDFFT_OK;
}

int64_t crdfft_uneven_offsets(const int64_t* sizes, int64_t count, int64_t* offsets)
{
    if (sizes == nullptr || count < 0)
        return -1;
    int64_t off = 0;
    for (int64_t t = 0; t < count; ++t)
    {
        if (offsets != nullptr)
            offsets[t] = off;
        off += (sizes[t] + 1) / 2 * 2; // each transform starts on a 16-byte boundary
    }
    return off;
}

crdfft_status crdfft_plan_create_uneven(const int64_t* sizes, int64_t count, const int64_t* offsets,
                                        crdfft_plan** plan)
{
    if (plan == nullptr || sizes == nullptr || count < 1)
        return CRDFFT_INVALID_ARG;
    *plan = nullptr;
    Plan* p = nullptr;
    const crdfft_status st = create_uneven(sizes, count, offsets, &p);
    if (st == CRDFFT_OK)
        *plan = reinterpret_cast<crdfft_plan*>(p);
    return st;
}

static crdfft_status copy_out(const std::string& s, char* buf, size_t cap, size_t* needed)
{
    if (needed != nullptr)
        *needed = s.size() + 1;
    if (buf == nullptr || cap == 0)
        return CRDFFT_OK;
    if (cap < s.size() + 1)
        return CRDFFT_INVALID_ARG;
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return CRDFFT_OK;
}

crdfft_status crdfft_wisdom_export(char* buf, size_t cap, size_t* needed)
{
    return copy_out(wisdom_export(), buf, cap, needed);
}

crdfft_status crdfft_wisdom_import(const char* text)
{
    if (text == nullptr)
        return CRDFFT_INVALID_ARG;
    return wisdom_import(text) < 0 ? CRDFFT_INVALID_ARG : CRDFFT_OK;
}

void crdfft_wisdom_forget(void) { wisdom_forget(); }

crdfft_status crdfft_planner_log(char* buf, size_t cap, size_t* needed)
{
    return copy_out(planner_log_export(), buf, cap, needed);
}

int32_t crdfft_pass_feature_count(void) { return kPassFeatures; }

crdfft_status crdfft_learned_model_import(const char* text)
{
    if (text == nullptr)
        return CRDFFT_INVALID_ARG;
    return learned_import(text) < 0 ? CRDFFT_INVALID_ARG : CRDFFT_OK;
}

crdfft_status crdfft_learned_model_export(char* buf, size_t cap, size_t* needed)
{
    return copy_out(learned_export(), buf, cap, needed);
}

void crdfft_learned_model_forget(void) { learned_forget(); }

crdfft_status crdfft_learned_predict(const float* features, float* out)
{
    if (features == nullptr || out == nullptr)
        return CRDFFT_INVALID_ARG;
    if (!learned_ready())
        return CRDFFT_INVALID_ARG;
    *out = learned_predict(features);
    return CRDFFT_OK;
}

crdfft_status crdfft_device_status(crdfft_plan* plan, void* stream)
{
    if (plan == nullptr)
        return CRDFFT_INVALID_ARG;
    Plan& p = *as_plan(plan);
    int flag = 0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (cudaMemcpyAsync(&flag, p.err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return CRDFFT_LAUNCH;
    if (flag != 0)
    {
        if (cudaMemsetAsync(p.err, 0, sizeof(int), s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
            return CRDFFT_LAUNCH;
        return CRDFFT_DEVICE_TIMEOUT;
    }
    for (auto& kv : p.batched)
    {
        const crdfft_status st = crdfft_device_status(reinterpret_cast<crdfft_plan*>(kv.second), stream);
        if (st != CRDFFT_OK)
            return st;
    }
    return CRDFFT_OK;
}

} // extern "C"
