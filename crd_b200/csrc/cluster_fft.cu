// Cluster-fused four-step: one thread-block cluster of C CTAs transforms one line of length N = N1 * N2 that is too
// long for one CTA's shared memory but fits the cluster's, with one HBM read and one HBM write per element.
//
//   phase A  CTA c transforms columns n2 in [c N2/C, (c+1) N2/C): length-N1 DFTs over n1 of x[n1 N2 + n2],
//            read straight from HBM (coalesced across the CTA's adjacent columns), result kept in shared memory
//   exchange cluster barrier; CTA c gathers rows k1 in [c N1/C, (c+1) N1/C) of all columns from the other CTAs'
//            shared memory (distributed shared memory reads), multiplying by the four-step twiddle W_N^{n2 k1}
//            (factored into two 32 KiB tables that stay in L1, shared by every transform);
//            a second cluster barrier, then it stores them into its own (reused) shared memory
//   phase B  CTA c transforms its rows: length-N2 DFTs over n2, written straight to X[k1 + N1 k2] (coalesced across
//            its adjacent rows)
//
// It replaces the reference's four-step / deep-split passes at these sizes (engine/numerics/hesap-fft/kernels/
// fft_kernels.cpp:359-515, 2363-2658), whose intermediate round-trips through memory. The stage code is the
// line-FFT kernel's (line_fft.cuh). The cluster barriers are hardware barriers; nothing here spins on a flag.

#include "kernels.hpp"
#include "line_fft.cuh"

#include <cooperative_groups.h>

#include <cstdlib>

namespace cg = cooperative_groups;

// Cluster barrier, every thread of every CTA: arrive with release semantics (this CTA's shared-memory writes become
// visible to the cluster), wait with acquire semantics. The .aligned forms (all threads of the warp execute them
// together, which holds here) skip the per-thread convergence handling of the generic barrier.
__device__ __forceinline__ void cluster_barrier()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

namespace crdfft
{
namespace lfft
{
namespace
{

// Launched with a cluster of C CTAs (a launch attribute: 16 is above the portable size and needs the kernel's
// non-portable opt-in). Two CTAs an SM at C = 8 (512 threads), five at C = 16 (256 threads).
template <class S1, class S2, int C, int P, bool EPI, int MINB>
__global__ void __launch_bounds__((S1::n * S2::n) / (P * C), MINB)
    cluster_fft_kernel(const PassDesc dA, const PassDesc dB, const float2* __restrict__ gin, float2* __restrict__ gout)
{
    constexpr int N1 = S1::n;
    constexpr int N2 = S2::n;
    constexpr int N = N1 * N2;
    constexpr int LA = N2 / C; // columns a CTA transforms in phase A
    constexpr int LB = N1 / C; // rows a CTA transforms in phase B
    constexpr int TA = (N1 + P - 1) / P;
    constexpr int TB = (N2 + P - 1) / P;
    constexpr int THREADS = N / (P * C);
    static_assert(TA * LA == THREADS && TB * LB == THREADS, "both phases use every thread");
    constexpr int PA = LA + 1; // odd pitches: conflict-free column access
    constexpr int PB = LB + 1;
    extern __shared__ float2 buf[];

    cg::cluster_group cluster = cg::this_cluster();
    const int rank = static_cast<int>(cluster.block_rank());
    const long long t = blockIdx.x / C; // transform
    const int tid = threadIdx.x;

    // ---- phase A: columns
    {
        Ctx c;
        init_scales(dA, c);
        const int jt = tid / LA;
        const int ll = tid - jt * LA;
        c.jt = jt;
        c.T = TA;
        c.ok = true;
        c.q = rank * LA + ll;
        c.in = gin + t * N + rank * LA + ll;
        c.out = nullptr;
        const LayCol lay{buf + ll, PA};
        SchedRun<S1>::template go<P, true, false, false, Kind<PassMap::Col, EPI>>(dA, c, lay, N1);
    }
    cluster_barrier(); // every CTA's columns are in its shared memory

    // ---- exchange: rows k1 of this CTA, all n2, times W_N^{n2 k1}. A thread keeps one column n2 (THREADS is a
    // multiple of N2), so it reads one remote CTA's shared memory, and the twiddle W_N^{n2 k1} is
    // hi[(n2>>4) N1 + k1] * lo[16 k1 + (n2&15)]: for one k1, a warp's 32 columns read two hi entries and 16
    // consecutive lo entries (L1-resident tables).
    static_assert(THREADS % N2 == 0, "a thread keeps one column through the exchange");
    constexpr int PER = (LB * N2) / THREADS;
    constexpr int KSTEP = THREADS / N2;
    float2 v[PER];
    const int n2 = tid % N2;
    const int kl0 = tid / N2;
    const int src = n2 / LA;
    const float2* remote = cluster.map_shared_rank(buf, src) + (n2 - src * LA);
    const float2* twh = static_cast<const float2*>(dA.ftw_hi) + (n2 >> 4) * N1;
    const float2* twl = static_cast<const float2*>(dA.ftw_lo) + (n2 & 15);
#pragma unroll
    for (int i = 0; i < PER; ++i)
    {
        const int k1 = rank * LB + kl0 + i * KSTEP;
        v[i] = cmul(remote[k1 * PA], cmul(__ldg(twh + k1), __ldg(twl + k1 * 16)));
    }
    cluster_barrier(); // every CTA's remote reads are performed (release); shared memory may be reused
#pragma unroll
    for (int i = 0; i < PER; ++i)
        buf[n2 * PB + kl0 + i * KSTEP] = v[i];
    __syncthreads();

    // ---- phase B: rows, stored transposed to X[k1 + N1 k2]
    {
        Ctx c;
        init_scales(dB, c);
        const int jt = tid / LB;
        const int ll = tid - jt * LB;
        c.jt = jt;
        c.T = TB;
        c.ok = true;
        c.q = 0;
        c.in = nullptr;
        c.out = gout + t * N + rank * LB + ll;
        const LayCol lay{buf + ll, PB};
        SchedRun<S2>::template go<P, false, true, false, Kind<PassMap::Col, EPI>>(dB, c, lay, N2);
    }
}

using ClusterFn = void (*)(const PassDesc, const PassDesc, const float2*, float2*);

// MINB: CTAs an SM the registers are sized for (the kernel is latency-bound: more resident clusters hide the cluster
// barriers better).
template <class S1, class S2, int C, int P, int MINB> struct ClusterInst
{
    static constexpr int threads = (S1::n * S2::n) / (P * C);
    static constexpr int smem_elems =
        (S1::n * (S2::n / C + 1)) > (S2::n * (S1::n / C + 1)) ? (S1::n * (S2::n / C + 1)) : (S2::n * (S1::n / C + 1));
    static ClusterFn get(bool epi)
    {
        return epi ? cluster_fft_kernel<S1, S2, C, P, true, MINB> : cluster_fft_kernel<S1, S2, C, P, false, MINB>;
    }
};

struct ClusterEntry
{
    int n1, n2, cluster, threads, smem_bytes;
    ClusterFn fn_epi, fn_plain;
    int minb;
};

template <class I> ClusterEntry entry(int n1, int n2, int c, int minb)
{
    return ClusterEntry{n1, n2, c, I::threads, I::smem_elems * 8, I::get(true), I::get(false), minb};
}

const ClusterEntry* find(long long n1, long long n2)
{
    static const ClusterEntry table[] = {
        entry<ClusterInst<Sched<16, 16>, Sched<16, 16>, 8, 16, 2>>(256, 256, 8, 2),    // 65536
        // 65536, 16-CTA clusters at five CTAs an SM (48 registers, no spills; 1.68 -> 1.60 ms per 2 GiB over four;
        // six spill and are slower), four kept for comparison (CRDFFT_CLUSTER_OCC=4)
        entry<ClusterInst<Sched<16, 16>, Sched<16, 16>, 16, 16, 5>>(256, 256, 16, 5),
        entry<ClusterInst<Sched<16, 16>, Sched<16, 16>, 16, 16, 4>>(256, 256, 16, 4),
    };
    static const int want = [] {
        const char* e = std::getenv("CRDFFT_CLUSTER_SIZE");
        return e != nullptr ? std::atoi(e) : 16;
    }();
    const int occ = [] {
        const char* e = std::getenv("CRDFFT_CLUSTER_OCC");
        return e != nullptr ? std::atoi(e) : 0;
    }();
    const ClusterEntry* any = nullptr;
    for (const ClusterEntry& e : table)
        if (e.n1 == n1 && e.n2 == n2)
        {
            if (e.cluster == want && (occ == 0 || e.minb == occ))
                return &e;
            if (any == nullptr)
                any = &e;
        }
    return any;
}

} // namespace
} // namespace lfft

bool cluster_split(long long n, long long* n1, long long* n2)
{
    for (long long a : {256LL})
        if (n % a == 0 && lfft::find(a, n / a) != nullptr)
        {
            *n1 = a;
            *n2 = n / a;
            return true;
        }
    return false;
}

cudaError_t launch_cluster_fft(const PassDesc& a, const PassDesc& b, long long batch, const void* in, void* out,
                               cudaStream_t stream)
{
    const lfft::ClusterEntry* e = lfft::find(a.n, b.n);
    if (e == nullptr || batch < 1)
        return cudaErrorInvalidConfiguration;
    // The four-step twiddle is applied in the exchange, so only conjugation and scale select the EPI instance.
    const bool epi = a.conj_in != 0 || b.conj_out != 0 || b.scale != 1.0f;
    lfft::ClusterFn fn = epi ? e->fn_epi : e->fn_plain;
    if (e->smem_bytes > 48 * 1024)
    {
        const cudaError_t err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, e->smem_bytes);
        if (err != cudaSuccess)
            return err;
    }
    const long long grid = batch * e->cluster;
    if (grid > 0x7fffffffLL)
        return cudaErrorInvalidConfiguration;
    if (e->cluster > 8)
    {
        const cudaError_t err = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (err != cudaSuccess)
            return err;
    }
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(static_cast<unsigned>(grid), 1, 1);
    cfg.blockDim = dim3(static_cast<unsigned>(e->threads), 1, 1);
    cfg.dynamicSmemBytes = static_cast<size_t>(e->smem_bytes);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = static_cast<unsigned>(e->cluster);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, fn, a, b, static_cast<const float2*>(in), static_cast<float2*>(out));
}

} // namespace crdfft
