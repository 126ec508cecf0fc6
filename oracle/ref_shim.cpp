// Test infrastructure: a C ABI over the reference's own crd-hesap-fft plans, compiled together with the reference's
// sources by oracle/Makefile into oracle/_ref/libcrdref.so. Tests and the CPU-baseline leg of bench.py load it with
// ctypes; the product never links it. Every function forwards to the reference class named in its comment and adds
// only the batching loop the reference's batch semantics describe: a batch of independent transforms is split into
// contiguous ranges, one range and one plan per thread (engine/numerics/hesap-fft/include/crd/hesap/fft/detail/
// batch_arms.hpp:59-77).

#include <crd/hesap/complex.hpp>
#include <crd/hesap/dsp/spectral.hpp>
#include <crd/hesap/fft/bluestein.hpp>
#include <crd/hesap/fft/fft.hpp>
#include <crd/hesap/fft/fft_dispatch.hpp>
#include <crd/hesap/fft/nd_fft.hpp>
#include <crd/hesap/fft/real_fft.hpp>
#include <crd/hesap/wavelet/cwt.hpp>
#include <crd/memory/allocators/malloc_allocator.hpp>

#include <cstddef>
#include <cstdint>
#include <map>
#include <memory>
#include <thread>
#include <vector>

namespace fft = crd::hesap::fft;
namespace cont = crd::containers;
using crd::hesap::Complex;

namespace
{

// Never destroyed: plans kept in the caches below deallocate through it, and static destructors at process exit
// run in an order that could otherwise destroy the allocator first.
crd::memory::MallocAllocator& alloc()
{
    static crd::memory::MallocAllocator* a = new crd::memory::MallocAllocator("crdref-shim");
    return *a;
}

fft::FftDirection dir_of(int dir)
{
    return dir == 0 ? fft::FftDirection::Forward : fft::FftDirection::Inverse;
}

bool is_pow2(std::size_t n)
{
    return n != 0 && (n & (n - 1)) == 0;
}

// Runs fn(first, last) over [0, count) in `threads` contiguous ranges, one std::thread each (range j is
// [j*count/threads, (j+1)*count/threads)), the partition of batch_arms.hpp:59-77.
template <typename F> void fan_out(int threads, std::size_t count, const F& fn)
{
    if (threads <= 1 || count <= 1)
    {
        fn(std::size_t{0}, count);
        return;
    }
    const std::size_t t = static_cast<std::size_t>(threads) < count ? static_cast<std::size_t>(threads) : count;
    std::vector<std::thread> pool;
    pool.reserve(t);
    for (std::size_t j = 0; j < t; ++j)
    {
        pool.emplace_back([&fn, j, t, count]() { fn(j * count / t, (j + 1) * count / t); });
    }
    for (auto& th : pool)
    {
        th.join();
    }
}

// fan_out with the range index passed to fn(j, first, last).
template <typename F> void fan_out_indexed(std::size_t t, std::size_t count, const F& fn)
{
    if (t <= 1)
    {
        fn(std::size_t{0}, std::size_t{0}, count);
        return;
    }
    std::vector<std::thread> pool;
    pool.reserve(t);
    for (std::size_t j = 0; j < t; ++j)
    {
        pool.emplace_back([&fn, j, t, count]() { fn(j, j * count / t, (j + 1) * count / t); });
    }
    for (auto& th : pool)
    {
        th.join();
    }
}

// A batch of contiguous size-n complex transforms of type T, in place. Power-of-two sizes run FftPlan<T>::execute
// (fft.hpp:409-413, unnormalised both ways); other sizes run BluesteinPlan<T>::execute (bluestein.hpp:87-136, whose
// inverse is normalised by 1/n).
template <typename T> int c2c(std::size_t n, std::size_t batch, T* data, int dir, int threads)
{
    if (n == 0)
    {
        return -1;
    }
    auto* x = reinterpret_cast<Complex<T>*>(data);
    fan_out(threads, batch,
            [&](std::size_t first, std::size_t last)
            {
                if (is_pow2(n))
                {
                    const fft::FftPlan<T> plan(&alloc(), n);
                    for (std::size_t t = first; t < last; ++t)
                    {
                        plan.execute(cont::Span<Complex<T>>(x + t * n, n), dir_of(dir));
                    }
                }
                else
                {
                    const fft::BluesteinPlan<T> plan(&alloc(), n);
                    for (std::size_t t = first; t < last; ++t)
                    {
                        plan.execute(cont::Span<Complex<T>>(x + t * n, n), dir_of(dir));
                    }
                }
            });
    return 0;
}

} // namespace

namespace
{
template <typename T, typename F> int spectral_rows(std::size_t n, std::size_t count, const T* x, T* out,
                                                    std::size_t row, int threads, const F& one)
{
    fan_out(threads, count,
            [&](std::size_t first, std::size_t last)
            {
                for (std::size_t g = first; g < last; ++g)
                {
                    const auto r = one(cont::ConstSpan<T>(x + g * n, n));
                    for (std::size_t k = 0; k < row && k < r.size(); ++k)
                    {
                        out[g * row + k] = r[k];
                    }
                }
            });
    return 0;
}
} // namespace

extern "C"
{

// The CPU level the reference's runtime dispatch selected (crd::CpuLevel value: 0 portable .. 4 avx512). The first
// call runs the reference's known-answer self-check (src/fft_self_check.cpp) on the selected table.
int crdref_level(void)
{
    return static_cast<int>(fft::fft_kernels().level);
}

// Reference's known-answer self-check over a level's table: 0 when both golden digests match, 1 otherwise
// (src/fft_self_check.cpp:153-211, kAnswers64/kAnswers32 at :96-97).
int crdref_self_check_level(int level)
{
    for (const auto& entry : fft::fft_kernel_levels())
    {
        if (static_cast<int>(entry.level) == level)
        {
            return fft::fft_self_check(*entry.table) == nullptr ? 0 : 1;
        }
    }
    return -1;
}

// The algorithm name FftPlan<float>(n) runs forward (fft.hpp:224-227 planner; fft_kernels.hpp fft_algorithm_name).
const char* crdref_plan_algorithm_f32(std::size_t n)
{
    if (!is_pow2(n))
    {
        return "bluestein";
    }
    const fft::FftPlan<float> plan(&alloc(), n);
    return fft::fft_algorithm_name(plan.state().forward);
}

int crdref_c2c_f32(std::size_t n, std::size_t batch, float* data, int dir, int threads)
{
    return c2c<float>(n, batch, data, dir, threads);
}

int crdref_c2c_f64(std::size_t n, std::size_t batch, double* data, int dir, int threads)
{
    return c2c<double>(n, batch, data, dir, threads);
}

// FftPlan<T>::execute_reference: the reference's own radix-2 in-place oracle (fft.hpp:417-460). Power of two only.
int crdref_execute_reference_f32(std::size_t n, float* data, int dir)
{
    if (!is_pow2(n))
    {
        return -1;
    }
    const fft::FftPlan<float> plan(&alloc(), n);
    plan.execute_reference(cont::Span<Complex<float>>(reinterpret_cast<Complex<float>*>(data), n), dir_of(dir));
    return 0;
}

int crdref_execute_reference_f64(std::size_t n, double* data, int dir)
{
    if (!is_pow2(n))
    {
        return -1;
    }
    const fft::FftPlan<double> plan(&alloc(), n);
    plan.execute_reference(cont::Span<Complex<double>>(reinterpret_cast<Complex<double>*>(data), n), dir_of(dir));
    return 0;
}

// FftPlan<float>::execute_batched: element-major batch, element i of transform t at data[i*batch + t]
// (fft.hpp:462-470).
int crdref_execute_batched_f32(std::size_t n, std::size_t batch, float* data, int dir)
{
    if (!is_pow2(n))
    {
        return -1;
    }
    const fft::FftPlan<float> plan(&alloc(), n);
    plan.execute_batched(cont::Span<Complex<float>>(reinterpret_cast<Complex<float>*>(data), n * batch), batch,
                         dir_of(dir));
    return 0;
}

// The Stockham plan of the self-check (FftPlan(alloc, n, FftAlgorithm::Stockham)), so its known-answer cases can be
// dumped as golden vectors. n is a power of two from 2 to 128.
int crdref_stockham_f32(std::size_t n, std::size_t batch, float* data, int dir)
{
    if (!is_pow2(n))
    {
        return -1;
    }
    const fft::FftPlan<float> plan(&alloc(), n, fft::FftAlgorithm::Stockham);
    auto* x = reinterpret_cast<Complex<float>*>(data);
    if (batch == 0)
    {
        plan.execute(cont::Span<Complex<float>>(x, n), dir_of(dir));
    }
    else
    {
        plan.execute_batched(cont::Span<Complex<float>>(x, n * batch), batch, dir_of(dir));
    }
    return 0;
}

// RealFftPlan<float>::rfft over a batch: real[n] -> complex[n/2+1] per transform (real_fft.hpp:41-64).
int crdref_rfft_f32(std::size_t n, std::size_t batch, const float* in, float* out, int threads)
{
    if (n < 4 || !is_pow2(n))
    {
        return -1;
    }
    const std::size_t h = n / 2 + 1;
    fan_out(threads, batch,
            [&](std::size_t first, std::size_t last)
            {
                const fft::RealFftPlan<float> plan(&alloc(), n);
                for (std::size_t t = first; t < last; ++t)
                {
                    plan.rfft(cont::ConstSpan<float>(in + t * n, n),
                              cont::Span<Complex<float>>(reinterpret_cast<Complex<float>*>(out) + t * h, h));
                }
            });
    return 0;
}

// RealFftPlan<float>::irfft over a batch: complex[n/2+1] -> real[n], normalised by 1/n (real_fft.hpp:67-92).
int crdref_irfft_f32(std::size_t n, std::size_t batch, const float* in, float* out, int threads)
{
    if (n < 4 || !is_pow2(n))
    {
        return -1;
    }
    const std::size_t h = n / 2 + 1;
    fan_out(threads, batch,
            [&](std::size_t first, std::size_t last)
            {
                const fft::RealFftPlan<float> plan(&alloc(), n);
                for (std::size_t t = first; t < last; ++t)
                {
                    plan.irfft(
                        cont::ConstSpan<Complex<float>>(reinterpret_cast<const Complex<float>*>(in) + t * h, h),
                        cont::Span<float>(out + t * n, n));
                }
            });
    return 0;
}

// An uneven batch: transform t of length sizes[t] at complex offset offsets[t], in place, forward or inverse;
// contiguous ranges of transforms per thread (batch_arms.hpp:59-77), each thread keeping one plan per size across
// calls (FftPlan<float> for powers of two, BluesteinPlan<float> otherwise) the way a caller with a plan cache would.
int crdref_uneven_f32(std::size_t count, const std::int64_t* sizes, const std::int64_t* offsets, float* data, int dir,
                      int threads)
{
    auto* x = reinterpret_cast<Complex<float>*>(data);
    struct Cache
    {
        std::map<std::size_t, std::unique_ptr<fft::FftPlan<float>>> pow2;
        std::map<std::size_t, std::unique_ptr<fft::BluesteinPlan<float>>> other;
    };
    // One cache per range index (ranges are stable for a given count and thread count), kept across calls and never
    // destroyed (its plans would otherwise be freed at exit, after or during the allocator's own teardown).
    static std::map<std::size_t, Cache>& caches = *new std::map<std::size_t, Cache>();
    const std::size_t nt = threads < 1 ? 1 : (static_cast<std::size_t>(threads) < count ? threads : count);
    for (std::size_t j = 0; j < nt; ++j)
        (void)caches[j]; // created here, on one thread; each range then touches only its own
    fan_out_indexed(nt, count,
            [&](std::size_t j, std::size_t first, std::size_t last)
            {
                Cache& cache = caches.at(j);
                for (std::size_t t = first; t < last; ++t)
                {
                    const std::size_t n = static_cast<std::size_t>(sizes[t]);
                    cont::Span<Complex<float>> span(x + offsets[t], n);
                    if (is_pow2(n))
                    {
                        auto& pl = cache.pow2[n];
                        if (!pl)
                            pl = std::make_unique<fft::FftPlan<float>>(&alloc(), n);
                        pl->execute(span, dir_of(dir));
                    }
                    else
                    {
                        auto& pl = cache.other[n];
                        if (!pl)
                            pl = std::make_unique<fft::BluesteinPlan<float>>(&alloc(), n);
                        pl->execute(span, dir_of(dir));
                    }
                }
            });
    return 0;
}

// NdFftPlan<T>::execute, in place on a row-major array of ndim dims (nd_fft.hpp:105-147; inverse normalised by
// 1/prod(dims)). Runs on the calling thread (one set of axis plans).
int crdref_nd_f32(std::size_t ndim, const std::size_t* dims, float* data, int dir)
{
    if (ndim == 0)
    {
        return -1;
    }
    std::size_t total = 1;
    for (std::size_t i = 0; i < ndim; ++i)
    {
        total *= dims[i];
    }
    const fft::NdFftPlan<float> plan(&alloc(), cont::ConstSpan<std::size_t>(dims, ndim));
    plan.execute(cont::Span<Complex<float>>(reinterpret_cast<Complex<float>*>(data), total), dir_of(dir));
    return 0;
}

int crdref_nd_f64(std::size_t ndim, const std::size_t* dims, double* data, int dir)
{
    if (ndim == 0)
    {
        return -1;
    }
    std::size_t total = 1;
    for (std::size_t i = 0; i < ndim; ++i)
    {
        total *= dims[i];
    }
    const fft::NdFftPlan<double> plan(&alloc(), cont::ConstSpan<std::size_t>(dims, ndim));
    plan.execute(cont::Span<Complex<double>>(reinterpret_cast<Complex<double>*>(data), total), dir_of(dir));
    return 0;
}

// hesap-dsp's spectral estimators over `count` signals of `n` samples each, one signal at a time per thread
// (contiguous ranges, as above); each call runs the reference's own segment loop (spectral.hpp:44-120) on the
// calling thread. welch_psd (spectral.hpp:141-172): out = count x (nperseg/2 + 1). spectrogram (spectral.hpp:177-183):
// out = count x nseg x (nperseg/2 + 1). periodogram (spectral.hpp:188-220): out = count x (n/2 + 1).

// RealFftPlan takes powers of two only (real_fft.hpp); other segment lengths are refused here, not aborted on.
int crdref_welch_f32(std::size_t n, std::size_t count, const float* x, double fs, std::size_t nperseg,
                     std::size_t noverlap, float* out, int threads)
{
    if (nperseg < 4 || !is_pow2(nperseg))
        return -1;
    return spectral_rows<float>(n, count, x, out, nperseg / 2 + 1, threads,
                                [&](cont::ConstSpan<float> s)
                                { return crd::hesap::dsp::welch_psd<float>(&alloc(), s, static_cast<float>(fs),
                                                                           nperseg, noverlap); });
}

int crdref_welch_f64(std::size_t n, std::size_t count, const double* x, double fs, std::size_t nperseg,
                     std::size_t noverlap, double* out, int threads)
{
    if (nperseg < 4 || !is_pow2(nperseg))
        return -1;
    return spectral_rows<double>(n, count, x, out, nperseg / 2 + 1, threads,
                                 [&](cont::ConstSpan<double> s)
                                 { return crd::hesap::dsp::welch_psd<double>(&alloc(), s, fs, nperseg, noverlap); });
}

int crdref_spectrogram_f64(std::size_t n, std::size_t count, const double* x, double fs, std::size_t nperseg,
                           std::size_t noverlap, double* out, int threads)
{
    if (nperseg < 4 || !is_pow2(nperseg))
        return -1;
    const std::size_t hop = nperseg - noverlap;
    const std::size_t nseg = n < nperseg ? 0 : (n - noverlap) / hop;
    return spectral_rows<double>(n, count, x, out, nseg * (nperseg / 2 + 1), threads,
                                 [&](cont::ConstSpan<double> s)
                                 {
                                     std::size_t ns = 0, nf = 0;
                                     return crd::hesap::dsp::spectrogram<double>(&alloc(), s, fs, nperseg, noverlap,
                                                                                 ns, nf);
                                 });
}

int crdref_periodogram_f64(std::size_t n, std::size_t count, const double* x, double fs, double* out, int threads)
{
    if (n < 4 || !is_pow2(n))
        return -1;
    return spectral_rows<double>(n, count, x, out, n / 2 + 1, threads,
                                 [&](cont::ConstSpan<double> s)
                                 { return crd::hesap::dsp::periodogram<double>(&alloc(), s, fs); });
}

// hesap-wavelet's cwt<float> (cwt.hpp:616-621) over `count` signals of `n` samples, one signal at a time per thread
// (contiguous ranges, as above): out = count x nscales x n interleaved complex values, freqs = nscales values.
int crdref_cwt_f32(std::size_t n, std::size_t count, const float* x, const float* scales, std::size_t nscales,
                   const char* wavelet, float* out, double* freqs, int threads)
{
    if (n == 0 || nscales == 0 || wavelet == nullptr)
        return -1;
    const auto w = crd::hesap::wavelet::continuous_wavelet(wavelet);
    fan_out(threads, count,
            [&](std::size_t first, std::size_t last)
            {
                for (std::size_t g = first; g < last; ++g)
                {
                    const auto r = crd::hesap::wavelet::cwt<float>(&alloc(), cont::ConstSpan<float>(x + g * n, n),
                                                                   cont::ConstSpan<float>(scales, nscales), w);
                    float* o = out + g * nscales * n * 2;
                    for (std::size_t k = 0; k < nscales * n; ++k)
                    {
                        o[2 * k] = r.coeffs[k].re;
                        o[2 * k + 1] = r.coeffs[k].im;
                    }
                    if (g == 0 && freqs != nullptr)
                        for (std::size_t s = 0; s < nscales; ++s)
                            freqs[s] = r.frequencies[s];
                }
            });
    return 0;
}

} // extern "C"
