// crdfft_self_check: the device known-answer check. It has the role of the reference's fft_self_check
// (engine/numerics/hesap-fft/src/fft_self_check.cpp:153-211), which runs a table's routines on small integer inputs
// before first use. Here the answers come from a host FP64 DFT computed on the spot (the reference's outputs were
// checked once against an mpmath DFT, :1-6), and the cases cover every codelet radix (9 included), a four-step, a real transform
// and a Bluestein size. Tolerance: max|gpu - dft| <= 1e-5 * (1 + max|dft|), the FP32 error of these sizes with room.

#include "../../include/crdfft.h"

#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <map>
#include <mutex>
#include <complex>
#include <cstdlib>
#include <cstdint>
#include <vector>

namespace
{

using cd = std::complex<double>;

double small_value(std::size_t k, std::size_t salt)
{
    static const int kValues[7] = {1, -2, 2, -1, -2, 1, 2};
    return kValues[(k * (salt % 5U + 2U) + salt * 3U + k / 7U) % 7U];
}

std::vector<cd> dft(const std::vector<cd>& x, int dir)
{
    const std::size_t n = x.size();
    std::vector<cd> y(n);
    const double sg = dir ? 1.0 : -1.0;
    for (std::size_t k = 0; k < n; ++k)
    {
        cd acc(0.0, 0.0);
        for (std::size_t j = 0; j < n; ++j)
        {
            const double ang = sg * 6.283185307179586476925286766559 * static_cast<double>((j * k) % n) /
                               static_cast<double>(n);
            acc += x[j] * cd(std::cos(ang), std::sin(ang));
        }
        y[k] = acc;
    }
    return y;
}

// FP64 radix-2 FFT for the four-step case (power of two).
std::vector<cd> fft_pow2(std::vector<cd> a, int dir)
{
    const std::size_t n = a.size();
    std::size_t lg = 0;
    while ((std::size_t{1} << lg) < n)
        ++lg;
    for (std::size_t i = 0; i < n; ++i)
    {
        std::size_t r = 0;
        for (std::size_t b = 0; b < lg; ++b)
            if (i & (std::size_t{1} << b))
                r |= std::size_t{1} << (lg - 1 - b);
        if (i < r)
            std::swap(a[i], a[r]);
    }
    const double sg = dir ? 1.0 : -1.0;
    for (std::size_t len = 2; len <= n; len <<= 1)
        for (std::size_t k = 0; k < len / 2; ++k)
        {
            const double ang = sg * 6.283185307179586476925286766559 * static_cast<double>(k) / static_cast<double>(len);
            const cd w(std::cos(ang), std::sin(ang));
            for (std::size_t s = 0; s < n; s += len)
            {
                const cd u = a[s + k], v = a[s + k + len / 2] * w;
                a[s + k] = u + v;
                a[s + k + len / 2] = u - v;
            }
        }
    return a;
}

std::atomic<int> g_plant_mismatch{0};

bool close(const std::vector<float>& got, const std::vector<cd>& want, double scale)
{
    // test hook: a mistake planted in the host answer, on the CPU (crdfft_debug_self_check_mismatch)
    const double planted = g_plant_mismatch.load() ? 1.0 : 0.0;
    double maxref = 0.0, maxerr = 0.0;
    for (std::size_t k = 0; k < want.size(); ++k)
    {
        const cd w = want[k] * scale + cd(k == 0 ? planted : 0.0, 0.0);
        maxref = std::max(maxref, std::abs(w));
        maxerr = std::max(maxerr, std::abs(cd(got[2 * k], got[2 * k + 1]) - w));
    }
    return std::isfinite(maxerr) && maxerr <= 1e-5 * (1.0 + maxref);
}

bool run_c2c(long long n, int dir, std::size_t salt, void* dbuf)
{
    std::vector<cd> x(static_cast<std::size_t>(n));
    std::vector<float> h(static_cast<std::size_t>(2 * n));
    for (long long i = 0; i < n; ++i)
    {
        x[i] = cd(small_value(i, 2 * salt), small_value(i, 2 * salt + 1));
        h[2 * i] = static_cast<float>(x[i].real());
        h[2 * i + 1] = static_cast<float>(x[i].imag());
    }
    if (cudaMemcpy(dbuf, h.data(), h.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess)
        return false;
    crdfft_plan* p = nullptr;
    if (crdfft_fft_plan_create(n, &p) != CRDFFT_OK)
        return false;
    const crdfft_status st = crdfft_fft_execute(p, dbuf, dir, nullptr);
    const bool synced = cudaDeviceSynchronize() == cudaSuccess;
    crdfft_plan_destroy(p);
    if (st != CRDFFT_OK || !synced)
        return false;
    if (cudaMemcpy(h.data(), dbuf, h.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return false;
    const std::vector<cd> want = (n > 8192) ? fft_pow2(x, dir) : dft(x, dir);
    return close(h, want, 1.0);
}

} // namespace

namespace
{
// Per device: 0 not checked yet, 1 passed, 2 failed (plans on that device are refused from then on).
std::mutex g_first_use_mu;
std::map<int, int> g_first_use;
thread_local bool t_in_self_check = false;
} // namespace

namespace crdfft
{
// The known-answer check at the first plan creation on each device, as the reference checks each kernel table
// before its first use (src/fft_kernel_dispatch.cpp:48-52 through process_checked_kernel_level). The check itself
// creates plans; those skip it (t_in_self_check). CRDFFT_SELF_CHECK=0 turns it off.
crdfft_status first_use_self_check(int dev)
{
    static const bool off = [] {
        const char* e = std::getenv("CRDFFT_SELF_CHECK");
        return e != nullptr && std::atoi(e) == 0;
    }();
    if (off || t_in_self_check)
        return CRDFFT_OK;
    std::lock_guard<std::mutex> lk(g_first_use_mu);
    int& state = g_first_use[dev];
    if (state == 1)
        return CRDFFT_OK;
    if (state == 2)
        return CRDFFT_NUMERIC_SELFCHECK;
    t_in_self_check = true;
    const crdfft_status st = crdfft_self_check();
    t_in_self_check = false;
    if (st == CRDFFT_OK)
        state = 1;
    else if (st == CRDFFT_NUMERIC_SELFCHECK)
        state = 2;
    return st; // other failures (out of memory, launch) leave the device unchecked: the next creation retries
}
} // namespace crdfft

extern "C" void crdfft_debug_self_check_mismatch(int32_t on) { g_plant_mismatch.store(on ? 1 : 0); }

extern "C" void crdfft_debug_self_check_reset(void)
{
    std::lock_guard<std::mutex> lk(g_first_use_mu);
    g_first_use.clear();
}

extern "C" crdfft_status crdfft_self_check(void)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return CRDFFT_NO_DEVICE;
    void* dbuf = nullptr;
    const long long maxn = 32768;
    if (cudaMalloc(&dbuf, static_cast<std::size_t>(maxn) * 8) != cudaSuccess)
        return CRDFFT_OOM;
    struct Case
    {
        long long n;
        int dir;
    };
    static const Case kCases[] = {{2, 0},    {4, 0},    {8, 1},   {16, 0},   {3, 0},   {5, 1},    {7, 0},   {9, 0},
                                  {81, 1},   {2187, 0},
                                  {105, 0},  {105, 1},  {240, 0}, {1024, 0}, {1024, 1}, {4096, 0}, {17, 0},
                                  {32768, 0}, {32768, 1}};
    bool ok = true;
    std::size_t salt = 0;
    for (const Case& c : kCases)
    {
        if (!run_c2c(c.n, c.dir, salt++, dbuf))
        {
            ok = false;
            break;
        }
    }
    cudaFree(dbuf);
    return ok ? CRDFFT_OK : CRDFFT_NUMERIC_SELFCHECK;
}
