// The continuous wavelet transform of crd-hesap-wavelet (cwt.hpp:461-614, cwt_arm) as a device plan over `count`
// real signals (crdfft_cwt_*).
//
// Plan time, on the host in FP64 as the reference does once a call: the wavelet on its grid (sample_psi,
// cwt.hpp:149-280), its cumulative integral (conjugated for complex wavelets, cwt.hpp:470-477), each scale's tap
// count (cwt.hpp:479-501), the FFT length lfft (the power of two >= n + the longest kernel, cwt.hpp:502-506), and
// each scale's kernel: the integral sampled at floor(m / (a step)) and reversed, narrowed to FP32
// (cwt.hpp:569-581). The kernels do not depend on the signal, so their spectra are computed once, on the device, and
// kept for every execute (the reference transforms each kernel again on every call, cwt.hpp:582).
//
// Execute, all on the caller's stream: the signals zero-padded to lfft (cwt.cu) and transformed in one batched FFT
// plan; then, over chunks of signals, the product of every signal's spectrum with every kernel spectrum as one grid
// of (signal, scale) lines (cwt.cu, cwt.hpp:583-587), one batched unnormalised inverse FFT over those lines, and the
// epilogue -sqrt(a) (w[t+1] - w[t]) / lfft (cwt.cu, cwt.hpp:589-596). A chunk's lines fill the GPU in each launch,
// where a launch per signal would give one CTA per scale. Where the FFT length has a compile-time line schedule
// (256 .. 8192), one kernel (conv.cu, cwt_line_kernel) does the product, the inverse FFT in shared memory and the
// epilogue for every line, so only the coefficients are written.
#include "../../include/crdfft.h"
#include "kernels.hpp"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <new>
#include <numbers>
#include <string>
#include <vector>

struct crdfft_cwt_plan
{
    int device = -1;
    long long n = 0, count = 0, nscales = 0, lfft = 0;
    long long chunk = 0;                 // signals a product / inverse FFT / epilogue round takes
    bool fused = false;                  // one line kernel over all (signal, scale) lines (conv.cu)
    crdfft_plan* lines_plan = nullptr;   // fused: the convolution plan whose line pass (stages, twiddles) it runs
    crdfft::PassDesc pass{};             // fused: that line pass, lines = count x nscales
    crdfft_plan* forward = nullptr;      // the signals' FFTs (batch count, in place on X)
    crdfft_plan* inverse = nullptr;      // chunk x nscales inverse FFTs, in place on W
    crdfft_plan* inverse_tail = nullptr; // (count mod chunk) x nscales, when the last chunk is shorter
    void* spectra = nullptr;             // nscales x lfft complex: the kernels' spectra
    void* X = nullptr;                   // count x lfft complex: the signals' spectra
    void* W = nullptr;                   // chunk x nscales x lfft complex: the filtered sequences
    crdfft::CwtScale* scales = nullptr;

    ~crdfft_cwt_plan()
    {
        for (crdfft_plan* p : {forward, inverse, inverse_tail, lines_plan})
            if (p != nullptr)
                crdfft_plan_destroy(p);
        for (void* b : {spectra, X, W, static_cast<void*>(scales)})
            if (b != nullptr)
                cudaFree(b);
    }
};

namespace
{

using cd = std::complex<double>;

enum class Kind
{
    Mexh,
    Morl,
    Cmor,
    Gaus,
    Cgau,
    Shan,
    Fbsp,
    Paul
};

struct Wavelet
{
    Kind kind = Kind::Mexh;
    double lower = -8.0, upper = 8.0;
    double bandwidth = 1.0, center = 1.0;
    int order = 0;
    bool complex_valued = false;
    bool l2_normalize = false;
};

// A non-negative decimal with an optional leading '-' (cwt.hpp:282-306); `pos` moves past it.
double number_at(const std::string& s, size_t& pos)
{
    double sign = 1.0;
    if (pos < s.size() && s[pos] == '-')
    {
        sign = -1.0;
        ++pos;
    }
    double v = 0.0;
    for (; pos < s.size() && s[pos] >= '0' && s[pos] <= '9'; ++pos)
        v = v * 10.0 + (s[pos] - '0');
    if (pos < s.size() && s[pos] == '.')
    {
        ++pos;
        for (double f = 0.1; pos < s.size() && s[pos] >= '0' && s[pos] <= '9'; ++pos, f *= 0.1)
            v += (s[pos] - '0') * f;
    }
    return sign * v;
}

void skip_dash(const std::string& s, size_t& pos)
{
    if (pos < s.size() && s[pos] == '-')
        ++pos;
}

// pywt-style names (continuous_wavelet, cwt.hpp:300-407); a name that matches none is the Mexican hat, as there.
Wavelet parse_wavelet(const std::string& name)
{
    Wavelet w;
    auto starts = [&](const char* p) { return name.rfind(p, 0) == 0; };
    size_t pos = 4;
    if (name == "morl")
        w.kind = Kind::Morl;
    else if (starts("cmor"))
    {
        w.kind = Kind::Cmor;
        w.bandwidth = number_at(name, pos);
        skip_dash(name, pos);
        w.center = number_at(name, pos);
        w.complex_valued = true;
    }
    else if (starts("cgau") || starts("gaus"))
    {
        w.kind = starts("cgau") ? Kind::Cgau : Kind::Gaus;
        w.lower = -5.0;
        w.upper = 5.0;
        w.order = static_cast<int>(number_at(name, pos));
        w.complex_valued = w.kind == Kind::Cgau;
        w.l2_normalize = true;
    }
    else if (starts("shan"))
    {
        w.kind = Kind::Shan;
        w.lower = -20.0;
        w.upper = 20.0;
        w.bandwidth = number_at(name, pos);
        skip_dash(name, pos);
        w.center = number_at(name, pos);
        w.complex_valued = true;
    }
    else if (starts("fbsp"))
    {
        w.kind = Kind::Fbsp;
        w.lower = -20.0;
        w.upper = 20.0;
        w.order = static_cast<int>(number_at(name, pos));
        skip_dash(name, pos);
        w.bandwidth = number_at(name, pos);
        skip_dash(name, pos);
        w.center = number_at(name, pos);
        w.complex_valued = true;
    }
    else if (starts("paul"))
    {
        w.kind = Kind::Paul;
        w.lower = -12.0;
        w.upper = 12.0;
        w.order = pos < name.size() ? static_cast<int>(number_at(name, pos)) : 4;
        w.complex_valued = true;
    }
    return w;
}

// Ascending coefficients of the polynomial P_p with d^p/dx^p e^{g(x)} = P_p(x) e^{g(x)}, for g = -x^2 (phase 0) or
// g = -x^2 - i x (phase -i): P_{k+1} = P_k' + g'(x) P_k, P_0 = 1 (cwt.hpp:86-147).
std::vector<cd> gauss_poly(int p, cd phase)
{
    std::vector<cd> c{cd(1.0, 0.0)};
    for (int s = 0; s < p; ++s)
    {
        std::vector<cd> nxt(c.size() + 1, cd(0.0, 0.0));
        for (size_t k = 1; k < c.size(); ++k)
            nxt[k - 1] += static_cast<double>(k) * c[k];
        for (size_t k = 0; k < c.size(); ++k)
        {
            nxt[k + 1] += -2.0 * c[k];
            nxt[k] += phase * c[k];
        }
        c.swap(nxt);
    }
    return c;
}

double sinc_pi(double x) { return x == 0.0 ? 1.0 : std::sin(std::numbers::pi * x) / (std::numbers::pi * x); }

// The wavelet on linspace(lower, upper, grid_n), L2-normalised for gaus / cgau (cwt.hpp:149-280).
std::vector<cd> sample_psi(const Wavelet& w, long long grid_n)
{
    const double pi = std::numbers::pi;
    const double step = (w.upper - w.lower) / static_cast<double>(grid_n - 1);
    std::vector<cd> poly;
    if (w.kind == Kind::Gaus)
        poly = gauss_poly(w.order, cd(0.0, 0.0));
    else if (w.kind == Kind::Cgau)
        poly = gauss_poly(w.order, cd(0.0, -1.0));
    const double gsign = ((w.order / 2) & 1) ? -1.0 : 1.0;
    double paul_norm = 0.0;
    cd paul_im(1.0, 0.0);
    if (w.kind == Kind::Paul)
    {
        double fm = 1.0, f2m = 1.0;
        for (int j = 2; j <= w.order; ++j)
            fm *= j;
        for (int j = 2; j <= 2 * w.order; ++j)
            f2m *= j;
        paul_norm = std::pow(2.0, w.order) * fm / std::sqrt(pi * f2m);
        for (int j = 0; j < w.order; ++j)
            paul_im *= cd(0.0, 1.0);
    }
    std::vector<cd> out(static_cast<size_t>(grid_n));
    for (long long k = 0; k < grid_n; ++k)
    {
        const double t = w.lower + static_cast<double>(k) * step;
        cd v;
        switch (w.kind)
        {
        case Kind::Mexh:
            v = 2.0 / (std::sqrt(3.0) * std::pow(pi, 0.25)) * (1.0 - t * t) * std::exp(-t * t / 2.0);
            break;
        case Kind::Morl:
            v = std::exp(-t * t / 2.0) * std::cos(5.0 * t);
            break;
        case Kind::Cmor:
            v = std::pow(pi * w.bandwidth, -0.5) * std::exp(-t * t / w.bandwidth) * std::polar(1.0, 2.0 * pi * w.center * t);
            break;
        case Kind::Gaus:
        case Kind::Cgau:
        {
            cd p(0.0, 0.0);
            for (size_t j = poly.size(); j-- > 0;)
                p = p * t + poly[j];
            v = w.kind == Kind::Gaus ? gsign * p.real() * std::exp(-t * t)
                                     : p * (std::exp(-t * t) * cd(std::cos(t), -std::sin(t)));
            break;
        }
        case Kind::Shan:
            v = std::sqrt(w.bandwidth) * sinc_pi(w.bandwidth * t) * std::polar(1.0, 2.0 * pi * w.center * t);
            break;
        case Kind::Fbsp:
            v = std::sqrt(w.bandwidth) * std::pow(sinc_pi(w.bandwidth * t / w.order), w.order) *
                std::polar(1.0, 2.0 * pi * w.center * t);
            break;
        case Kind::Paul:
        {
            // (1 - i t)^-(m+1) in polar form
            const double r = std::hypot(1.0, t), th = std::atan2(-t, 1.0);
            v = paul_norm * paul_im * std::polar(std::pow(r, -(w.order + 1.0)), -(w.order + 1.0) * th);
            break;
        }
        }
        out[static_cast<size_t>(k)] = v;
    }
    if (w.l2_normalize)
    {
        double e = 0.0;
        for (const cd& v : out)
            e += std::norm(v) * step;
        const double inv = 1.0 / std::sqrt(e);
        for (cd& v : out)
            v *= inv;
    }
    return out;
}

// In-place radix-2 FP64 FFT (forward), for the central frequency only.
void fft64(std::vector<cd>& a)
{
    const size_t n = a.size();
    for (size_t i = 1, j = 0; i < n; ++i)
    {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1)
            j ^= bit;
        j |= bit;
        if (i < j)
            std::swap(a[i], a[j]);
    }
    for (size_t len = 2; len <= n; len <<= 1)
        for (size_t i = 0; i < n; i += len)
            for (size_t k = 0; k < len / 2; ++k)
            {
                const cd w = std::polar(1.0, -2.0 * std::numbers::pi * static_cast<double>(k) / static_cast<double>(len));
                const cd u = a[i + k], v = a[i + k + len / 2] * w;
                a[i + k] = u + v;
                a[i + k + len / 2] = u - v;
            }
}

// The bin of the largest |FFT(psi)|^2 over k >= 1 (the first one), folded, over the interval (cwt.hpp:410-438).
double central_frequency(const Wavelet& w, int precision)
{
    const long long n = 1LL << precision;
    std::vector<cd> psi = sample_psi(w, n);
    fft64(psi);
    long long bin = 1;
    double best = -1.0;
    for (long long k = 1; k < n; ++k)
    {
        const double m = std::norm(psi[static_cast<size_t>(k)]);
        if (m > best)
        {
            best = m;
            bin = k;
        }
    }
    long long index = bin + 1;
    if (static_cast<double>(index) > static_cast<double>(n) / 2.0)
        index = n - index + 2;
    return static_cast<double>(index - 1) / (w.upper - w.lower);
}

struct Geometry
{
    Wavelet w;
    int precision = 12;
    long long grid_n = 0;
    double step = 0.0;
    std::vector<long long> taps;
    long long lfft = 0;
};

// Validates the descriptor and computes the scales' taps and the FFT length (cwt.hpp:464-506).
crdfft_status geometry(const crdfft_cwt_desc* d, Geometry* g)
{
    if (d == nullptr || d->wavelet == nullptr || d->scales == nullptr)
        return CRDFFT_INVALID_ARG;
    const int precision = d->precision == 0 ? 12 : d->precision;
    if (d->nsamples < 1 || d->count < 1 || d->nscales < 1 || d->nscales > 65535 || precision < 1 || precision > 20 ||
        d->sampling_period < 0.0)
        return CRDFFT_INVALID_DESC;
    g->w = parse_wavelet(d->wavelet);
    if (g->w.order < 0 || g->w.order > 15 || (g->w.kind == Kind::Fbsp && g->w.order < 1))
        return CRDFFT_INVALID_DESC;
    g->precision = precision;
    g->grid_n = 1LL << precision;
    const double xrange = g->w.upper - g->w.lower;
    g->step = xrange / static_cast<double>(g->grid_n - 1);
    long long kmax = 1;
    g->taps.assign(static_cast<size_t>(d->nscales), 0);
    for (long long s = 0; s < d->nscales; ++s)
    {
        const double a = d->scales[s];
        if (!(a > 0.0) || !std::isfinite(a))
            return CRDFFT_INVALID_DESC;
        if (a * xrange > static_cast<double>(1LL << 27))
            return CRDFFT_UNSUPPORTED_SIZE; // a kernel of more than 2^27 taps
        const long long count_raw = static_cast<long long>(std::ceil(a * xrange + 1.0));
        long long kk = 0;
        for (long long m = 0; m < count_raw; ++m, ++kk)
            if (static_cast<unsigned long long>(static_cast<double>(m) / (a * g->step)) >=
                static_cast<unsigned long long>(g->grid_n))
                break;
        g->taps[static_cast<size_t>(s)] = kk;
        kmax = std::max(kmax, kk);
    }
    g->lfft = 1;
    while (g->lfft < d->nsamples + kmax)
        g->lfft <<= 1;
    if (g->lfft > (1LL << 30))
        return CRDFFT_UNSUPPORTED_SIZE;
    return CRDFFT_OK;
}

crdfft_desc line_desc(long long lfft, long long batch)
{
    crdfft_desc d{};
    d.rank = 1;
    d.kind = CRDFFT_C2C;
    d.precision = CRDFFT_PREC_FP32;
    d.norm = CRDFFT_NORM_NONE;
    d.dims[0] = lfft;
    d.batch = batch;
    return d;
}

crdfft_status build(const crdfft_cwt_desc* d, const Geometry& g, crdfft_cwt_plan* p)
{
    const long long ns = d->nscales, lfft = g.lfft;
    p->n = d->nsamples;
    p->count = d->count;
    p->nscales = ns;
    p->lfft = lfft;
    if (cudaGetDevice(&p->device) != cudaSuccess)
        return CRDFFT_NO_DEVICE;

    // the integrated wavelet (cwt.hpp:470-477), each scale's reversed kernel narrowed to FP32 (cwt.hpp:569-581)
    std::vector<cd> ipsi = sample_psi(g.w, g.grid_n);
    cd acc(0.0, 0.0);
    for (cd& v : ipsi)
    {
        acc += v;
        v = g.w.complex_valued ? std::conj(acc * g.step) : acc * g.step;
    }
    std::vector<float> table(static_cast<size_t>(ns * lfft) * 2, 0.0f);
    std::vector<crdfft::CwtScale> sc(static_cast<size_t>(ns));
    for (long long s = 0; s < ns; ++s)
    {
        const double a = d->scales[s];
        const long long kk = g.taps[static_cast<size_t>(s)];
        crdfft::CwtScale& c = sc[static_cast<size_t>(s)];
        c.taps_ok = kk >= 2 ? 1 : 0;
        c.off = kk >= 2 ? (kk - 2) / 2 : 0;
        c.amp = -static_cast<float>(std::sqrt(a));
        if (c.off + d->nsamples >= lfft)
            return CRDFFT_INVALID_DESC; // cannot happen: lfft >= n + kk
        if (kk < 2)
            continue;
        float* row = table.data() + static_cast<size_t>(s * lfft) * 2;
        for (long long i = 0; i < kk; ++i)
        {
            const long long m = kk - 1 - i;
            const cd v = ipsi[static_cast<size_t>(static_cast<double>(m) / (a * g.step))];
            row[2 * i] = static_cast<float>(v.real());
            row[2 * i + 1] = static_cast<float>(v.imag());
        }
    }

    // the fused line kernel where the FFT length has a compile-time schedule: one launch, no filtered-sequence scratch
    const long long line_bytes = lfft * 8;
    crdfft_desc ld = line_desc(lfft, d->count * ns);
    if (crdfft_conv_plan_create(&ld, 0, 1.0, &p->lines_plan) == CRDFFT_OK)
    {
        p->fused = crdfft::conv_line_pass(p->lines_plan, &p->pass) && crdfft::cwt_lines_supported(p->pass);
        if (!p->fused)
        {
            crdfft_plan_destroy(p->lines_plan);
            p->lines_plan = nullptr;
        }
    }
    // otherwise signals a round: the filtered sequences within 512 MiB, the grid rows (lines) within 65535
    p->chunk = p->fused ? d->count
                        : std::max<long long>(1, std::min<long long>({static_cast<long long>(d->count),
                                                                      (512LL << 20) / (ns * line_bytes), 65535 / ns}));
    const size_t kbytes = static_cast<size_t>(ns * line_bytes);
    if (cudaMalloc(&p->spectra, kbytes) != cudaSuccess ||
        (!p->fused && cudaMalloc(&p->W, static_cast<size_t>(p->chunk) * kbytes) != cudaSuccess) ||
        cudaMalloc(&p->X, static_cast<size_t>(d->count * line_bytes)) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void**>(&p->scales), sizeof(crdfft::CwtScale) * static_cast<size_t>(ns)) !=
            cudaSuccess)
    {
        cudaGetLastError();
        return CRDFFT_OOM;
    }
    if (cudaMemcpy(p->spectra, table.data(), kbytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(p->scales, sc.data(), sizeof(crdfft::CwtScale) * static_cast<size_t>(ns),
                   cudaMemcpyHostToDevice) != cudaSuccess)
        return CRDFFT_LAUNCH;

    crdfft_desc fd = line_desc(lfft, d->count);
    crdfft_status st = crdfft_plan_create(&fd, &p->forward);
    if (st != CRDFFT_OK)
        return st;
    // the kernels' spectra, once: a forward plan over the table in place
    crdfft_desc kd = line_desc(lfft, ns);
    crdfft_plan* kf = nullptr;
    st = crdfft_plan_create(&kd, &kf);
    if (st != CRDFFT_OK)
        return st;
    st = crdfft_execute(kf, p->spectra, p->spectra, CRDFFT_FORWARD, nullptr);
    const cudaError_t e = cudaStreamSynchronize(nullptr);
    crdfft_plan_destroy(kf);
    if (st != CRDFFT_OK)
        return st;
    if (e != cudaSuccess)
        return CRDFFT_LAUNCH;
    if (p->fused)
        return CRDFFT_OK;
    crdfft_desc id = line_desc(lfft, p->chunk * ns);
    st = crdfft_plan_create(&id, &p->inverse);
    if (st != CRDFFT_OK)
        return st;
    const long long tail = d->count % p->chunk;
    if (tail != 0)
    {
        crdfft_desc td = line_desc(lfft, tail * ns);
        st = crdfft_plan_create(&td, &p->inverse_tail);
    }
    return st;
}

} // namespace

extern "C" {

crdfft_status crdfft_cwt_plan_create(const crdfft_cwt_desc* desc, crdfft_cwt_plan** plan)
{
    if (plan == nullptr)
        return CRDFFT_INVALID_ARG;
    *plan = nullptr;
    Geometry g;
    crdfft_status st = geometry(desc, &g);
    if (st != CRDFFT_OK)
        return st;
    auto* p = new (std::nothrow) crdfft_cwt_plan();
    if (p == nullptr)
        return CRDFFT_OOM;
    try
    {
        st = build(desc, g, p);
    }
    catch (const std::bad_alloc&)
    {
        st = CRDFFT_OOM; // the host kernel table
    }
    if (st != CRDFFT_OK)
    {
        delete p;
        return st;
    }
    *plan = p;
    return CRDFFT_OK;
}

crdfft_status crdfft_cwt_plan_destroy(crdfft_cwt_plan* plan)
{
    delete plan;
    return CRDFFT_OK;
}

crdfft_status crdfft_cwt_execute(crdfft_cwt_plan* plan, const float* x, void* coeffs, void* stream)
{
    if (plan == nullptr || x == nullptr || coeffs == nullptr)
        return CRDFFT_INVALID_ARG;
    crdfft_cwt_plan& p = *plan;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev != p.device)
        return CRDFFT_NO_DEVICE;
    const auto s = static_cast<cudaStream_t>(stream);
    if (crdfft::launch_cwt_pad(x, p.X, p.n, p.lfft, p.count, s) != cudaSuccess)
        return CRDFFT_LAUNCH;
    crdfft_status st = crdfft_execute(p.forward, p.X, p.X, CRDFFT_FORWARD, stream);
    if (st != CRDFFT_OK)
        return st;
    if (p.fused)
        return crdfft::launch_cwt_lines(p.pass, p.X, p.spectra, p.scales, p.nscales, p.n, coeffs, s) == cudaSuccess
                   ? CRDFFT_OK
                   : CRDFFT_LAUNCH;
    for (long long c0 = 0; c0 < p.count; c0 += p.chunk)
    {
        const long long cc = std::min(p.chunk, p.count - c0);
        const void* spec = static_cast<const char*>(p.X) + static_cast<size_t>(c0 * p.lfft) * 8;
        if (crdfft::launch_cwt_product(spec, p.spectra, p.W, p.lfft, p.nscales, cc, s) != cudaSuccess)
            return CRDFFT_LAUNCH;
        st = crdfft_execute(cc == p.chunk ? p.inverse : p.inverse_tail, p.W, p.W, CRDFFT_INVERSE, stream);
        if (st != CRDFFT_OK)
            return st;
        void* out = static_cast<char*>(coeffs) + static_cast<size_t>(c0 * p.nscales * p.n) * 8;
        if (crdfft::launch_cwt_diff(p.W, p.scales, out, p.n, p.lfft, p.nscales, cc, s) != cudaSuccess)
            return CRDFFT_LAUNCH;
    }
    return CRDFFT_OK;
}

crdfft_status crdfft_cwt_frequencies(const crdfft_cwt_desc* desc, double* frequencies)
{
    if (frequencies == nullptr)
        return CRDFFT_INVALID_ARG;
    Geometry g;
    const crdfft_status st = geometry(desc, &g);
    if (st != CRDFFT_OK)
        return st;
    const double fc = central_frequency(g.w, g.precision);
    const double period = desc->sampling_period == 0.0 ? 1.0 : desc->sampling_period;
    for (long long s = 0; s < desc->nscales; ++s)
        frequencies[s] = fc / (desc->scales[s] * period);
    return CRDFFT_OK;
}

int64_t crdfft_cwt_fft_length(const crdfft_cwt_desc* desc)
{
    Geometry g;
    return geometry(desc, &g) == CRDFFT_OK ? g.lfft : -1;
}

crdfft_status crdfft_cwt_plan_info(const crdfft_cwt_plan* plan, int64_t* fft_length, int64_t* signals_per_round,
                                   int32_t* fused)
{
    if (plan == nullptr)
        return CRDFFT_INVALID_ARG;
    if (fft_length != nullptr)
        *fft_length = plan->lfft;
    if (signals_per_round != nullptr)
        *signals_per_round = plan->chunk;
    if (fused != nullptr)
        *fused = plan->fused ? 1 : 0;
    return CRDFFT_OK;
}

} // extern "C"
