/* crdfft.hpp — C++20 wrappers over the C ABI of crdfft.h, with crd-hesap-fft's class names and verbs.
 *
 * The reference's plans (engine/numerics/hesap-fft/include/crd/hesap/fft/: FftPlan fft.hpp:224-470, RealFftPlan
 * real_fft.hpp:18-101, BluesteinPlan bluestein.hpp:29-149, NdFftPlan nd_fft.hpp:28-194) own their tables and
 * transform CPU memory; these own a device plan and transform device memory (or host memory through
 * execute_host), ordered on the CUDA stream passed (nullptr: the legacy default stream). Errors throw crdfft::Error
 * with the library's status instead of the reference's fatal asserts. Header only: link libcrdfft.so.
 */
#pragma once

#include "crdfft.h"

#include <complex>
#include <cstdint>
#include <span>
#include <stdexcept>
#include <string>
#include <utility>

namespace crdfft
{

enum class Direction : int32_t
{
    Forward = CRDFFT_FORWARD,
    Inverse = CRDFFT_INVERSE,
};

class Error : public std::runtime_error
{
public:
    Error(crdfft_status s, const char* what)
        : std::runtime_error(std::string(what) + ": " + crdfft_status_string(s)), m_status(s)
    {
    }
    crdfft_status status() const noexcept { return m_status; }

private:
    crdfft_status m_status;
};

inline void check(crdfft_status s, const char* what)
{
    if (s != CRDFFT_OK)
        throw Error(s, what);
}

// A device plan handle: move-only, destroyed with the object.
class Handle
{
public:
    Handle() = default;
    explicit Handle(crdfft_plan* p) noexcept : m_p(p) {}
    Handle(Handle&& o) noexcept : m_p(std::exchange(o.m_p, nullptr)) {}
    Handle& operator=(Handle&& o) noexcept
    {
        if (this != &o)
        {
            reset();
            m_p = std::exchange(o.m_p, nullptr);
        }
        return *this;
    }
    Handle(const Handle&) = delete;
    Handle& operator=(const Handle&) = delete;
    ~Handle() { reset(); }

    crdfft_plan* get() const noexcept { return m_p; }
    crdfft_plan** out() noexcept
    {
        reset();
        return &m_p;
    }
    crdfft_plan_info info() const
    {
        crdfft_plan_info i{};
        check(crdfft_plan_info_get(m_p, &i), "plan_info_get");
        return i;
    }

private:
    void reset() noexcept
    {
        if (m_p != nullptr)
            crdfft_plan_destroy(m_p);
        m_p = nullptr;
    }
    crdfft_plan* m_p = nullptr;
};

using cfloat = std::complex<float>; // layout-compatible with the reference's Complex<float> and CUDA's float2

// The general descriptor plan (crdfft_plan_create): batched 1-D/2-D/3-D C2C, R2C or C2R.
class Plan
{
public:
    explicit Plan(const crdfft_desc& d) { check(crdfft_plan_create(&d, m_h.out()), "plan_create"); }
    void execute(const void* in, void* out, Direction dir, void* stream = nullptr) const
    {
        check(crdfft_execute(m_h.get(), in, out, static_cast<int32_t>(dir), stream), "execute");
    }
    // host buffers (pinned for overlap); synchronise `stream` before reading `out`
    void execute_host(const void* in, void* out, Direction dir, void* stream = nullptr) const
    {
        check(crdfft_execute_host(m_h.get(), in, out, static_cast<int32_t>(dir), stream), "execute_host");
    }
    // split-complex planes (C2C plans whose transforms tile the planes: packed, or rank-1 element-major)
    void execute_planar(const float* re_in, const float* im_in, float* re_out, float* im_out, Direction dir,
                        void* stream = nullptr) const
    {
        check(crdfft_execute_planar(m_h.get(), re_in, im_in, re_out, im_out, static_cast<int32_t>(dir), stream),
              "execute_planar");
    }
    crdfft_plan_info info() const { return m_h.info(); }
    crdfft_plan* handle() const noexcept { return m_h.get(); }

private:
    Handle m_h;
};

// The CEIR tensor.fft lowering (crdfft_ceir_fft_desc): a plan and a direction for the op, or nullopt-like `ok` false
// with the reject reason when the op is outside the envelope (the provider keeps its own path then).
struct TensorFftLowering
{
    bool ok = false;
    int32_t reject = 0;
    int32_t direction = 0;
    crdfft_desc desc{};
};
inline TensorFftLowering lower_tensor_fft(const crdfft_ceir_fft_op& op)
{
    TensorFftLowering l;
    l.ok = crdfft_ceir_fft_desc(&op, &l.desc, &l.direction, &l.reject) == CRDFFT_OK;
    return l;
}

// FftPlan<float>(alloc, n): one size-n complex transform, in place, unnormalised both ways (fft.hpp:224, 409-413).
class FftPlan
{
public:
    explicit FftPlan(int64_t n) : m_n(n) { check(crdfft_fft_plan_create(n, m_h.out()), "FftPlan"); }
    int64_t size() const noexcept { return m_n; }
    void execute(cfloat* device_data, Direction dir, void* stream = nullptr) const
    {
        check(crdfft_fft_execute(m_h.get(), device_data, static_cast<int32_t>(dir), stream), "execute");
    }
    // element i of transform t at data[i * batch + t] (fft.hpp:462-470)
    void execute_batched(cfloat* device_data, int64_t batch, Direction dir, void* stream = nullptr) const
    {
        check(crdfft_fft_execute_batched(m_h.get(), device_data, batch, static_cast<int32_t>(dir), stream),
              "execute_batched");
    }

private:
    int64_t m_n;
    Handle m_h;
};

// RealFftPlan<float>(alloc, n): real[n] <-> complex[n/2 + 1]; rfft unnormalised, irfft normalised
// (real_fft.hpp:41-92).
class RealFftPlan
{
public:
    explicit RealFftPlan(int64_t n) : m_n(n) { check(crdfft_real_plan_create(n, m_h.out()), "RealFftPlan"); }
    int64_t size() const noexcept { return m_n; }
    void rfft(const float* in, cfloat* out, void* stream = nullptr) const
    {
        check(crdfft_rfft(m_h.get(), in, out, stream), "rfft");
    }
    void irfft(const cfloat* in, float* out, void* stream = nullptr) const
    {
        check(crdfft_irfft(m_h.get(), in, out, stream), "irfft");
    }

private:
    int64_t m_n;
    Handle m_h;
};

// BluesteinPlan<float>(alloc, n): any n; inverse normalised by 1/n (bluestein.hpp:29-149).
class BluesteinPlan
{
public:
    explicit BluesteinPlan(int64_t n) { check(crdfft_bluestein_plan_create(n, m_h.out()), "BluesteinPlan"); }
    void execute(cfloat* device_data, Direction dir, void* stream = nullptr) const
    {
        check(crdfft_bluestein_execute(m_h.get(), device_data, static_cast<int32_t>(dir), stream), "execute");
    }

private:
    Handle m_h;
};

// NdFftPlan<float>(alloc, dims): row-major N-D in place; inverse normalised by 1/prod(dims) (nd_fft.hpp:28-194).
class NdFftPlan
{
public:
    explicit NdFftPlan(std::span<const int64_t> dims)
    {
        check(crdfft_nd_plan_create(static_cast<int32_t>(dims.size()), dims.data(), m_h.out()), "NdFftPlan");
    }
    void execute(cfloat* device_data, Direction dir, void* stream = nullptr) const
    {
        check(crdfft_nd_execute(m_h.get(), device_data, static_cast<int32_t>(dir), stream), "execute");
    }

private:
    Handle m_h;
};

// The fused FFT convolution (crdfft_conv_plan_create): desc.kind C2C for complex signals, R2C for real signals with
// a half spectrum.
class ConvPlan
{
public:
    ConvPlan(const crdfft_desc& d, bool filter_per_signal = false, double scale = -1.0)
    {
        check(crdfft_conv_plan_create(&d, filter_per_signal ? 1 : 0, scale, m_h.out()), "ConvPlan");
    }
    void execute(const void* in, const cfloat* spectrum, void* out, void* stream = nullptr) const
    {
        check(crdfft_conv_execute(m_h.get(), in, spectrum, out, stream), "conv_execute");
    }

private:
    Handle m_h;
};

// hesap-dsp's welch_psd / spectrogram / periodogram on the device (crdfft_spectral_plan_create).
class SpectralPlan
{
public:
    explicit SpectralPlan(const crdfft_spectral_desc& d)
        : m_segments(crdfft_spectral_segments(&d))
    {
        check(crdfft_spectral_plan_create(&d, m_h.out()), "SpectralPlan");
    }
    int64_t segments() const noexcept { return m_segments; }
    void execute(const float* x, float* out, void* stream = nullptr) const
    {
        check(crdfft_spectral_execute(m_h.get(), x, out, stream), "spectral_execute");
    }

private:
    int64_t m_segments;
    Handle m_h;
};

// hesap-wavelet's cwt on the device (crdfft_cwt_plan_create): count x nscales x nsamples complex coefficients.
class CwtPlan
{
public:
    CwtPlan(const char* wavelet, std::span<const double> scales, int64_t nsamples, int64_t count = 1,
            int32_t precision = 12)
    {
        crdfft_cwt_desc d{};
        d.wavelet = wavelet;
        d.scales = scales.data();
        d.nsamples = nsamples;
        d.count = count;
        d.nscales = static_cast<int64_t>(scales.size());
        d.precision = precision;
        check(crdfft_cwt_plan_create(&d, &m_p), "CwtPlan");
    }
    CwtPlan(CwtPlan&& o) noexcept : m_p(std::exchange(o.m_p, nullptr)) {}
    CwtPlan& operator=(CwtPlan&& o) noexcept
    {
        if (this != &o)
        {
            crdfft_cwt_plan_destroy(m_p);
            m_p = std::exchange(o.m_p, nullptr);
        }
        return *this;
    }
    CwtPlan(const CwtPlan&) = delete;
    CwtPlan& operator=(const CwtPlan&) = delete;
    ~CwtPlan() { crdfft_cwt_plan_destroy(m_p); }

    void execute(const float* device_x, cfloat* device_coeffs, void* stream = nullptr) const
    {
        check(crdfft_cwt_execute(m_p, device_x, device_coeffs, stream), "cwt_execute");
    }
    int64_t fft_length() const
    {
        int64_t n = 0;
        check(crdfft_cwt_plan_info(m_p, &n, nullptr, nullptr), "cwt_plan_info");
        return n;
    }

private:
    crdfft_cwt_plan* m_p = nullptr;
};

// One-shot helpers (fft.hpp:1006-1029).
inline void fft(cfloat* device_data, int64_t n, Direction dir, void* stream = nullptr)
{
    check(crdfft_fft(device_data, n, static_cast<int32_t>(dir), stream), "fft");
}
inline void ifft_normalized(cfloat* device_data, int64_t n, void* stream = nullptr)
{
    check(crdfft_ifft_normalized(device_data, n, stream), "ifft_normalized");
}

} // namespace crdfft
