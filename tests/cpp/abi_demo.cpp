// C++20 host code through include/crdfft.hpp: the crd-hesap-fft class names over the C ABI. Test infrastructure:
// tests/test_zz_cpp_binding.py compiles it with g++ against libcrdfft.so and runs it.
//   abi_demo host            device-free paths (status codes, descriptor validation, the spectral segment rule)
//   abi_demo device IN OUT   FftPlan(4096) forward of the complex64 file IN into OUT, RealFftPlan(4096) rfft of the
//                            real parts of IN appended to OUT, a 3-segment Welch PSD of them appended after that,
//                            then the re and im planes of a lowered tensor.fft of IN's split planes
#include <crdfft.hpp>

#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <fstream>
#include <vector>

namespace
{

int host_checks()
{
    // an invalid descriptor is refused before any device is touched
    crdfft_desc d{};
    d.rank = 0;
    d.batch = 1;
    try
    {
        crdfft::Plan p(d);
        std::puts("FAIL: rank 0 accepted");
        return 1;
    }
    catch (const crdfft::Error& e)
    {
        if (e.status() != CRDFFT_INVALID_DESC)
        {
            std::printf("FAIL: status %d\n", static_cast<int>(e.status()));
            return 1;
        }
    }
    crdfft_spectral_desc s{};
    s.mode = CRDFFT_SPECTRAL_WELCH;
    s.detrend = 1;
    s.nsamples = 512;
    s.count = 1;
    s.nperseg = 64;
    s.noverlap = 0; // Welch reads 0 as nperseg / 2
    s.fs = 100.0;
    if (crdfft_spectral_segments(&s) != 15)
    {
        std::puts("FAIL: segments");
        return 1;
    }
    // the CWT's FFT length (the morl kernel at scale 16 has 257 taps) and a negative scale refused without a device
    const double scales[2] = {1.0, 16.0};
    crdfft_cwt_desc c{};
    c.wavelet = "morl";
    c.scales = scales;
    c.nsamples = 100;
    c.count = 1;
    c.nscales = 2;
    if (crdfft_cwt_fft_length(&c) != 512)
    {
        std::puts("FAIL: cwt fft length");
        return 1;
    }
    const double bad[2] = {1.0, -2.0};
    try
    {
        crdfft::CwtPlan p("morl", std::span<const double>(bad, 2), 100);
        std::puts("FAIL: negative scale accepted");
        return 1;
    }
    catch (const crdfft::Error& e)
    {
        if (e.status() != CRDFFT_INVALID_DESC)
        {
            std::printf("FAIL: cwt status %d\n", static_cast<int>(e.status()));
            return 1;
        }
    }
    // the CEIR tensor.fft lowering: a rank-2 [6, 4096] op along its innermost axis is a batch of six 4096-point
    // transforms; a dynamic extent is refused with the reference's reason
    crdfft_ceir_fft_op op{};
    op.num_operands = 2;
    op.num_results = 2;
    op.operand_is_tensor = 1;
    op.element_is_f32 = 1;
    op.rank = 2;
    op.axis = -1;
    op.shape[0] = 6;
    op.shape[1] = 4096;
    op.direction = "inverse";
    const crdfft::TensorFftLowering l = crdfft::lower_tensor_fft(op);
    if (!l.ok || l.desc.dims[0] != 4096 || l.desc.batch != 6 || l.direction != CRDFFT_INVERSE ||
        l.desc.norm != CRDFFT_NORM_NONE)
    {
        std::puts("FAIL: tensor.fft lowering");
        return 1;
    }
    op.shape[0] = -1;
    if (crdfft::lower_tensor_fft(op).ok || crdfft::lower_tensor_fft(op).reject != CRDFFT_CEIR_SHAPE_NOT_STATIC)
    {
        std::puts("FAIL: dynamic extent accepted");
        return 1;
    }
    std::printf("host ok: %s\n", crdfft_status_string(CRDFFT_OK));
    return 0;
}

int device_run(const char* in_path, const char* out_path)
{
    constexpr int64_t n = 4096;
    std::vector<crdfft::cfloat> x(n);
    {
        std::ifstream f(in_path, std::ios::binary);
        f.read(reinterpret_cast<char*>(x.data()), static_cast<std::streamsize>(n * sizeof(crdfft::cfloat)));
        if (!f)
            return 2;
    }
    std::vector<float> xr(n);
    for (int64_t i = 0; i < n; ++i)
        xr[static_cast<size_t>(i)] = x[static_cast<size_t>(i)].real();
    std::vector<float> xi(n);
    for (int64_t i = 0; i < n; ++i)
        xi[static_cast<size_t>(i)] = x[static_cast<size_t>(i)].imag();
    crdfft::cfloat* dx = nullptr;
    crdfft::cfloat* ds = nullptr;
    float* dr = nullptr;
    float* dp = nullptr;
    float* di = nullptr; // the imaginary plane (the real plane is dr)
    float* dpr = nullptr;
    float* dpi = nullptr;
    cudaMalloc(&di, n * sizeof(float));
    cudaMalloc(&dpr, n * sizeof(float));
    cudaMalloc(&dpi, n * sizeof(float));
    cudaMemcpy(di, xi.data(), n * sizeof(float), cudaMemcpyHostToDevice);
    cudaMalloc(&dx, n * sizeof(crdfft::cfloat));
    cudaMalloc(&ds, (n / 2 + 1) * sizeof(crdfft::cfloat));
    cudaMalloc(&dr, n * sizeof(float));
    cudaMalloc(&dp, 33 * sizeof(float));
    cudaMemcpy(dx, x.data(), n * sizeof(crdfft::cfloat), cudaMemcpyHostToDevice);
    cudaMemcpy(dr, xr.data(), n * sizeof(float), cudaMemcpyHostToDevice);
    try
    {
        crdfft::FftPlan plan(n);
        plan.execute(dx, crdfft::Direction::Forward);
        crdfft::RealFftPlan real(n);
        real.rfft(dr, ds);
        crdfft_spectral_desc s{};
        s.mode = CRDFFT_SPECTRAL_WELCH;
        s.detrend = 1;
        s.nsamples = 128;
        s.count = 1;
        s.nperseg = 64;
        s.noverlap = 32;
        s.fs = 1.0;
        crdfft::SpectralPlan welch(s);
        welch.execute(dr, dp);
        // a forward tensor.fft op on [4096] split-complex planes, lowered and run on the planes
        crdfft_ceir_fft_op op{};
        op.num_operands = 2;
        op.num_results = 2;
        op.operand_is_tensor = 1;
        op.element_is_f32 = 1;
        op.rank = 1;
        op.axis = -1;
        op.shape[0] = n;
        op.direction = "forward";
        const crdfft::TensorFftLowering l = crdfft::lower_tensor_fft(op);
        if (!l.ok)
            return 4;
        crdfft::Plan tp(l.desc);
        tp.execute_planar(dr, di, dpr, dpi, static_cast<crdfft::Direction>(l.direction));
    }
    catch (const crdfft::Error& e)
    {
        std::printf("FAIL: %s\n", e.what());
        return 1;
    }
    if (cudaDeviceSynchronize() != cudaSuccess)
        return 3;
    std::vector<crdfft::cfloat> y(n), sp(n / 2 + 1);
    std::vector<float> psd(33), pre(n), pim(n);
    cudaMemcpy(pre.data(), dpr, n * sizeof(float), cudaMemcpyDeviceToHost);
    cudaMemcpy(pim.data(), dpi, n * sizeof(float), cudaMemcpyDeviceToHost);
    cudaMemcpy(y.data(), dx, n * sizeof(crdfft::cfloat), cudaMemcpyDeviceToHost);
    cudaMemcpy(sp.data(), ds, (n / 2 + 1) * sizeof(crdfft::cfloat), cudaMemcpyDeviceToHost);
    cudaMemcpy(psd.data(), dp, 33 * sizeof(float), cudaMemcpyDeviceToHost);
    std::ofstream o(out_path, std::ios::binary);
    o.write(reinterpret_cast<const char*>(y.data()), static_cast<std::streamsize>(y.size() * sizeof(crdfft::cfloat)));
    o.write(reinterpret_cast<const char*>(sp.data()), static_cast<std::streamsize>(sp.size() * sizeof(crdfft::cfloat)));
    o.write(reinterpret_cast<const char*>(psd.data()), static_cast<std::streamsize>(psd.size() * sizeof(float)));
    o.write(reinterpret_cast<const char*>(pre.data()), static_cast<std::streamsize>(pre.size() * sizeof(float)));
    o.write(reinterpret_cast<const char*>(pim.data()), static_cast<std::streamsize>(pim.size() * sizeof(float)));
    cudaFree(di);
    cudaFree(dpr);
    cudaFree(dpi);
    cudaFree(dx);
    cudaFree(ds);
    cudaFree(dr);
    cudaFree(dp);
    std::puts("device ok");
    return 0;
}

} // namespace

int main(int argc, char** argv)
{
    if (argc >= 2 && std::strcmp(argv[1], "host") == 0)
        return host_checks();
    if (argc >= 4 && std::strcmp(argv[1], "device") == 0)
        return device_run(argv[2], argv[3]);
    std::puts("usage: abi_demo host | abi_demo device IN OUT");
    return 2;
}
