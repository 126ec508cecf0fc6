// Test infrastructure: launchers for the reference's own GPU FFT kernels, the CUDA C its CKIR compiler emitted
// (bench/gpu-fft/generated/fft1024_r{16,4}_batched.cu, included from where they lie in the reference tree; nothing is
// copied). They are the reference's same-box GPU comparator for the N = 1024 batched FFT (bench/gpu-fft/
// ckir_fft_profilee.cu:46-56 launches them the same way: one 1024-point transform per block, split re/im planes,
// the full W_1024 table as two planes). Built by `make -C oracle ckir` with --fmad=false, as the reference builds
// them (bench/CMakeLists.txt:64).

#include <cuda_runtime.h>

#define ckir ckref_fft1024_r16_kernel
#include "fft1024_r16_batched.cu"
#undef ckir
#define ckir ckref_fft1024_r4_kernel
#include "fft1024_r4_batched.cu"
#undef ckir

extern "C" {

// in_re/in_im: batch x 1024 floats each; tw_re/tw_im: 1024 floats (W_1024^k); out_re/out_im: batch x 1024 floats.
int ckref_fft1024_r16(float* in_re, float* in_im, float* tw_re, float* tw_im, float* out_re, float* out_im, int batch,
                      void* stream)
{
    ckref_fft1024_r16_kernel<<<batch, 64, 0, static_cast<cudaStream_t>(stream)>>>(in_re, in_im, tw_re, tw_im, out_re,
                                                                                   out_im);
    return static_cast<int>(cudaGetLastError());
}

int ckref_fft1024_r4(float* in_re, float* in_im, float* tw_re, float* tw_im, float* out_re, float* out_im, int batch,
                     void* stream)
{
    ckref_fft1024_r4_kernel<<<batch, 256, 0, static_cast<cudaStream_t>(stream)>>>(in_re, in_im, tw_re, tw_im, out_re,
                                                                                  out_im);
    return static_cast<int>(cudaGetLastError());
}

} // extern "C"
