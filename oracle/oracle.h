/*
 * TEST INFRASTRUCTURE ONLY - the CPU oracle of the GPU FFT path. Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load it, as the checker; the product (crd_b200/) never links or calls it.
 *
 * Plain-C restatements of the reference's FFT algorithms (yatiyr/CRD, engine/numerics/hesap-fft), each citing the
 * reference file:line it follows. Complex arrays are interleaved {re, im}. Directions: 0 forward (exp(-2πi jk/n)),
 * 1 inverse (exp(+2πi jk/n)).
 */
#ifndef CRD_ORACLE_H
#define CRD_ORACLE_H

#include <stddef.h>
#include <stdint.h>

/* The reference tests' LCG: s = s*6364136223846793005 + 1442695040888963407, u = (s>>11)/2^53*2-1 in [-1, 1)
 * (tests/numerics/hesap-fft/test_fft.cpp:31-44). Fills count doubles. */
void orc_lcg_fill_f64(uint64_t seed, size_t count, double* out);
void orc_lcg_fill_f32(uint64_t seed, size_t count, float* out);
/* Standard normal draws by Box-Muller over pairs of the same LCG's (0, 1] uniforms. */
void orc_gauss_fill_f32(uint64_t seed, size_t count, float* out);

/* Brute-force FP64 DFT with the (j*k) % n angle reduction (test_fft.cpp:47-65). Unnormalised. */
void orc_naive_dft(size_t n, const double* x, double* y, int dir);

/* FP64 mixed-radix self-sorting FFT for any n (any prime factor; O(n * sum of factors)). Validated against
 * orc_naive_dft by the tests, the way the reference gates execute_reference (test_fft.cpp:215-219). Unnormalised. */
int orc_fft_f64(size_t n, const double* x, double* y, int dir);
/* Same, over `batch` contiguous transforms, split over `threads` POSIX threads (0 = 1). */
int orc_fft_batch_f64(size_t n, size_t batch, const double* x, double* y, int dir, int threads);

/* Restatement of FftPlan<T>::execute_reference, the reference's radix-2 in-place DIT oracle with a twiddle table
 * computed in f64 and narrowed to T (fft.hpp:251-260, 417-460). Power of two only; returns -1 otherwise. */
int orc_execute_reference_f32(size_t n, float* data, int dir);
int orc_execute_reference_f64(size_t n, double* data, int dir);

/* Restatement of BluesteinPlan<double>::execute (bluestein.hpp:29-136): forward unnormalised, inverse normalised by
 * 1/n, chirp exp(+iπ k²/n) with k² mod 2n, M = pow2 >= 2n-1. In place. */
int orc_bluestein_f64(size_t n, double* data, int dir);

/* Restatement of RealFftPlan<double>::rfft / irfft (real_fft.hpp:41-92): rfft real[n] -> complex[n/2+1]
 * unnormalised; irfft complex[n/2+1] -> real[n] normalised by 1/n. n even >= 2. */
int orc_rfft_f64(size_t n, const double* x, double* y);
int orc_irfft_f64(size_t n, const double* x, double* y);

/* Restatement of NdFftPlan<double>::execute (nd_fft.hpp:105-182): per-axis forward line transforms, the inverse by
 * conj(FFT(conj x)) / prod(dims). Row-major, in place. */
int orc_nd_f64(size_t ndim, const size_t* dims, double* data, int dir);

/* Error metrics against an FP64 truth over count complex values:
 *   rel_l2   = ||a - b||_2 / ||b||_2
 *   max_rel  = max|a - b| / (1 + max|b|)   (the reference tests' metric, test_fft.cpp:68-96) */
double orc_rel_l2_f32(size_t count, const float* a, const double* b);
double orc_max_rel_f32(size_t count, const float* a, const double* b);

#endif
