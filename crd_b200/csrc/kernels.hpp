// Host-side entry points of the CUDA translation units, called by the planner (plan.cpp).

#pragma once

#include "chain_list.hpp"
#include "pass_desc.hpp"
#include "../../include/crdfft.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace crdfft
{

// One launch of the line-FFT kernel (line_fft.cu).
cudaError_t launch_line_pass(const PassDesc& d, const PassShape& sh, const void* in, void* out, cudaStream_t stream);

// Fused FFT convolution of the lines of a pass (conv.cu): out = conj(FFT(conj(FFT(in) * H))) * scale, with H's
// element e of line l at line_offset(smap, l) + e * smap.estride, the pass's conj_out set and its scale.
bool conv_supported(const PassDesc& d);
cudaError_t launch_conv(const PassDesc& d, PassMap map, const LineMap& smap, const void* in, const void* spec,
                        void* out, cudaStream_t stream);
// Lines a CTA, points a thread and shared memory of a fused convolution pass (conv.cu).
void conv_shape(const PassDesc& d, PassMap map, int* P, int* lpc, int* smem);

// Real-data line kernels (real_line.cu): the pass describes the M-point complex lines (n = 2M reals), row map,
// unit stride. R2C: in = M real pairs a line, out = M + 1 complex. C2R: in = M + 1 complex, out = M real pairs,
// conj_out set. Conv: real pairs in and out, the half spectrum (M + 1 values a line) at line_offset(smap, l),
// conj_out set. wn holds W_n^k for k = 0 .. M/2 at least.
enum : int
{
    kRealR2C = 0,
    kRealC2R = 1,
    kRealConv = 2,
};
struct RealLineAux
{
    const void* wn;
    LineMap smap;
};
bool real_line_supported(const PassDesc& d);

// The row pass of a half-length four-step (M = n1 n2 complex points of z[m] = x[2m] + i x[2m+1]) fused with the R2C
// recombination (real_line.cu): a CTA transforms rows p and n1 - p of the column pass's output, which hold the
// pairs Z[k], Z[M-k] (k = p + n1 k2), and writes the real input's spectrum X[k], k = 0 .. M, at out + t odist.
struct RowR2CDesc
{
    long long M;      // half length
    long long odist;  // complex elements between transforms of the output
    long long batch;  // transforms of this launch
    int n1, n2;       // column and row lengths of the four-step
    const void* wn;   // float2 W_{2M}^k, k = 0 .. M
    float scale;
};
bool row_r2c_supported(const PassDesc& row);

cudaError_t launch_row_r2c(const PassDesc& row, const RowR2CDesc& r, const void* ws, void* out,
                           cudaStream_t stream);
cudaError_t launch_real_line(const PassDesc& d, int mode, const RealLineAux& r, const void* in, const void* spec,
                             void* out, cudaStream_t stream);
// Segment periodograms (spectral.cu): the pass describes the M-point complex lines of one segment (nperseg = 2M).
// welch = 0: out = count x nseg x (M + 1) rows; welch = 1: out = count x ntiles per-CTA sums, then
// launch_welch_finish adds them into count x (M + 1).
struct SpectralDesc
{
    long long nsamples; // samples a signal (the distance between signals)
    long long count;    // signals
    long long nseg;     // segments a signal
    long long hop;      // nperseg - noverlap
    int nperseg;
    int lpc;            // segments a CTA
    int ntiles;         // CTAs a signal
    int detrend;        // subtract each segment's mean
    int welch;
    float scale;        // 1 / (fs sum w^2)
    const float* win;   // nperseg window values
    const void* wn;     // float2 W_nperseg^k, k = 0 .. M/2 at least
};
bool spectral_shape(const PassDesc& d, int* P, int* lpc, int* threads, int* smem);
cudaError_t launch_spectral(const PassDesc& d, const SpectralDesc& sd, int threads, int smem, const void* x,
                            void* out, cudaStream_t stream);
cudaError_t launch_welch_finish(const SpectralDesc& sd, const void* part, void* psd, cudaStream_t stream);
// The four-step column pass as a persistent kernel fed by 2-D tensor copies (tma_col.cu).
bool tma_col_supported(const PassDesc& d);
cudaError_t launch_tma_col(const PassDesc& d, const void* in, void* out, cudaStream_t stream);
// The four-step row pass with its transposed tile stored by the Tensor Memory Accelerator (tma_col.cu).
bool row_tstore_supported(const PassDesc& d, const PassShape& sh);
cudaError_t launch_row_tstore(const PassDesc& d, const PassShape& sh, const void* in, void* out, cudaStream_t stream);
int pass_lines_per_cta_limit();
int pass_line_pitch(int n);
int pass_cta_line_pitch(int n, int lpc); // the compile-time-schedule kernel's line pitch (complex elements)
int pass_threads_limit(int points_per_thread, long long n); // classic kernel CTA size limit
int pass_pipe_threads();
int pass_pipe_smem(int n, PassMap map, int lpc);
bool pass_has_kernel(const PassDesc& d, const PassShape& sh);
// A compile-time schedule exists for the pass's radices at this many points a thread.
bool pass_has_static(const PassDesc& d, int points_per_thread);

// Real <-> half-length complex recombination (real_ops.cu), the math of the reference's RealFftPlan
// (include/crd/hesap/fft/real_fft.hpp:41-92), over `batch` transforms of real length n = 2h.
//   r2c_post: z (h complex per transform, zdist apart) -> out (h+1 complex per transform, odist apart)
//   c2r_pre:  in (h+1 complex, idist apart) -> z (h complex, zdist apart), ready for the inverse half FFT
struct RealRecombine
{
    long long h;
    long long batch;
    long long zdist;
    long long xdist; // the (h+1)-element spectrum side
    const void* wn;  // float2 W_n^k, k = 0 .. h
    float scale;     // applied to the output
};
cudaError_t launch_r2c_post(const RealRecombine& p, const void* z, void* out, cudaStream_t stream);
cudaError_t launch_c2r_pre(const RealRecombine& p, const void* in, void* z, cudaStream_t stream);

// Bluestein helpers (real_ops.cu): chirp pre-multiply with zero padding, pointwise spectrum product, chirp
// post-multiply. The math of include/crd/hesap/fft/bluestein.hpp:87-136.
struct ChirpDesc
{
    long long n;      // transform length
    long long m;      // padded power-of-two length (>= 2n - 1)
    long long batch;
    long long xdist;  // distance between transforms on the n side
    long long wdist;  // distance between transforms on the m side (scratch)
    const void* chirp; // float2 exp(+iπ k²/n), k < n
    const void* bfft;  // float2 FFT_m(b_circ), length m
    int conj;          // inverse direction: conjugate x on the way in and the result on the way out
    float scale;       // final scale (1/m, times 1/n for the normalised inverse)
};
cudaError_t launch_chirp_pre(const ChirpDesc& p, const void* x, void* w, cudaStream_t stream);
cudaError_t launch_spectrum_mul(const ChirpDesc& p, void* w, cudaStream_t stream);
cudaError_t launch_chirp_post(const ChirpDesc& p, const void* w, void* x, cudaStream_t stream);

// Cluster-fused four-step (cluster_fft.cu): one thread-block cluster per transform of n = a.n * b.n, columns of
// length a.n (descriptor a: in.estride = b.n, stage twiddles, four-step twiddle tables), rows of length b.n
// (descriptor b: out.estride = a.n), contiguous transforms n apart. cluster_split names the split when a compiled
// instance exists for n.
bool cluster_split(long long n, long long* n1, long long* n2);
cudaError_t launch_cluster_fft(const PassDesc& a, const PassDesc& b, long long batch, const void* in, void* out,
                               cudaStream_t stream);

// A bump arena of device memory: while bound to the calling thread, plan creation takes every device allocation
// (tables, status word, workspace) from it instead of cudaMalloc, and plans built so never free.
crdfft_status first_use_self_check(int dev); // selfcheck.cpp

struct Arena
{
    char* base;
    size_t size;
    size_t used;
};
void arena_bind(Arena* a);

// Tensor-core line pass (tc_fft.cu): the first radix-16 stage as a tcgen05 GEMM. prec 1 = split-BF16 (3 terms),
// 2 = FP16 with a per-line scale. Row-contiguous passes of n = 512 (16.8.4), 1024 (16.16.4), 4096 (16.16.16).
bool tc_pass_supported(const PassDesc& d, int prec);
void tc_build_a(int prec, std::vector<uint16_t>* out);
cudaError_t launch_tc_pass(const PassDesc& d, int prec, const void* amat, const void* in, void* out,
                           cudaStream_t stream);

// The continuous wavelet transform's element-wise kernels (cwt.cu). CwtScale: one scale's epilogue parameters.
struct CwtScale
{
    long long off; // (taps - 2) / 2: the first filtered sample a coefficient reads
    float amp;     // -sqrt(scale)
    int taps_ok;   // taps >= 2; otherwise the scale's coefficients are 0
};
cudaError_t launch_cwt_pad(const float* x, void* X, long long n, long long lfft, long long count, cudaStream_t stream);
// product: W (signals x nscales x lfft) = X (signals x lfft) times K (nscales x lfft), line by line;
// diff: out (signals x nscales x n) from W.
cudaError_t launch_cwt_product(const void* X, const void* K, void* W, long long lfft, long long nscales,
                               long long signals, cudaStream_t stream);
cudaError_t launch_cwt_diff(const void* W, const CwtScale* scales, void* out, long long n, long long lfft,
                            long long nscales, long long signals, cudaStream_t stream);
// The CWT's lines in one kernel (conv.cu): load conj(X[c] K[s]) into shared memory, the forward stages of `d` (a
// fused-convolution plan's line pass, conv_line_pass), and the differenced, conjugated, scaled store of n samples.
// d.lines = signals x nscales lines of this launch. cwt_lines_supported: a compile-time schedule exists for d.
bool conv_line_pass(crdfft_plan* plan, PassDesc* out);
bool cwt_lines_supported(const PassDesc& d);
cudaError_t launch_cwt_lines(const PassDesc& d, const void* X, const void* K, const CwtScale* scales, long long nscales,
                             long long n, void* out, cudaStream_t stream);

// The two-pass four-step as one persistent launch over L2-sized waves (chain_fft.cu). col: the column pass of wave 0
// (lines wave_t * n2, maps relative to the wave's first transform, the four-step twiddle on); row: its row pass
// (lines wave_t * n1, input in the wave's slot). ctr: 1 + 2 waves ints, zero before the launch (the tile ticket, then
// each wave's finished column tiles, then its finished row tiles).
struct ChainDesc
{
    PassDesc col;
    PassDesc row;
    long long waves;      // W = ceil(batch / wave_t)
    long long wave_t;     // transforms a wave
    long long batch;
    long long idist;      // complex elements between transforms, input and output
    long long odist;
    long long slot_elems; // wave_t * n: one wave's intermediate
    int slots;            // intermediate slots (waves in flight)
    int lag;              // a wave's row tiles follow the column tiles of the wave `lag` later; 1 <= lag < slots
    int col_lpc;          // lines a column tile (chain_lines_per_tile(n1))
    int row_lpc;          // lines a row tile
    long long col_items;  // column tiles a wave: ceil(wave_t * n2 / col_lpc)
    long long row_items;  // row tiles a wave: ceil(wave_t * n1 / row_lpc)
    int* ctr;
    int spin_limit;       // polls a dependency wait may take before it gives up (status word |= 1)
};
bool chain_supported(const PassDesc& col, const PassDesc& row);
cudaError_t launch_chain(const ChainDesc& cd, const void* in, void* out, void* ws, cudaStream_t stream);

// Elementwise scale of `count` complex values (used by normalisations that no pass can absorb).
cudaError_t launch_scale(void* data, long long count, float s, cudaStream_t stream);
cudaError_t launch_planar_gather(const void* re, const void* im, void* out, long long count, cudaStream_t stream);
cudaError_t launch_planar_scatter(const void* in, void* re, void* im, long long count, cudaStream_t stream);

} // namespace crdfft
