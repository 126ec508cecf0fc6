/*
 * crdfft.h - C ABI of the B200 FFT execution path (plan creation + execute), a drop-in for crd-hesap-fft's
 * plan/execute surface (reference: engine/numerics/hesap-fft/include/crd/hesap/fft/).
 *
 * Data are device pointers to interleaved single-precision complex values ({float re; float im;}, the layout of
 * crd::hesap::Complex<f32>, engine/numerics/hesap/include/crd/hesap/complex.hpp:30-35) or to plain floats for the
 * real side of R2C/C2R. Every call is stream-ordered on the CUDA stream passed as `stream` (NULL = legacy default
 * stream). No function aborts: each returns a crdfft_status. Plans are immutable after creation; one plan may be
 * executed from several threads only on distinct workspaces (crdfft_set_workspace), as the reference's "one plan
 * per thread" rule (fft.hpp:17-18) asks of its scratch.
 *
 * Sign and normalisation follow the reference:
 *   forward  X_k = sum_j x_j exp(-2 pi i j k / n)           (fft.hpp:257-259)
 *   inverse  x_j = sum_k X_k exp(+2 pi i j k / n) * s       s = 1 (CRDFFT_NORM_NONE, FftPlan, fft.hpp:16)
 *                                                           s = 1/n (CRDFFT_NORM_INVERSE: BluesteinPlan,
 *                                                           bluestein.hpp:84-86; RealFftPlan::irfft,
 *                                                           real_fft.hpp:87-91; NdFftPlan, nd_fft.hpp:138-146)
 */
#ifndef CRDFFT_H
#define CRDFFT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. The reference's preconditions are CRD_ASSERTs and its out-of-memory is fatal (fft.hpp:237,411,468,
 * 480-483); here each becomes a returned code. */
typedef enum crdfft_status
{
    CRDFFT_OK = 0,
    CRDFFT_INVALID_DESC = 1,      /* malformed descriptor (rank, dims, strides, kind) */
    CRDFFT_UNSUPPORTED_SIZE = 2,  /* a size or layout this build does not plan */
    CRDFFT_OOM = 3,               /* a device allocation for tables or workspace failed */
    CRDFFT_LAUNCH = 4,            /* a kernel launch or CUDA runtime call failed */
    CRDFFT_DEVICE_TIMEOUT = 5,    /* a bounded device-side wait gave up (persistent kernels) */
    CRDFFT_NUMERIC_SELFCHECK = 6, /* the device known-answer check disagreed with the host FP64 DFT */
    CRDFFT_INVALID_ARG = 7,       /* null plan/pointer, wrong direction, size mismatch */
    CRDFFT_NO_DEVICE = 8          /* no CUDA device, or the plan's device is not current */
} crdfft_status;

/* FftDirection (include/crd/hesap/fft/fft_kernels.hpp:20-24). */
typedef enum crdfft_direction
{
    CRDFFT_FORWARD = 0,
    CRDFFT_INVERSE = 1
} crdfft_direction;

typedef enum crdfft_kind
{
    CRDFFT_C2C = 0, /* complex -> complex */
    CRDFFT_R2C = 1, /* real[n] -> complex[n/2+1] (RealFftPlan::rfft, real_fft.hpp:41-64); forward only */
    CRDFFT_C2R = 2  /* complex[n/2+1] -> real[n] (RealFftPlan::irfft, real_fft.hpp:67-92); inverse only */
} crdfft_kind;

typedef enum crdfft_precision
{
    CRDFFT_PREC_FP32 = 0,       /* FP32 butterflies, FP32 data */
    CRDFFT_PREC_SPLIT_BF16 = 1,   /* first radix-16 stage as a tensor-core GEMM on three-term bf16 splits, six
                                     products, FP32 accumulate (rel-L2 about 4e-7) */
    CRDFFT_PREC_FP16_SCALED = 2,  /* the same on fp16 with a per-line power-of-two scale, one term (about 2e-4) */
    CRDFFT_PREC_SPLIT_BF16_2 = 3, /* bf16 hi+lo, three products (about 16 bits of the data: above 1e-6) */
    CRDFFT_PREC_SPLIT_FP16_2 = 4  /* fp16 hi+lo with a per-line scale, three products (about 22 bits) */
} crdfft_precision;

typedef enum crdfft_norm
{
    CRDFFT_NORM_NONE = 0,   /* unnormalised both ways (FftPlan) */
    CRDFFT_NORM_INVERSE = 1 /* inverse scaled by 1/prod(dims) (Bluestein, Real, Nd plans) */
} crdfft_norm;

/* A plan descriptor. dims are row-major (dims[rank-1] varies fastest). For R2C/C2R, dims[rank-1] is the real
 * length n and the complex side holds n/2+1 values along that axis (rank 2 and 3 real plans: packed batches, n/2 at
 * most 8192; the reference's real plan is 1-D and its NdFftPlan complex). Strides and distances count elements of the
 * side they describe (complex elements, or floats on the real side); 0 selects the packed layout:
 *   istride = 1, idist = prod(input dims).
 * The reference's element-major execute_batched (fft.hpp:462-470) is istride = ostride = batch, idist = odist = 1. */
typedef struct crdfft_desc
{
    int32_t rank;      /* 1, 2 or 3 */
    int32_t kind;      /* crdfft_kind */
    int32_t precision; /* crdfft_precision */
    int32_t norm;      /* crdfft_norm */
    int64_t dims[3];
    int64_t batch;     /* >= 1 */
    int64_t istride;   /* rank 1 only; 0 = 1 */
    int64_t idist;     /* 0 = packed */
    int64_t ostride;   /* rank 1 only; 0 = 1 */
    int64_t odist;     /* 0 = packed */
} crdfft_desc;

typedef struct crdfft_plan crdfft_plan;

typedef struct crdfft_plan_info
{
    char algorithm[64];      /* "single-pass", "four-step", "bluestein", "real+single-pass", "nd-axes", ... */
    int32_t passes;          /* kernel launches one forward execute issues */
    int32_t device;          /* the CUDA device the plan lives on */
    int64_t workspace_bytes; /* scratch one execute needs */
    int64_t table_bytes;     /* device twiddle / chirp tables the plan owns */
    int64_t factors[8];      /* the line lengths of the passes (e.g. n1, n2 of the four-step), 0-terminated */
} crdfft_plan_info;

/* ---- General plan (cuFFT-style descriptor) ------------------------------------------------------------------ */

/* Build a plan on the current CUDA device. Computes twiddle tables in FP64 on the host and narrows them to FP32
 * (the reference's convention, fft.hpp:251-260), uploads them and allocates the workspace. Replaces the FftPlan /
 * RealFftPlan / BluesteinPlan / NdFftPlan constructors (fft.hpp:224-304, real_fft.hpp:21-36, bluestein.hpp:31-75,
 * nd_fft.hpp:31-79). */
crdfft_status crdfft_plan_create(const crdfft_desc* desc, crdfft_plan** plan);

/* Release a plan, its tables and its owned workspace. NULL is accepted. */
crdfft_status crdfft_plan_destroy(crdfft_plan* plan);

/* Run the plan: `in` -> `out` (in == out allowed for C2C, the reference's in-place execute, fft.hpp:409-413).
 * `direction` is crdfft_direction; R2C plans accept only CRDFFT_FORWARD and C2R plans only CRDFFT_INVERSE. */
crdfft_status crdfft_execute(crdfft_plan* plan, const void* in, void* out, int32_t direction, void* stream);

/* Run the plan on HOST buffers, the way the reference's plans are called (FftPlan::execute transforms a span of CPU
 * memory in place, fft.hpp:409-413): `in` and `out` are host memory laid out as the plan's descriptor says (element
 * stride 1; in == out allowed). The batch is cut into chunks (an eighth of the batch, 4 to 64 MiB of input) that run
 * through a three-stage pipeline, each stage on its own internal stream (copy to the device, transform, copy back)
 * with three staging slots, so the copies in both directions and the transforms of different chunks overlap. Convolution plans are not supported. Use page-locked host memory (cudaHostAlloc / pinned tensors): with
 * pageable memory the result is the same but the copies do not overlap. The work is ordered after everything
 * already queued on `stream`, and `stream` waits for all of it: synchronise `stream` before reading `out`. The first
 * call on a plan allocates its device staging buffers (three chunks each way) and the chunk plans; calls on one plan
 * must not overlap. Uneven-batch plans are not supported (CRDFFT_INVALID_ARG). */
crdfft_status crdfft_execute_host(crdfft_plan* plan, const void* in, void* out, int32_t direction, void* stream);

/* Run a C2C plan on split-complex (planar) operands: separate re and im planes of float, each laid out as the
 * plan's descriptor says for complex elements (in == out planes allowed). The layouts whose transforms tile the
 * planes exactly are accepted: packed batches, and the rank-1 element-major batch (istride = ostride = batch,
 * idist = odist = 1); others return CRDFFT_INVALID_ARG. The split-complex tensors of the reference's CEIR
 * `tensor.fft` op (operands re_in, im_in; results re_out, im_out; engine/execution/ceir-gpu/src/ckir_synth.cpp:331)
 * and of its CKIR FFT kernels (engine/gpu/kir/include/crd/kir/ckir_fft.hpp:61-66) take this entry point. The planes
 * are interleaved into a staging buffer the plan allocates at its first planar call (prod(dims) * batch * 8 bytes),
 * transformed there in place and split again: two streaming passes around the plan's own. */
crdfft_status crdfft_execute_planar(crdfft_plan* plan, const float* re_in, const float* im_in, float* re_out,
                                    float* im_out, int32_t direction, void* stream);

crdfft_status crdfft_plan_info_get(const crdfft_plan* plan, crdfft_plan_info* info);

/* Bytes of scratch one execute of this plan uses (0 when it needs none). */
size_t crdfft_workspace_size(const crdfft_plan* plan);

/* Point the plan at caller-owned device scratch of at least crdfft_workspace_size bytes (256-byte aligned); the
 * plan frees the workspace it allocated. NULL restores a plan-owned workspace. */
crdfft_status crdfft_set_workspace(crdfft_plan* plan, void* workspace, size_t bytes);

const char* crdfft_status_string(crdfft_status status);

/* ---- The reference's plan classes, verb for verb ------------------------------------------------------------- */

/* FftPlan<float>(alloc, n) (fft.hpp:224): one size-n complex transform, unnormalised both ways. */
crdfft_status crdfft_fft_plan_create(int64_t n, crdfft_plan** plan);
/* FftPlan::execute(data, dir) (fft.hpp:409-413): in place. */
crdfft_status crdfft_fft_execute(crdfft_plan* plan, void* data, int32_t direction, void* stream);
/* FftPlan::execute_batched(data, batch, dir) (fft.hpp:462-470): `batch` transforms, element i of transform t at
 * data[i*batch + t], in place. */
crdfft_status crdfft_fft_execute_batched(crdfft_plan* plan, void* data, int64_t batch, int32_t direction,
                                         void* stream);

/* RealFftPlan<float>(alloc, n) (real_fft.hpp:21-36); n even, >= 2. */
crdfft_status crdfft_real_plan_create(int64_t n, crdfft_plan** plan);
/* RealFftPlan::rfft(real_in[n], out[n/2+1]) (real_fft.hpp:41-64), unnormalised. */
crdfft_status crdfft_rfft(crdfft_plan* plan, const float* real_in, void* out, void* stream);
/* RealFftPlan::irfft(in[n/2+1], real_out[n]) (real_fft.hpp:67-92), normalised by 1/n. */
crdfft_status crdfft_irfft(crdfft_plan* plan, const void* in, float* real_out, void* stream);

/* BluesteinPlan<float>(alloc, n) (bluestein.hpp:31): any n >= 1; forward unnormalised, inverse normalised by 1/n.
 * 7-smooth n run natively in mixed radix; other n run the chirp-z algorithm over a power-of-two plan. */
crdfft_status crdfft_bluestein_plan_create(int64_t n, crdfft_plan** plan);
/* BluesteinPlan::execute(data, dir) (bluestein.hpp:87-136): in place. */
crdfft_status crdfft_bluestein_execute(crdfft_plan* plan, void* data, int32_t direction, void* stream);

/* NdFftPlan<float>(alloc, dims) (nd_fft.hpp:31): row-major ndim in 1..3; inverse normalised by 1/prod(dims). */
crdfft_status crdfft_nd_plan_create(int32_t ndim, const int64_t* dims, crdfft_plan** plan);
/* NdFftPlan::execute(data, dir) (nd_fft.hpp:105-147): in place. */
crdfft_status crdfft_nd_execute(crdfft_plan* plan, void* data, int32_t direction, void* stream);

/* One-shot fft(alloc, data, dir) (fft.hpp:1006-1012) and ifft_normalized (fft.hpp:1015-1029): build a transient
 * plan, run it in place, release it (synchronises the stream before releasing). */
crdfft_status crdfft_fft(void* data, int64_t n, int32_t direction, void* stream);
crdfft_status crdfft_ifft_normalized(void* data, int64_t n, void* stream);

/* ---- Fused FFT convolution ---------------------------------------------------------------------------------- */

/* y = IFFT(FFT(x) * H) * scale for a batch of 1-D (rank 1) or 2-D (rank 2, rows x cols) complex signals: the circular
 * convolution with the filter whose spectrum H = FFT(h) the caller supplies. No counterpart in crd-hesap-fft's CPU
 * API; it follows the reference's GPU fused convolution (engine/gpu/kir/include/crd/kir/ckir_fft.hpp:279-296,
 * 2075-2090: scale 1/N by default, one filter shared by the batch or one per signal), where the vendor route takes
 * three global passes (bench/gpu-fft/cufft_conv_bench.cu:3-5). Rank 1 runs in one launch (each signal's forward
 * FFT, product and inverse FFT in shared memory: one read and one write per point); rank 2 runs the row FFTs, the
 * fused convolution along the columns, then the inverse row FFTs. desc: C2C, packed (element stride 1, distance
 * the signal size), each dimension up to 8192 and 7-smooth. filter_per_transform: 0 for one spectrum (rank 1: n
 * values; rank 2: rows x cols, row-major) shared by the batch, 1 for one per signal (batch times that). scale < 0
 * means 1 / (number of points of one signal).
 * desc.kind = CRDFFT_R2C: real signals (float in and out) and the half spectrum H (n/2 + 1 complex values along the
 * last axis: rank 1 n/2 + 1, rank 2 rows x (cols/2 + 1)); the last dimension even with half at most 8192. Rank 1
 * is one launch; rank 2 is R2C rows, the fused convolution along the half-width columns and C2R rows, the order of
 * the reference's real 2-D convolution (ckir_fft.hpp:2300-2308). */
crdfft_status crdfft_conv_plan_create(const crdfft_desc* desc, int32_t filter_per_transform, double scale,
                                      crdfft_plan** plan);
/* in == out allowed. crdfft_execute rejects convolution plans (CRDFFT_INVALID_ARG). */
crdfft_status crdfft_conv_execute(crdfft_plan* plan, const void* in, const void* spectrum, void* out, void* stream);

/* ---- Spectral estimators ------------------------------------------------------------------------------------ */

/* The segment periodograms of hesap-dsp (engine/numerics/hesap-dsp/include/crd/hesap/dsp/spectral.hpp) over `count`
 * real signals of `nsamples` floats each (packed), in one launch: each segment minus its mean ('constant' detrend),
 * times the window, real FFT, one-sided density |X|^2 / (fs sum w^2), doubled except at DC and Nyquist.
 *   CRDFFT_SPECTRAL_WELCH        welch_psd (spectral.hpp:141-172): the average over segments, count x nfreq;
 *                                noverlap 0 means nperseg / 2, as there
 *   CRDFFT_SPECTRAL_SPECTROGRAM  spectrogram (spectral.hpp:177-183): count x nseg x nfreq, row s = segment s
 *   CRDFFT_SPECTRAL_PERIODOGRAM  periodogram (spectral.hpp:188-220): one segment of the whole signal, boxcar
 *                                window, count x nfreq (nperseg, noverlap and window ignored)
 * nfreq = nperseg / 2 + 1, nseg = (nsamples - noverlap) / (nperseg - noverlap), 0 when nsamples < nperseg (Welch
 * then writes zeros). nperseg even, at least 4, half at most 8192. The Welch average adds the segments in a fixed
 * order, so its result is the same on every run. */
#define CRDFFT_SPECTRAL_WELCH 0
#define CRDFFT_SPECTRAL_SPECTROGRAM 1
#define CRDFFT_SPECTRAL_PERIODOGRAM 2
typedef struct crdfft_spectral_desc
{
    int32_t mode;
    int32_t detrend;      /* 1: subtract each segment's mean (the reference's 'constant'); 0: none */
    int64_t nsamples;
    int64_t count;
    int64_t nperseg;
    int64_t noverlap;
    double fs;
    const float* window;  /* host, nperseg values; NULL: the periodic Hann window (windows.hpp:120-124) */
} crdfft_spectral_desc;
crdfft_status crdfft_spectral_plan_create(const crdfft_spectral_desc* desc, crdfft_plan** plan);
/* Segments a signal under the descriptor (after the Welch noverlap default), or -1 for an invalid one. */
int64_t crdfft_spectral_segments(const crdfft_spectral_desc* desc);
/* x: count x nsamples floats on the device; out as above. crdfft_execute rejects spectral plans. */
crdfft_status crdfft_spectral_execute(crdfft_plan* plan, const float* x, float* out, void* stream);

/* ---- Continuous wavelet transform ------------------------------------------------------------------------- */

/* crd-hesap-wavelet's cwt (engine/numerics/hesap-wavelet/include/crd/hesap/wavelet/cwt.hpp:461-621) over `count`
 * real signals of nsamples samples. The plan builds the wavelet's integral and each scale's kernel in FP64 on the
 * host (sample_psi, cwt.hpp:149-280; the kernels at cwt.hpp:569-581) and keeps the kernels' spectra on the device;
 * an execute zero-pads and transforms the signals, then for every (signal, scale) line multiplies the two spectra,
 * inverse-transforms and forms -sqrt(a) (w[t+1] - w[t]) / lfft (cwt.hpp:583-596): in one kernel with the line in
 * shared memory for FFT lengths 256 .. 8192 that have a compile-time schedule, else as a product kernel, a batched
 * inverse FFT plan and an epilogue kernel in rounds of as many signals as 512 MiB of scratch holds. */
typedef struct crdfft_cwt_desc
{
    const char* wavelet;    /* "mexh", "morl", "cmorB-C", "gausP", "cgauP", "shanB-C", "fbspM-B-C", "paulM"
                             * (continuous_wavelet, cwt.hpp:300-407); a name matching none is "mexh", as there */
    const double* scales;   /* host memory: nscales scales > 0 */
    int64_t nsamples;       /* n >= 1 */
    int64_t count;          /* signals >= 1 */
    int64_t nscales;        /* 1 .. 65535 */
    double sampling_period; /* for the frequencies only; 0 = 1 */
    int32_t precision;      /* log2 of the wavelet grid, 1 .. 20; 0 = 12 (the reference's default) */
    int32_t reserved;       /* 0 */
} crdfft_cwt_desc;

typedef struct crdfft_cwt_plan crdfft_cwt_plan;

crdfft_status crdfft_cwt_plan_create(const crdfft_cwt_desc* desc, crdfft_cwt_plan** plan);
crdfft_status crdfft_cwt_plan_destroy(crdfft_cwt_plan* plan);
/* x: count x nsamples floats on the device; coeffs: count x nscales x nsamples complex values on the device, signal
 * c's CwtResult::coeffs[s * n + i] (cwt.hpp:446-456) at coeffs[(c * nscales + s) * n + i]. Stream-ordered; the plan's
 * scratch serves one execute at a time. */
crdfft_status crdfft_cwt_execute(crdfft_cwt_plan* plan, const float* x, void* coeffs, void* stream);
/* Host only, no device: CwtResult::frequencies, central_frequency / (scale * sampling_period) (cwt.hpp:410-444). */
crdfft_status crdfft_cwt_frequencies(const crdfft_cwt_desc* desc, double* frequencies);
/* Host only, no device: the FFT length, the power of two >= n + the longest kernel (cwt.hpp:479-506); -1 for an
 * invalid descriptor. */
int64_t crdfft_cwt_fft_length(const crdfft_cwt_desc* desc);
/* The plan's FFT length, the signals one round takes, and whether one fused line kernel runs each execute (FFT
 * lengths with a compile-time line schedule) or the product / inverse FFT / epilogue rounds. Any pointer may be NULL. */
crdfft_status crdfft_cwt_plan_info(const crdfft_cwt_plan* plan, int64_t* fft_length, int64_t* signals_per_round,
                                   int32_t* fused);

/* ---- Uneven batches ---------------------------------------------------------------------------------------- */

/* `count` independent forward/inverse complex transforms of different lengths (7-smooth, 2 .. 8192^2), transform t
 * at element offset offsets[t] of the input and of the output (NULL: packed, see crdfft_uneven_offsets). The
 * reference runs such a batch as a loop of per-size plans over crd-jobs ranges (detail/batch_arms.hpp:59-77); here
 * one persistent launch walks a device work list, captured once per (in, out, direction) into a CUDA graph.
 * Execute with crdfft_execute; both directions unnormalised. */
crdfft_status crdfft_plan_create_uneven(const int64_t* sizes, int64_t count, const int64_t* offsets,
                                        crdfft_plan** plan);
/* Packed offsets for an uneven batch (each transform starting on a 16-byte boundary) into offsets[count] (may be
 * NULL); returns the total number of complex elements the buffer needs, or -1. */
int64_t crdfft_uneven_offsets(const int64_t* sizes, int64_t count, int64_t* offsets);

/* ---- Planner ----------------------------------------------------------------------------------------------- */

/* How plan creation picks each pass's launch shape (kernel variant, points a thread, lines a CTA):
 *   CRDFFT_PLANNER_ESTIMATE  remembered wisdom for the pass's geometry class, else a fixed heuristic (default)
 *   CRDFFT_PLANNER_MEASURE   remembered wisdom, else time every candidate on the device (scratch buffers of up to
 *                            512 MiB per pass, 64 MiB when the device is short of memory, each timed launch after
 *                            an L2-sized read so that its input comes from HBM) and remember the fastest
 * Two levels are planned this way: the decomposition of each 1-D transform length (one pass, the cluster four-step,
 * or the two-pass four-step n1 x n2 for every split whose halves fit one CTA; timed as whole executes of a sample of
 * the batch, up to 256 MiB) and the launch shape of each pass. The reference plans from the size alone from a board
 * measured offline (detail/level_plans_gen.hpp:33-148); here the board is measured on the device and kept as wisdom.
 * The environment variable CRDFFT_PLANNER=measure sets the initial mode. Once a class has wisdom, every later plan of
 * that class makes the same choice. */
#define CRDFFT_PLANNER_ESTIMATE 0
#define CRDFFT_PLANNER_MEASURE 1
/*   CRDFFT_PLANNER_LEARNED   remembered wisdom, else the imported learned models (crdfft_learned_model_import)
 *                            rank the candidates (decompositions and launch shapes) and the measuring planner times
 *                            only their top proposals (CRDFFT_LEARNED_TOP_K, default 2) and keeps the fastest: the
 *                            model proposes, the measurement judges. Without a model for a level, that level is
 *                            planned as in CRDFFT_PLANNER_MEASURE. */
#define CRDFFT_PLANNER_LEARNED 2
void crdfft_set_planner_mode(int32_t mode);

/* Force the decomposition of 1-D transforms of length n in plans created from now on (whatever the planner mode):
 * kind 1 one pass, 2 the cluster four-step, 3 the two-pass four-step with columns of n1 (rows of n / n1); kind 0
 * removes the override. A decomposition the length does not admit is ignored at plan creation (the planner
 * decides). Returns CRDFFT_INVALID_ARG for a kind outside 0..3. */
crdfft_status crdfft_set_decomposition(int64_t n, int32_t kind, int64_t n1);

/* Wisdom as text ("crdfft-wisdom 1" then one line per pass class: key, pipelined, points a thread, lines a CTA,
 * measured ms, and a trailing "w" when the pass runs the 80-register build of its kernel; decompositions on lines
 * starting "D|": key, kind, n1, ms), keyed by device name. Export writes a NUL-terminated string into buf when cap
 * suffices and reports the size needed; import merges entries and rejects a malformed text (CRDFFT_INVALID_ARG)
 * without changes. */
crdfft_status crdfft_wisdom_export(char* buf, size_t cap, size_t* needed);
crdfft_status crdfft_wisdom_import(const char* text);
void crdfft_wisdom_forget(void);

/* Every timing the measuring planner took in this process, one line per candidate ("<key> pipelined=.. P=.. lpc=..
 * lines=.. ms=.. feat=f0,..,f31", the winner marked "best", the heuristic's own choice marked "heur"): the training
 * data of the learned cost model. crdfft_wisdom_forget clears it too. */
crdfft_status crdfft_planner_log(char* buf, size_t cap, size_t* needed);

/* ---- Learned cost model -------------------------------------------------------------------------------------- */

/* No counterpart in the reference (its planner reads a board of per-level winners measured offline,
 * detail/level_plans_gen.hpp:33-148). A 3-layer MLP (FP32, ReLU) predicts the log-time of a pass under a candidate
 * launch shape from a feature vector of crdfft_pass_feature_count() floats (the "feat=" field of the planner log).
 * The model text is "crdfft-mlp 1", then "dims D H", "mean" and "std" (D feature normalisers each), "target m s"
 * (log(ms) = m + s * output) and "params P" followed by the P parameters of crdfft_mlp_param_count's layout.
 * Import rejects a malformed text (CRDFFT_INVALID_ARG) and keeps the current model. */
int32_t crdfft_pass_feature_count(void);
crdfft_status crdfft_learned_model_import(const char* text);
crdfft_status crdfft_learned_model_export(char* buf, size_t cap, size_t* needed);
void crdfft_learned_model_forget(void);
/* Host evaluation of the imported model on one feature vector: predicted log(ms) in *out. */
crdfft_status crdfft_learned_predict(const float* features, float* out);

/* Device kernels that train the model (no library call, no floating-point atomics: bit-reproducible). Every pointer
 * is device memory; parameters are one flat array [W1 (H x D)][b1 (H)][W2 (H x H)][b2 (H)][W3 (H)][b3 (1)],
 * weights row-major (out x in); x is rows x D row-major (already normalised); workspace holds
 * crdfft_mlp_workspace_floats(D, H, rows) floats. */
size_t crdfft_mlp_param_count(int32_t in_dim, int32_t hidden);
size_t crdfft_mlp_workspace_floats(int32_t in_dim, int32_t hidden, int64_t rows);
/* y[rows] = W3 relu(W2 relu(W1 x + b1) + b2) + b3 */
crdfft_status crdfft_mlp_forward(int32_t in_dim, int32_t hidden, const float* params, const float* x, int64_t rows,
                                 float* y, float* workspace, void* stream);
/* loss[0] = mean((y - target)^2) and grad = d loss / d params (same layout as params). */
crdfft_status crdfft_mlp_gradients(int32_t in_dim, int32_t hidden, const float* params, const float* x,
                                   const float* target, int64_t rows, float* grad, float* loss, float* workspace,
                                   void* stream);
/* One Adam step (bias-corrected moments, step >= 1) over count parameters. */
crdfft_status crdfft_mlp_adam(float* params, const float* grad, float* m, float* v, int64_t count, int32_t step,
                              float lr, float beta1, float beta2, float eps, void* stream);

/* ---- The CEIR tensor.fft lowering -------------------------------------------------------------------------- */

/* What the reference's GPU provider knows about a `tensor.fft` op when it lowers it (synth_fft,
 * engine/execution/ceir-gpu/src/ckir_synth.cpp:318-366; the op contract, engine/execution/ceir/src/tensor.cpp:174-192,
 * 344). The provider fills it from the op and its operand re_in. */
#define CRDFFT_CEIR_MAX_RANK 8
typedef struct crdfft_ceir_fft_op
{
    int32_t num_operands;      /* the op's operand count (re_in, im_in) */
    int32_t num_results;       /* the op's result count (re_out, im_out) */
    int32_t operand_is_tensor; /* re_in is Tensor-kinded */
    int32_t element_is_f32;    /* re_in's element type is f32 */
    int32_t rank;              /* rank of re_in's shape */
    int32_t axis;              /* the `axis` attribute; -1 when absent (the innermost axis) */
    int64_t shape[CRDFFT_CEIR_MAX_RANK]; /* static extents; a dynamic extent as -1 */
    const char* direction;     /* the `direction` attribute's string, NULL when it is not a string */
} crdfft_ceir_fft_op;

/* Why an op was not lowered. The first six have the reference's SynthReject names (OpNotSupported,
 * OperandNotTensor, ElementNotF32, FftRankUnsupported, ShapeNotStatic, FftDirectionUnknown); its FftLengthNotPow2
 * does not occur here: every static length >= 1 is planned. */
typedef enum crdfft_ceir_reject
{
    CRDFFT_CEIR_NONE = 0,
    CRDFFT_CEIR_OP_NOT_SUPPORTED = 1,
    CRDFFT_CEIR_OPERAND_NOT_TENSOR = 2,
    CRDFFT_CEIR_ELEMENT_NOT_F32 = 3,
    CRDFFT_CEIR_RANK_UNSUPPORTED = 4,
    CRDFFT_CEIR_SHAPE_NOT_STATIC = 5,
    CRDFFT_CEIR_DIRECTION_UNKNOWN = 6,
    CRDFFT_CEIR_AXIS_UNSUPPORTED = 7
} crdfft_ceir_reject;

/* Map a tensor.fft op to a plan descriptor and a direction (host only, no device needed). The transform runs along
 * `axis`: the innermost axis of any rank (batch = product of the other extents, packed) or axis 0 of a rank-2
 * tensor (the element-major batch); FP32, unnormalised both ways like the op (the 1/N is the caller's,
 * engine/gpu/kir/include/crd/kir/ckir_fft.hpp:21). The plan then runs with crdfft_execute_planar on the op's four
 * planes. On a rejection *reject says why (the status is CRDFFT_INVALID_DESC or CRDFFT_UNSUPPORTED_SIZE) and the
 * provider keeps its own path for the op. */
crdfft_status crdfft_ceir_fft_desc(const crdfft_ceir_fft_op* op, crdfft_desc* desc, int32_t* direction,
                                   int32_t* reject);

/* ---- Without device allocation ----------------------------------------------------------------------------- */

/* No counterpart in the reference (its plans always allocate their tables from the caller's allocator).
 * For callers that cannot allocate device memory (work enqueued while a stream is being captured, real-time
 * callbacks that must never enter an allocator, processes whose device memory belongs to a pool they do not own):
 * `batch` contiguous size-n complex transforms (FftPlan semantics: unnormalised both ways; in == out allowed), with
 * every table and intermediate taken from a 64 MiB device array that the library holds on each GPU it is loaded on.
 * Allocates no device memory. n up to 2^22 (larger: CRDFFT_UNSUPPORTED_SIZE); a length with a prime factor above 7
 * (Bluestein, padded length m >= 2n - 1) is accepted while its ~8 m (batch + 3) bytes fit the array, else also
 * CRDFFT_UNSUPPORTED_SIZE. All calls on a device share the array: the last call's plan stays in it, and calls whose
 * GPU work overlaps race, so order them on one stream. A call with a new (n, batch) rebuilds the array: it waits for
 * all work queued on the device (cudaDeviceSynchronize), so the previous call's kernels finish first on any stream,
 * and during a stream capture it returns CRDFFT_INVALID_ARG without queuing anything: make the first call with each
 * (n, batch) outside the capture. A captured graph reads the array as it was when captured: it is valid only until
 * a call with another (n, batch). The first call on a device looks up the array's address; make it before any
 * stream capture. */
crdfft_status crdfft_execute_static_scratch(const void* in, void* out, int64_t n, int64_t batch, int32_t direction,
                                            void* stream);

/* ---- Self-check and fault injection ------------------------------------------------------------------------- */

/* The device known-answer check (the role of the reference's fft_self_check, src/fft_self_check.cpp:153-211):
 * runs a set of small transforms (radices 2..16, 3, 5, 7, a four-step and a real transform) on the current device
 * and compares them with a host FP64 DFT: max|gpu - dft| <= 1e-5 (1 + max|dft|). CRDFFT_OK or
 * CRDFFT_NUMERIC_SELFCHECK. The library also runs it once per device at the first plan creation there, as the
 * reference checks its kernel table before first use (src/fft_kernel_dispatch.cpp:48-52): if it disagrees, that
 * creation and every later one on the device return CRDFFT_NUMERIC_SELFCHECK. CRDFFT_SELF_CHECK=0 in the environment
 * turns the first-use check off; crdfft_execute_static_scratch (which allocates nothing) does not run it. */
crdfft_status crdfft_self_check(void);

/* Test hooks for the first-use check: plant a mistake in the check's host FP64 answers (on: every comparison
 * disagrees), and forget which devices were checked, so the next plan creation checks again. */
void crdfft_debug_self_check_mismatch(int32_t on);
void crdfft_debug_self_check_reset(void);

/* Test hook: uneven-batch plans created from now on run their power-of-two line lengths on the run-time stages (0)
 * or on the compile-time stages (1); -1 returns the choice to the planner. */
void crdfft_debug_uneven_variant(int32_t variant);

/* Test hook: make the k-th device allocation from now fail (k >= 1), as if the device were out of memory; 0 turns
 * it off. The reference tests its out-of-memory paths with a refusing allocator in a child process
 * (tests/numerics/hesap-fft/CMakeLists.txt:26-36); here plan creation returns CRDFFT_OOM instead. */
void crdfft_debug_fail_alloc_after(int32_t k);

/* Read and clear the plan's device status word, after the work queued on `stream`: CRDFFT_DEVICE_TIMEOUT when a
 * kernel of this plan gave up a bounded wait since the last call (its outputs are then incomplete), else CRDFFT_OK.
 * Synchronises the stream. */
crdfft_status crdfft_device_status(crdfft_plan* plan, void* stream);

/* Test hook: plans created while this is on make each CTA of their pipelined kernels first wait on a shared-memory
 * barrier that nothing completes, so the bounded wait runs out; the CTA then lets its own copies land and returns,
 * and crdfft_device_status reports CRDFFT_DEVICE_TIMEOUT. 0 turns it off. */
void crdfft_debug_stall_waits(int32_t on);

#ifdef __cplusplus
}
#endif

#endif /* CRDFFT_H */
