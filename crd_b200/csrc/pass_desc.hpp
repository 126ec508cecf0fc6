// One launch of the line-FFT kernel family: `lines` independent DFTs of length n, each read from and written to
// global memory through a two-level (group, line-in-group, element) address map, with optional conjugation,
// four-step twiddle and scale fused into the store. Every plan in this library is a short sequence of these passes
// (one for n that fits a CTA's shared memory, two for the four-step above that), which replaces the reference's
// per-algorithm CPU engines (engine/numerics/hesap-fft/kernels/fft_kernels.cpp:187-354 Stockham,
// :2363-2658 four-step).
//
// Shared between the host planner (C++20) and the CUDA translation unit; plain data only.

#pragma once

#include <cstdint>

namespace crdfft
{

inline constexpr int kMaxStages = 12;

// Element e of line l = g * lines_per_group + q sits at  g*gdist + q*ldist + e*estride  (complex elements).
struct LineMap
{
    long long gdist;
    long long ldist;
    long long estride;
};

struct PassDesc
{
    int n;                       // line length
    int nstages;                 // number of radix stages (product of radix[] == n)
    int radix[kMaxStages];       // stage radices in execution order (each of 2,3,4,5,7,8,9,16, or 32)
    long long lines;             // total lines this launch transforms
    long long lines_per_group;   // lines per address group (a transform, for multi-line-per-transform passes)
    LineMap in;
    LineMap out;
    const void* tw;              // float2 stage-ordered twiddles: for each stage after the first (radix R, after
                                 // radices multiplying to L), W_{LR}^{r k} at (r-1) L + k, stages back to back
    // Four-step twiddle, fused into the store: output element k of line q is multiplied by W_M^{q*k}
    // (q < n2, k < n1 = n) = hi[(q>>4) n + k] * lo[16 k + (q&15)] with hi = W_M^{16 a k}, lo = W_M^{b k}.
    // Off when ftw_M == 0. The twiddle row q of a line is (its index within its group) / ftw_div: 1 for a 1-D
    // four-step (lines of a group are the columns), the column count for a split column pass of a 2-D array (the
    // lines of a group are (q, column) pairs, column fastest).
    const void* ftw_hi;
    const void* ftw_lo;
    long long ftw_M;
    int ftw_div;
    int discard_in;              // the input is dead once this pass has read it (a four-step intermediate read from
                                 // L2): the classic row kernel drops its 128-byte L2 lines without a write-back
    int conj_in;                 // conjugate every input element (inverse via conj(DFT(conj x)))
    int conj_out;                // conjugate every output element
    float scale;                 // multiply every output element (1 = off)
    // Pipelined kernel only: a device word the kernel ORs 1 into when a bounded shared-memory barrier wait gives up
    // (the host reads it with crdfft_device_status), the wait's iteration limit, and a test hook that makes the
    // first wait of every CTA target a barrier nothing completes, so that the wait runs out without any fault.
    int* err;
    int spin_limit;
    int debug_stall;
};

// The kernel variants the planner can pick for a pass.
enum class PassMap : int
{
    Row = 0, // threads run along the elements of a line; lines are contiguous (estride == 1 on the loading side)
    Col = 1, // threads run across adjacent lines (ldist == 1): strided columns, four-step pass 1 and N-D axes
};

// How a launch is shaped. Chosen by the host planner from n and the two line maps.
struct PassShape
{
    bool pipelined;         // persistent CTAs, input lines brought into shared memory by bulk async copies
    PassMap map;
    int threads_per_line;   // T
    int lines_per_cta;      // LPC
    int points_per_thread;  // P (template instance: 8, 16 or 32)
    bool direct_load;       // first stage reads global memory itself (coalesced for this map)
    bool direct_store;      // last stage writes global memory itself
    int smem_bytes;
    bool wide_regs;         // compile-time schedules at 16 points a thread: the 80-register build (fewer resident
                            // warps, no spill) instead of the 64-register one
    bool tma_store;         // the row pass of a four-step: the transposed tile leaves by tensor stores (tma_col.cu)
};

} // namespace crdfft
