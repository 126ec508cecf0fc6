// Device work list of the uneven-batch kernel (uneven.cu), built by the planner (plan.cpp).

#pragma once

#include "pass_desc.hpp"

#include <cuda_runtime.h>

namespace crdfft
{

enum UnevenKind : int
{
    kUnevenSmall = 0, // up to `lines` whole transforms of one length, at offsets line_off[line_table + a]
    kUnevenCol = 1,   // columns q0 .. q0+lines-1 of one long transform -> its workspace region (+ four-step twiddle)
    kUnevenRow = 2,   // rows of one long transform's workspace region -> the output (waits for its COL items)
};

// One line length's run-time radix schedule and stage-ordered twiddle table.
struct UnevenSched
{
    int n;
    int nstages;
    int radix[kMaxStages];
    const void* tw;
    int variant; // 0: the run-time stages (every length); 1: the length's compile-time schedule (uneven_static_ok)
};

struct UnevenItem
{
    int kind;
    int sched;       // index into the schedule table (the item's line length)
    int lines;
    int line_table;  // SMALL: first index into line_off; else -1
    long long in_base, in_ldist, in_estride;
    long long out_base, out_ldist, out_estride;
    int transform;   // COL/ROW: index of the long transform (completion counter)
    int need;        // ROW: COL items of that transform
    int q0;          // COL: first column (four-step twiddle row)
    int ftw;         // COL: index of the long transform's four-step tables; else -1
};

struct UnevenTables
{
    const void* const* ftw_hi; // per long length: hi[(q>>4) n1 + k1] = W_n^{16 (q>>4) k1}
    const void* const* ftw_lo; // lo[16 k1 + (q&15)] = W_n^{(q&15) k1}
};

struct UnevenDesc
{
    const UnevenItem* items;
    const UnevenSched* scheds;
    const long long* line_off;
    UnevenTables tables;
    int* counter;   // next item; followed in memory by done[ntransforms] (zeroed together before each launch)
    int* done;
    int* err;
    int nitems;
    int ntransforms;
    int spin_limit;
    int slot_elems; // float2 elements of one item slot of shared memory (two slots, then the stages' buffer)
    int conj;       // inverse: conjugate in and out
    float scale;
};

int uneven_threads();
// Line lengths the persistent kernel also has as compile-time stage sequences (the powers of two 16 .. 4096).
bool uneven_static_ok(int n);
cudaError_t launch_uneven(const UnevenDesc& u, int smem_bytes, const void* in, void* out, void* scratch,
                          cudaStream_t stream);

} // namespace crdfft
