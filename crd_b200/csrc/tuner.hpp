// The measuring planner: times the candidate launch shapes of a pass on the device and keeps the fastest as
// "wisdom" (keyed by device name and the pass's geometry class), which later plans reuse without measuring and which
// can be exported and imported as text. Every measurement is also appended to a log (the training data of the
// learned cost model). The reference plans from the size alone (its board of per-level winners was measured
// offline, include/crd/hesap/fft/detail/level_plans_gen.hpp:33-148); here the board is measured on the device.

#pragma once

#include "pass_desc.hpp"

#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace crdfft
{

enum PlannerMode : int
{
    kPlannerEstimate = 0, // wisdom if present, else the heuristic
    kPlannerMeasure = 1,  // wisdom if present, else time every candidate and remember the fastest
    kPlannerLearned = 2,  // wisdom if present, else the candidate the learned cost model ranks first
};

int planner_mode();
void set_planner_mode(int mode);

struct WisdomEntry
{
    bool pipelined = false;
    int points_per_thread = 16;
    int lines_per_cta = 1;
    float ms = 0.0f;
    bool wide_regs = false;
    bool tma_store = false;
};

// The geometry class of a pass: line length and radices, thread map, direct load/store, epilogue, line counts
// bucketed by powers of two, and the parities the pipelined kernel's eligibility depends on.
std::string pass_key(const PassDesc& d, PassMap map, bool dl, bool ds);

bool wisdom_lookup(const std::string& key, WisdomEntry* e);
void wisdom_store(const std::string& key, const WisdomEntry& e);
std::string wisdom_export();
int wisdom_import(const std::string& text); // entries read, or -1 on a malformed line
void wisdom_forget();

// Bytes of input the measuring planner times a candidate on (a pass's lines, or a decomposition's transforms): large
// enough that a launch runs in the steady state of a large batch. On 64 MiB samples the ramp and tail of a 30 us
// launch decided the ranking (the 4096-point pass ranked 32 points a thread first; on 2 GiB it is 2-3 % slower).
// Falls back to 64 MiB when the device cannot hold two sample buffers.
inline constexpr long long kPlannerSampleBytes = 512LL << 20;
inline constexpr long long kPlannerSmallSampleBytes = 64LL << 20;

// Times each candidate (1 warm-up, min of 3 launches, CUDA events, each after an L2-sized read so that the input
// comes from HBM as in a large batch) on scratch buffers sized for up to kPlannerSampleBytes of the pass's lines;
// returns the index of the fastest, or -1 if none could run. ms receives each candidate's time
// (or a negative value when it failed). Appends every timing to the planner log.
// `heuristic` is the index of the heuristic's own choice among the candidates (or -1), marked in the log.
int measure_shapes(const PassDesc& d, const std::string& key, const std::vector<PassShape>& cands,
                   std::vector<float>* ms, int heuristic = -1);
std::string planner_log_export();
void planner_log_append(const std::string& line);

// Decomposition wisdom: for a 1-D transform class (device, length, batch and layout class), the decomposition the
// planner settled on (kind 1 single pass, 2 cluster four-step, 3 two-pass four-step with columns of n1) and its
// measured time. Exported and imported with the pass wisdom (lines whose key starts with "D|").
struct DecompEntry
{
    int kind = 0;
    long long n1 = 0;
    float ms = 0.0f;
};
bool decomp_lookup(const std::string& key, DecompEntry* e);
void decomp_store(const std::string& key, const DecompEntry& e);
std::string decomp_key(long long n, long long batch, bool packed_unit, bool padded, int precision);

// Times `run` (which queues one execute on the stream it is given): 1 warm-up, then the minimum of 3 runs, each
// after an L2-sized read so that inputs come from HBM. Milliseconds, or a negative value when a run failed.
float time_cold_fn(cudaError_t (*run)(void*, cudaStream_t), void* ctx);
template <class F> float time_cold(F& run)
{
    return time_cold_fn([](void* c, cudaStream_t s) { return (*static_cast<F*>(c))(s); }, &run);
}

} // namespace crdfft
