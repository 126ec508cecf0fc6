// The learned cost model of the planner: a 3-layer MLP (FP32, ReLU, 64 hidden units by default) that predicts the
// log-time of a pass under a candidate launch shape from the pass geometry and the shape. Trained offline on the
// measuring planner's timings (the planner log carries each candidate's feature vector) with the CUDA kernels of
// mlp.cu; evaluated here on the host at plan creation, where it ranks a pass's candidates in microseconds instead of
// timing them on the device.

#pragma once

#include "pass_desc.hpp"

#include <string>

namespace crdfft
{

constexpr int kPassFeatures = 32;

// Feature vector of (pass, candidate shape); the layout is documented at its definition (learned.cpp).
void pass_features(const PassDesc& d, const PassShape& sh, float* f);

// Model as text ("crdfft-mlp 1"): dims, feature normalisation, target normalisation, parameters.
int learned_import(const std::string& text); // 0, or -1 on a malformed text (the current model is kept)
std::string learned_export();
bool learned_ready();
void learned_forget();
// Predicted log(ms) of the whole pass.
float learned_predict(const float* feat);

// The decomposition model (a second model in the same text, tag "crdfft-mlp-decomp"): the predicted log(ms) of a
// whole 1-D transform batch under a decomposition (single pass, cluster four-step, or two-pass four-step n1 x n2).
bool learned_decomp_ready();
float learned_decomp_predict(const float* feat);
// Feature vector of a decomposition (kind 1 single pass, 2 cluster, 3 four-step with columns of n1); radices of the
// two line lengths r1[s1], r2[s2]; layout documented at the definition (learned.cpp).
void decomp_features(long long n, int kind, long long n1, long long batch, bool packed_unit, bool padded,
                     int precision, const int* r1, int s1, const int* r2, int s2, bool stat1, bool stat2,
                     bool tma_col, float* f);

} // namespace crdfft
