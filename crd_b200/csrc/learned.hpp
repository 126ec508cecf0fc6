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

} // namespace crdfft
