// Learned cost model (a small MLP) that ranks candidate plans for a shape,
// and the candidate lists it ranks.
#pragma once

#include <cstddef>

#include "maxmulsk.h"

namespace mmsk {

// Candidate plans of class 0 (FP32) or 1 (split precision); returns the count.
int candidate_plans(int cls, maxmulsk_plan* out, int cap);

// Features of a shape (MAXMULSK_MLP_FEATURES floats).
void mlp_features(size_t M, size_t K, size_t N, int cls, float* x);
int mlp_load(const char* path);
void mlp_unload();
// Host forward pass of the loaded model: predicted log-time per candidate.
bool mlp_predict_host(size_t M, size_t K, size_t N, int cls, float* y);
// Picks the candidate with the lowest predicted time, if a model is loaded;
// with `margin`, also the predicted log-time gap between it and the
// runner-up (how sure the model is of its choice).
bool mlp_predict_plan(size_t M, size_t K, size_t N, int precision, maxmulsk_plan* out, float* margin = nullptr);

}  // namespace mmsk
