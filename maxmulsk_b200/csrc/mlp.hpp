// Learned cost model (a small MLP) that ranks plans for a shape.
#pragma once

#include <cstddef>

#include "maxmulsk.h"

namespace mmsk {

// Picks the candidate with the lowest predicted time, if a model is loaded.
bool mlp_predict_plan(size_t M, size_t K, size_t N, int precision, maxmulsk_plan* out);

}  // namespace mmsk
