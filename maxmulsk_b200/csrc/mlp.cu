// Learned cost model: placeholder until the model kernels land.
#include "mlp.hpp"

namespace mmsk {

bool mlp_predict_plan(size_t, size_t, size_t, int, maxmulsk_plan*) { return false; }

}  // namespace mmsk
