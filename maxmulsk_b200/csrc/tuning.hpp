// Tuning database and learned cost model used by the picker.
#pragma once

#include <cstddef>

#include "maxmulsk.h"

namespace mmsk {

// Exact-shape lookup in the loaded tuning database (MAXMULSK_TUNING_DB, read
// once under a mutex, or maxmulsk_tuning_load()).
bool tuning_lookup(size_t M, size_t K, size_t N, int precision, maxmulsk_plan* out);

// Prediction of the learned cost model, if one is loaded.
bool tuning_predict(size_t M, size_t K, size_t N, int precision, maxmulsk_plan* out);

// Loads (replaces) the database from a text file; returns entries read or -1.
int tuning_load_db(const char* path);
// Adds or replaces one entry in memory, under the requested precision `key`.
void tuning_put(size_t M, size_t K, size_t N, int key, const maxmulsk_plan& p, double time_us);
// Writes the in-memory database; returns entries written or -1.
int tuning_save_db(const char* path);
void tuning_clear();

}  // namespace mmsk
