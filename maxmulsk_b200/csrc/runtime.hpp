// Host runtime: per-device state, workspace cache, per-thread host staging,
// plan validation and dispatch. C++ only; the C ABI in capi.cpp wraps it.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <cuda_runtime.h>

#include "maxmulsk.h"

namespace mmsk {

// Records a CUDA error message for maxmulsk_last_error_message() and maps it
// to a status (allocation failures to MAXMULSK_ERR_ALLOC).
maxmulsk_status cuda_status(cudaError_t e, const char* where);
void set_error_message(const std::string& msg);
const char* last_error_message();

// Plan helpers (plan.cpp).
maxmulsk_status classify_plan(size_t M, size_t K, size_t N, const maxmulsk_plan* plan);
size_t workspace_bytes(size_t M, size_t K, size_t N, const maxmulsk_plan& plan);
maxmulsk_plan choose_rule(size_t M, size_t K, size_t N, int precision, int sms);
maxmulsk_plan choose_tuned(size_t M, size_t K, size_t N, int precision, int sms);
bool parse_config_env(maxmulsk_plan& out);
// Exhaustive search as the picker's fallback. picker_doubt says why the
// learned model should not decide this shape (no model loaded, a shape
// outside its training range, two plans predicted within
// MAXMULSK_AUTOTUNE_MARGIN, default 0.005 in ln-time), or nullptr when the
// model (or a tuning database entry) decides. MAXMULSK_AUTOTUNE=0 turns the
// fallback off.
const char* picker_doubt(size_t M, size_t K, size_t N, int precision);
bool autotune_fallback_enabled();
// Runs the search on these device operands when it is due (enabled, no
// database entry, picker_doubt, `s` not being captured into a graph) and
// stores the winner in the tuning database; C is overwritten by the search.
// Failures leave the picker to the model or the rule.
void autotune_fallback(const float* dA, const float* dB, float* dC, size_t M, size_t K, size_t N, int precision,
                       cudaStream_t s);
// Host-pointer form: copies A and B to this thread's device staging first.
void autotune_fallback_host(const float* A, const float* B, size_t M, size_t K, size_t N, int precision);
// The library-managed workspace of (current device, stream), grown to at
// least `need` bytes (it may synchronise `s` to grow); nullptr on failure.
void* managed_workspace(cudaStream_t s, size_t need, size_t* bytes, maxmulsk_status* st);

// Runs a validated plan on device pointers with a caller-provided workspace.
// b_planes (split-precision plans only): B's operand planes, already written
// by split_one(as_b); only A is split then.
maxmulsk_status run_plan_dev(const float* dA, const float* dB, float* dC, size_t M, size_t K, size_t N,
                             const maxmulsk_plan& plan, void* ws, size_t ws_bytes, cudaStream_t s,
                             void* b_planes = nullptr);

// Runs a plan with the library-managed workspace of (current device, stream).
maxmulsk_status run_plan_managed(const float* dA, const float* dB, float* dC, size_t M, size_t K, size_t N,
                                 const maxmulsk_plan& plan, cudaStream_t s, void* b_planes = nullptr);

// Host-pointer form: copy in, run, copy out, wait, check the error word.
// Large products with page-locked A and C run as a pipeline of row blocks, so
// that copies in, the GEMM and copies out overlap.
maxmulsk_status run_plan_host(const float* A, const float* B, float* C, size_t M, size_t K, size_t N,
                              const maxmulsk_plan& plan);

// Empty-shape contract of the reference (capi/maxmulsk.cpp:13-20), on device
// memory: true when handled. K == 0 zeroes C.
bool handle_empty_dev(float* dC, size_t M, size_t K, size_t N, cudaStream_t s, maxmulsk_status* st);

// Waits for `s`, then reports and clears the device error word.
maxmulsk_status stream_status(cudaStream_t s);

}  // namespace mmsk
