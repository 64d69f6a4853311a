// Phase timing: the counterpart of the reference's lab hooks, macros at fixed
// scopes of its blocked driver (allocation, pack_a, pack_b, compute,
// writeback: sme/support/lab_hooks.hpp:1-22, used in
// sme/v3/sme-1x4-acc-kcout.cpp:453-561), and of the per-phase timing
// breakdown of its test harness (sme/support/test_sme.cpp:580-678).
//
// Off by default (one relaxed atomic load per scope). Switched on by
// MAXMULSK_PHASE_TIMING=1 in the environment or maxmulsk_phase_timing(1).
// While on, a PhaseScope records a CUDA event pair around its work on its
// stream (device time, summed per phase by maxmulsk_phase_report) and an NVTX
// range on the host thread (for a profiler). Streams being captured into a
// CUDA graph record nothing: a captured launch runs later, from the graph.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

namespace mmsk {

enum Phase : int {
    kPhaseSplit = 0,     // operand planes (split pre-pass)            ~ pack_a / pack_b
    kPhaseGemm,          // the GEMM kernel                            ~ compute + writeback
    kPhaseReduce,        // split-K reduction of the partial tiles     ~ later Kc panels' add
    kPhaseGrouped,       // one grouped batch (its CUDA graph)
    kPhaseH2D,           // host entry points: operands to the device
    kPhaseD2H,           // host entry points: C back to the host
    kPhaseCount
};

bool phase_timing_on();
void phase_set(bool on);
// Waits for the recorded scopes, writes {"phase": {"calls": n, "ms": t}, ...}
// (device time per phase since the last report) into buf, NUL-terminated and
// truncated to len, forgets them, and returns the length of the whole text.
size_t phase_report(char* buf, size_t len);

// While a PhaseMute lives, scopes on this host thread record nothing (the
// autotuner's timing runs are not phases of the caller's call).
class PhaseMute {
public:
    PhaseMute();
    ~PhaseMute();
    PhaseMute(const PhaseMute&) = delete;
    PhaseMute& operator=(const PhaseMute&) = delete;
};

class PhaseScope {
public:
    PhaseScope(Phase phase, cudaStream_t stream);
    ~PhaseScope();
    PhaseScope(const PhaseScope&) = delete;
    PhaseScope& operator=(const PhaseScope&) = delete;

private:
    Phase phase_;
    cudaStream_t stream_;
    cudaEvent_t begin_ = nullptr;
    bool nvtx_ = false;
};

}  // namespace mmsk
