// Exposes the reference's own portable CPU GEMM and checker with a C ABI so
// Python (ctypes) can call them. TEST INFRASTRUCTURE ONLY.
//
// Nothing of the reference is copied here: the recipe in oracle/Makefile puts
// the reference checkout's root on the include path and this file includes
// common/utils.hpp from where it lies. Built into oracle/_ref/ (git-ignored).
//
//   Utils::multiply_scalar     common/utils.hpp:50-61  (argument order M, N, K)
//   Utils::check_correctness   common/utils.hpp:24-48
//   Utils::compute_gflops      common/utils.hpp:20-22
#include "common/utils.hpp"

#include <cstddef>
#include <sstream>
#include <iostream>

extern "C" {

void ref_multiply_scalar(const float* A, const float* B, float* C,
                         size_t M, size_t N, size_t K) {
    Utils::multiply_scalar(A, B, C, M, N, K);
}

// Returns 1 when every |ref - target| <= tol. The reference prints its
// mismatches to std::cout; they are swallowed here.
int ref_check_correctness(const float* ref, const float* target, size_t size, float tol) {
    std::ostringstream sink;
    std::streambuf* old = std::cout.rdbuf(sink.rdbuf());
    bool ok = Utils::check_correctness(ref, target, size, "ref", tol);
    std::cout.rdbuf(old);
    return ok ? 1 : 0;
}

double ref_compute_gflops(size_t M, size_t N, size_t K, double time_ms) {
    return Utils::compute_gflops(M, N, K, time_ms);
}

}  // extern "C"
