"""CPU oracle for the FP32 GEMM (test infrastructure only).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package. It is the checker, never the product.

* ``liboracle.so`` (oracle/oracle.c, built by oracle/Makefile): the C
  restatement: FP32 scalar GEMM (Utils::multiply_scalar), the v3 outer-Kc
  panel order, FP64 truth, error measures, split planes, seeded generators.
* ``libmaxmulsk_ref.so`` (oracle/_ref/, built from the reference checkout's
  common/utils.hpp by ``make -C oracle ref REFERENCE_ROOT=<checkout>``): the reference's own
  multiply_scalar / check_correctness, used to pin the restatement and as the
  timed CPU baseline. Present only where it was built.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_float, c_int, c_int64, c_size_t, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libmaxmulsk_ref.so")
REF_FMA_LIB = os.path.join(HERE, "_ref", "libmaxmulsk_ref_fma.so")

_lib = None
_ref = None
_ref_fma = None


def build(reference_root: str | None = None) -> None:
    """Compiles the oracle, and the reference's own common/utils.hpp into
    oracle/_ref when `reference_root` names a reference checkout that has it."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if reference_root and os.path.exists(os.path.join(reference_root, "common", "utils.hpp")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REFERENCE_ROOT={reference_root}"], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        fp = POINTER(c_float)
        dp = POINTER(c_double)
        L.oracle_fill_uniform.argtypes = [fp, c_size_t, c_uint64]
        L.oracle_fill_normal.argtypes = [fp, c_size_t, c_uint64, c_float]
        L.oracle_fill_wide.argtypes = [fp, c_size_t, c_uint64]
        L.oracle_sgemm_scalar.argtypes = [fp, fp, fp, c_size_t, c_size_t, c_size_t]
        L.oracle_sgemm_panels.argtypes = [fp, fp, fp, c_size_t, c_size_t, c_size_t, c_size_t, c_int]
        L.oracle_dgemm.argtypes = [fp, fp, dp, c_size_t, c_size_t, c_size_t, c_int]
        L.oracle_dgemm_abs.argtypes = [fp, fp, dp, c_size_t, c_size_t, c_size_t]
        L.oracle_dgemm_rows.argtypes = [fp, fp, dp, c_size_t, c_size_t, POINTER(c_int64), c_size_t]
        L.oracle_errors.argtypes = [fp, dp, fp, fp, c_size_t, c_size_t, c_size_t, dp]
        L.oracle_relfrob.argtypes = [fp, fp, c_size_t]
        L.oracle_relfrob.restype = c_double
        L.oracle_check_correctness.argtypes = [fp, fp, c_size_t, c_float, fp]
        L.oracle_check_correctness.restype = c_size_t
        L.oracle_split_tf32.argtypes = [fp, fp, fp, c_size_t]
        L.oracle_split_bf16.argtypes = [fp, fp, fp, fp, c_size_t]
        L.oracle_sgemm_split_exact.argtypes = [fp, fp, fp, c_size_t, c_size_t, c_size_t, c_int]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def _load_ref(path: str) -> ctypes.CDLL:
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built (make -C oracle ref)")
    R = ctypes.CDLL(path)
    fp = POINTER(c_float)
    R.ref_multiply_scalar.argtypes = [fp, fp, fp, c_size_t, c_size_t, c_size_t]
    R.ref_check_correctness.argtypes = [fp, fp, c_size_t, c_float]
    R.ref_check_correctness.restype = c_int
    R.ref_compute_gflops.argtypes = [c_size_t, c_size_t, c_size_t, c_double]
    R.ref_compute_gflops.restype = c_double
    return R


def ref() -> ctypes.CDLL:
    """The reference's own compiled common/utils.hpp (oracle/_ref), no contraction."""
    global _ref
    if _ref is None:
        _ref = _load_ref(REF_LIB)
    return _ref


def ref_fma_available() -> bool:
    return os.path.exists(REF_FMA_LIB)


def ref_fma() -> ctypes.CDLL:
    """The same reference source built with multiply-add contraction (FMA)."""
    global _ref_fma
    if _ref_fma is None:
        _ref_fma = _load_ref(REF_FMA_LIB)
    return _ref_fma


def _f(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(POINTER(c_float))


def _d(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(POINTER(c_double))


# ------------------------------------------------------------------ inputs
def fill_uniform(n: int, seed: int) -> np.ndarray:
    x = np.empty(n, np.float32)
    lib().oracle_fill_uniform(_f(x), n, seed)
    return x


def fill_normal(n: int, seed: int, scale: float) -> np.ndarray:
    x = np.empty(n, np.float32)
    lib().oracle_fill_normal(_f(x), n, seed, float(np.float32(scale)))
    return x


def fill_wide(n: int, seed: int) -> np.ndarray:
    x = np.empty(n, np.float32)
    lib().oracle_fill_wide(_f(x), n, seed)
    return x


# ------------------------------------------------------------------ products
def sgemm_scalar(A: np.ndarray, B: np.ndarray, M: int, K: int, N: int) -> np.ndarray:
    """Restatement of Utils::multiply_scalar (called with its (M, N, K) order)."""
    C = np.empty(M * N, np.float32)
    lib().oracle_sgemm_scalar(_f(A), _f(B), _f(C), M, N, K)
    return C.reshape(M, N)


def sgemm_panels(A: np.ndarray, B: np.ndarray, M: int, K: int, N: int, kc: int = 0, fma: bool = True) -> np.ndarray:
    C = np.empty(M * N, np.float32)
    lib().oracle_sgemm_panels(_f(A), _f(B), _f(C), M, K, N, kc, 1 if fma else 0)
    return C.reshape(M, N)


def dgemm(A: np.ndarray, B: np.ndarray, M: int, K: int, N: int, threads: int | None = None) -> np.ndarray:
    C = np.empty(M * N, np.float64)
    lib().oracle_dgemm(_f(A), _f(B), _d(C), M, K, N, threads or min(8, os.cpu_count() or 1))
    return C.reshape(M, N)


def dgemm_abs(A: np.ndarray, B: np.ndarray, M: int, K: int, N: int) -> np.ndarray:
    """(|A||B|)_ij in FP64, k upward (the max-relative floor's sums)."""
    C = np.empty(M * N, np.float64)
    lib().oracle_dgemm_abs(_f(A), _f(B), _d(C), M, K, N)
    return C.reshape(M, N)


def dgemm_rows(A: np.ndarray, B: np.ndarray, K: int, N: int, rows) -> np.ndarray:
    r = np.ascontiguousarray(np.asarray(rows, dtype=np.int64))
    C = np.empty(len(r) * N, np.float64)
    lib().oracle_dgemm_rows(_f(A), _f(B), _d(C), K, N, r.ctypes.data_as(POINTER(c_int64)), len(r))
    return C.reshape(len(r), N)


def errors(C: np.ndarray, C64: np.ndarray, A: np.ndarray, B: np.ndarray, M: int, K: int, N: int) -> dict:
    out = np.zeros(4, np.float64)
    lib().oracle_errors(_f(np.ascontiguousarray(C, np.float32)), _d(np.ascontiguousarray(C64)), _f(A), _f(B),
                        M, K, N, _d(out))
    return {"normwise": out[0], "max_rel": out[1], "rel_frob": out[2], "max_abs": out[3]}


def relfrob(a: np.ndarray, b: np.ndarray) -> float:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return float(lib().oracle_relfrob(_f(a), _f(b), a.size))


def check_correctness(ref_: np.ndarray, got: np.ndarray, tol: float = 1e-3) -> tuple[int, float]:
    md = np.zeros(1, np.float32)
    r = np.ascontiguousarray(ref_, np.float32)
    g = np.ascontiguousarray(got, np.float32)
    bad = lib().oracle_check_correctness(_f(r), _f(g), r.size, tol, _f(md))
    return int(bad), float(md[0])


def split_tf32(x: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    x = np.ascontiguousarray(x, np.float32).ravel()
    hi = np.empty_like(x)
    lo = np.empty_like(x)
    lib().oracle_split_tf32(_f(x), _f(hi), _f(lo), x.size)
    return hi, lo


def split_bf16(x: np.ndarray) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    x = np.ascontiguousarray(x, np.float32).ravel()
    l0, l1, l2 = np.empty_like(x), np.empty_like(x), np.empty_like(x)
    lib().oracle_split_bf16(_f(x), _f(l0), _f(l1), _f(l2), x.size)
    return l0, l1, l2


def sgemm_split_exact(A: np.ndarray, B: np.ndarray, M: int, K: int, N: int, mode: int) -> np.ndarray:
    C = np.empty(M * N, np.float32)
    lib().oracle_sgemm_split_exact(_f(A), _f(B), _f(C), M, K, N, mode)
    return C.reshape(M, N)


# ------------------------------------------------------------------ the reference itself
def ref_multiply_scalar(A: np.ndarray, B: np.ndarray, M: int, K: int, N: int) -> np.ndarray:
    C = np.empty(M * N, np.float32)
    ref().ref_multiply_scalar(_f(A), _f(B), _f(C), M, N, K)
    return C.reshape(M, N)


def ref_fma_multiply_scalar(A: np.ndarray, B: np.ndarray, M: int, K: int, N: int) -> np.ndarray:
    C = np.empty(M * N, np.float32)
    ref_fma().ref_multiply_scalar(_f(A), _f(B), _f(C), M, N, K)
    return C.reshape(M, N)


def ref_check_correctness(ref_: np.ndarray, got: np.ndarray, tol: float = 1e-3) -> bool:
    r = np.ascontiguousarray(ref_, np.float32)
    g = np.ascontiguousarray(got, np.float32)
    return bool(ref().ref_check_correctness(_f(r), _f(g), r.size, tol))
