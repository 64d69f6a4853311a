"""ctypes bindings for libmaxmulsk_b200.so (the C ABI in include/maxmulsk.h).

The library is built in-tree by ``maxmulsk_b200.build``. Loading fails loudly
when it is missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_float, c_int32, c_size_t, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libmaxmulsk_b200.so")


class Plan(ctypes.Structure):
    """maxmulsk_plan: how one GEMM is cut into work."""

    _fields_ = [
        ("precision", c_int32),
        ("tile_m", c_int32),
        ("tile_n", c_int32),
        ("split_k", c_int32),
        ("variant", c_int32),
        ("chunk", c_int32),
        ("reserved", c_int32 * 2),
    ]

    def __repr__(self) -> str:
        return (f"Plan(precision={self.precision}, tile_m={self.tile_m}, tile_n={self.tile_n}, "
                f"split_k={self.split_k}, variant={self.variant}"
                + (f", chunk={self.chunk})" if self.chunk else ")"))

    def as_tuple(self) -> tuple[int, int, int, int, int]:
        return (self.precision, self.tile_m, self.tile_n, self.split_k, self.variant)


class Problem(ctypes.Structure):
    """maxmulsk_problem: one GEMM of a grouped launch (device pointers)."""

    _fields_ = [
        ("A", c_void_p),
        ("B", c_void_p),
        ("C", c_void_p),
        ("M", c_size_t),
        ("K", c_size_t),
        ("N", c_size_t),
    ]


class ErrorReport(ctypes.Structure):
    """maxmulsk_error_report: error measures of an FP32 result against FP64."""

    _fields_ = [
        ("normwise", ctypes.c_double),
        ("max_rel", ctypes.c_double),
        ("rel_frob", ctypes.c_double),
        ("max_abs", ctypes.c_double),
        ("norm_a", ctypes.c_double),
        ("norm_b", ctypes.c_double),
        ("norm_diff", ctypes.c_double),
        ("norm_c64", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: float(getattr(self, name)) for name, _ in self._fields_}


# name -> (restype, argtypes)
_SIGNATURES: dict[str, tuple] = {
    "maxmulsk_sgemm_v3": (c_int32, [c_void_p, c_void_p, c_void_p, c_size_t, c_size_t, c_size_t]),
    "maxmulsk_sgemm_v4": (c_int32, [c_void_p, c_void_p, c_void_p, c_size_t, c_size_t, c_size_t]),
    "maxmulsk_sgemm_v3_dev": (c_int32, [c_void_p, c_void_p, c_void_p, c_size_t, c_size_t, c_size_t, c_void_p]),
    "maxmulsk_sgemm_v4_dev": (c_int32, [c_void_p, c_void_p, c_void_p, c_size_t, c_size_t, c_size_t, c_void_p]),
    "maxmulsk_classify": (c_int32, [c_size_t, c_size_t, c_size_t, POINTER(Plan)]),
    "maxmulsk_choose": (c_int32, [c_size_t, c_size_t, c_size_t, c_int32, POINTER(Plan)]),
    "maxmulsk_picker_doubt": (c_char_p, [c_size_t, c_size_t, c_size_t, c_int32]),
    "maxmulsk_choose_rule": (c_int32, [c_size_t, c_size_t, c_size_t, c_int32, POINTER(Plan)]),
    "maxmulsk_workspace_bytes": (c_size_t, [c_size_t, c_size_t, c_size_t, POINTER(Plan)]),
    "maxmulsk_sgemm_plan_dev": (c_int32, [c_void_p, c_void_p, c_void_p, c_size_t, c_size_t, c_size_t,
                                          POINTER(Plan), c_void_p, c_size_t, c_void_p]),
    "maxmulsk_sgemm_plan": (c_int32, [c_void_p, c_void_p, c_void_p, c_size_t, c_size_t, c_size_t,
                                      POINTER(Plan)]),
    "maxmulsk_sgemm_split": (c_int32, [c_void_p, c_void_p, c_void_p, c_size_t, c_size_t, c_size_t, c_int32]),
    "maxmulsk_sgemm_split_dev": (c_int32, [c_void_p, c_void_p, c_void_p, c_size_t, c_size_t, c_size_t,
                                           c_int32, c_void_p]),
    "maxmulsk_sgemm_plan_static_dev": (c_int32, [c_void_p, c_void_p, c_void_p, c_size_t, c_size_t, c_size_t,
                                                 POINTER(Plan), c_void_p]),
    "maxmulsk_grouped_create": (c_int32, [POINTER(Problem), c_size_t, POINTER(Plan), POINTER(c_void_p)]),
    "maxmulsk_grouped_launch": (c_int32, [c_void_p, c_void_p]),
    "maxmulsk_grouped_info": (c_int32, [c_void_p, POINTER(Plan), POINTER(c_int32), POINTER(c_size_t)]),
    "maxmulsk_grouped_plans": (c_int32, [c_void_p, POINTER(Plan)]),
    "maxmulsk_grouped_destroy": (None, [c_void_p]),
    "maxmulsk_sgemm_grouped_dev": (c_int32, [POINTER(Problem), c_size_t, c_void_p]),
    "maxmulsk_candidates": (c_size_t, [c_int32, POINTER(Plan), c_size_t]),
    "maxmulsk_autotune_time_dev": (c_int32, [c_void_p, c_void_p, c_void_p, c_size_t, c_size_t, c_size_t,
                                             POINTER(Plan), c_size_t, c_void_p, c_size_t, c_int32,
                                             POINTER(c_float), c_void_p]),
    "maxmulsk_autotune_dev": (c_int32, [c_void_p, c_void_p, c_void_p, c_size_t, c_size_t, c_size_t, c_int32,
                                        c_void_p, c_size_t, POINTER(Plan), POINTER(c_float), c_void_p]),
    "maxmulsk_tuning_load": (c_int32, [c_char_p]),
    "maxmulsk_tuning_save": (c_int32, [c_char_p]),
    "maxmulsk_tuning_clear": (None, []),
    "maxmulsk_model_load": (c_int32, [c_char_p]),
    "maxmulsk_mlp_features": (c_int32, [c_size_t, c_size_t, c_size_t, c_int32, POINTER(c_float)]),
    "maxmulsk_mlp_predict_host": (c_int32, [c_size_t, c_size_t, c_size_t, c_int32, POINTER(c_float)]),
    "maxmulsk_mlp_forward_dev": (c_int32, [c_void_p, c_void_p, c_int32, c_void_p, c_void_p, c_void_p, c_void_p,
                                           c_void_p, c_void_p]),
    "maxmulsk_mlp_backward_dev": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                            c_void_p, c_void_p, c_int32, c_float, c_void_p, c_void_p, c_void_p,
                                            c_void_p]),
    "maxmulsk_mlp_adam_dev": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_float, c_float, c_float, c_float,
                                        c_int32, c_void_p]),
    "maxmulsk_mlp_predict_dev": (c_int32, [c_void_p, c_void_p, c_void_p, c_int32, c_void_p, c_void_p, c_void_p,
                                           c_void_p]),
    "maxmulsk_probe_split_bytes": (c_size_t, [c_size_t, c_size_t, c_int32, c_int32]),
    "maxmulsk_probe_split_dev": (c_int32, [c_void_p, c_size_t, c_size_t, c_int32, c_int32, c_void_p, c_void_p]),
    "maxmulsk_probe_timeout_dev": (c_int32, [ctypes.c_int64, c_void_p]),
    "maxmulsk_check_dgemm_dev": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_size_t, c_size_t,
                                           c_void_p]),
    "maxmulsk_check_errors_work_bytes": (c_size_t, []),
    "maxmulsk_check_errors_dev": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_size_t,
                                            c_size_t, c_void_p, c_size_t, POINTER(ErrorReport), c_void_p]),
    "maxmulsk_stream_status": (c_int32, [c_void_p]),
    "maxmulsk_status_string": (c_char_p, [c_int32]),
    "maxmulsk_last_error_message": (c_char_p, []),
    "maxmulsk_version": (c_char_p, []),
    "maxmulsk_phase_timing": (None, [c_int32]),
    "maxmulsk_phase_report": (c_size_t, [c_char_p, c_size_t]),
}

_lib: ctypes.CDLL | None = None


def load() -> ctypes.CDLL:
    """Loads the CUDA library once; raises ImportError if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m maxmulsk_b200.build` "
            "(nvcc, sm_100a). There is no CPU fallback.")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    """Names every header in include/ declares (parsed from the header text)."""
    import re
    inc = os.path.join(os.path.dirname(HERE), "include")
    names: list[str] = []
    for f in sorted(os.listdir(inc)):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(inc, f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b(maxmulsk_[a-z0-9_]+)\s*\(", text):
            if m.group(1) not in names:
                names.append(m.group(1))
    return names


__all__ = ["Plan", "Problem", "ErrorReport", "load", "exported_symbols", "LIB_PATH", "c_float"]
