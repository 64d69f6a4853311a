"""MaxMulSK-B200: row-major FP32 GEMM C = A*B on NVIDIA B200 (sm_100a).

Python mirror of the C ABI in include/maxmulsk.h (itself the drop-in for the
reference's capi/maxmulsk.h). Same names, same (M, K, N) argument order, same
status codes; C is overwritten and never read.

Host entry points take numpy float32 arrays (C-contiguous); device entry
points take torch CUDA tensors or raw device pointers (int). Every call goes
through libmaxmulsk_b200.so; nothing here computes a product on the CPU.
"""
from __future__ import annotations

import ctypes
import enum
from typing import Any

from . import _lib
from ._lib import ErrorReport, Plan, Problem

__version__ = "0.1.0"


class Status(enum.IntEnum):
    OK = 0
    ERR_UNSUPPORTED = 1
    ERR_ALLOC = 2
    ERR_CUDA = 3
    ERR_INVALID = 4
    ERR_TIMEOUT = 5


class Precision(enum.IntEnum):
    FP32 = 0
    TF32X3 = 1
    BF16X6 = 2
    BF16X9 = 3
    SPLIT_AUTO = 4


FP32_FMA = 0
FP32_SCALAR = 1
TC_SPLIT_INPUTS = 0
TC_REUSE_PLANES = 1
TC_FUSED_SPLIT = 2
PHASE_REPORT_BYTES = 1024   # MAXMULSK_PHASE_REPORT_BYTES


class MaxMulSKError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = Status(status) if status in Status._value2member_map_ else status
        msg = lib().maxmulsk_last_error_message()
        super().__init__(f"{where}: {self.status!s} ({(msg or b'').decode(errors='replace')})")


def lib() -> ctypes.CDLL:
    return _lib.load()


def _host_ptr(x: Any, n: int, name: str, writable: bool = False) -> int | None:
    if x is None:
        return None
    if isinstance(x, int):
        return x
    import numpy as np
    if not isinstance(x, np.ndarray):
        raise TypeError(f"{name} must be a numpy array or an int pointer")
    if x.dtype != np.float32 or not x.flags.c_contiguous:
        raise TypeError(f"{name} must be a C-contiguous float32 array")
    if x.size < n:
        raise ValueError(f"{name} has {x.size} elements, needs {n}")
    if writable and not x.flags.writeable:
        raise ValueError(f"{name} is read-only")
    return x.ctypes.data


def _dev_ptr(x: Any, n: int, name: str) -> int | None:
    if x is None:
        return None
    if isinstance(x, int):
        return x
    try:
        import torch
    except ImportError as e:  # pragma: no cover
        raise TypeError(f"{name}: device entry points take torch tensors or int pointers") from e
    if not isinstance(x, torch.Tensor) or not x.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor or an int pointer")
    if x.dtype != torch.float32 or not x.is_contiguous():
        raise TypeError(f"{name} must be a contiguous float32 CUDA tensor")
    if x.numel() < n:
        raise ValueError(f"{name} has {x.numel()} elements, needs {n}")
    return x.data_ptr()


def _stream_ptr(stream: Any) -> int | None:
    if stream is None:
        try:
            import torch
            if torch.cuda.is_available():
                return torch.cuda.current_stream().cuda_stream
        except ImportError:  # pragma: no cover
            pass
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


# --------------------------------------------------------------------------- host
def sgemm_v3(A, B, C, M: int, K: int, N: int) -> Status:
    """C = A*B on host buffers; the tuned FP32 SIMT plan (capi/maxmulsk.h:32-33)."""
    return Status(lib().maxmulsk_sgemm_v3(_host_ptr(A, M * K, "A"), _host_ptr(B, K * N, "B"),
                                          _host_ptr(C, M * N, "C", True), M, K, N))


def sgemm_v4(A, B, C, M: int, K: int, N: int) -> Status:
    """C = A*B on host buffers; the fixed-rule FP32 SIMT plan (capi/maxmulsk.h:36-37)."""
    return Status(lib().maxmulsk_sgemm_v4(_host_ptr(A, M * K, "A"), _host_ptr(B, K * N, "B"),
                                          _host_ptr(C, M * N, "C", True), M, K, N))


def sgemm_plan(A, B, C, M: int, K: int, N: int, plan: Plan) -> Status:
    return Status(lib().maxmulsk_sgemm_plan(_host_ptr(A, M * K, "A"), _host_ptr(B, K * N, "B"),
                                            _host_ptr(C, M * N, "C", True), M, K, N, ctypes.byref(plan)))


def sgemm_split(A, B, C, M: int, K: int, N: int, precision: int = Precision.TF32X3) -> Status:
    return Status(lib().maxmulsk_sgemm_split(_host_ptr(A, M * K, "A"), _host_ptr(B, K * N, "B"),
                                             _host_ptr(C, M * N, "C", True), M, K, N, int(precision)))


# --------------------------------------------------------------------------- device
def sgemm_v3_dev(dA, dB, dC, M: int, K: int, N: int, stream=None) -> Status:
    return Status(lib().maxmulsk_sgemm_v3_dev(_dev_ptr(dA, M * K, "A"), _dev_ptr(dB, K * N, "B"),
                                              _dev_ptr(dC, M * N, "C"), M, K, N, _stream_ptr(stream)))


def sgemm_v4_dev(dA, dB, dC, M: int, K: int, N: int, stream=None) -> Status:
    return Status(lib().maxmulsk_sgemm_v4_dev(_dev_ptr(dA, M * K, "A"), _dev_ptr(dB, K * N, "B"),
                                              _dev_ptr(dC, M * N, "C"), M, K, N, _stream_ptr(stream)))


def sgemm_plan_dev(dA, dB, dC, M: int, K: int, N: int, plan: Plan, ws=None, ws_bytes: int = 0,
                   stream=None) -> Status:
    wsp = None
    if ws is not None:
        wsp = ws if isinstance(ws, int) else ws.data_ptr()
        if not isinstance(ws, int) and not ws_bytes:
            ws_bytes = ws.numel() * ws.element_size()
    return Status(lib().maxmulsk_sgemm_plan_dev(_dev_ptr(dA, M * K, "A"), _dev_ptr(dB, K * N, "B"),
                                                _dev_ptr(dC, M * N, "C"), M, K, N, ctypes.byref(plan),
                                                wsp, ws_bytes, _stream_ptr(stream)))


def sgemm_split_dev(dA, dB, dC, M: int, K: int, N: int, precision: int = Precision.TF32X3,
                    stream=None) -> Status:
    return Status(lib().maxmulsk_sgemm_split_dev(_dev_ptr(dA, M * K, "A"), _dev_ptr(dB, K * N, "B"),
                                                 _dev_ptr(dC, M * N, "C"), M, K, N, int(precision),
                                                 _stream_ptr(stream)))


# --------------------------------------------------------------------------- plans
def make_plan(precision: int = Precision.FP32, tile_m: int = 128, tile_n: int = 128, split_k: int = 1,
              variant: int = 0, chunk: int = 0) -> Plan:
    p = Plan()
    p.precision, p.tile_m, p.tile_n, p.split_k, p.variant = int(precision), tile_m, tile_n, split_k, variant
    p.chunk = chunk
    return p


def classify(M: int, K: int, N: int, plan: Plan) -> Status:
    return Status(lib().maxmulsk_classify(M, K, N, ctypes.byref(plan)))


def choose(M: int, K: int, N: int, precision: int = Precision.FP32) -> Plan:
    p = Plan()
    st = lib().maxmulsk_choose(M, K, N, int(precision), ctypes.byref(p))
    if st != 0:
        raise MaxMulSKError(st, "maxmulsk_choose")
    return p


def picker_doubt(M: int, K: int, N: int, precision: int = Precision.FP32) -> str | None:
    """Why the GEMM entry points would search exhaustively for this shape
    instead of trusting the learned model (maxmulsk_picker_doubt), or None."""
    r = lib().maxmulsk_picker_doubt(M, K, N, int(precision))
    return r.decode() if r else None


def choose_rule(M: int, K: int, N: int, precision: int = Precision.FP32) -> Plan:
    p = Plan()
    st = lib().maxmulsk_choose_rule(M, K, N, int(precision), ctypes.byref(p))
    if st != 0:
        raise MaxMulSKError(st, "maxmulsk_choose_rule")
    return p


def workspace_bytes(M: int, K: int, N: int, plan: Plan) -> int:
    return int(lib().maxmulsk_workspace_bytes(M, K, N, ctypes.byref(plan)))


def slice_len(K: int, split_k: int) -> int:
    """K slice length of a plan (the kernels' rule, internal.hpp slice_len)."""
    if split_k <= 1 or K == 0:
        return K
    per = (K + split_k - 1) // split_k
    per = (per + 31) // 32 * 32
    return min(per, K)


def slice_count(K: int, split_k: int) -> int:
    """K slices a plan actually runs (the kernels' rule, internal.hpp slice_count)."""
    kc = slice_len(K, split_k)
    return (K + kc - 1) // kc if kc else 1


def stream_status(stream=None) -> Status:
    return Status(lib().maxmulsk_stream_status(_stream_ptr(stream)))


def status_string(s: int) -> str:
    return lib().maxmulsk_status_string(int(s)).decode()


def last_error_message() -> str:
    return (lib().maxmulsk_last_error_message() or b"").decode(errors="replace")


def version() -> str:
    return lib().maxmulsk_version().decode()


def phase_timing(on: bool = True) -> None:
    """Turns phase timing on or off (maxmulsk_phase_timing)."""
    lib().maxmulsk_phase_timing(1 if on else 0)


def phase_report() -> dict:
    """Device time per phase since the last report, {"gemm": {"calls": n, "ms": t}, ...}
    (maxmulsk_phase_report); the recorded phases are then forgotten."""
    import json
    buf = ctypes.create_string_buffer(PHASE_REPORT_BYTES)
    lib().maxmulsk_phase_report(buf, PHASE_REPORT_BYTES)
    return json.loads(buf.value.decode())


# --------------------------------------------------------------------------- FP64 checking
def check_dgemm_dev(dA, dB, dC64, dCabs, M: int, K: int, N: int, stream=None) -> Status:
    """C64 = A*B in FP64 on the device (and |A||B| when dCabs is given):
    maxmulsk_check_dgemm_dev. dC64 / dCabs: float64 CUDA tensors or pointers."""
    def ptr(x):
        return None if x is None else (x if isinstance(x, int) else x.data_ptr())
    return Status(lib().maxmulsk_check_dgemm_dev(_dev_ptr(dA, M * K, "A"), _dev_ptr(dB, K * N, "B"), ptr(dC64),
                                                 ptr(dCabs), M, K, N, _stream_ptr(stream)))


def check_errors_dev(dC, dC64, dCabs, dA, dB, M: int, K: int, N: int, stream=None) -> dict:
    """Error measures of an FP32 result against C64 (maxmulsk_check_errors_dev):
    {"normwise", "max_rel", "rel_frob", "max_abs", "norm_a", ...}."""
    import torch

    def ptr(x):
        return None if x is None else (x if isinstance(x, int) else x.data_ptr())
    nb = int(lib().maxmulsk_check_errors_work_bytes())
    work = torch.empty(nb // 8 + 1, dtype=torch.float64, device="cuda")
    rep = ErrorReport()
    st = lib().maxmulsk_check_errors_dev(_dev_ptr(dC, M * N, "C"), ptr(dC64), ptr(dCabs), _dev_ptr(dA, M * K, "A"),
                                         _dev_ptr(dB, K * N, "B"), M, K, N, work.data_ptr(), nb, ctypes.byref(rep),
                                         _stream_ptr(stream))
    check(st, "maxmulsk_check_errors_dev")
    return rep.as_dict()


class Fp64Check:
    """FP64 truth of one product on the device, computed once, against which
    several FP32 results are measured (the GPU form of the reference's FP64
    checks). dA, dB: float32 CUDA tensors holding A (M x K) and B (K x N)."""

    def __init__(self, dA, dB, M: int, K: int, N: int, with_abs: bool = True, stream=None):
        import torch
        self.dA, self.dB, self.M, self.K, self.N = dA, dB, M, K, N
        self.c64 = torch.empty(M * N, dtype=torch.float64, device="cuda")
        self.cabs = torch.empty(M * N, dtype=torch.float64, device="cuda") if with_abs else None
        check(check_dgemm_dev(dA, dB, self.c64, self.cabs, M, K, N, stream), "maxmulsk_check_dgemm_dev")

    def errors(self, dC, stream=None) -> dict:
        return check_errors_dev(dC, self.c64, self.cabs, self.dA, self.dB, self.M, self.K, self.N, stream)


def check(status: int, where: str = "maxmulsk") -> None:
    if status != 0:
        raise MaxMulSKError(status, where)


class Grouped:
    """A captured grouped launch (maxmulsk_grouped_create). `problems` is a list
    of (dA, dB, dC, M, K, N) with torch CUDA tensors or int device pointers."""

    def __init__(self, problems, plan: Plan | None = None):
        n = len(problems)
        arr = (Problem * max(1, n))()
        self._keep = []
        for i, (a, b, c, M, K, N) in enumerate(problems):
            arr[i].A = _dev_ptr(a, M * K, "A") if M * K else 0
            arr[i].B = _dev_ptr(b, K * N, "B") if K * N else 0
            arr[i].C = _dev_ptr(c, M * N, "C") if M * N else 0
            arr[i].M, arr[i].K, arr[i].N = M, K, N
            self._keep.append((a, b, c))
        self.count = n
        h = ctypes.c_void_p()
        st = lib().maxmulsk_grouped_create(arr, n, ctypes.byref(plan) if plan is not None else None, ctypes.byref(h))
        check(st, "maxmulsk_grouped_create")
        self.handle = h

    def launch(self, stream=None) -> Status:
        return Status(lib().maxmulsk_grouped_launch(self.handle, _stream_ptr(stream)))

    def info(self):
        p = Plan()
        sk = (ctypes.c_int32 * max(1, self.count))()
        units = ctypes.c_size_t()
        check(lib().maxmulsk_grouped_info(self.handle, ctypes.byref(p), sk, ctypes.byref(units)), "grouped_info")
        return p, list(sk)[: self.count], units.value

    def plans(self) -> list:
        """The plan each problem runs (maxmulsk_grouped_plans)."""
        arr = (Plan * max(1, self.count))()
        check(lib().maxmulsk_grouped_plans(self.handle, arr), "grouped_plans")
        return [arr[i] for i in range(self.count)]

    def close(self):
        if getattr(self, "handle", None):
            lib().maxmulsk_grouped_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def matmul(a, b, precision: int = Precision.FP32, plan: Plan | None = None, stream=None):
    """torch convenience: returns a new CUDA tensor C = a @ b (float32, row-major)."""
    import torch
    M, K = a.shape
    K2, N = b.shape
    if K != K2:
        raise ValueError("inner dimensions differ")
    c = torch.empty((M, N), device=a.device, dtype=torch.float32)
    if plan is not None:
        st = sgemm_plan_dev(a, b, c, M, K, N, plan, stream=stream) if workspace_bytes(M, K, N, plan) == 0 \
            else _plan_with_ws(a, b, c, M, K, N, plan, stream)
    elif int(precision) == Precision.FP32:
        st = sgemm_v3_dev(a, b, c, M, K, N, stream)
    else:
        st = sgemm_split_dev(a, b, c, M, K, N, precision, stream)
    check(st, "matmul")
    return c


def _plan_with_ws(a, b, c, M, K, N, plan, stream):
    """sgemm_plan_dev with a fresh workspace on the current CUDA device."""
    import torch
    nb = workspace_bytes(M, K, N, plan)
    if nb == 0:
        return sgemm_plan_dev(a, b, c, M, K, N, plan, None, 0, stream)
    dev = a.device if hasattr(a, "device") else torch.device("cuda", torch.cuda.current_device())
    ws = torch.empty(nb + 256, dtype=torch.uint8, device=dev)
    off = (-ws.data_ptr()) % 256
    st = sgemm_plan_dev(a, b, c, M, K, N, plan, ws.data_ptr() + off, nb, stream)
    if st == 0 and stream is not None:
        # Once `ws` is dropped the caching allocator may hand its block to
        # work on the current stream; order that after this call's kernels.
        ws.record_stream(torch.cuda.ExternalStream(stream) if isinstance(stream, int) else stream)
    return st


__all__ = [
    "Status", "Precision", "Plan", "Problem", "FP32_FMA", "FP32_SCALAR", "TC_SPLIT_INPUTS", "TC_REUSE_PLANES", "TC_FUSED_SPLIT",
    "MaxMulSKError",
    "sgemm_v3", "sgemm_v4", "sgemm_plan", "sgemm_split",
    "sgemm_v3_dev", "sgemm_v4_dev", "sgemm_plan_dev", "sgemm_split_dev",
    "make_plan", "classify", "choose", "picker_doubt", "choose_rule", "workspace_bytes", "slice_len", "slice_count",
    "stream_status", "status_string", "last_error_message", "version", "check", "matmul", "lib", "Grouped",
    "ErrorReport", "check_dgemm_dev", "check_errors_dev", "Fp64Check",
]
