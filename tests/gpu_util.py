"""Helpers for the GPU tests: device buffers (torch, plumbing only), calls
through the C ABI, and result read-back."""
from __future__ import annotations

import numpy as np

import maxmulsk_b200 as mm

SENTINEL = 3.75   # the reference checker's never-written marker (check_nb.cpp:54)


def to_dev(torch, x: np.ndarray):
    return torch.from_numpy(np.ascontiguousarray(x).ravel()).cuda()


def run_plan(torch, A: np.ndarray, B: np.ndarray, M: int, K: int, N: int, plan, guard: int = 64,
             dA=None, dB=None, offset: int = 0):
    """C = A*B through maxmulsk_sgemm_plan_dev with a caller workspace.
    C sits between guard bands prefilled with the sentinel; returns
    (status, C, guard bands intact)."""
    if dA is None:
        dA = to_dev(torch, A)
    if dB is None:
        dB = to_dev(torch, B)
    buf = torch.full((M * N + 2 * guard + offset,), SENTINEL, dtype=torch.float32, device="cuda")
    c_ptr = buf.data_ptr() + 4 * (guard + offset)
    nb = mm.workspace_bytes(M, K, N, plan)
    ws = torch.empty(nb + 512, dtype=torch.uint8, device="cuda")
    ws_ptr = ws.data_ptr() + ((-ws.data_ptr()) % 256)
    st = mm.sgemm_plan_dev(dA.data_ptr(), dB.data_ptr(), c_ptr, M, K, N, plan, ws_ptr, nb, None)
    st2 = mm.stream_status(None)
    host = buf.cpu().numpy()
    C = host[guard + offset: guard + offset + M * N].reshape(M, N).copy()
    bands_ok = bool(np.all(host[:guard + offset] == SENTINEL) and np.all(host[guard + offset + M * N:] == SENTINEL))
    return (st if st != 0 else st2), C, bands_ok


def bits(x: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
