"""Autotuner driver: times every candidate plan of a set of shapes on the
device and writes the timings (the picker's training data) and a tuning
database of the best plan per shape.

    python -m maxmulsk_b200.autotune --train 2000 --test 500 --out timings.npz --db tuning_db.txt

Shapes: M, N, K each log-uniform in [1, 16384] (fixed seeds). Per shape and
class (0 FP32, 1 split precision) every candidate of maxmulsk_candidates() is
timed by maxmulsk_autotune_time_dev (a CUDA graph of repeated calls, median of
three replays). The rule picker's plan (maxmulsk_choose_rule) is timed beside
them, so the learned picker can be compared with the method it replaces.
"""
from __future__ import annotations

import argparse
import ctypes
import math
import os
import sys
import time

import numpy as np

from . import Plan, Precision, choose_rule, lib, workloads

WS_LIMIT = 24 << 30          # candidates needing more workspace are skipped (timed as +inf)


def candidates(cls: int) -> list[Plan]:
    n = lib().maxmulsk_candidates(cls, None, 0)
    arr = (Plan * n)()
    lib().maxmulsk_candidates(cls, arr, n)
    return [arr[i] for i in range(n)]


def time_plans(dA, dB, dC, M, K, N, plans, ws_ptr, ws_bytes, stream=None) -> np.ndarray:
    arr = (Plan * len(plans))(*plans)
    out = (ctypes.c_float * len(plans))()
    st = lib().maxmulsk_autotune_time_dev(dA, dB, dC, M, K, N, arr, len(plans), ws_ptr, ws_bytes, 0, out, stream)
    if st != 0:
        raise RuntimeError(f"autotune failed with status {st} for {(M, K, N)}")
    return np.array(out, dtype=np.float32)


def collect(shapes, log=print) -> dict:
    import torch
    mx = max(max(m * k, k * n, m * n) for m, k, n in shapes)
    big = torch.empty(mx, dtype=torch.float32, device="cuda")
    dA = torch.empty(mx, dtype=torch.float32, device="cuda").uniform_(-1, 1)
    dB = torch.empty(mx, dtype=torch.float32, device="cuda").uniform_(-1, 1)
    free = torch.cuda.mem_get_info()[0]
    ws_bytes = int(min(WS_LIMIT, free * 0.8)) // 256 * 256
    ws = torch.empty(ws_bytes + 256, dtype=torch.uint8, device="cuda")
    wp = ws.data_ptr() + ((-ws.data_ptr()) % 256)
    c0, c1 = candidates(0), candidates(1)
    t0 = np.full((len(shapes), len(c0)), np.inf, np.float32)
    t1 = np.full((len(shapes), len(c1)), np.inf, np.float32)
    r0 = np.full(len(shapes), np.inf, np.float32)
    r1 = np.full(len(shapes), np.inf, np.float32)
    start = time.time()
    for i, (M, K, N) in enumerate(shapes):
        a, b, c = dA.data_ptr(), dB.data_ptr(), big.data_ptr()
        t0[i] = time_plans(a, b, c, M, K, N, c0, wp, ws_bytes)
        t1[i] = time_plans(a, b, c, M, K, N, c1, wp, ws_bytes)
        r0[i] = time_plans(a, b, c, M, K, N, [choose_rule(M, K, N, Precision.FP32)], wp, ws_bytes)[0]
        r1[i] = time_plans(a, b, c, M, K, N, [choose_rule(M, K, N, Precision.SPLIT_AUTO)], wp, ws_bytes)[0]
        if (i + 1) % 100 == 0:
            log(f"  {i + 1}/{len(shapes)} shapes, {time.time() - start:.0f} s")
    return {"shapes": np.array(shapes, np.int64), "t_fp32": t0, "t_split": t1, "t_rule_fp32": r0,
            "t_rule_split": r1,
            "cand_fp32": np.array([p.as_tuple() for p in c0], np.int32),
            "cand_split": np.array([p.as_tuple() for p in c1], np.int32)}


def write_db(path: str, d: dict) -> int:
    """Best measured plan per (shape, class) in the tuning-database format of
    tuning.cpp: M K N requested precision tile_m tile_n split_k variant time_us."""
    n = 0
    with open(path, "w") as f:
        f.write("# maxmulsk tuning database: M K N requested precision tile_m tile_n split_k variant time_us\n")
        for (M, K, N), t0, t1 in zip(d["shapes"], d["t_fp32"], d["t_split"]):
            for req, t, cands in ((int(Precision.FP32), t0, d["cand_fp32"]),
                                  (int(Precision.SPLIT_AUTO), t1, d["cand_split"])):
                if not np.isfinite(t).any():
                    continue
                j = int(np.argmin(t))
                prec, tm, tn, sk, var = (int(x) for x in cands[j])
                f.write(f"{M} {K} {N} {req} {prec} {tm} {tn} {sk} {var} {float(t[j]):.3f}\n")
                n += 1
    return n


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--test", type=int, default=500)
    ap.add_argument("--out", required=True)
    ap.add_argument("--db", default=None)
    a = ap.parse_args()
    shapes = workloads.picker_shapes(a.train, seed=5001) + workloads.picker_shapes(a.test, seed=5002)
    d = collect(shapes)
    d["n_train"] = np.array(a.train)
    np.savez_compressed(a.out, **d)
    print("wrote", a.out)
    if a.db:
        print("db entries written:", write_db(a.db, d))


if __name__ == "__main__":
    main()
