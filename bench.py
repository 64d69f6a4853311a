"""Benchmark: split-precision tensor-core FP32 GEMM vs the FP32 SIMT kernel.

One step = one C = A*B of the workload through the library (split pre-pass +
tcgen05 GEMM for the headline), inputs resident in HBM. Default workload: the
square 4096^3 FP32 GEMM of the square sweep (uniform [-1, 1) inputs, fixed
seed), the shape the speed target is stated on.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--size S] [--precision auto|fp32|tf32x3|bf16x6|bf16x9]

Multi-GPU (one rank per GPU): under torchrun, or `--gpus N` alone, which
starts the N ranks itself through torch.distributed.run. Every rank
multiplies its own M-row shard (a 4096 x 4096 block of A and the whole B); no
collective touches the data path. Timing is on the device (CUDA events), max
over ranks; a line is printed only when the ranks started match --gpus.

The reference arm (--impl reference) times the reference's own CPU GEMM,
Utils::multiply_scalar (common/utils.hpp:50-61) compiled into oracle/_ref, on
the host's cores over a bounded sample of rows of the same product.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GFLOP/s & %roofline: split-precision TC vs FP32 SIMT GEMM at stated FP64 error"
PREC = {"tf32x3": 1, "bf16x6": 2, "bf16x9": 3}
PRODUCTS = {1: 3, 2: 6, 3: 9}


def env_int(name: str, default: int) -> int:
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def measured_peaks() -> tuple[dict, str]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "sm_max_mhz": 1965.0}, \
        "fallback"


def traffic_from_profiles(name: str) -> float | None:
    """DRAM bytes per launch of the dominant kernel, from a committed ncu summary."""
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for line in f:
            if line.startswith("dram_bytes_per_launch:"):
                try:
                    return float(line.split(":", 1)[1].split()[0])
                except ValueError:
                    return None
    return None


def resolved_split(plan, M: int, N: int) -> int:
    """The K split a plan runs: its split_k, or for split_k 0 (tensor-core
    plans) as many slices per tile as the device has work slots per tile
    (SMs, or CTA pairs for 256-row tiles), 1..64."""
    if plan.split_k:
        return plan.split_k
    import torch
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    slots = sms // 2 if plan.tile_m == 256 else sms
    tiles = -(-M // plan.tile_m) * -(-N // plan.tile_n)
    return max(1, min(64, slots // tiles))


def launches_per_step(plan, M: int, K: int, N: int) -> int:
    """Kernels of this library one call of `plan` launches: the split pre-pass
    (one per operand) and the tensor-core GEMM, the fused-split GEMM, or the
    SIMT GEMM; plus the split-K reduction when every tile is cut into 3 or
    more K slices."""
    import maxmulsk_b200 as mm
    n = 1 if plan.precision == 0 or plan.variant == mm.TC_FUSED_SPLIT else 3
    if mm.slice_count(K, resolved_split(plan, M, N)) >= 3:
        n += 1
    return n


# ----------------------------------------------------------------------------- ranks
def launch_ranks(n: int) -> int:
    """Runs this script again as n ranks, one process per GPU, under
    torch.distributed.run on 127.0.0.1 (the form `bench.py --gpus n` takes
    when no launcher set WORLD_SIZE); returns their exit status. NCCL's log
    stays on (NCCL_DEBUG=INFO unless set), so the communicator's ranks show."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    env = dict(os.environ)
    env.setdefault("NCCL_DEBUG", "INFO")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.run(cmd, env=env).returncode


class Ranks:
    """One rank per GPU (RANK / WORLD_SIZE / LOCAL_RANK from the launcher):
    barriers and the max over ranks of a per-rank time. Nothing on the data
    path is exchanged: each rank multiplies its own shard."""

    def __init__(self, backend: str = "nccl", device=None):
        self.rank = env_int("RANK", 0)
        self.world = env_int("WORLD_SIZE", 1)
        self.local = env_int("LOCAL_RANK", 0)
        self.backend = backend
        self.device = device
        if self.world > 1:
            from datetime import timedelta

            import torch.distributed as dist
            kw = {"device_id": device} if backend == "nccl" else {}
            dist.init_process_group(backend, timeout=timedelta(seconds=120), **kw)

    def barrier(self) -> None:
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max(self, x: float) -> float:
        from maxmulsk_b200 import shard
        return shard.max_over_ranks(x, self.device if self.backend == "nccl" else None)

    def timed(self, fn, steps: int, start, stop) -> float:
        """Seconds per step of fn, the max over ranks: barrier, t0 = start(),
        `steps` calls, stop(t0) -> seconds, barrier."""
        self.barrier()
        t0 = start()
        for _ in range(steps):
            fn()
        secs = stop(t0)
        self.barrier()
        return self.max(secs / steps)

    def close(self) -> None:
        if self.world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


def check_world(gpus: int, world: int) -> None:
    """A line's n_gpus must be what --gpus asked for."""
    if world != gpus:
        print(f"bench.py: --gpus {gpus} but the launcher started {world} rank(s); no line printed",
              file=sys.stderr)
        sys.exit(2)


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.marks: list[tuple[float, float]] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu=timestamp,{self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", self.gpu_id], stdout=self.out, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        try:
            with open(self.out.name) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) < 10:
                        continue
                    try:
                        rows.append({"sm": float(parts[2]), "max": float(parts[3]), "power": float(parts[4]),
                                     "active": parts[5], "hw": parts[6], "hwt": parts[7], "swt": parts[8],
                                     "pcap": parts[9]})
                    except ValueError:
                        continue
        finally:
            os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        loaded = [r for r in rows if r["power"] > 300.0] or rows
        reasons = set()
        for r in loaded:
            if r["hw"].lower() == "active":
                reasons.add("hw_slowdown")
            if r["hwt"].lower() == "active":
                reasons.add("hw_thermal_slowdown")
            if r["swt"].lower() == "active":
                reasons.add("sw_thermal_slowdown")
            if r["pcap"].lower() == "active":
                reasons.add("sw_power_cap")
        return {"sm_mhz": statistics.median(r["sm"] for r in loaded), "sm_max_mhz": max(r["max"] for r in rows),
                "reasons": sorted(reasons), "samples": len(loaded),
                "power_w_max": max(r["power"] for r in loaded)}


# ----------------------------------------------------------------------------- CPU baseline
def cpu_rows_gflops(A, B, K: int, N: int, budget_s: float, threads: int, start_row: int = 0) -> dict:
    """The reference's multiply_scalar (oracle/_ref, else the oracle's
    restatement) on whole rows of the product, `threads` host threads, for
    about budget_s seconds. Returns GFLOP/s and what was sampled."""
    import numpy as np
    import oracle
    if oracle.ref_available():
        fn = oracle.ref().ref_multiply_scalar
        kind = "reference"
    else:
        fn = oracle.lib().oracle_sgemm_scalar
        kind = "port"
    fp = ctypes.POINTER(ctypes.c_float)
    Bp = B.ctypes.data_as(fp)
    M = A.shape[0]
    done_rows = [0] * threads
    stop = time.perf_counter() + budget_s
    out = np.empty((threads, N), np.float32)

    def worker(t: int):
        r = start_row + t
        while time.perf_counter() < stop:
            row = r % M
            fn(A[row].ctypes.data_as(fp), Bp, out[t].ctypes.data_as(fp), 1, N, K)
            done_rows[t] += 1
            r += threads

    t0 = time.perf_counter()
    ths = [threading.Thread(target=worker, args=(t,)) for t in range(threads)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    dt = time.perf_counter() - t0
    rows = sum(done_rows)
    return {"value": 2.0 * rows * K * N / dt / 1e9, "unit": "GFLOP/s", "cores": threads, "kind": kind,
            "sample": f"{rows} rows of the {M}x{K}x{N} product (1 x {K} x {N} each) in {dt:.1f} s",
            "seconds": dt}


def run_reference(args) -> None:
    rank = env_int("RANK", 0)
    world = env_int("WORLD_SIZE", 1)
    if rank != 0:
        return
    import numpy as np
    import oracle
    from maxmulsk_b200 import datagen
    S = args.size
    A = datagen.uniform(S * S, 11).reshape(S, S)
    B = datagen.uniform(S * S, 12).reshape(S, S)
    threads = os.cpu_count() or 1
    oracle.lib()
    # Each step: a bounded sample of rows, one row per host thread per step
    # at least, sized so the whole run stays within a few minutes.
    budget = max(0.05, min(2.0, 150.0 / max(1, args.steps + args.warmup)))
    for w in range(args.warmup):
        cpu_rows_gflops(A, B, S, S, budget, threads, start_row=w * threads)
    vals, rows_total, secs = [], 0, 0.0
    for s in range(args.steps):
        r = cpu_rows_gflops(A, B, S, S, budget, threads, start_row=(args.warmup + s) * threads)
        vals.append(r["value"])
        secs += r["seconds"]
        rows_total += int(r["sample"].split()[0])
    value = 2.0 * rows_total * S * S / secs / 1e9
    kind = "reference" if oracle.ref_available() else "port"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / max(1, args.steps),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded uniform [-1, 1))",
        "config": {"workload": f"square {S}^3 FP32 GEMM, reference CPU path (Utils::multiply_scalar) on "
                               f"row samples", "M": S, "K": S, "N": S},
        "cpu_baseline": {"value": value, "unit": "GFLOP/s", "cores": threads, "kind": kind,
                         "sample": f"{rows_total} rows of the {S}^3 product over {args.steps} steps, "
                                   f"{threads} threads"},
        "e2e": {"value": value, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- tables
def graph_time(torch, fn, reps: int) -> float:
    """Seconds per call of fn, measured by replaying a CUDA graph of `reps`
    calls (no host launch overhead in the measurement)."""
    fn()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        fn()                                          # warm on the capture stream
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    with torch.cuda.graph(g):
        for _ in range(reps):
            fn()
    g.replay()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(3):
        g.replay()
    e1.record()
    torch.cuda.synchronize()
    del g
    return e0.elapsed_time(e1) / 1e3 / (3 * reps)


def run_tables(args) -> None:
    """Per-cell measurements of the other benchmark configurations (one JSON
    line per cell): the square sweep with uniform and wide inputs, the narrow-M
    shapes, the grouped batch."""
    import numpy as np
    import torch

    import maxmulsk_b200 as mm
    from maxmulsk_b200 import datagen, workloads

    torch.cuda.set_device(env_int("LOCAL_RANK", 0))
    peaks, peak_src = measured_peaks()
    fp32_peak = 148 * 128 * 2 * peaks.get("sm_max_mhz", 1965.0) * 1e6 / 1e12
    kernels = [("simt", 0), ("tf32x3", 1), ("bf16x6", 2), ("bf16x9", 3)]

    def run_plan(dA, dB, dC, M, K, N, plan):
        nb = mm.workspace_bytes(M, K, N, plan)
        ws = torch.empty(nb + 256, dtype=torch.uint8, device="cuda")
        wp = ws.data_ptr() + ((-ws.data_ptr()) % 256)

        def fn():
            mm.check(mm.sgemm_plan_dev(dA, dB, dC, M, K, N, plan, wp, nb), "plan")
        return fn, ws

    def errors(chk, dC):
        e = chk.errors(dC)
        return e["normwise"], e["max_rel"]

    def emit(d):
        print(json.dumps(d), flush=True)

    if args.workload in ("sweep", "narrow"):
        if args.workload == "sweep":
            cells = [(S, S, S, dist) for S in workloads.SQUARE for dist in ("uniform", "wide")]
        else:
            cells = [(M, K, N, "normal") for (M, K, N) in workloads.NARROW_M]
        for (M, K, N, dist) in cells:
            if dist == "normal":
                A = datagen.normal(M * K, 31, 1.0 / np.sqrt(K)); B = datagen.normal(K * N, 32, 1.0 / np.sqrt(K))
            elif dist == "wide":
                A = datagen.wide(M * K, 31); B = datagen.wide(K * N, 32)
            else:
                A = datagen.uniform(M * K, 31); B = datagen.uniform(K * N, 32)
            dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
            chk = mm.Fp64Check(dA, dB, M, K, N)         # the library's FP64 check product
            flops = 2.0 * M * N * K
            bytes_min = 4.0 * (M * K + K * N + M * N)
            # The plain FP32 kernel: one FMA chain per output (split_k = 1; the
            # tile does not change the bits), the error bar of the split modes.
            # The picker's SIMT plan may cut K into slices, which is faster
            # and also shortens the chains, so its error moves with the plan.
            dCp = torch.empty(M * N, device="cuda")
            fn_p, ws_p = run_plan(dA, dB, dCp, M, K, N, mm.make_plan(0, 128, 128, 1))
            fn_p()
            plain_err, _ = errors(chk, dCp)
            del ws_p, dCp
            simt_err = None
            for name, pc in kernels:
                dC = torch.empty(M * N, device="cuda")
                plan = mm.choose(M, K, N, pc)
                fn, ws = run_plan(dA, dB, dC, M, K, N, plan)
                reps = int(max(3, min(200, 2e10 / flops)))
                t = graph_time(torch, fn, reps)
                nw, mr = errors(chk, dC)
                if pc == 0:
                    simt_err = nw
                peak = fp32_peak if pc == 0 else peaks["bf16_tflops"] / (2.0 if pc == 1 else 1.0) / PRODUCTS[pc]
                emit({"workload": args.workload, "M": M, "K": K, "N": N, "dist": dist, "kernel": name,
                      "plan": list(plan.as_tuple()), "ms": t * 1e3, "gflops": flops / t / 1e9,
                      "frac_compute_roofline": flops / t / 1e12 / peak,
                      "hbm_gbs_at_min_bytes": bytes_min / t / 1e9,
                      "frac_hbm_roofline": bytes_min / t / 1e9 / peaks["hbm_gbs"],
                      "normwise": nw, "max_rel": mr, "normwise_over_simt": nw / simt_err,
                      "normwise_over_plain_fp32": nw / plain_err,
                      "peak_basis": ("FP32 FMA nominal at max clock" if pc == 0 else
                                     f"{peak_src} bf16 {peaks['bf16_tflops']} TF/s / {PRODUCTS[pc]}"
                                     + (" / 2 (TF32)" if pc == 1 else ""))})
                del ws, dC
        return

    # grouped batch: one persistent launch from a CUDA graph vs one launch per GEMM
    shapes = workloads.grouped_problems()[: max(1, args.problems)]
    probs, keep = [], []
    for i, (M, K, N) in enumerate(shapes):
        a = torch.from_numpy(datagen.uniform(M * K, 1000 + 2 * i)).cuda()
        b = torch.from_numpy(datagen.uniform(K * N, 1001 + 2 * i)).cuda()
        c = torch.empty(M * N, device="cuda")
        probs.append((a, b, c, M, K, N))
    flops = sum(2.0 * M * K * N for M, K, N in shapes)
    g = mm.Grouped(probs)
    gp, splits, units = g.info()
    for _ in range(3):
        g.launch()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    reps = 20
    e0.record()
    for _ in range(reps):
        g.launch()
    e1.record()
    torch.cuda.synchronize()
    t_group = e0.elapsed_time(e1) / 1e3 / reps
    # one launch per GEMM, same tile shape and K split per problem, replayed from a graph
    fns = []
    for (a, b, c, M, K, N), s in zip(probs, splits):
        plan = mm.make_plan(0, gp.tile_m, gp.tile_n, max(1, s))
        fn, ws = run_plan(a, b, c, M, K, N, plan)
        fns.append(fn)
        keep.append(ws)
    t_seq = graph_time(torch, lambda: [f() for f in fns], 1)
    emit({"workload": "grouped", "precision": "fp32", "problems": len(shapes), "gflop": flops / 1e9, "units": units,
          "plan": {"tile_m": gp.tile_m, "tile_n": gp.tile_n, "split_k_max": max(splits)},
          "grouped_ms": t_group * 1e3, "grouped_gflops": flops / t_group / 1e9,
          "per_gemm_launches_ms": t_seq * 1e3, "per_gemm_launches_gflops": flops / t_seq / 1e9,
          "frac_fp32_roofline": flops / t_group / 1e12 / fp32_peak})
    g.close()
    # split precision: the fused-split tcgen05 kernel over the group (A with K
    # not a multiple of 4 is repacked in the graph; N not a multiple of 4
    # would run in the FP32 part of the same graph)
    for name, pc in (("bf16x6", 2), ("bf16x9", 3), ("split_auto", 4)):
        gt = mm.Grouped(probs, mm.make_plan(pc, 128, 128, 0))
        tp, tsplits, tunits = gt.info()
        tplans = gt.plans()
        singles = [i for i, p in enumerate(tplans) if p.precision != 0 and p.variant != mm.TC_FUSED_SPLIT]
        for _ in range(3):
            gt.launch()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            gt.launch()
        e1.record()
        torch.cuda.synchronize()
        t_tc = e0.elapsed_time(e1) / 1e3 / reps
        nw = []
        for i in np.random.default_rng(0).choice(len(shapes), 16, replace=False):
            a, b, c, M, K, N = probs[i]
            nw.append(mm.Fp64Check(a, b, M, K, N, with_abs=False).errors(c)["normwise"])
        # the same problems as one launch each (the picker's plan of each
        # problem for this precision), replayed from one CUDA graph
        pfns, pkeep = [], []
        for (a, b, c, M, K, N) in probs:
            fn, ws = run_plan(a, b, c, M, K, N, mm.choose(M, K, N, pc))
            pfns.append(fn)
            pkeep.append(ws)
        t_per = graph_time(torch, lambda: [f() for f in pfns], 1)
        del pkeep
        peak_b = peaks["bf16_tflops"] / PRODUCTS[3 if pc == 3 else 2]
        emit({"workload": "grouped", "precision": name, "problems": len(shapes), "gflop": flops / 1e9,
              "units": tunits, "fp32_fallback_problems": sum(1 for M, K, N in shapes if N % 4),
              "a_repacked_problems": sum(1 for M, K, N in shapes if K % 4 and not N % 4),
              "plan": {"fused_tile": "128x128", "split_k_max": max(tsplits),
                       "own_launch_problems": len(singles),
                       "own_launch_gflop": sum(2.0 * shapes[i][0] * shapes[i][1] * shapes[i][2] for i in singles) / 1e9,
                       "search": "group configurations timed at creation"},
              "grouped_ms": t_tc * 1e3, "grouped_gflops": flops / t_tc / 1e9,
              "frac_split_roofline": flops / t_tc / 1e12 / peak_b,
              "per_gemm_launches_ms": t_per * 1e3, "per_gemm_launches_gflops": flops / t_per / 1e9,
              "normwise_max_of_16_sampled": max(nw)})
        gt.close()


# ----------------------------------------------------------------------------- ours
def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--size", type=int, default=4096)
    ap.add_argument("--precision", choices=["auto", "fp32"] + list(PREC), default="auto",
                    help="split mode; auto = the fastest mode on this device, picked during warm-up; "
                         "fp32 = the SIMT kernel as the timed step (profiling runs: no extras)")
    ap.add_argument("--no-extras", action="store_true",
                    help="headline timing only, with the picker's plans (for profiling runs)")
    ap.add_argument("--shape", default=None, help="M,K,N instead of the square workload (profiling runs; "
                                                   "implies --no-extras)")
    ap.add_argument("--plan", default=None, help="precision,tile_m,tile_n,split_k instead of the picker's plan "
                                                  "(profiling runs)")
    ap.add_argument("--problems", type=int, default=256,
                    help="grouped workload: the first N problems of the 256-GEMM batch (profiling runs)")
    ap.add_argument("--workload", choices=["square4096", "sweep", "narrow", "grouped"], default="square4096",
                    help="square4096 (default, one JSON line) or a per-cell table of the other configurations")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        sys.exit(launch_ranks(args.gpus))
    check_world(args.gpus, env_int("WORLD_SIZE", 1))

    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload != "square4096":
        run_tables(args)
        return

    import numpy as np
    import torch

    import maxmulsk_b200 as mm
    from maxmulsk_b200 import datagen

    local = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ranks = Ranks("nccl", dev)
    rank, world = ranks.rank, ranks.world

    S = args.size
    M = K = N = S
    if args.shape:
        M, K, N = (int(x) for x in args.shape.split(","))
        args.no_extras = True
    fixed_plan = None
    if args.plan:
        fixed_plan = mm.make_plan(*(int(x) for x in args.plan.split(",")))
        args.precision = {0: "fp32", 1: "tf32x3", 2: "bf16x6", 3: "bf16x9"}[fixed_plan.precision]
    # This rank's M-row shard of an (world*S) x S x S product: its own rows of A.
    A = datagen.uniform(M * K, 11 + 1000 * rank).reshape(M, K)
    B = datagen.uniform(K * N, 12).reshape(K, N)
    dA = torch.from_numpy(A).to(dev)
    dB = torch.from_numpy(B).to(dev)
    dC = torch.empty((M, N), dtype=torch.float32, device=dev)
    dCs = torch.empty((M, N), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    barrier = ranks.barrier
    max_over_ranks = ranks.max

    def timed(fn, steps: int) -> float:
        """Seconds per step: CUDA events on the launching stream, synchronize
        on both sides, barriers around, the max over ranks."""
        def start():
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            return e0, e1

        def stop(ev):
            ev[1].record(stream)
            torch.cuda.synchronize(dev)
            return ev[0].elapsed_time(ev[1]) / 1e3
        return ranks.timed(fn, steps, start, stop)

    def mode_step(pc: int, out):
        mp = mm.choose(M, K, N, pc)
        mb = mm.workspace_bytes(M, K, N, mp)
        mws = torch.empty(mb + 256, dtype=torch.uint8, device=dev)
        mwp = mws.data_ptr() + ((-mws.data_ptr()) % 256)

        def step():
            mm.check(mm.sgemm_plan_dev(dA, dB, out, M, K, N, mp, mwp, mb, stream), "mode step")
        return step, mp, mws

    # Plans: each kernel at its best plan for this shape, found by exhaustive
    # search over the autotuner's candidates (maxmulsk_autotune_dev, untimed
    # warm-up). The results go into the library's in-process tuning database,
    # so maxmulsk_choose -- and the end-to-end call below -- return them.
    tuned = {}
    if fixed_plan is None and not args.no_extras:     # profiling runs keep the picker's plans
        tws_bytes = 2 << 30
        tws = torch.empty(tws_bytes + 256, dtype=torch.uint8, device=dev)
        twp = tws.data_ptr() + ((-tws.data_ptr()) % 256)
        for pc in (0, 1, 2):
            best, us = mm.Plan(), ctypes.c_float()
            mm.check(mm.lib().maxmulsk_autotune_dev(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), M, K, N, pc, twp,
                                                    tws_bytes, ctypes.byref(best), ctypes.byref(us),
                                                    stream.cuda_stream), "autotune")
            tuned[pc] = (best.as_tuple(), float(us.value))
        del tws
        torch.cuda.synchronize(dev)

    # Split mode: the one given, or the fastest on this device (picked during
    # warm-up, untimed; every mode meets the accuracy bar at this shape).
    if args.precision == "auto":
        # The modes are within a few per cent of each other at this shape:
        # five interleaved rounds of 100 steps over all of them, each mode's
        # best round decides.
        steps = {name: mode_step(pc, dC) for name, pc in PREC.items()}
        for fn, _, _ in steps.values():
            for _ in range(3):
                fn()
        best_t = {name: float("inf") for name in steps}
        for _ in range(5):
            for name, (fn, _, _) in steps.items():
                best_t[name] = min(best_t[name], timed(fn, 100))
        args.precision = min(best_t, key=best_t.get)
        del steps
    prec = 0 if args.precision == "fp32" else PREC[args.precision]
    if prec == 0:
        args.no_extras = True

    plan = fixed_plan if fixed_plan is not None else mm.choose(M, K, N, prec)
    ws_bytes = mm.workspace_bytes(M, K, N, plan)
    ws = torch.empty(ws_bytes + 256, dtype=torch.uint8, device=dev)
    wsp = ws.data_ptr() + ((-ws.data_ptr()) % 256)
    reuse = mm.make_plan(plan.precision, plan.tile_m, plan.tile_n, plan.split_k, mm.TC_REUSE_PLANES)

    def step_tc():
        mm.check(mm.sgemm_plan_dev(dA, dB, dC, M, K, N, plan, wsp, ws_bytes, stream), "tc step")

    def step_gemm_only():
        mm.check(mm.sgemm_plan_dev(dA, dB, dC, M, K, N, reuse, wsp, ws_bytes, stream), "tc gemm")

    splan = mm.choose(M, K, N, mm.Precision.FP32)
    sws_bytes = mm.workspace_bytes(M, K, N, splan)
    sws = torch.empty(sws_bytes + 256, dtype=torch.uint8, device=dev)
    swsp = sws.data_ptr() + ((-sws.data_ptr()) % 256)

    def step_simt():
        mm.check(mm.sgemm_plan_dev(dA, dB, dCs, M, K, N, splan, swsp, sws_bytes, stream), "simt step")

    gpu_uuid = str(local)
    try:
        gpu_uuid = str(torch.cuda.get_device_properties(dev).uuid)
        if not gpu_uuid.startswith("GPU-"):
            gpu_uuid = "GPU-" + gpu_uuid
    except Exception:
        pass

    # ---- headline: split pre-pass + tcgen05 GEMM, K timed steps
    for _ in range(args.warmup):
        step_tc()
    mm.check(mm.stream_status(stream), "warm-up status")
    sampler = ClockSampler(gpu_uuid)
    sampler.start()
    time.sleep(0.3)
    t_step = timed(step_tc, args.steps)
    sampler.stop()
    mm.check(mm.stream_status(stream), "timed status")
    clocks = sampler.summary()
    flops = 2.0 * M * N * K
    value = flops * world / t_step / 1e9

    out = {
        "metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded uniform [-1, 1), SplitMix64)",
        "config": {"workload": (f"{M}x{K}x{N}" if args.shape else f"square {S}^3") + " FP32 GEMM, " + (
                       "FP32 SIMT kernel" if prec == 0 else
                       f"{args.precision} split tensor-core kernel (split pre-pass + tcgen05 GEMM)") +
                       "; per-rank M-row shard",
                   "M": M, "K": K, "N": N, "precision": args.precision,
                   "plan": {"tile_m": plan.tile_m, "tile_n": plan.tile_n, "split_k": plan.split_k,
                            "variant": plan.variant},
                   "plan_search": "exhaustive over the autotuner's candidates at this shape (warm-up, untimed)"
                                  if tuned else "given",
                   "l2": f"A+B+C = {4 * (M * K + K * N + M * N) / 2**20:.0f} MiB, workspace "
                         f"{ws_bytes / 2**20:.0f} MiB (L2 126 MB)", "parallelism": f"replicas x{world} (M-row shards)"},
        "clocks": clocks,
        "gpu_launches": launches_per_step(plan, M, K, N) * args.steps,
    }

    if not args.no_extras:
        peaks, peak_src = measured_peaks()
        # ---- the GEMM kernel alone (planes already split), for the roofline
        n_k = max(20, min(args.steps, 200))
        for _ in range(3):
            step_gemm_only()
        t_gemm = timed(step_gemm_only, n_k)
        tf32_peak = peaks["bf16_tflops"] / 2.0         # TF32 dense = half the BF16 rate
        mode_peak = (tf32_peak if prec == 1 else peaks["bf16_tflops"]) / PRODUCTS[prec]
        achieved = flops / t_gemm / 1e12
        pair = plan.tile_m == 256
        traffic = traffic_from_profiles(f"tc_gemm_{'pair_' if pair else ''}{args.precision}_{S}.txt")
        out["roofline"] = {
            "bound": "tensor", "achieved": achieved, "peak": mode_peak, "unit": "TFLOP/s",
            "frac": achieved / mode_peak, "traffic": traffic,
            "kernel": f"{'tc_gemm_pair_kernel' if pair else 'tc_gemm_kernel'} (GEMM alone, planes already split)",
            "peak_basis": f"{peak_src} bf16 burst {peaks['bf16_tflops']} TF/s"
                          f"{' / 2 (TF32 rate)' if prec == 1 else ''} / {PRODUCTS[prec]} products; useful 2MNK flops",
            "gemm_ms": t_gemm * 1e3, "prepass_ms": max(0.0, (t_step - t_gemm) * 1e3),
        }
        # ---- phase breakdown of the headline step (maxmulsk_phase_report: CUDA
        # events around the split pre-pass and the GEMM; outside the timed region)
        mm.phase_report()
        mm.phase_timing(True)
        for _ in range(20):
            step_tc()
        torch.cuda.synchronize(dev)
        phases = mm.phase_report()
        mm.phase_timing(False)
        out["phases"] = {k: {"calls_per_step": v["calls"] / 20, "ms_per_step": v["ms"] / 20}
                         for k, v in phases.items()}
        # ---- the FP32 SIMT kernel on the same inputs
        for _ in range(3):
            step_simt()
        t_simt = timed(step_simt, max(10, min(args.steps, 100)))
        simt_gf = flops / t_simt / 1e9
        sm_mhz = clocks.get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
        fp32_peak_max = 148 * 128 * 2 * peaks.get("sm_max_mhz", 1965.0) * 1e6 / 1e12
        out["simt"] = {"gflops": simt_gf, "ms_per_step": t_simt * 1e3,
                       "plan": {"tile_m": splan.tile_m, "tile_n": splan.tile_n, "split_k": splan.split_k},
                       "peak_tflops": fp32_peak_max, "frac": simt_gf / 1e3 / fp32_peak_max,
                       "peak_basis": "nominal FP32 FMA: 148 SMs x 128 lanes x 2 x max SM clock"}
        # ---- the other split modes, same inputs (pre-pass + GEMM per step)
        modes = {}
        for name, pc in PREC.items():
            dCm = torch.empty((M, N), dtype=torch.float32, device=dev)
            step_mode, mp, mws = mode_step(pc, dCm)
            for _ in range(3):
                step_mode()
            t_m = timed(step_mode, max(10, min(args.steps, 50)))
            modes[name] = {"gflops": flops / t_m / 1e9, "ms_per_step": t_m * 1e3,
                           "plan": {"tile_m": mp.tile_m, "tile_n": mp.tile_n, "split_k": mp.split_k},
                           "_C": dCm}
            del mws
        out["speedup_vs_simt"] = (flops / t_step) / (flops / t_simt)
        out["speedup_vs_simt_gemm_only"] = t_simt / t_gemm
        # ---- FP64-measured error of both kernels (the library's FP64 check product, outside timing);
        # the plain FP32 kernel (one FMA chain per output, split_k 1) is the error bar
        dCp = torch.empty((M, N), dtype=torch.float32, device=dev)
        mm.check(mm.sgemm_plan_dev(dA, dB, dCp, M, K, N, mm.make_plan(0, 128, 128, 1), None, 0, stream), "plain")
        if rank == 0:
            # the library's FP64 check product and device error reduction
            chk = mm.Fp64Check(dA, dB, M, K, N, stream=stream)
            errs = {}
            for name, Cx in [("tc", dC), ("simt", dCs), ("plain_fp32", dCp)] + [(k, v["_C"]) for k, v in modes.items()]:
                e = chk.errors(Cx, stream=stream)
                errs[name] = {"normwise": e["normwise"], "max_rel": e["max_rel"]}
            del chk
            errs["tc_over_simt_normwise"] = errs["tc"]["normwise"] / errs["simt"]["normwise"]
            out["fp64_error"] = {"tc": errs["tc"], "simt": errs["simt"], "plain_fp32": errs["plain_fp32"],
                                 "tc_over_simt_normwise": errs["tc_over_simt_normwise"],
                                 "tc_over_plain_fp32_normwise": errs["tc"]["normwise"] / errs["plain_fp32"]["normwise"]}
            for k in modes:
                modes[k]["normwise_over_simt"] = errs[k]["normwise"] / errs["simt"]["normwise"]
        for k in modes:
            modes[k].pop("_C", None)
        out["split_modes"] = modes
        # ---- end to end through the public host-pointer API (pinned host buffers)
        hA = torch.from_numpy(A).pin_memory()
        hB = torch.from_numpy(B).pin_memory()
        hC = torch.empty((M, N), dtype=torch.float32).pin_memory()
        e2e_steps = max(3, min(args.steps, 30))
        lib = mm.lib()
        for _ in range(2):
            mm.check(lib.maxmulsk_sgemm_split(hA.data_ptr(), hB.data_ptr(), hC.data_ptr(), M, K, N, prec), "e2e")
        barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            mm.check(lib.maxmulsk_sgemm_split(hA.data_ptr(), hB.data_ptr(), hC.data_ptr(), M, K, N, prec), "e2e")
        t_e2e = max_over_ranks((time.perf_counter() - t0) / e2e_steps)
        out["e2e"] = {"value": flops * world / t_e2e / 1e9, "unit": "GFLOP/s",
                      "h2d_bytes_per_step": 4 * (M * K + K * N), "d2h_bytes_per_step": 4 * M * N,
                      "ms_per_step": t_e2e * 1e3, "steps": e2e_steps,
                      "api": "maxmulsk_sgemm_split (host pointers, synchronous, pinned buffers)"}
        # ---- the reference's CPU path, rank 0 at N = 1 only
        if world == 1 and rank == 0:
            out["cpu_baseline"] = cpu_rows_gflops(A, B, K, N, budget_s=12.0, threads=1)
            out["cpu_baseline"].pop("seconds", None)

    if rank == 0:
        print(json.dumps(out), flush=True)
    ranks.close()


if __name__ == "__main__":
    main()
