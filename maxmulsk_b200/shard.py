"""Multi-GPU sharding of the GEMM path, one process per GPU.

The path has no exchange step, so no collective touches the data:

* one product C = A*B shards by M-row blocks: each rank holds its rows of A
  and C and the whole of B, and multiplies them in its own HBM;
* a grouped batch shards by problem: problems are dealt to ranks greedily,
  heaviest first, to balance 2*M*N*K per rank.

The only collective is on timings (the max over ranks of a measured time).
The reference is single-threaded (capi/maxmulsk.h:9-17) and has no
multi-device path; its one-stream batch (run_batch,
sme/v3/sme-1x4-acc-kcout-onestream.hpp:61-63) is what a problem shard runs.
"""
from __future__ import annotations

import heapq
from typing import Sequence

from . import Plan, Precision, Status, _plan_with_ws, choose

ROW_ALIGN = 256     # a multiple of every kernel's tile height


def row_shard(M: int, world: int, rank: int, align: int = ROW_ALIGN) -> tuple[int, int]:
    """Rows [r0, r1) of an M-row product owned by `rank`. Shards are whole
    multiples of `align` rows except the last non-empty one; trailing ranks
    may get none when M is small."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank out of range")
    blocks = -(-M // align)
    per = -(-blocks // world)
    r0 = min(M, rank * per * align)
    r1 = min(M, (rank + 1) * per * align)
    return r0, r1


def balance_problems(shapes: Sequence[tuple[int, int, int]], world: int) -> list[list[int]]:
    """Problem indices per rank: longest-processing-time-first by 2*M*N*K,
    each problem to the least loaded rank (ties to the lowest rank)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(shapes)), key=lambda i: (-2 * shapes[i][0] * shapes[i][1] * shapes[i][2], i))
    heap = [(0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        M, K, N = shapes[i]
        out[r].append(i)
        heapq.heappush(heap, (load + 2 * M * N * K, r))
    for lst in out:
        lst.sort()
    return out


def sgemm_rows_dev(dA, dB, dC, M: int, K: int, N: int, rank: int, world: int,
                   precision: int = Precision.FP32, plan: Plan | None = None, stream=None) -> Status:
    """This rank's rows of C = A*B, with A, B, C the whole matrices on this
    device (torch CUDA tensors or int pointers). Only rows r0..r1 of A are
    read and of C written. The shard runs the plan of the whole product
    (chosen for (M, K, N) unless given), so its rows are the ones a
    single-device launch of that plan writes."""
    r0, r1 = row_shard(M, world, rank)
    if r1 <= r0:
        return Status.OK
    if plan is None:
        plan = choose(M, K, N, precision)
    pa = dA if isinstance(dA, int) else dA.data_ptr()
    pb = dB if isinstance(dB, int) else dB.data_ptr()
    pc = dC if isinstance(dC, int) else dC.data_ptr()
    pa += 4 * r0 * K
    pc += 4 * r0 * N
    return Status(_plan_with_ws(pa, pb, pc, r1 - r0, K, N, plan, stream))


def max_over_ranks(x: float, device=None) -> float:
    """The max of a per-rank number (a step time) over the default process
    group; x itself without one."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
