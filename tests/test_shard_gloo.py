"""Multi-rank host logic on CPU: two gloo ranks on 127.0.0.1.

Row shards partition the product with no overlap, problem shards deal every
grouped problem to exactly one rank with balanced flops, each rank's row
shard of the oracle product reassembles the whole product bit for bit, and
the timing collective returns the max over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as tmp

from maxmulsk_b200 import shard, workloads


def _port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out_dir: str):
    import torch
    import torch.distributed as dist

    import oracle
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        om = oracle
        M, K, N = 700, 96, 130
        A = om.fill_uniform(M * K, 1).reshape(M, K)
        B = om.fill_uniform(K * N, 2)
        r0, r1 = shard.row_shard(M, world, rank, align=64)
        part = om.sgemm_scalar(np.ascontiguousarray(A[r0:r1]).ravel(), B, r1 - r0, K, N) if r1 > r0 \
            else np.zeros(0, np.float32)
        # gather the row blocks (test plumbing only: the product path has no collective)
        sizes = [None] * world
        dist.all_gather_object(sizes, (r0, r1, part.tobytes()))
        full = np.zeros((M, N), np.float32)
        covered = np.zeros(M, int)
        for a, b, raw in sizes:
            if b > a:
                full[a:b] = np.frombuffer(raw, np.float32).reshape(b - a, N)
            covered[a:b] += 1
        ok_cover = bool(np.all(covered == 1))
        want = om.sgemm_scalar(A.ravel(), B, M, K, N).reshape(M, N)
        ok_bits = bool(np.array_equal(full.view(np.uint32), want.view(np.uint32)))
        t = shard.max_over_ranks(1.0 + rank)
        shapes = workloads.grouped_problems()
        mine = shard.balance_problems(shapes, world)[rank]
        everyone = [None] * world
        dist.all_gather_object(everyone, mine)
        with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
            f.write(f"{ok_cover} {ok_bits} {t} {sorted(sum(everyone, [])) == list(range(len(shapes)))}\n")
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    world = 2
    tmp.start_processes(_worker, args=(world, _port(), str(tmp_path)), nprocs=world, join=True,
                        start_method="spawn")
    for r in range(world):
        cover, bits, t, dealt = (tmp_path / f"r{r}.txt").read_text().split()
        assert cover == "True" and bits == "True" and dealt == "True"
        assert float(t) == float(world)


@pytest.mark.parametrize("M", [0, 1, 255, 256, 257, 4096, 4096 + 77, 100000])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_row_shards_partition(M, world):
    got = [shard.row_shard(M, world, r) for r in range(world)]
    pos = 0
    for r0, r1 in got:
        assert r0 == pos or r1 == r0
        assert r0 % shard.ROW_ALIGN == 0 or r0 == M
        pos = max(pos, r1)
    assert pos == M
    assert sum(r1 - r0 for r0, r1 in got) == M


def test_problem_balance():
    shapes = workloads.grouped_problems()
    for world in (2, 4, 8):
        parts = shard.balance_problems(shapes, world)
        assert sorted(sum(parts, [])) == list(range(len(shapes)))
        loads = [sum(2 * shapes[i][0] * shapes[i][1] * shapes[i][2] for i in p) for p in parts]
        biggest = max(2 * M * N * K for M, K, N in shapes)
        assert max(loads) - min(loads) <= biggest
