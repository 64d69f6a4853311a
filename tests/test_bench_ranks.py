"""bench.py's multi-rank path on CPU.

* `Ranks` (barriers and the max over ranks of a per-rank step time) on two
  gloo ranks with a stub step whose duration differs by rank: both ranks
  report the slower rank's time.
* `bench.py --gpus 2` with no launcher starts two ranks itself through
  torch.distributed.run and prints one line with n_gpus 2 (the reference arm,
  which runs on the host's cores, so the launch is exercised without a GPU).
* A line is refused when the ranks started differ from --gpus.
"""
import json
import os
import socket
import subprocess
import sys
import time

import torch.multiprocessing as tmp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out_dir: str):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    ranks = bench.Ranks("gloo")
    try:
        def step():
            time.sleep(0.004 * (rank + 1))
        t = ranks.timed(step, 5, time.perf_counter, lambda t0: time.perf_counter() - t0)
        with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
            f.write(f"{ranks.rank} {ranks.world} {t!r}\n")
    finally:
        ranks.close()


def test_ranks_time_is_the_max_over_two_gloo_ranks(tmp_path):
    world = 2
    tmp.start_processes(_worker, args=(world, _port(), str(tmp_path)), nprocs=world, join=True,
                        start_method="spawn")
    got = [(tmp_path / f"r{r}.txt").read_text().split() for r in range(world)]
    assert [g[:2] for g in got] == [["0", "2"], ["1", "2"]]
    t0, t1 = float(got[0][2]), float(got[1][2])
    assert t0 == t1                     # every rank reports the same number
    assert t0 >= 0.008                  # ... the slower rank's


def _clean_env():
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "LOCAL_WORLD_SIZE", "MASTER_ADDR", "MASTER_PORT",
              "TORCHELASTIC_RUN_ID", "GROUP_RANK", "ROLE_RANK"):
        env.pop(k, None)
    return env


def test_gpus_two_starts_two_ranks_itself():
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--impl", "reference",
           "--steps", "1", "--warmup", "3", "--size", "128"]
    r = subprocess.run(cmd, cwd=ROOT, env=_clean_env(), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, r.stdout
    assert lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2


def test_line_refused_when_ranks_differ_from_gpus():
    env = _clean_env()
    env["WORLD_SIZE"] = "1"
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--impl", "reference",
           "--steps", "1", "--warmup", "3", "--size", "128"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 2
    assert not [x for x in r.stdout.splitlines() if x.startswith("{")]
