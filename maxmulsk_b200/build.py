"""Builds the CUDA library in-tree: maxmulsk_b200/lib/libmaxmulsk_b200.so.

Every kernel is compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``);
nvcc cross-compiles without a GPU. Objects go to maxmulsk_b200/_build/ and are
rebuilt when their source or any header is newer.

    python -m maxmulsk_b200.build [--force] [-j N]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libmaxmulsk_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++20", "-lineinfo", "-Xcompiler", "-fPIC,-Wall", "-I", CSRC,
          "-I", os.path.join(ROOT, "include")]
CUFLAGS = ARCH + COMMON + ["--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def sources() -> list[str]:
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    hs.append(os.path.join(ROOT, "include", "maxmulsk.h"))
    return hs


def _compile(src: str, force: bool, newest_header: float) -> tuple[str, str]:
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src + ".o")
    if not force and os.path.exists(obj):
        mt = os.path.getmtime(obj)
        if mt >= os.path.getmtime(path) and mt >= newest_header:
            return obj, ""
    cmd = [NVCC] + (CUFLAGS if src.endswith(".cu") else ARCH + COMMON) + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, (r.stdout + r.stderr).strip()


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    newest_header = max(os.path.getmtime(h) for h in headers())
    srcs = sources()
    with ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, force, newest_header), srcs))
    objs = [o for o, _ in results]
    for (o, msg), s in zip(results, srcs):
        if msg and verbose:
            print(f"[{s}] {msg}", file=sys.stderr)
    relink = force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs)
    if relink:
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.j, verbose=a.v))


if __name__ == "__main__":
    main()
