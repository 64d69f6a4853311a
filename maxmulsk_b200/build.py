"""Builds the CUDA library in-tree: maxmulsk_b200/lib/libmaxmulsk_b200.so.

Every kernel is compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``);
nvcc cross-compiles without a GPU. Objects go to maxmulsk_b200/_build/. An
object is rebuilt unless the SHA-256 stamp beside it matches the hash of its
source, every header and the compiler flags; the library is relinked unless
its stamp matches the hash of the object stamps and the link flags. Stale
objects or a stale library shipped beside newer sources are therefore never
reused, whatever their file times say.

    python -m maxmulsk_b200.build [--force] [-j N]
"""
from __future__ import annotations

import argparse
import hashlib
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
CXXFLAGS = ARCH + COMMON
LINKFLAGS = ARCH + ["-shared"]
LIBS = ["-lpthread", "-ldl"]


def sources() -> list[str]:
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers() -> list[str]:
    hs = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h")))
    hs.append(os.path.join(ROOT, "include", "maxmulsk.h"))
    return hs


def _sha(*parts: bytes) -> str:
    h = hashlib.sha256()
    for p in parts:
        h.update(len(p).to_bytes(8, "little"))
        h.update(p)
    return h.hexdigest()


def _read(path: str) -> bytes:
    with open(path, "rb") as f:
        return f.read()


def _stamp_ok(path: str, key: str) -> bool:
    try:
        with open(path + ".sha256") as f:
            return f.read().strip() == key
    except OSError:
        return False


def _write_stamp(path: str, key: str) -> None:
    with open(path + ".sha256", "w") as f:
        f.write(key + "\n")


def _compile(src: str, force: bool, header_key: str) -> tuple[str, str, str]:
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src + ".o")
    flags = CUFLAGS if src.endswith(".cu") else CXXFLAGS
    key = _sha(_read(path), header_key.encode(), " ".join([NVCC] + flags).encode())
    if not force and os.path.exists(obj) and _stamp_ok(obj, key):
        return obj, "", key
    cmd = [NVCC] + flags + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    _write_stamp(obj, key)
    return obj, (r.stdout + r.stderr).strip(), key


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    header_key = _sha(*(os.path.basename(h).encode() + b"\0" + _read(h) for h in headers()))
    srcs = sources()
    with ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, force, header_key), srcs))
    objs = [o for o, _, _ in results]
    for (o, msg, _), s in zip(results, srcs):
        if msg and verbose:
            print(f"[{s}] {msg}", file=sys.stderr)
    lib_key = _sha(*(k.encode() for _, _, k in results), " ".join(LINKFLAGS + LIBS).encode())
    if force or not os.path.exists(LIB) or not _stamp_ok(LIB, lib_key):
        cmd = [NVCC] + LINKFLAGS + ["-o", LIB] + objs + LIBS
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        _write_stamp(LIB, lib_key)
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
