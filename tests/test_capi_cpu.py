"""The C-ABI library without a GPU: it loads, exports every symbol the
headers declare, and its pure host logic (plan validation, workspace sizing,
status names) behaves. No compute call is made here."""
import ctypes
import subprocess

import pytest

import maxmulsk_b200 as mm
from maxmulsk_b200 import _lib


def test_library_exports_every_declared_symbol(built_lib):
    declared = _lib.exported_symbols()
    assert "maxmulsk_sgemm_v3" in declared and "maxmulsk_sgemm_v4" in declared
    missing = [n for n in declared if not hasattr(built_lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    for n in declared:
        assert f" T {n}" in out, n


def test_binding_table_covers_header(built_lib):
    assert set(_lib.exported_symbols()) <= set(_lib._SIGNATURES) | {"maxmulsk_stream_status"}


def test_library_is_built_for_sm100a_only(built_lib):
    # Every CUDA source is compiled with exactly one target, sm_100a (no PTX
    # for other architectures, no multi-arch fat binary): the flags build.py
    # passes to nvcc for .cu sources, host sources and the link.
    from maxmulsk_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    for flags in (build.CUFLAGS, build.CXXFLAGS, build.LINKFLAGS):
        gencodes = [flags[i + 1] for i, f in enumerate(flags) if f == "-gencode"]
        assert gencodes == ["arch=compute_100a,code=sm_100a"], flags
        assert not any(f.startswith(("-arch", "--gpu-architecture")) for f in flags), flags


def test_status_codes_keep_reference_values(built_lib):
    # capi/maxmulsk.h:24-28: OK = 0, ERR_UNSUPPORTED = 1, ERR_ALLOC = 2
    assert (mm.Status.OK, mm.Status.ERR_UNSUPPORTED, mm.Status.ERR_ALLOC) == (0, 1, 2)
    assert mm.status_string(0) == "MAXMULSK_OK"
    assert mm.status_string(2) == "MAXMULSK_ERR_ALLOC"
    assert mm.status_string(5) == "MAXMULSK_ERR_TIMEOUT"
    assert mm.version() == mm.__version__


@pytest.mark.parametrize("plan,ok", [
    ((0, 128, 128, 1, 0), True), ((0, 128, 64, 4, 1), True), ((0, 64, 64, 64, 0), True),
    ((0, 64, 128, 1, 0), False), ((0, 128, 128, 0, 0), False), ((0, 128, 128, 65, 0), False),
    ((0, 128, 128, 1, 2), False), ((1, 128, 256, 1, 0), True), ((2, 128, 64, 8, 0), True),
    ((3, 128, 128, 1, 0), True), ((1, 64, 128, 1, 0), False), ((1, 128, 96, 1, 0), False),
    ((1, 256, 256, 1, 0), True), ((2, 256, 128, 3, 0), True), ((1, 256, 64, 1, 0), False),
    ((1, 128, 128, 1, 1), True), ((1, 128, 128, 1, 2), False), ((4, 128, 128, 1, 0), False), ((-1, 128, 128, 1, 0), False),
    # split_k 0: one K slice per SM for every tile, tensor-core plans only
    ((1, 128, 256, 0, 0), True), ((2, 256, 256, 0, 0), True), ((2, 128, 128, 0, 2), True), ((3, 128, 128, 0, 2), True),
    ((2, 128, 128, -1, 0), False),
])
def test_classify(built_lib, plan, ok):
    p = mm.make_plan(*plan)
    st = mm.classify(256, 256, 256, p)
    assert (st == mm.Status.OK) == ok
    if not ok:
        assert st == mm.Status.ERR_UNSUPPORTED


def test_classify_null_plan(built_lib):
    assert built_lib.maxmulsk_classify(16, 16, 16, None) == mm.Status.ERR_INVALID


def test_workspace_bytes(built_lib):
    # FP32 without split: no workspace.
    assert mm.workspace_bytes(512, 512, 512, mm.make_plan(0, 128, 128, 1)) == 0
    # FP32 with 4 slices: counters + 4 partial C's.
    M, K, N = 128, 8192, 512
    ws = mm.workspace_bytes(M, K, N, mm.make_plan(0, 64, 64, 4))
    assert ws >= 4 * M * N * 4 and ws % 256 == 0
    # 3xTF32: two FP32 planes of A and of B at least.
    ws = mm.workspace_bytes(M, K, N, mm.make_plan(1, 128, 128, 1))
    assert ws >= 2 * 4 * (M * K + K * N)
    # BF16 x6: three BF16 planes.
    ws6 = mm.workspace_bytes(M, K, N, mm.make_plan(2, 128, 128, 1))
    assert 3 * 2 * (M * K + K * N) <= ws6 < ws
    # invalid plan -> 0
    assert mm.workspace_bytes(M, K, N, mm.make_plan(0, 32, 32, 1)) == 0


def test_slice_rule():
    assert mm.slice_len(8192, 1) == 8192
    assert mm.slice_len(8192, 4) == 2048
    assert mm.slice_len(100, 3) == 64          # rounded up to 32, fewer slices result
    assert mm.slice_len(20, 8) == 20           # never longer than K
    for K in (1, 31, 33, 1000, 32768):
        for s in (1, 2, 3, 7, 64):
            kc = mm.slice_len(K, s)
            n = -(-K // kc)
            assert 1 <= n <= s and (n - 1) * kc < K


def test_probe_bytes(built_lib):
    # As A (R x C = M x K): C padded to 16 bytes, planes 1 KiB aligned.
    assert built_lib.maxmulsk_probe_split_bytes(4, 5, 1, 0) == 2 * 1024
    # As B (K x N), TF32: transposed N x Kp, Kp = K padded to 4 floats.
    assert built_lib.maxmulsk_probe_split_bytes(1000, 10, 1, 1) == 2 * ((10 * 1000 * 4 + 1023) // 1024 * 1024)
    # As B, BF16: N padded to 64 elements (128 bytes), 3 planes.
    assert built_lib.maxmulsk_probe_split_bytes(1000, 10, 2, 1) == 3 * ((1000 * 64 * 2 + 1023) // 1024 * 1024)
    assert built_lib.maxmulsk_probe_split_bytes(10, 10, 0, 1) == 0


def test_fused_split_plan_rules(built_lib):
    import maxmulsk_b200 as mm
    ok = mm.make_plan(mm.Precision.BF16X6, 128, 128, 4, mm.TC_FUSED_SPLIT)
    assert mm.classify(128, 8192, 512, ok) == mm.Status.OK
    assert mm.classify(128, 8190, 512, ok) == mm.Status.ERR_UNSUPPORTED      # K % 4
    assert mm.classify(128, 8192, 510, ok) == mm.Status.ERR_UNSUPPORTED      # N % 4
    for bad in (mm.make_plan(mm.Precision.TF32X3, 128, 128, 1, mm.TC_FUSED_SPLIT),
                mm.make_plan(mm.Precision.BF16X6, 128, 256, 1, mm.TC_FUSED_SPLIT),
                mm.make_plan(mm.Precision.BF16X9, 256, 128, 1, mm.TC_FUSED_SPLIT)):
        assert mm.classify(256, 256, 256, bad) == mm.Status.ERR_UNSUPPORTED


def test_phase_report_without_records(built_lib):
    # Nothing recorded: the empty report and its length; the switch and the
    # report touch no device when there is nothing to wait for.
    buf = ctypes.create_string_buffer(64)
    assert built_lib.maxmulsk_phase_report(buf, 64) == 2 and buf.value == b"{}"
    built_lib.maxmulsk_phase_timing(1)
    built_lib.maxmulsk_phase_timing(0)
    assert mm.phase_report() == {}
    small = ctypes.create_string_buffer(1)
    assert built_lib.maxmulsk_phase_report(small, 1) == 2 and small.value == b""


@pytest.mark.parametrize("compiler", [["gcc", "-std=c99", "-x", "c"], ["g++", "-std=c++17", "-x", "c++"]])
def test_c_caller_compiles_links_and_runs(built_lib, tmp_path, compiler):
    # A C (and a C++) caller of the header: it compiles with -Wall -Werror,
    # links every entry point against the library and runs its host-only
    # calls (no device work).
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    inc = os.path.join(os.path.dirname(here), "include")
    libdir = os.path.dirname(_lib.LIB_PATH)
    exe = str(tmp_path / "c_abi_check")
    cmd = compiler + ["-Wall", "-Wextra", "-Werror", "-I", inc, os.path.join(here, "c_abi_check.c"),
                      "-x", "none", "-L", libdir, "-lmaxmulsk_b200", f"-Wl,-rpath,{libdir}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert r.stdout.startswith("c-abi ok")
