"""FP32 SIMT kernel on the GPU against the oracle, through the C ABI.

Bit-exact bars:
* SCALAR variant == the reference's Utils::multiply_scalar (golden SHA-256s,
  generated from the reference itself), every tile shape.
* FMA variant with split_k slices == oracle_sgemm_panels: one fused
  multiply-add chain per slice, slices added in order (the reference's v3
  outer-Kc panel order).
Contract checks follow the reference's own checker (check_nb.cpp): sentinel
prefill, repeat with a new B, refusal of bad plans with C untouched, plus the
capi empty-shape rules (capi/maxmulsk.cpp:13-20).
"""
import hashlib

import numpy as np
import pytest

import maxmulsk_b200 as mm
from gpu_util import SENTINEL, bits, run_plan, to_dev

pytestmark = pytest.mark.gpu

TILES = [(128, 128), (128, 64), (64, 64)]


def _inputs(oracle_mod, M, K, N, seed=1, kind="uniform"):
    if kind == "uniform":
        return oracle_mod.fill_uniform(M * K, seed), oracle_mod.fill_uniform(K * N, seed + 1)
    if kind == "wide":
        return oracle_mod.fill_wide(M * K, seed), oracle_mod.fill_wide(K * N, seed + 1)
    sc = 1.0 / np.sqrt(K)
    return oracle_mod.fill_normal(M * K, seed, sc), oracle_mod.fill_normal(K * N, seed + 1, sc)


@pytest.mark.parametrize("tile", TILES)
def test_scalar_variant_matches_reference_golden(cuda, oracle_mod, golden_cases, tile):
    for c in golden_cases:
        M, K, N = c["M"], c["K"], c["N"]
        A = oracle_mod.fill_uniform(M * K, c["seed_a"])
        B = oracle_mod.fill_uniform(K * N, c["seed_b"])
        plan = mm.make_plan(mm.Precision.FP32, tile[0], tile[1], 1, mm.FP32_SCALAR)
        st, C, bands = run_plan(cuda, A, B, M, K, N, plan)
        assert st == 0, mm.last_error_message()
        assert bands, c["tag"]
        assert hashlib.sha256(C.tobytes()).hexdigest() == c["sha256"], (c["tag"], tile)


@pytest.mark.parametrize("tile", TILES)
def test_fma_variant_matches_contracted_reference_golden(cuda, oracle_mod, golden_cases, tile):
    for c in golden_cases:
        M, K, N = c["M"], c["K"], c["N"]
        A = oracle_mod.fill_uniform(M * K, c["seed_a"])
        B = oracle_mod.fill_uniform(K * N, c["seed_b"])
        plan = mm.make_plan(mm.Precision.FP32, tile[0], tile[1], 1, mm.FP32_FMA)
        st, C, bands = run_plan(cuda, A, B, M, K, N, plan)
        assert st == 0 and bands
        assert hashlib.sha256(C.tobytes()).hexdigest() == c["sha256_fma"], (c["tag"], tile)


SHAPES = [(16, 16, 16), (67, 67, 67), (20, 35, 41), (128, 128, 128), (1, 1, 1), (1, 300, 7), (129, 65, 257),
          (64, 1100, 128), (300, 257, 130), (5, 4096, 3)]


@pytest.mark.parametrize("tile", TILES)
@pytest.mark.parametrize("split_k", [1, 2, 3, 7])
def test_fma_variant_bit_exact_vs_panel_oracle(cuda, oracle_mod, tile, split_k):
    for i, (M, K, N) in enumerate(SHAPES):
        A, B = _inputs(oracle_mod, M, K, N, seed=10 + i)
        plan = mm.make_plan(mm.Precision.FP32, tile[0], tile[1], split_k)
        st, C, bands = run_plan(cuda, A, B, M, K, N, plan)
        assert st == 0, mm.last_error_message()
        assert bands
        ref = oracle_mod.sgemm_panels(A, B, M, K, N, kc=mm.slice_len(K, split_k), fma=True)
        assert np.array_equal(bits(C), bits(ref)), ((M, K, N), tile, split_k)


def test_narrow_m_split_bit_exact(cuda, oracle_mod):
    # The narrow-M LLM shapes of the reference's sweep (bench_sweep_shapes.h:4-6),
    # K shortened to keep the oracle quick; N(0, 1/K) inputs.
    for (M, K, N) in [(64, 8192, 512), (128, 4096, 512)]:
        A, B = _inputs(oracle_mod, M, K, N, seed=3, kind="normal")
        plan = mm.choose_rule(M, K, N)
        assert plan.split_k > 1
        st, C, bands = run_plan(cuda, A, B, M, K, N, plan)
        assert st == 0 and bands
        ref = oracle_mod.sgemm_panels(A, B, M, K, N, kc=mm.slice_len(K, plan.split_k), fma=True)
        assert np.array_equal(bits(C), bits(ref))


def test_unaligned_pointers_take_the_scalar_load_path(cuda, oracle_mod):
    M, K, N = 70, 96, 72
    A, B = _inputs(oracle_mod, M, K, N, seed=5)
    Abuf = cuda.zeros(M * K + 1, device="cuda")
    Abuf[1:] = to_dev(cuda, A)
    dA = Abuf[1:]                           # 4-byte aligned, not 16
    plan = mm.make_plan(0, 128, 128, 2)
    st, C, bands = run_plan(cuda, A, B, M, K, N, plan, dA=dA, offset=1)
    assert st == 0 and bands
    ref = oracle_mod.sgemm_panels(A, B, M, K, N, kc=mm.slice_len(K, 2), fma=True)
    assert np.array_equal(bits(C), bits(ref))


def test_repeat_with_new_b_same_buffers(cuda, oracle_mod):
    # check_nb.cpp:61-66: no stale state may survive between calls.
    M, K, N = 200, 300, 100
    A, B = _inputs(oracle_mod, M, K, N, seed=7)
    B2 = oracle_mod.fill_uniform(K * N, 99)
    plan = mm.make_plan(0, 64, 64, 3)
    dA = to_dev(cuda, A)
    for Bx in (B, B2):
        st, C, bands = run_plan(cuda, A, Bx, M, K, N, plan, dA=dA)
        assert st == 0 and bands
        ref = oracle_mod.sgemm_panels(A, Bx, M, K, N, kc=mm.slice_len(K, 3), fma=True)
        assert np.array_equal(bits(C), bits(ref))


@pytest.mark.parametrize("bad", [(0, 96, 128, 1, 0), (0, 128, 128, 0, 0), (0, 128, 128, 100, 0),
                                 (1, 128, 80, 1, 0), (7, 128, 128, 1, 0)])
def test_bad_plan_refused_and_c_untouched(cuda, oracle_mod, bad):
    # check_nb.cpp:70-79
    M = K = N = 256
    A, B = _inputs(oracle_mod, M, K, N)
    dA, dB = to_dev(cuda, A), to_dev(cuda, B)
    dC = cuda.full((M * N,), 9.0, device="cuda")
    st = mm.sgemm_plan_dev(dA, dB, dC, M, K, N, mm.make_plan(*bad))
    assert st == mm.Status.ERR_UNSUPPORTED
    cuda.cuda.synchronize()
    assert bool((dC == 9.0).all())
    C = np.full(M * N, 9.0, np.float32)
    assert mm.sgemm_plan(A, B, C, M, K, N, mm.make_plan(*bad)) == mm.Status.ERR_UNSUPPORTED
    assert np.all(C == 9.0)


def test_empty_shapes(cuda):
    # capi/maxmulsk.cpp:13-20: M or N == 0 -> OK, untouched; K == 0 -> C = 0.
    C = np.full(12, SENTINEL, np.float32)
    A = np.ones(12, np.float32)
    assert mm.sgemm_v3(A, A, C, 0, 4, 3) == 0 and np.all(C == SENTINEL)
    assert mm.sgemm_v4(A, A, C, 3, 4, 0) == 0 and np.all(C == SENTINEL)
    assert mm.sgemm_v3(A, A, C, 3, 0, 4) == 0 and np.all(C == 0)
    C[:] = SENTINEL
    assert mm.sgemm_v4(A, A, C, 4, 0, 3) == 0 and np.all(C == 0)
    dC = cuda.full((12,), SENTINEL, device="cuda")
    assert mm.sgemm_v3_dev(0, 0, dC, 3, 0, 4) == 0
    cuda.cuda.synchronize()
    assert bool((dC == 0).all())
    C[:] = SENTINEL
    assert mm.sgemm_split(A, A, C, 3, 0, 4, mm.Precision.TF32X3) == 0 and np.all(C == 0)


def test_null_pointers_rejected(cuda):
    assert mm.sgemm_v3_dev(0, 0, 0, 4, 4, 4) == mm.Status.ERR_INVALID
    C = np.zeros(16, np.float32)
    assert mm.sgemm_v3(None, None, C, 4, 4, 4) == mm.Status.ERR_INVALID


@pytest.mark.parametrize("entry", ["v3", "v4"])
def test_host_entry_points_vs_reference_checks(cuda, oracle_mod, golden_cases, entry):
    fn = mm.sgemm_v3 if entry == "v3" else mm.sgemm_v4
    for c in golden_cases:
        M, K, N = c["M"], c["K"], c["N"]
        A = oracle_mod.fill_uniform(M * K, c["seed_a"])
        B = oracle_mod.fill_uniform(K * N, c["seed_b"])
        C = np.full(M * N, SENTINEL, np.float32)
        assert fn(A, B, C, M, K, N) == 0, mm.last_error_message()
        ref = oracle_mod.sgemm_scalar(A, B, M, K, N)
        # Utils::check_correctness (common/utils.hpp:24-48): |ref - got| <= 1e-3
        bad, _ = oracle_mod.check_correctness(ref, C, 1e-3)
        assert bad == 0, c["tag"]
        # check_nb.cpp:58-59: relative Frobenius distance < 5e-6
        assert oracle_mod.relfrob(C, ref) < 5e-6, c["tag"]


def test_fp64_error_of_simt(cuda, oracle_mod):
    M = K = N = 512
    for kind in ("uniform", "wide"):
        A, B = _inputs(oracle_mod, M, K, N, seed=21, kind=kind)
        C = np.empty(M * N, np.float32)
        assert mm.sgemm_v3(A, B, C, M, K, N) == 0
        e = oracle_mod.errors(C, oracle_mod.dgemm(A, B, M, K, N), A, B, M, K, N)
        # FP32 class: a few units of 2^-24 times sqrt(K) at most.
        assert e["normwise"] < 4 * 2.0 ** -24 * np.sqrt(K), (kind, e)


def test_deterministic_repeat(cuda, oracle_mod):
    M, K, N = 96, 4000, 200
    A, B = _inputs(oracle_mod, M, K, N, seed=8)
    plan = mm.make_plan(0, 64, 64, 16)
    _, C1, _ = run_plan(cuda, A, B, M, K, N, plan)
    _, C2, _ = run_plan(cuda, A, B, M, K, N, plan)
    assert np.array_equal(bits(C1), bits(C2))


@pytest.mark.parametrize("prec", [mm.Precision.FP32, mm.Precision.TF32X3, mm.Precision.BF16X6])
def test_host_entry_pipelined_path_matches_device_path(cuda, oracle_mod, prec):
    # Page-locked A and C of >= 32 MiB with M >= 1024 take the row-block
    # pipeline of the host entry points (B split once, A and C in blocks, a
    # ragged last block). FP32: bit for bit the device entry's result.
    # Split modes: the same plan on row blocks; only the tail-wave K split of
    # the schedule may differ, so the results agree to the accumulation bound.
    torch = cuda
    M, K, N = 2048 + 77, 2048, 2048
    A = oracle_mod.fill_uniform(M * K, 201)
    B = oracle_mod.fill_uniform(K * N, 202)
    pA = torch.from_numpy(A).pin_memory()
    pB = torch.from_numpy(B).pin_memory()
    pC = torch.full((M * N,), SENTINEL).pin_memory()
    dA, dB = pA.cuda(), pB.cuda()
    dC = torch.empty(M * N, device="cuda")
    if prec == mm.Precision.FP32:
        assert mm.sgemm_v3(pA.data_ptr(), pB.data_ptr(), pC.data_ptr(), M, K, N) == 0, mm.last_error_message()
        assert mm.sgemm_v3_dev(dA, dB, dC, M, K, N) == 0
    else:
        assert mm.sgemm_split(pA.data_ptr(), pB.data_ptr(), pC.data_ptr(), M, K, N, prec) == 0, \
            mm.last_error_message()
        assert mm.sgemm_split_dev(dA, dB, dC, M, K, N, prec) == 0
    assert mm.stream_status() == 0
    got, want = pC.numpy(), dC.cpu().numpy()
    if prec == mm.Precision.FP32:
        assert np.array_equal(bits(got), bits(want))
    else:
        assert np.max(np.abs(got - want)) <= K * 2.0 ** -22
        assert not np.any(got == SENTINEL)


@pytest.mark.parametrize("world", [2, 3, 8])
def test_row_shards_reassemble_the_product(cuda, oracle_mod, world):
    # Each rank's M-row shard (shard.sgemm_rows_dev), run here one after the
    # other on one device, writes exactly its rows; together they equal the
    # whole-matrix launch of the same plan bit for bit (FP32: the same chain
    # per output). The plan is the picker's for the whole product, which the
    # shards run; the whole launch is given it too, since a device-pointer
    # v3 call may replace a doubtful pick by an exhaustive search's.
    from maxmulsk_b200 import shard
    torch = cuda
    M, K, N = 1000, 384, 200
    A, B = _inputs(oracle_mod, M, K, N, seed=31)
    dA, dB = to_dev(torch, A), to_dev(torch, B)
    dC = torch.full((M * N,), SENTINEL, device="cuda")
    plan = mm.choose(M, K, N, mm.Precision.FP32)
    for r in range(world):
        assert shard.sgemm_rows_dev(dA, dB, dC, M, K, N, r, world) == 0
    st, whole, _ = run_plan(torch, A, B, M, K, N, plan, dA=dA, dB=dB)
    assert st == 0 and mm.stream_status() == 0
    assert np.array_equal(bits(dC.cpu().numpy()), bits(whole.ravel()))
