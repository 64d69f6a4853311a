"""Split-precision tensor-core path on the GPU against the oracle.

* The split pre-pass planes are compared bit for bit with the oracle's
  definitions (oracle_split_tf32 / oracle_split_bf16), in the layouts the
  kernel reads (the counterpart of the reference's pack-layout probes,
  sme/v4/sme-1x4-kcout-ncblock-apack4za.hpp:44-49, check_nb.cpp:22-39).
* The tcgen05 GEMM is compared with the oracle's exact split product (the
  same kept limb pairs, accumulated in FP64): the only difference allowed is
  the FP32 accumulation, bounded below.
* Against the FP64 truth, every split mode must stay within 2x the FP32 SIMT
  kernel's normwise error (plus a floor of 2^-24 for tiny K).
"""
import numpy as np
import pytest

import maxmulsk_b200 as mm
from gpu_util import bits, run_plan, to_dev

pytestmark = pytest.mark.gpu

MODES = [mm.Precision.TF32X3, mm.Precision.BF16X6, mm.Precision.BF16X9]


def _planes_from_probe(cuda, X: np.ndarray, R: int, C: int, prec: int, as_b: bool):
    nb = mm.lib().maxmulsk_probe_split_bytes(R, C, int(prec), int(as_b))
    out = cuda.zeros(nb // 4 + 256, dtype=cuda.float32, device="cuda")
    base = out.data_ptr() + ((-out.data_ptr()) % 1024)
    dX = to_dev(cuda, X)
    st = mm.lib().maxmulsk_probe_split_dev(dX.data_ptr(), R, C, int(prec), int(as_b), base, None)
    assert st == 0
    cuda.cuda.synchronize()
    off = (base - out.data_ptr()) // 4
    return out.cpu().numpy()[off: off + nb // 4].view(np.uint8)[:nb]


@pytest.mark.parametrize("prec", [mm.Precision.TF32X3, mm.Precision.BF16X6])
@pytest.mark.parametrize("as_b", [False, True])
@pytest.mark.parametrize("shape", [(5, 7), (67, 67), (128, 33), (3, 200)])
def test_split_planes_bit_exact(cuda, oracle_mod, prec, as_b, shape):
    R, C = shape
    X = np.concatenate([oracle_mod.fill_uniform(R * C // 2, 1), oracle_mod.fill_wide(R * C - R * C // 2, 2)])
    raw = _planes_from_probe(cuda, X, R, C, prec, as_b)
    tf32 = prec == mm.Precision.TF32X3
    es = 4 if tf32 else 2
    P = 2 if tf32 else 3
    if tf32:
        want = [p.reshape(R, C) for p in oracle_mod.split_tf32(X)]
    else:
        want = [p.reshape(R, C) for p in oracle_mod.split_bf16(X)]
    if as_b and tf32:
        # transposed: [P][C][Rp], K-major
        Rp = -(-R // 4) * 4
        plane_bytes = -(-(C * Rp * es) // 1024) * 1024
    else:
        Cp = -(-C // (128 // es)) * (128 // es) if as_b else -(-C // (16 // es)) * (16 // es)
        plane_bytes = -(-(R * Cp * es) // 1024) * 1024
    for p in range(P):
        if tf32:
            w = want[p].view(np.uint32)
        else:
            w = (want[p].view(np.uint32) >> 16).astype(np.uint16)
        if as_b and tf32:
            v = raw[p * plane_bytes: p * plane_bytes + C * Rp * es].view(np.uint32).reshape(C, Rp)
            assert np.array_equal(v[:, :R].T, w), p
            assert np.all(v[:, R:] == 0)
            continue
        chunk = raw[p * plane_bytes: p * plane_bytes + R * Cp * es]
        v = chunk.view(np.uint32) if tf32 else chunk.view(np.uint16)
        if as_b:
            nbe = 128 // es
            v = v.reshape(Cp // nbe, R, nbe).transpose(1, 0, 2).reshape(R, Cp)
        else:
            v = v.reshape(R, Cp)
        assert np.array_equal(v[:, :C], w), p
        assert np.all(v[:, C:] == 0)


SHAPES = [(128, 128, 128), (67, 67, 67), (20, 35, 41), (300, 520, 200), (256, 1024, 512), (1, 64, 1), (130, 16, 300)]


TC_TILES = [(128, 64), (128, 128), (128, 256), (256, 128), (256, 256)]


@pytest.mark.parametrize("prec", MODES)
@pytest.mark.parametrize("tile", TC_TILES)
@pytest.mark.parametrize("split_k", [1, 3, 0])
def test_tc_gemm_vs_exact_split_product(cuda, oracle_mod, prec, tile, split_k):
    for i, (M, K, N) in enumerate(SHAPES):
        A = oracle_mod.fill_uniform(M * K, 30 + i)
        B = oracle_mod.fill_uniform(K * N, 60 + i)
        plan = mm.make_plan(prec, tile[0], tile[1], split_k)
        st, C, bands = run_plan(cuda, A, B, M, K, N, plan)
        assert st == 0, mm.last_error_message()
        assert bands, ((M, K, N), plan)
        ideal = oracle_mod.sgemm_split_exact(A, B, M, K, N, int(prec))
        # Only FP32 accumulation separates the two: bounded by K units of
        # 2^-24 of sum |a||b| <= K for U[-1,1) inputs, far looser in practice.
        C64 = oracle_mod.dgemm(A, B, M, K, N)
        e = oracle_mod.errors(C, C64, A, B, M, K, N)
        e_ideal = oracle_mod.errors(ideal, C64, A, B, M, K, N)
        assert e["normwise"] <= 4 * e_ideal["normwise"] + 8 * 2.0 ** -24, ((M, K, N), plan, e, e_ideal)
        assert np.max(np.abs(C - ideal)) <= K * 2.0 ** -22 + 1e-6


WRITEBACK_SHAPES = [(300, 256, 200), (1, 64, 4), (129, 96, 260), (257, 128, 36), (128, 64, 128)]


@pytest.mark.parametrize("prec", MODES)
@pytest.mark.parametrize("tile", TC_TILES)
def test_tma_store_writeback_equals_register_writeback(cuda, oracle_mod, prec, tile):
    # Whole tiles leave through TMA stores when C is 16-byte aligned and N is
    # a multiple of 4 (tile configurations with shared memory for the store
    # boxes), and from registers otherwise -- here by placing C one float off
    # its alignment. The sums are the same, so the bits are; the boxes
    # clipped at the M and N edges write nothing outside C (guard bands).
    variants = [0] + ([mm.TC_FUSED_SPLIT] if prec != mm.Precision.TF32X3 and tile == (128, 128) else [])
    for i, (M, K, N) in enumerate(WRITEBACK_SHAPES):
        A = oracle_mod.fill_uniform(M * K, 600 + i)
        B = oracle_mod.fill_uniform(K * N, 700 + i)
        dA, dB = to_dev(cuda, A), to_dev(cuda, B)
        for var in variants:
            plan = mm.make_plan(prec, tile[0], tile[1], 1, var)
            st1, C1, b1 = run_plan(cuda, A, B, M, K, N, plan, dA=dA, dB=dB)
            st2, C2, b2 = run_plan(cuda, A, B, M, K, N, plan, dA=dA, dB=dB, offset=1)
            assert st1 == 0 and st2 == 0, mm.last_error_message()
            assert b1 and b2, ((M, K, N), var)
            assert np.array_equal(bits(C1), bits(C2)), ((M, K, N), var)


@pytest.mark.parametrize("kind", ["uniform", "wide"])
def test_split_error_within_twice_simt(cuda, oracle_mod, kind):
    # The bar is the plain FP32 kernel: one FMA chain per output (split_k 1).
    # A K-split SIMT plan shortens the chains and so its error; the bar does
    # not move with the picker's plan choice.
    M = K = N = 1024
    fill = oracle_mod.fill_uniform if kind == "uniform" else oracle_mod.fill_wide
    A, B = fill(M * K, 71), fill(K * N, 72)
    C64 = oracle_mod.dgemm(A, B, M, K, N)
    _, Cs, _ = run_plan(cuda, A, B, M, K, N, mm.make_plan(mm.Precision.FP32, 128, 128, 1))
    e_simt = oracle_mod.errors(Cs, C64, A, B, M, K, N)
    for prec in MODES:
        C = np.empty(M * N, np.float32)
        assert mm.sgemm_split(A, B, C, M, K, N, prec) == 0, mm.last_error_message()
        e = oracle_mod.errors(C, C64, A, B, M, K, N)
        print(kind, int(prec), e, "simt", e_simt)
        assert e["normwise"] <= 2 * e_simt["normwise"] + 2.0 ** -24, (kind, int(prec), e, e_simt)


@pytest.mark.parametrize("tile", [(128, 128), (256, 256)])
def test_split_k_deterministic(cuda, oracle_mod, tile):
    M, K, N = 300, 6000, 384
    A = oracle_mod.fill_uniform(M * K, 81)
    B = oracle_mod.fill_uniform(K * N, 82)
    plan = mm.make_plan(mm.Precision.TF32X3, tile[0], tile[1], 8)
    _, C1, _ = run_plan(cuda, A, B, M, K, N, plan)
    _, C2, _ = run_plan(cuda, A, B, M, K, N, plan)
    assert np.array_equal(bits(C1), bits(C2))


@pytest.mark.parametrize("prec", MODES)
@pytest.mark.parametrize("tile", TC_TILES)
def test_tail_wave_split_matches_whole_tiles(cuda, oracle_mod, prec, tile):
    # 4352 x 512 x 4352 gives tile counts that leave a partial last wave, so
    # the schedule splits the K of the tail tiles; results must stay within
    # the same error of the exact split product as whole tiles.
    M, K, N = 1280 + 64, 512, 2304
    A = oracle_mod.fill_uniform(M * K, 91)
    B = oracle_mod.fill_uniform(K * N, 92)
    st, C, bands = run_plan(cuda, A, B, M, K, N, mm.make_plan(prec, tile[0], tile[1], 1))
    assert st == 0 and bands
    ideal = oracle_mod.sgemm_split_exact(A, B, M, K, N, int(prec))
    assert np.max(np.abs(C - ideal)) <= K * 2.0 ** -22


def test_split_device_entry_and_picker(cuda, oracle_mod):
    M, K, N = 128, 8192, 512
    sc = 1.0 / np.sqrt(K)
    A = oracle_mod.fill_normal(M * K, 91, sc)
    B = oracle_mod.fill_normal(K * N, 92, sc)
    dA, dB = to_dev(cuda, A), to_dev(cuda, B)
    dC = cuda.empty(M * N, device="cuda")
    assert mm.sgemm_split_dev(dA, dB, dC, M, K, N, mm.Precision.TF32X3) == 0
    assert mm.stream_status() == 0
    C = dC.cpu().numpy()
    C64 = oracle_mod.dgemm(A, B, M, K, N)
    e = oracle_mod.errors(C, C64, A, B, M, K, N)
    assert e["rel_frob"] < 1e-5, e


FUSED_SHAPES = [(128, 128, 128), (68, 68, 68), (20, 36, 40), (300, 520, 200), (256, 1024, 512), (4, 64, 4),
                (130, 16, 300), (128, 8192, 512), (1344, 512, 2304)]


@pytest.mark.parametrize("prec", [mm.Precision.BF16X6, mm.Precision.BF16X9])
@pytest.mark.parametrize("split_k", [1, 2, 5, 0])
def test_fused_split_equals_split_inputs(cuda, oracle_mod, prec, split_k):
    # The fused kernel splits FP32 tiles into limbs itself (A's into tensor
    # memory, B's into shared memory); the products, their order and the
    # chunked accumulation are those of the split-inputs path on the same
    # tiles, so C must agree bit for bit.
    for i, (M, K, N) in enumerate(FUSED_SHAPES):
        A = np.concatenate([oracle_mod.fill_uniform(M * K // 2, 200 + i),
                            oracle_mod.fill_wide(M * K - M * K // 2, 300 + i)])
        B = oracle_mod.fill_uniform(K * N, 400 + i)
        dA, dB = to_dev(cuda, A), to_dev(cuda, B)
        st1, C1, b1 = run_plan(cuda, A, B, M, K, N, mm.make_plan(prec, 128, 128, split_k), dA=dA, dB=dB)
        st2, C2, b2 = run_plan(cuda, A, B, M, K, N, mm.make_plan(prec, 128, 128, split_k, mm.TC_FUSED_SPLIT),
                               dA=dA, dB=dB)
        assert st1 == 0 and st2 == 0, mm.last_error_message()
        assert b1 and b2, (M, K, N)
        assert np.array_equal(bits(C1), bits(C2)), ((M, K, N), split_k)


def test_fused_split_unaligned_inputs_take_the_split_inputs_path(cuda, oracle_mod):
    M, K, N = 96, 256, 128
    A = oracle_mod.fill_uniform(M * K, 501)
    B = oracle_mod.fill_uniform(K * N, 502)
    Abuf = cuda.zeros(M * K + 1, device="cuda")
    Abuf[1:] = to_dev(cuda, A)
    plan = mm.make_plan(mm.Precision.BF16X6, 128, 128, 1, mm.TC_FUSED_SPLIT)
    st, C, bands = run_plan(cuda, A, B, M, K, N, plan, dA=Abuf[1:])
    assert st == 0 and bands
    _, Cref, _ = run_plan(cuda, A, B, M, K, N, mm.make_plan(mm.Precision.BF16X6, 128, 128, 1))
    assert np.array_equal(bits(C), bits(Cref))


@pytest.mark.parametrize("variant", [mm.TC_SPLIT_INPUTS, mm.TC_FUSED_SPLIT])
@pytest.mark.parametrize("shape", [(128, 32768, 512), (64, 8192, 512), (300, 2048, 700)])
def test_fill_split_is_the_slots_per_tile_split(cuda, oracle_mod, variant, shape):
    # split_k 0 cuts every tile into as many K slices as the device has SMs
    # per tile (at most 64): the same schedule, and so the same bits, as the
    # plan that names that split.
    torch = cuda
    M, K, N = shape
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    tiles = -(-M // 128) * -(-N // 128)
    want = max(1, min(64, sms // tiles))
    A = oracle_mod.fill_uniform(M * K, 501)
    B = oracle_mod.fill_uniform(K * N, 502)
    dA, dB = to_dev(torch, A), to_dev(torch, B)
    prec = mm.Precision.BF16X6
    st0, C0, b0 = run_plan(torch, A, B, M, K, N, mm.make_plan(prec, 128, 128, 0, variant), dA=dA, dB=dB)
    st1, C1, b1 = run_plan(torch, A, B, M, K, N, mm.make_plan(prec, 128, 128, want, variant), dA=dA, dB=dB)
    assert st0 == 0 and st1 == 0, mm.last_error_message()
    assert b0 and b1
    assert np.array_equal(bits(C0), bits(C1)), (shape, want)
