"""FP64-measured accuracy on the GPU, at every configuration cell.

* The FP64 check product (maxmulsk_check_dgemm_dev: one FMA chain per output
  in double, k upward) equals the oracle's FP64 product bit for bit, and the
  device error reduction agrees with the oracle's error measures.
* The split modes' accuracy bar: normwise error <= 2x the plain FP32 kernel's
  (one FMA chain per output, split_k 1) on every cell of the benchmark
  configurations -- the six narrow-M shapes with N(0, 1/K) inputs, and the
  square sweep with uniform and wide-range inputs -- for every candidate plan
  the autotuner or the picker may run, each split mode. The reference checks
  every library against an FP64 product before timing
  (docs/BENCHMARKS.md:112-120, :395-399).
* Each mode's product set is pinned exactly: on inputs built so that every
  limb product and every partial sum is exact in FP32 (k pairs whose leading
  limbs cancel inside one MMA), the tensor-core result equals the oracle's
  exact split product (oracle_sgemm_split_exact) bit for bit, so a missing or
  extra limb product changes the bits.
"""
import numpy as np
import pytest

import maxmulsk_b200 as mm
from maxmulsk_b200 import datagen, workloads
from gpu_util import bits, run_plan, to_dev
from pinning import pinning_inputs as _pinning_inputs

pytestmark = pytest.mark.gpu

MODES = [mm.Precision.TF32X3, mm.Precision.BF16X6, mm.Precision.BF16X9]


# --------------------------------------------------------------------------- the FP64 check itself
@pytest.mark.parametrize("shape", [(1, 1, 1), (67, 67, 67), (20, 35, 41), (130, 513, 70), (64, 2048, 96),
                                   (3, 0, 5)])
def test_fp64_check_product_bit_exact(cuda, oracle_mod, shape):
    torch = cuda
    M, K, N = shape
    A = np.concatenate([oracle_mod.fill_uniform(M * K // 2, 11), oracle_mod.fill_wide(M * K - M * K // 2, 12)])
    B = oracle_mod.fill_wide(K * N, 13)
    dA, dB = to_dev(torch, A) if M * K else torch.zeros(1, device="cuda"), \
        to_dev(torch, B) if K * N else torch.zeros(1, device="cuda")
    c64 = torch.full((M * N,), 7.0, dtype=torch.float64, device="cuda")
    cab = torch.full((M * N,), 7.0, dtype=torch.float64, device="cuda")
    assert mm.check_dgemm_dev(dA.data_ptr(), dB.data_ptr(), c64, cab, M, K, N) == 0, mm.last_error_message()
    assert mm.stream_status() == 0
    want = oracle_mod.dgemm(A, B, M, K, N).ravel()
    want_abs = oracle_mod.dgemm_abs(A, B, M, K, N).ravel()
    assert np.array_equal(c64.cpu().numpy().view(np.uint64), want.view(np.uint64))
    assert np.array_equal(cab.cpu().numpy().view(np.uint64), want_abs.view(np.uint64))


@pytest.mark.parametrize("kind", ["uniform", "wide"])
def test_fp64_error_reduction_matches_oracle(cuda, oracle_mod, kind):
    torch = cuda
    M, K, N = 300, 700, 260
    fill = oracle_mod.fill_uniform if kind == "uniform" else oracle_mod.fill_wide
    A, B = fill(M * K, 21), fill(K * N, 22)
    dA, dB = to_dev(torch, A), to_dev(torch, B)
    _, C, _ = run_plan(torch, A, B, M, K, N, mm.make_plan(mm.Precision.BF16X6, 128, 128, 1))
    chk = mm.Fp64Check(dA, dB, M, K, N)
    got = chk.errors(to_dev(torch, C))
    want = oracle_mod.errors(C, oracle_mod.dgemm(A, B, M, K, N), A, B, M, K, N)
    for key in ("normwise", "max_rel", "rel_frob", "max_abs"):
        assert abs(got[key] - want[key]) <= 1e-12 * abs(want[key]), (key, got[key], want[key])
    # deterministic: the same bits on a second reduction
    again = chk.errors(to_dev(torch, C))
    assert again == got


# --------------------------------------------------------------------------- the 2x bar at every cell
def _cells():
    out = [("normal", M, K, N) for (M, K, N) in workloads.NARROW_M]
    for S in workloads.SQUARE:
        out += [("uniform", S, S, S), ("wide", S, S, S)]
    return out


def _inputs(kind, M, K, N):
    if kind == "normal":
        return datagen.normal(M * K, 31, 1.0 / np.sqrt(K)), datagen.normal(K * N, 32, 1.0 / np.sqrt(K))
    if kind == "wide":
        return datagen.wide(M * K, 31), datagen.wide(K * N, 32)
    return datagen.uniform(M * K, 31), datagen.uniform(K * N, 32)


def _plans_of_mode(prec):
    """Every plan of a split mode the autotuner or the picker may run: the
    candidates of that precision (BF16X9: the BF16X6 candidates' tiles, K
    splits and variants) and the picker's own choice."""
    cands = []
    arr = (mm.Plan * 64)()
    n = mm.lib().maxmulsk_candidates(1, arr, 64)
    for p in arr[:n]:
        if prec == mm.Precision.BF16X9 and p.precision == mm.Precision.BF16X6:
            cands.append(mm.make_plan(prec, p.tile_m, p.tile_n, p.split_k, p.variant))
        elif p.precision == prec:
            cands.append(mm.make_plan(p.precision, p.tile_m, p.tile_n, p.split_k, p.variant))
    return cands


@pytest.mark.parametrize("cell", _cells(), ids=lambda c: f"{c[0]}-{c[1]}x{c[2]}x{c[3]}")
def test_split_modes_within_twice_plain_fp32_at_every_cell(cuda, cell):
    torch = cuda
    kind, M, K, N = cell
    A, B = _inputs(kind, M, K, N)
    dA, dB = to_dev(torch, A), to_dev(torch, B)
    chk = mm.Fp64Check(dA, dB, M, K, N)
    dC = torch.empty(M * N, device="cuda")

    def err_of(plan):
        nb = mm.workspace_bytes(M, K, N, plan)
        ws = torch.empty(nb + 256, dtype=torch.uint8, device="cuda")
        wp = ws.data_ptr() + ((-ws.data_ptr()) % 256)
        st = mm.sgemm_plan_dev(dA, dB, dC, M, K, N, plan, wp, nb)
        assert st == 0 and mm.stream_status() == 0, (plan, mm.last_error_message())
        return chk.errors(dC)["normwise"]

    plain = err_of(mm.make_plan(mm.Precision.FP32, 128, 128, 1))
    picked_simt = err_of(mm.choose(M, K, N, mm.Precision.FP32))
    worst = {}
    for prec in MODES:
        plans = _plans_of_mode(prec) + [mm.choose(M, K, N, prec)]
        for plan in plans:
            if mm.classify(M, K, N, plan) != 0:
                continue
            e = err_of(plan)
            assert e <= 2.0 * plain, (cell, plan, e, plain)
            worst[int(prec)] = max(worst.get(int(prec), 0.0), e)
        # the drop-in entry for split precision (the picker's plan)
        assert mm.sgemm_split_dev(dA, dB, dC, M, K, N, prec) == 0 and mm.stream_status() == 0
        e = chk.errors(dC)["normwise"]
        assert e <= 2.0 * plain, (cell, int(prec), e, plain)
    print(cell, "plain", plain, "picked SIMT", picked_simt,
          {k: (v, v / plain, v / picked_simt) for k, v in worst.items()})


# --------------------------------------------------------------------------- exact product sets
PIN_TILES = [(128, 64), (128, 128), (128, 256), (256, 128), (256, 256)]


@pytest.mark.parametrize("prec", MODES)
@pytest.mark.parametrize("side", ["a", "b"])
def test_product_set_pinned_exactly(cuda, oracle_mod, prec, side):
    torch = cuda
    rng = np.random.default_rng(100 + int(prec) * 10 + (side == "b"))
    levels = [1] if prec == mm.Precision.TF32X3 else [1, 2]
    for level in levels:
        for (M, K, N) in [(130, 64, 200), (64, 32, 64), (257, 64, 36)]:
            A, B = _pinning_inputs(rng, M, K, N, prec, side, level)
            want = oracle_mod.sgemm_split_exact(A, B, M, K, N, int(prec))
            # the exact split product differs from the full product here:
            # the pins would catch a mode that computed more (or fewer) pairs
            dA, dB = to_dev(torch, A), to_dev(torch, B)
            for tile in PIN_TILES:
                variants = [mm.TC_SPLIT_INPUTS]
                if prec != mm.Precision.TF32X3 and tile == (128, 128):
                    variants.append(mm.TC_FUSED_SPLIT)
                for var in variants:
                    for sk in (1, 2):
                        plan = mm.make_plan(prec, tile[0], tile[1], sk, var)
                        st, C, bands = run_plan(torch, A, B, M, K, N, plan, dA=dA, dB=dB)
                        assert st == 0 and bands, (plan, mm.last_error_message())
                        assert np.array_equal(bits(C), bits(want)), (int(prec), side, level, (M, K, N), plan)
