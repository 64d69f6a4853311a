"""Grouped launch (one persistent kernel over many GEMMs, replayed from a CUDA
graph) against the oracle: every problem bit for bit equal to the oracle's
panel sum with that problem's K split, like a per-GEMM launch; C regions
between problems untouched; graph replays identical. The counterpart of the
reference's run_batch (sme/v3/sme-1x4-acc-kcout-onestream.hpp:61-63)."""
import numpy as np
import pytest

import maxmulsk_b200 as mm
from maxmulsk_b200 import workloads
from gpu_util import run_plan

pytestmark = pytest.mark.gpu

SENT = 3.75


def _group(cuda, oracle_mod, shapes, seed, plan=None):
    torch = cuda
    problems, host, offs = [], [], []
    total = sum(m * n for m, k, n in shapes) + 64 * (len(shapes) + 1)
    cbuf = torch.full((total,), SENT, device="cuda")
    off = 64
    for i, (M, K, N) in enumerate(shapes):
        A = oracle_mod.fill_uniform(M * K, seed + 2 * i) if M * K else np.zeros(1, np.float32)
        B = oracle_mod.fill_uniform(K * N, seed + 2 * i + 1) if K * N else np.zeros(1, np.float32)
        dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
        problems.append((dA, dB, cbuf.data_ptr() + 4 * off, M, K, N))
        host.append((A, B))
        offs.append(off)
        off += M * N + 64
    g = mm.Grouped(problems, plan)
    return g, cbuf, host, offs


def _check(cuda, oracle_mod, g, cbuf, host, offs, shapes):
    plan, splits, _ = g.info()
    plans = g.plans()
    assert [p.split_k for p in plans] == list(splits)
    assert all(p.precision == 0 and (p.tile_m, p.tile_n) == (plan.tile_m, plan.tile_n) for p in plans)
    c = cbuf.cpu().numpy()
    mask = np.ones(c.size, bool)
    for (M, K, N), (A, B), off, s in zip(shapes, host, offs, splits):
        got = c[off: off + M * N].reshape(M, N)
        mask[off: off + M * N] = False
        if M * N == 0:
            continue
        if K == 0:
            assert np.all(got == 0)
            continue
        want = oracle_mod.sgemm_panels(A, B, M, K, N, kc=mm.slice_len(K, s), fma=plan.variant == 0)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), ((M, K, N), s)
    assert np.all(c[mask] == SENT), "a grouped launch wrote outside its C matrices"


MIXED = [(1, 700, 3), (37, 5, 129), (128, 1024, 128), (67, 67, 67), (300, 2049, 90), (1, 8192, 1024),
         (511, 640, 512), (20, 35, 41), (0, 16, 16), (16, 0, 16), (129, 4000, 257), (3, 999, 1000)]


@pytest.mark.parametrize("tile", [None, (128, 128), (128, 64), (64, 64)])
def test_grouped_bit_exact_and_contained(cuda, oracle_mod, tile):
    plan = None if tile is None else mm.make_plan(0, tile[0], tile[1], 0)
    g, cbuf, host, offs = _group(cuda, oracle_mod, MIXED, 100, plan)
    assert g.launch() == 0
    assert mm.stream_status() == 0
    _check(cuda, oracle_mod, g, cbuf, host, offs, MIXED)
    g.close()


def test_grouped_graph_replays_identically(cuda, oracle_mod):
    shapes = MIXED[:8]
    g, cbuf, host, offs = _group(cuda, oracle_mod, shapes, 300)
    assert g.launch() == 0
    cuda.cuda.synchronize()
    first = cbuf.clone()
    for off, (M, K, N) in zip(offs, shapes):
        cbuf[off: off + M * N] = -7.0
    for _ in range(3):
        assert g.launch() == 0
    cuda.cuda.synchronize()
    assert bool(cuda.equal(first, cbuf))
    g.close()


def test_grouped_scalar_variant_and_fixed_split(cuda, oracle_mod):
    plan = mm.make_plan(0, 64, 64, 3, mm.FP32_SCALAR)
    g, cbuf, host, offs = _group(cuda, oracle_mod, MIXED, 500, plan)
    _, splits, _ = g.info()
    assert all(s == 3 or s == 1 for s in splits)
    assert g.launch() == 0
    cuda.cuda.synchronize()
    _check(cuda, oracle_mod, g, cbuf, host, offs, MIXED)


def test_grouped_benchmark_batch_sampled(cuda, oracle_mod):
    # The grouped batch of the benchmark (256 GEMMs); the FP64 error of a
    # sample of problems is FP32-class and every problem's C is written (C is
    # prefilled with NaN: with 38 M random outputs a finite marker such as
    # 3.75 would also come out of the products now and then).
    torch = cuda
    shapes = workloads.grouped_problems()
    probs, As, Bs, Cs = [], [], [], []
    for i, (M, K, N) in enumerate(shapes):
        a = torch.rand(M * K, device="cuda") * 2 - 1
        b = torch.rand(K * N, device="cuda") * 2 - 1
        c = torch.full((M * N,), float("nan"), device="cuda")
        probs.append((a, b, c, M, K, N))
        As.append(a); Bs.append(b); Cs.append(c)
    g = mm.Grouped(probs)
    assert g.launch() == 0
    assert mm.stream_status() == 0
    rng = np.random.default_rng(0)
    for i in rng.choice(len(shapes), 12, replace=False):
        M, K, N = shapes[i]
        err = mm.Fp64Check(As[i], Bs[i], M, K, N, with_abs=False).errors(Cs[i])["normwise"]
        assert err < 4 * 2.0 ** -24 * np.sqrt(K), (shapes[i], err)
    for c in Cs:
        assert not bool(torch.isnan(c).any())
    g.close()


# N not a multiple of 4 (129) runs in the FP32 part of the group; K not a
# multiple of 4 (5, 999) with a readable B runs on the tensor cores from a
# repacked copy of A.
MIXED_TC = [(128, 1024, 128), (67, 68, 132), (300, 2048, 92), (1, 8192, 1024), (511, 640, 512), (20, 36, 40),
            (3, 1000, 1000), (129, 4000, 256), (37, 5, 129), (64, 999, 100), (0, 16, 16), (16, 0, 16)]


@pytest.mark.parametrize("prec", [mm.Precision.BF16X6, mm.Precision.BF16X9])
def test_grouped_split_precision_matches_single_launches(cuda, oracle_mod, prec):
    # One persistent fused-split tcgen05 kernel over the group: each problem's
    # units are the tiles and K slices a single fused launch with the same K
    # split computes, with the same chunked accumulation and slice order, so
    # C is bit-identical to that launch (for K not a multiple of 4: to the
    # split-inputs launch, whose planes are zero-padded in K the same way).
    # Problems whose B the fused split cannot read run in the FP32 grouped
    # kernel of the same graph: bit-exact against the oracle's panel order.
    g, cbuf, host, offs = _group(cuda, oracle_mod, MIXED_TC, 700, mm.make_plan(prec, 128, 128, 0))
    plan, splits, units = g.info()
    assert plan.precision == int(prec) and plan.variant == mm.TC_FUSED_SPLIT and units > 0
    plans = g.plans()
    assert g.launch() == 0
    assert mm.stream_status() == 0
    c = cbuf.cpu().numpy()
    mask = np.ones(c.size, bool)
    for (M, K, N), (A, B), off, p in zip(MIXED_TC, host, offs, plans):
        got = c[off: off + M * N].reshape(M, N)
        mask[off: off + M * N] = False
        if M * N == 0:
            continue
        if K == 0:
            assert np.all(got == 0)
            continue
        if p.precision != 0:
            want_plan = p
            if p.variant == mm.TC_FUSED_SPLIT and K % 4:
                want_plan = mm.make_plan(p.precision, 128, 128, p.split_k, mm.TC_SPLIT_INPUTS)
            st, want, _ = run_plan(cuda, A, B, M, K, N, want_plan)
            assert st == 0
        else:
            assert N % 4 != 0
            want = oracle_mod.sgemm_panels(A, B, M, K, N, kc=mm.slice_len(K, p.split_k), fma=True)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), ((M, K, N), p)
    assert np.all(c[mask] == SENT), "a grouped launch wrote outside its C matrices"
    # replays reproduce the result
    first = cbuf.clone()
    for off, (M, K, N) in zip(offs, MIXED_TC):
        cbuf[off: off + M * N] = -7.0
    for _ in range(2):
        assert g.launch() == 0
    cuda.cuda.synchronize()
    assert bool(cuda.equal(first, cbuf))
    g.close()


def test_grouped_benchmark_batch_split_precision(cuda):
    # The benchmark's 256-GEMM batch with BF16x6: FP32-class FP64 error on a
    # sample, every C written (NaN prefill, as above).
    torch = cuda
    shapes = workloads.grouped_problems()
    probs, As, Bs, Cs = [], [], [], []
    for i, (M, K, N) in enumerate(shapes):
        a = torch.rand(M * K, device="cuda") * 2 - 1
        b = torch.rand(K * N, device="cuda") * 2 - 1
        c = torch.full((M * N,), float("nan"), device="cuda")
        probs.append((a, b, c, M, K, N))
        As.append(a); Bs.append(b); Cs.append(c)
    g = mm.Grouped(probs, mm.make_plan(mm.Precision.BF16X6, 128, 128, 0))
    assert g.launch() == 0
    assert mm.stream_status() == 0
    rng = np.random.default_rng(1)
    for i in rng.choice(len(shapes), 16, replace=False):
        M, K, N = shapes[i]
        err = mm.Fp64Check(As[i], Bs[i], M, K, N, with_abs=False).errors(Cs[i])["normwise"]
        assert err < 4 * 2.0 ** -24 * np.sqrt(K), (shapes[i], err)
    for c in Cs:
        assert not bool(torch.isnan(c).any())
    g.close()


def test_grouped_split_precision_big_problems_run_their_own_plans(cuda, oracle_mod):
    # A group with problems large enough to fill the GPU on their own: the
    # configuration search may run them as their own launches of their picked
    # plan inside the graph. Whatever it picks, every problem equals a single
    # launch of the plan maxmulsk_grouped_plans reports, bit for bit, and a
    # fixed split forces every problem onto the fused kernel.
    shapes = [(512, 4096, 3072), (384, 8192, 2048), (33, 2048, 512), (7, 512, 1024), (200, 1000, 2048),
              (129, 4096, 1024)]
    g, cbuf, host, offs = _group(cuda, oracle_mod, shapes, 900, mm.make_plan(mm.Precision.SPLIT_AUTO, 128, 128, 0))
    plans = g.plans()
    assert g.launch() == 0 and mm.stream_status() == 0
    c = cbuf.cpu().numpy()
    for (M, K, N), (A, B), off, p in zip(shapes, host, offs, plans):
        assert p.precision in (1, 2)
        st, want, _ = run_plan(cuda, A, B, M, K, N, p)
        assert st == 0
        assert np.array_equal(c[off: off + M * N].view(np.uint32), want.ravel().view(np.uint32)), ((M, K, N), p)
    g.close()
    g2, _, _, _ = _group(cuda, oracle_mod, shapes, 900, mm.make_plan(mm.Precision.BF16X6, 128, 128, 3))
    assert all(p.variant == mm.TC_FUSED_SPLIT and p.split_k == 3 for p in g2.plans())
    g2.close()
