"""The allocation-free entry point, maxmulsk_sgemm_plan_static_dev.

It exists for callers that cannot allocate device memory when they call (a
host application that owns the device memory budget and forbids plug-ins to
call cudaMalloc, or a latency-critical loop that cannot afford cudaMalloc and
cudaFree). It runs the FP32 SIMT split-K plan with its scratch in a static
device array instead of a workspace.

Its output must equal the workspace entry point's (maxmulsk_sgemm_plan_dev,
same plan) bit for bit, the bar every SIMT test here uses, on two calls in a
row with different inputs (the array keeps the previous call's contents, so
the second call shows nothing stale survives). This file is named to be
collected last, and passes alone in a fresh process or after the others.
"""
import ctypes

import numpy as np
import pytest

import maxmulsk_b200 as mm

pytestmark = pytest.mark.gpu

STATIC_BYTES = 16 << 20   # MAXMULSK_STATIC_SCRATCH_BYTES


def _static_call(dA, dB, dC, M, K, N, plan):
    return mm.lib().maxmulsk_sgemm_plan_static_dev(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), M, K, N,
                                                   ctypes.byref(plan), None)


def _workspace_call(torch, dA, dB, dC, M, K, N, plan):
    nb = mm.workspace_bytes(M, K, N, plan)
    ws = torch.empty(nb + 256, dtype=torch.uint8, device="cuda")
    wp = ws.data_ptr() + ((-ws.data_ptr()) % 256)
    st = mm.sgemm_plan_dev(dA, dB, dC, M, K, N, plan, wp, nb)
    torch.cuda.synchronize()
    return st


def test_static_scratch_matches_workspace_entry_on_two_calls(cuda, oracle_mod):
    torch = cuda
    M, K, N = 128, 8192, 512                  # a narrow-M shape of the reference's sweep
    plan = mm.make_plan(mm.Precision.FP32, 64, 64, 16)
    assert 0 < mm.workspace_bytes(M, K, N, plan) <= STATIC_BYTES
    sc = 1.0 / np.sqrt(K)
    for call, (sa, sb) in enumerate([(11, 12), (13, 14)]):
        A = oracle_mod.fill_normal(M * K, sa, sc)
        B = oracle_mod.fill_normal(K * N, sb, sc)
        dA = torch.from_numpy(A).cuda()
        dB = torch.from_numpy(B).cuda()
        d_static = torch.full((M * N,), 3.75, device="cuda")
        d_ws = torch.full((M * N,), -1.0, device="cuda")
        assert _static_call(dA, dB, d_static, M, K, N, plan) == 0, mm.last_error_message()
        assert mm.stream_status() == 0
        assert _workspace_call(torch, dA, dB, d_ws, M, K, N, plan) == 0
        got = d_static.cpu().numpy()
        want = d_ws.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"call {call}"


def _static_with_bands(torch, dA, dB, M, K, N, plan, guard=64):
    """The static entry with C between guard bands of the sentinel (3.75, the
    reference checker's marker, check_nb.cpp:54); returns (status, C, bands intact)."""
    buf = torch.full((M * N + 2 * guard,), 3.75, dtype=torch.float32, device="cuda")
    st = mm.lib().maxmulsk_sgemm_plan_static_dev(dA.data_ptr(), dB.data_ptr(), buf.data_ptr() + 4 * guard, M, K, N,
                                                 ctypes.byref(plan), None)
    st2 = mm.stream_status()
    host = buf.cpu().numpy()
    C = host[guard: guard + M * N].copy()
    bands = bool(np.all(host[:guard] == 3.75) and np.all(host[guard + M * N:] == 3.75))
    return (st if st != 0 else st2), C, bands


@pytest.mark.parametrize("plan_args", [(64, 64, 7), (128, 64, 3), (128, 128, 1), (64, 64, 1)])
def test_static_scratch_edges_and_no_split(cuda, oracle_mod, plan_args):
    # An odd shape (scalar loads and stores: K and N not multiples of 4,
    # partial tiles in M and N) with and without a K split, twice with new
    # inputs: the same bits as the workspace entry, nothing written outside C.
    from gpu_util import run_plan
    torch = cuda
    M, K, N = 97, 1000, 83
    plan = mm.make_plan(mm.Precision.FP32, *plan_args)
    assert mm.workspace_bytes(M, K, N, plan) <= STATIC_BYTES
    for seeds in ((21, 22), (23, 24)):
        A = oracle_mod.fill_uniform(M * K, seeds[0])
        B = oracle_mod.fill_wide(K * N, seeds[1])
        dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
        st, got, bands = _static_with_bands(torch, dA, dB, M, K, N, plan)
        assert st == 0 and bands, mm.last_error_message()
        st2, want, bands2 = run_plan(torch, A, B, M, K, N, plan, dA=dA, dB=dB)
        assert st2 == 0 and bands2
        assert np.array_equal(got.view(np.uint32), want.ravel().view(np.uint32)), (plan_args, seeds)


def test_static_scratch_rejects_plans_beyond_its_size(cuda, oracle_mod):
    torch = cuda
    M, K, N = 512, 8192, 1024
    plan = mm.make_plan(mm.Precision.FP32, 64, 64, 16)   # 16 partial C's of 2 MiB: 32 MiB
    assert mm.workspace_bytes(M, K, N, plan) > STATIC_BYTES
    dA = torch.zeros(M * K, device="cuda")
    dB = torch.zeros(K * N, device="cuda")
    dC = torch.full((M * N,), 9.0, device="cuda")
    assert _static_call(dA, dB, dC, M, K, N, plan) == mm.Status.ERR_UNSUPPORTED
    torch.cuda.synchronize()
    assert bool((dC == 9.0).all())
    assert "static" in mm.last_error_message()
