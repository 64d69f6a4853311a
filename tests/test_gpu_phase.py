"""Phase timing on the GPU (maxmulsk_phase_timing / maxmulsk_phase_report),
the counterpart of the reference's lab hooks and per-phase timing breakdown
(sme/support/lab_hooks.hpp:1-22, sme/support/test_sme.cpp:580-678): each
call records device time for the phases it runs -- and only those -- and the
results do not change with the timing on."""
import numpy as np
import pytest

import maxmulsk_b200 as mm
from gpu_util import bits, run_plan, to_dev

pytestmark = pytest.mark.gpu


def test_phases_recorded_per_call(cuda, oracle_mod):
    torch = cuda
    M, K, N = 512, 2048, 384
    A = oracle_mod.fill_uniform(M * K, 1)
    B = oracle_mod.fill_uniform(K * N, 2)
    dA, dB = to_dev(torch, A), to_dev(torch, B)
    split4 = mm.make_plan(mm.Precision.BF16X6, 128, 128, 4)
    _, C_off, _ = run_plan(torch, A, B, M, K, N, split4, dA=dA, dB=dB)
    mm.phase_report()                         # forget anything recorded before
    mm.phase_timing(True)
    try:
        # split precision, 4 K slices: pre-pass, GEMM, split-K reduction
        st, C_on, ok = run_plan(torch, A, B, M, K, N, split4, dA=dA, dB=dB)
        assert st == 0 and ok
        rep = mm.phase_report()
        assert set(rep) == {"split", "gemm", "reduce"}, rep
        assert all(v["calls"] == 1 and v["ms"] > 0 for v in rep.values()), rep
        assert np.array_equal(bits(C_on), bits(C_off))

        # FP32 SIMT without a K split: the GEMM only
        st, _, ok = run_plan(torch, A, B, M, K, N, mm.make_plan(mm.Precision.FP32, 128, 128, 1), dA=dA, dB=dB)
        assert st == 0 and ok
        assert set(mm.phase_report()) == {"gemm"}

        # host entry point: copies up, the GEMM, the copy down
        C_host = np.empty(M * N, np.float32)
        assert mm.sgemm_v3(A, B, C_host, M, K, N) == 0, mm.last_error_message()
        rep = mm.phase_report()
        assert {"h2d", "gemm", "d2h"} <= set(rep) <= {"h2d", "gemm", "reduce", "d2h"}, rep
        dC = torch.empty(M * N, device="cuda")
        assert mm.sgemm_v3_dev(dA, dB, dC, M, K, N) == 0
        assert np.array_equal(bits(C_host), bits(dC.cpu().numpy()))
        mm.phase_report()

        # a grouped batch: one "grouped" phase per launch, none from its capture
        probs = [(dA, dB, torch.empty(M * N, device="cuda"), M, K, N),
                 (dA, dB, torch.empty(M * N, device="cuda"), M, K, N)]
        g = mm.Grouped(probs)
        try:
            assert mm.phase_report() == {}
            assert g.launch() == 0 and g.launch() == 0
            rep = mm.phase_report()
            assert set(rep) == {"grouped"} and rep["grouped"]["calls"] == 2, rep
        finally:
            g.close()
    finally:
        mm.phase_timing(False)
    run_plan(torch, A, B, M, K, N, split4, dA=dA, dB=dB)
    assert mm.phase_report() == {}
