"""Failure detection on the GPU without a fault: every wait in this library's
kernels is bounded, and a wait that runs out records MAXMULSK_ERR_TIMEOUT in
the device error word instead of hanging. Here a probe kernel waits on a
barrier that nothing completes, with a limit of about a millisecond; the host
reads the status, and the context stays usable for the next GEMM."""
import numpy as np
import pytest

import maxmulsk_b200 as mm
from gpu_util import bits, run_plan

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_timeout_and_the_context_stays_usable(cuda, oracle_mod):
    assert mm.lib().maxmulsk_probe_timeout_dev(2_000_000, None) == 0
    assert mm.stream_status() == mm.Status.ERR_TIMEOUT
    assert mm.stream_status() == mm.Status.OK                 # the error word was cleared
    M, K, N = 96, 200, 80
    A = oracle_mod.fill_uniform(M * K, 601)
    B = oracle_mod.fill_uniform(K * N, 602)
    st, C, bands = run_plan(cuda, A, B, M, K, N, mm.make_plan(mm.Precision.FP32, 64, 64, 1))
    assert st == 0 and bands
    want = oracle_mod.sgemm_panels(A, B, M, K, N, kc=0, fma=True)
    assert np.array_equal(bits(C), bits(want))


def test_timeout_probe_rejects_out_of_range_limits(cuda):
    assert mm.lib().maxmulsk_probe_timeout_dev(0, None) == mm.Status.ERR_INVALID
    assert mm.lib().maxmulsk_probe_timeout_dev(3_000_000_000, None) == mm.Status.ERR_INVALID
