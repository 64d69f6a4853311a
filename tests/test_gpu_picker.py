"""The cost model's CUDA kernels against the FP64 oracle, GPU inference
against the host forward pass, and the exhaustive autotuner."""
import ctypes

import numpy as np
import pytest

import maxmulsk_b200 as mm
from maxmulsk_b200 import autotune, picker

pytestmark = pytest.mark.gpu


def test_backward_kernels_match_oracle_gradient(cuda):
    from oracle import mlp_ref
    torch = cuda
    rng = np.random.default_rng(3)
    B = 37
    p = rng.normal(0, 0.3, picker.NPARAM).astype(np.float32)
    X = rng.uniform(0, 1, (B, picker.F)).astype(np.float32)
    T = rng.normal(2, 1, (B, picker.O)).astype(np.float32)
    mask = (rng.random((B, picker.O)) > 0.25).astype(np.float32)
    L_ref, g_ref = mlp_ref.loss_and_grad(p.astype(np.float64), X.astype(np.float64), T, mask, float(mask.sum()))
    dp, dX, dT, dM = (torch.from_numpy(a).cuda() for a in (p, X, T, mask))
    Z1, H1, Z2, H2 = (torch.empty(B * picker.H, device="cuda") for _ in range(4))
    Y = torch.empty(B * picker.O, device="cuda")
    g = torch.empty(picker.NPARAM, device="cuda")
    work = torch.empty(B * (picker.O + 2 * picker.H), device="cuda")
    rl = torch.empty(B, device="cuda")
    L = mm.lib()
    assert L.maxmulsk_mlp_forward_dev(dp.data_ptr(), dX.data_ptr(), B, Z1.data_ptr(), H1.data_ptr(), Z2.data_ptr(),
                                      H2.data_ptr(), Y.data_ptr(), None) == 0
    assert L.maxmulsk_mlp_backward_dev(dp.data_ptr(), dX.data_ptr(), Z1.data_ptr(), H1.data_ptr(), Z2.data_ptr(),
                                       H2.data_ptr(), Y.data_ptr(), dT.data_ptr(), dM.data_ptr(), B,
                                       float(mask.sum()), g.data_ptr(), work.data_ptr(), rl.data_ptr(), None) == 0
    torch.cuda.synchronize()
    gg = g.cpu().numpy().astype(np.float64)
    assert abs(rl.sum().item() / mask.sum() - L_ref) <= 1e-4 * abs(L_ref)
    assert np.linalg.norm(gg - g_ref) <= 1e-4 * np.linalg.norm(g_ref)
    Yr = mlp_ref.forward(p.astype(np.float64), X.astype(np.float64))[-1]
    assert np.max(np.abs(Y.cpu().numpy().reshape(B, -1) - Yr)) < 1e-4


def test_adam_training_reduces_loss_and_gpu_inference_matches_host(cuda, tmp_path):
    rng = np.random.default_rng(4)
    X = rng.uniform(0, 1, (300, picker.F)).astype(np.float32)
    W = rng.normal(0, 1, (picker.F, picker.O))
    T = (X @ W + 3).astype(np.float32)
    mask = np.ones_like(T)
    tr = picker.Trainer(seed=1, out_bias=3.0)
    losses = tr.fit(X, T, mask, steps=400, lr=3e-3, log_every=100)
    assert losses[-1] < 0.1 * losses[0]
    Y, best = tr.predict(X[:20], mask[:20])
    assert np.array_equal(best, np.argmin(Y, axis=1))
    path = str(tmp_path / "m.bin")
    tr.save(path)
    assert mm.lib().maxmulsk_model_load(path.encode()) == 0
    try:
        out = (ctypes.c_float * picker.O)()
        for (M, K, N, cls) in [(1, 5000, 700, 0), (4096, 4096, 4096, 1)]:
            x = picker.features([(M, K, N)], cls)
            yg, _ = tr.predict(x, np.ones((1, picker.O), np.float32))
            assert mm.lib().maxmulsk_mlp_predict_host(M, K, N, cls, out) == 0
            assert np.max(np.abs(np.array(out) - yg[0])) < 1e-4
    finally:
        mm.lib().maxmulsk_model_load(None)


def test_autotuner_times_candidates_and_fills_the_database(cuda, tmp_path):
    torch = cuda
    M, K, N = 200, 3000, 300
    dA = torch.rand(M * K, device="cuda"); dB = torch.rand(K * N, device="cuda"); dC = torch.empty(M * N, device="cuda")
    ws = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    wp = ws.data_ptr() + ((-ws.data_ptr()) % 256)
    c0 = autotune.candidates(0)
    t = autotune.time_plans(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), M, K, N, c0, wp, (256 << 20) - 256)
    assert np.all(np.isfinite(t)) and np.all(t > 0)
    mm.lib().maxmulsk_tuning_clear()
    best = mm.Plan()
    us = ctypes.c_float()
    for prec in (mm.Precision.FP32, mm.Precision.SPLIT_AUTO):
        assert mm.lib().maxmulsk_autotune_dev(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), M, K, N, int(prec), wp,
                                              (256 << 20) - 256, ctypes.byref(best), ctypes.byref(us), None) == 0
        assert us.value > 0
        got = mm.choose(M, K, N, prec)
        assert got.as_tuple() == best.as_tuple()
    path = str(tmp_path / "db.txt")
    assert mm.lib().maxmulsk_tuning_save(path.encode()) == 2
    mm.lib().maxmulsk_tuning_clear()
    assert mm.lib().maxmulsk_tuning_load(path.encode()) == 2
    assert mm.choose(M, K, N, mm.Precision.FP32).as_tuple() == mm.choose(M, K, N, 0).as_tuple()
    mm.lib().maxmulsk_tuning_clear()


def test_trained_picker_regret_on_held_out_shapes(cuda):
    # The learned picker end to end: the MLP trained by the library's CUDA
    # forward/backward/Adam kernels on the autotuner's measured timings of
    # 2000 random shapes (M, N, K log-uniform in [1, 16384]; both classes),
    # then evaluated on the 500 held-out shapes against exhaustive search (the
    # seed is chosen on a validation part of the training shapes). Bar:
    # within 5% of exhaustive time per shape (mean, geometric mean) and in
    # total, and better than the hand-written rule it replaces, timed in the
    # same run.
    import os
    d = dict(np.load(os.path.join(os.path.dirname(picker.__file__), "data", "picker_timings.npz")))
    assert int(d["n_train"]) == 2000 and len(d["shapes"]) == 2500
    trainer, losses, r_mlp, r_rule = picker.train_and_evaluate(d)
    print("MLP", r_mlp, "rule", r_rule)
    assert losses[-1] < 0.2 * losses[0]
    assert r_mlp["rows"] == r_rule["rows"] == 1000
    assert r_mlp["mean"] <= 0.05 and r_mlp["geomean"] <= 0.05 and r_mlp["total_time"] <= 0.05, r_mlp
    assert r_mlp["total_time"] < r_rule["total_time"] and r_mlp["geomean"] < r_rule["geomean"], (r_mlp, r_rule)


# --------------------------------------------------------------------------- exhaustive search as the fallback
def _shipped_model():
    import os
    return os.path.join(os.path.dirname(picker.__file__), "data", "picker_model.bin").encode()


def _db_entries(tmp_path) -> int:
    path = str(tmp_path / "db_count.txt")
    return int(mm.lib().maxmulsk_tuning_save(path.encode()))


def _rand(torch, n):
    return torch.rand(n, device="cuda") * 2 - 1


@pytest.fixture
def clean_picker(monkeypatch):
    for v in ("MAXMULSK_AUTOTUNE", "MAXMULSK_AUTOTUNE_MARGIN", "MAXMULSK_CONFIG"):
        monkeypatch.delenv(v, raising=False)
    mm.lib().maxmulsk_tuning_clear()
    yield
    mm.lib().maxmulsk_tuning_clear()
    assert mm.lib().maxmulsk_model_load(_shipped_model()) == 0


def test_fallback_searches_without_a_model(cuda, clean_picker, tmp_path):
    # No learned model: the device entry searches the candidates on its own
    # operands, stores the winner, and runs it; the query then returns it.
    torch = cuda
    M, K, N = 300, 1500, 260
    mm.lib().maxmulsk_model_load(None)
    assert mm.picker_doubt(M, K, N) == "no learned model"
    rule = mm.choose(M, K, N).as_tuple()
    assert rule == mm.choose_rule(M, K, N).as_tuple()
    dA, dB, dC = _rand(torch, M * K), _rand(torch, K * N), torch.empty(M * N, device="cuda")
    assert mm.sgemm_v3_dev(dA, dB, dC, M, K, N) == 0 and mm.stream_status() == 0
    assert _db_entries(tmp_path) == 1
    assert mm.picker_doubt(M, K, N) is None                  # the database decides from now on
    tuned = mm.choose(M, K, N)
    # the call ran the stored plan: same bits as that plan run explicitly
    dC2 = torch.empty(M * N, device="cuda")
    nb = mm.workspace_bytes(M, K, N, tuned)
    ws = torch.empty(nb + 256, dtype=torch.uint8, device="cuda")
    assert mm.sgemm_plan_dev(dA, dB, dC2, M, K, N, tuned, ws.data_ptr() + ((-ws.data_ptr()) % 256), nb) == 0
    assert bool(torch.equal(dC, dC2))
    # split precision takes the same route (its own database key)
    assert mm.sgemm_split_dev(dA, dB, dC, M, K, N, mm.Precision.SPLIT_AUTO) == 0 and mm.stream_status() == 0
    assert _db_entries(tmp_path) == 2


def test_fallback_searches_outside_the_trained_range(cuda, clean_picker, tmp_path):
    torch = cuda
    M, K, N = 48, 20000, 40
    assert mm.picker_doubt(M, K, N) == "shape outside the trained range"
    dA, dB, dC = _rand(torch, M * K), _rand(torch, K * N), torch.empty(M * N, device="cuda")
    assert mm.sgemm_v3_dev(dA, dB, dC, M, K, N) == 0 and mm.stream_status() == 0
    assert _db_entries(tmp_path) == 1


def test_fallback_on_close_calls_and_its_switch(cuda, clean_picker, monkeypatch, tmp_path):
    torch = cuda
    M, K, N = 200, 700, 180
    dA, dB, dC = _rand(torch, M * K), _rand(torch, K * N), torch.empty(M * N, device="cuda")
    monkeypatch.setenv("MAXMULSK_AUTOTUNE_MARGIN", "0")          # the model decides
    assert mm.sgemm_v3_dev(dA, dB, dC, M, K, N) == 0 and mm.stream_status() == 0
    assert _db_entries(tmp_path) == 0
    monkeypatch.setenv("MAXMULSK_AUTOTUNE_MARGIN", "100")        # every shape is a close call
    monkeypatch.setenv("MAXMULSK_AUTOTUNE", "0")                 # ... but the fallback is off
    assert mm.sgemm_v3_dev(dA, dB, dC, M, K, N) == 0 and mm.stream_status() == 0
    assert _db_entries(tmp_path) == 0
    monkeypatch.delenv("MAXMULSK_AUTOTUNE")
    C_host = np.empty(M * N, np.float32)                          # the host entry searches too
    assert mm.sgemm_v3(dA.cpu().numpy(), dB.cpu().numpy(), C_host, M, K, N) == 0, mm.last_error_message()
    assert _db_entries(tmp_path) == 1


def test_fallback_never_runs_inside_a_stream_capture(cuda, clean_picker, monkeypatch, tmp_path):
    # A caller capturing its stream into a CUDA graph gets the model's (here,
    # with no model, the rule's) plan captured; nothing is timed or
    # synchronised during the capture, and the database stays empty.
    torch = cuda
    M, K, N = 160, 900, 96
    mm.lib().maxmulsk_model_load(None)
    dA, dB, dC = _rand(torch, M * K), _rand(torch, K * N), torch.empty(M * N, device="cuda")
    s = torch.cuda.Stream()
    # first call outside the capture with the search off: sizes the stream's workspace
    monkeypatch.setenv("MAXMULSK_AUTOTUNE", "0")
    assert mm.sgemm_v3_dev(dA, dB, dC, M, K, N, s) == 0
    torch.cuda.synchronize()
    want = dC.clone()
    monkeypatch.delenv("MAXMULSK_AUTOTUNE")
    assert mm.picker_doubt(M, K, N) == "no learned model"
    dC.zero_()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        st = mm.sgemm_v3_dev(dA, dB, dC, M, K, N, s)
    assert st == 0
    assert _db_entries(tmp_path) == 0
    g.replay()
    torch.cuda.synchronize()
    assert bool(torch.equal(dC, want))
    del g


def test_config_env_reaches_the_kernel(cuda, oracle_mod, clean_picker, monkeypatch):
    # MAXMULSK_CONFIG (the counterpart of MAXMULSK_BLOCKING,
    # sme/support/gemm_tuning.cpp:66-78) decides what maxmulsk_sgemm_v3 runs:
    # a 3-slice FP32 plan gives the oracle's 3-panel sum bit for bit; a
    # malformed value is ignored.
    M, K, N = 150, 1000, 90
    A = oracle_mod.fill_uniform(M * K, 5)
    B = oracle_mod.fill_uniform(K * N, 6)
    monkeypatch.setenv("MAXMULSK_CONFIG", "0,64,64,3")
    C = np.empty(M * N, np.float32)
    assert mm.sgemm_v3(A, B, C, M, K, N) == 0
    want = oracle_mod.sgemm_panels(A, B, M, K, N, kc=mm.slice_len(K, 3), fma=True)
    assert np.array_equal(C.view(np.uint32), want.ravel().view(np.uint32))
    monkeypatch.setenv("MAXMULSK_CONFIG", "0,64,64")
    monkeypatch.setenv("MAXMULSK_AUTOTUNE", "0")
    plan = mm.choose(M, K, N)
    C2 = np.empty(M * N, np.float32)
    assert mm.sgemm_v3(A, B, C2, M, K, N) == 0
    want2 = oracle_mod.sgemm_panels(A, B, M, K, N, kc=mm.slice_len(K, plan.split_k), fma=True)
    assert np.array_equal(C2.view(np.uint32), want2.ravel().view(np.uint32))


def test_live_regret_on_fresh_shapes(cuda, clean_picker):
    # The learned picker against exhaustive search, both timed now on this
    # GPU (the regret test above scores the committed timing table): 20 fresh
    # shapes, M, N, K log-uniform in [1, 16384] (product capped so the search
    # stays short), FP32 and split precision.
    from maxmulsk_b200 import workloads
    torch = cuda
    shapes = [s for s in workloads.picker_shapes(400, seed=9091) if s[0] * s[1] * s[2] <= 2 ** 35][:20]
    ws_bytes = 1 << 30
    ws = torch.empty(ws_bytes + 256, dtype=torch.uint8, device="cuda")
    wp = ws.data_ptr() + ((-ws.data_ptr()) % 256)
    regrets = {0: [], 1: []}
    totals = {0: [0.0, 0.0], 1: [0.0, 0.0]}
    for (M, K, N) in shapes:
        dA, dB, dC = _rand(torch, M * K), _rand(torch, K * N), torch.empty(M * N, device="cuda")
        for cls, prec in ((0, mm.Precision.FP32), (1, mm.Precision.SPLIT_AUTO)):
            cands = autotune.candidates(cls)
            t = autotune.time_plans(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), M, K, N, cands, wp, ws_bytes)
            pick = mm.choose(M, K, N, prec).as_tuple()
            idx = [i for i, c in enumerate(cands) if c.as_tuple() == pick]
            if idx and np.isfinite(t[idx[0]]):
                t_pick = float(t[idx[0]])
            else:   # the rule's plan, outside the candidate list: time it alone
                t_pick = float(autotune.time_plans(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), M, K, N,
                                                   [mm.choose(M, K, N, prec)], wp, ws_bytes)[0])
            best = float(np.min(t[np.isfinite(t)]))
            regrets[cls].append(t_pick / best - 1.0)
            totals[cls][0] += t_pick
            totals[cls][1] += best
    for cls in (0, 1):
        r = np.array(regrets[cls])
        total = totals[cls][0] / totals[cls][1] - 1.0
        print(f"class {cls}: {len(r)} shapes, mean regret {r.mean():.3f}, median {np.median(r):.3f}, "
              f"total-time {total:.3f}")
        # single live timings carry a few per cent of noise on both sides
        assert total <= 0.10 and r.mean() <= 0.10, (cls, r, total)
