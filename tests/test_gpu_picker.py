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
