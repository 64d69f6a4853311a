"""Cost-model pieces that need no GPU: the FP64 MLP oracle against finite
differences, the model file read by the library's host forward pass, the
features and the candidate lists."""
import ctypes
import math

import numpy as np
import pytest

import maxmulsk_b200 as mm
from maxmulsk_b200 import picker


def _oracle():
    from oracle import mlp_ref
    return mlp_ref


def test_oracle_gradient_matches_finite_differences():
    ref = _oracle()
    rng = np.random.default_rng(1)
    p = rng.normal(0, 0.3, picker.NPARAM)
    X = rng.uniform(0, 1, (5, picker.F))
    T = rng.normal(6, 1, (5, picker.O))
    mask = (rng.random((5, picker.O)) > 0.3).astype(float)
    L, g = ref.loss_and_grad(p, X, T, mask, mask.sum())
    for idx in rng.choice(picker.NPARAM, 25, replace=False):
        e = np.zeros_like(p); e[idx] = 1e-6
        num = (ref.loss_and_grad(p + e, X, T, mask, mask.sum())[0] -
               ref.loss_and_grad(p - e, X, T, mask, mask.sum())[0]) / 2e-6
        assert abs(num - g[idx]) <= 1e-6 + 1e-5 * abs(num), idx


def test_features_follow_their_definition(built_lib):
    x = picker.features([(3000, 77, 16384)], 1)[0]
    s = math.log(16384)
    want = [math.log(3000) / s, math.log(16384) / s, math.log(77) / s, 3000 % 16 / 16, 0.0, 77 % 16 / 16, 1.0]
    assert np.allclose(x, want, atol=1e-6)


def test_model_file_and_host_forward(built_lib, tmp_path):
    ref = _oracle()
    rng = np.random.default_rng(2)
    p = rng.normal(0, 0.2, picker.NPARAM).astype(np.float32)
    path = str(tmp_path / "m.bin")
    picker.save_params(path, p)
    assert mm.lib().maxmulsk_model_load(path.encode()) == 0
    try:
        for (M, K, N, cls) in [(1, 1, 1, 0), (4096, 4096, 4096, 1), (37, 16384, 512, 1), (500, 9, 3, 0)]:
            out = (ctypes.c_float * picker.O)()
            assert mm.lib().maxmulsk_mlp_predict_host(M, K, N, cls, out) == 0
            x = picker.features([(M, K, N)], cls)
            y = ref.forward(p.astype(np.float64), x.astype(np.float64))[-1][0]
            assert np.max(np.abs(np.array(out) - y)) < 1e-4
    finally:
        mm.lib().maxmulsk_model_load(None)
    out = (ctypes.c_float * picker.O)()
    assert mm.lib().maxmulsk_mlp_predict_host(8, 8, 8, 0, out) == mm.Status.ERR_UNSUPPORTED


def test_model_file_rejects_wrong_dims(built_lib, tmp_path):
    path = tmp_path / "bad.bin"
    path.write_bytes(b"MMSKMLP1" + np.array([7, 32, 48, 10], np.int32).tobytes() + b"\0" * 40)
    assert mm.lib().maxmulsk_model_load(str(path).encode()) == mm.Status.ERR_INVALID


def test_candidate_lists(built_lib):
    from maxmulsk_b200 import autotune
    c0, c1 = autotune.candidates(0), autotune.candidates(1)
    assert len(c0) == 24 and len(c1) == 48
    assert {p.precision for p in c0} == {0} and {p.precision for p in c1} == {1, 2}
    for p in c0 + c1:
        assert mm.classify(512, 512, 512, p) == mm.Status.OK


def _predict_in_fresh_process(env_value):
    import os
    import subprocess
    import sys
    env = dict(os.environ)
    env.pop("MAXMULSK_MODEL", None)
    if env_value is not None:
        env["MAXMULSK_MODEL"] = env_value
    code = ("import ctypes, maxmulsk_b200 as mm; out = (ctypes.c_float * 48)(); "
            "print(mm.lib().maxmulsk_mlp_predict_host(4096, 4096, 4096, 1, out))")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", code], env=env, cwd=root, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    return int(r.stdout.strip())


def test_default_model_beside_the_library(built_lib, tmp_path):
    # Unset MAXMULSK_MODEL: the weights shipped in maxmulsk_b200/data are
    # used; "none" turns the model off; a path names other weights.
    import os
    shipped = os.path.join(os.path.dirname(picker.__file__), "data", "picker_model.bin")
    if os.path.exists(shipped):
        assert _predict_in_fresh_process(None) == 0
    assert _predict_in_fresh_process("none") == mm.Status.ERR_UNSUPPORTED
    p = np.zeros(picker.NPARAM, np.float32)
    path = str(tmp_path / "zero.bin")
    picker.save_params(path, p)
    assert _predict_in_fresh_process(path) == 0


# --------------------------------------------------------------------------- MAXMULSK_CONFIG
# The counterpart of the reference's MAXMULSK_BLOCKING override
# (sme/support/gemm_tuning.cpp:66-78): a well-formed value wins over the
# picker, a malformed one is ignored.
SHAPE = (1000, 3000, 700)


def test_config_env_overrides_the_picker(built_lib, monkeypatch):
    M, K, N = SHAPE
    monkeypatch.delenv("MAXMULSK_CONFIG", raising=False)
    base_split = mm.choose(M, K, N, mm.Precision.BF16X6).as_tuple()
    monkeypatch.setenv("MAXMULSK_CONFIG", "2,256,256,4")
    assert mm.choose(M, K, N, mm.Precision.BF16X6).as_tuple() == (2, 256, 256, 4, 0)
    monkeypatch.setenv("MAXMULSK_CONFIG", "2,128,128,8,2")
    assert mm.choose(M, K, N, mm.Precision.BF16X6).as_tuple() == (2, 128, 128, 8, 2)
    # a configured plan of another precision leaves this precision's pick alone
    monkeypatch.setenv("MAXMULSK_CONFIG", "0,64,64,4")
    assert mm.choose(M, K, N, mm.Precision.BF16X6).as_tuple() == base_split
    assert mm.choose(M, K, N, mm.Precision.FP32).as_tuple() == (0, 64, 64, 4, 0)


@pytest.mark.parametrize("bad", ["", "2", "2,128,256", "a,b,c,d", "2,128,256,0", "2,0,256,4", "2,128,-1,4",
                                 ",,,", "2;128;256;4"])
def test_malformed_config_env_is_ignored(built_lib, monkeypatch, bad):
    M, K, N = SHAPE
    monkeypatch.delenv("MAXMULSK_CONFIG", raising=False)
    base = {p: mm.choose(M, K, N, p).as_tuple() for p in (mm.Precision.FP32, mm.Precision.BF16X6)}
    monkeypatch.setenv("MAXMULSK_CONFIG", bad)
    for p, want in base.items():
        assert mm.choose(M, K, N, p).as_tuple() == want, (bad, p)


# --------------------------------------------------------------------------- exhaustive fallback triggers
def _load_shipped_model():
    import os
    shipped = os.path.join(os.path.dirname(picker.__file__), "data", "picker_model.bin")
    assert mm.lib().maxmulsk_model_load(shipped.encode()) == 0


def test_picker_doubt_triggers(built_lib, monkeypatch):
    _load_shipped_model()
    # When the learned model is loaded and the shape is inside its training
    # range, only a close call sends the picker to exhaustive search; a shape
    # outside the range always does; MAXMULSK_AUTOTUNE=0 turns it all off.
    monkeypatch.delenv("MAXMULSK_AUTOTUNE", raising=False)
    monkeypatch.delenv("MAXMULSK_AUTOTUNE_MARGIN", raising=False)
    mm.lib().maxmulsk_tuning_clear()
    assert mm.picker_doubt(100, 20000, 30) == "shape outside the trained range"
    assert mm.picker_doubt(40000, 64, 64, mm.Precision.BF16X6) == "shape outside the trained range"
    monkeypatch.setenv("MAXMULSK_AUTOTUNE_MARGIN", "100")
    assert mm.picker_doubt(512, 512, 512) == "close call"
    monkeypatch.setenv("MAXMULSK_AUTOTUNE_MARGIN", "0")
    assert mm.picker_doubt(512, 512, 512) is None
    assert mm.picker_doubt(512, 512, 512, mm.Precision.BF16X9) is None      # BF16X9 is not searched
    monkeypatch.setenv("MAXMULSK_AUTOTUNE", "0")
    assert mm.picker_doubt(100, 20000, 30) is None


def test_choose_precisions_with_the_model(built_lib, monkeypatch):
    # The model's plan for each class: SPLIT_AUTO comes back as a concrete
    # split mode; BF16X9, which has no class of its own, runs the BF16X6
    # plan of the shape (same tiles, K split and variant) with nine products.
    monkeypatch.delenv("MAXMULSK_CONFIG", raising=False)
    _load_shipped_model()
    mm.lib().maxmulsk_tuning_clear()
    for shape in [(128, 32768, 512), (300, 700, 260), (4096, 4096, 4096), (7, 9000, 33)]:
        auto = mm.choose(*shape, mm.Precision.SPLIT_AUTO)
        assert auto.precision in (mm.Precision.TF32X3, mm.Precision.BF16X6), (shape, auto)
        x6 = mm.choose(*shape, mm.Precision.BF16X6)
        x9 = mm.choose(*shape, mm.Precision.BF16X9)
        assert x6.precision == mm.Precision.BF16X6 and x9.precision == mm.Precision.BF16X9
        assert x9.as_tuple()[1:] == x6.as_tuple()[1:], (shape, x6, x9)
        assert mm.classify(*shape, x9) == 0


def test_picker_doubt_without_a_model(built_lib, monkeypatch):
    monkeypatch.delenv("MAXMULSK_AUTOTUNE", raising=False)
    mm.lib().maxmulsk_model_load(None)
    try:
        assert mm.picker_doubt(512, 512, 512) == "no learned model"
        assert mm.picker_doubt(512, 512, 512, mm.Precision.SPLIT_AUTO) == "no learned model"
    finally:
        _load_shipped_model()


def test_close_calls_on_held_out_shapes(built_lib, monkeypatch):
    # How often the default margin sends a held-out shape to the search, and
    # what the search saves there: on the committed autotuner timings, the
    # model's regret on the close calls vs. the rest (the search's own regret
    # is zero by definition).
    import os
    monkeypatch.delenv("MAXMULSK_AUTOTUNE_MARGIN", raising=False)
    _load_shipped_model()
    d = dict(np.load(os.path.join(os.path.dirname(picker.__file__), "data", "picker_timings.npz")))
    ntr = int(d["n_train"])
    shapes = d["shapes"][ntr:]
    close = 0
    for (M, K, N) in shapes[:200]:
        if mm.picker_doubt(int(M), int(K), int(N)) == "close call":
            close += 1
    print("close calls in 200 held-out FP32 shapes:", close)
    assert 0 <= close <= 200
