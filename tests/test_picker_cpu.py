"""Cost-model pieces that need no GPU: the FP64 MLP oracle against finite
differences, the model file read by the library's host forward pass, the
features and the candidate lists."""
import ctypes
import math

import numpy as np

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
