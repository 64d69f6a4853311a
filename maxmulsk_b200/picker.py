"""The learned config picker: trains the cost-model MLP on the autotuner's
timings with the library's own CUDA kernels (maxmulsk_mlp_forward_dev /
_backward_dev / _adam_dev), evaluates its regret against exhaustive search on
held-out shapes, and writes the weights the library's picker loads
(maxmulsk_model_load or MAXMULSK_MODEL).

    python -m maxmulsk_b200.picker --data timings.npz --out model.bin

Inputs per (shape, class): the model's features (maxmulsk_mlp_features);
targets: ln(time in microseconds) of each candidate; candidates that could not
run are masked out of the loss and of the choice.
"""
from __future__ import annotations

import argparse
import ctypes
import struct

import numpy as np

from . import check, lib

F, H, O = 7, 64, 48
NPARAM = F * H + H + H * H + H + H * O + O


def features(shapes, cls: int) -> np.ndarray:
    out = np.empty((len(shapes), F), np.float32)
    buf = (ctypes.c_float * F)()
    for i, (M, K, N) in enumerate(shapes):
        check(lib().maxmulsk_mlp_features(int(M), int(K), int(N), cls, buf), "features")
        out[i] = np.frombuffer(buf, np.float32)
    return out


def dataset(d: dict, rows) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
    """X, T (ln us), mask, times (us, inf = not runnable) for both classes of the rows."""
    shapes = d["shapes"][rows]
    Xs, Ts, Ms, Ts_us = [], [], [], []
    for cls, key in ((0, "t_fp32"), (1, "t_split")):
        full = _padded(d[key][rows])
        mask = np.isfinite(full).astype(np.float32)
        T = np.where(mask > 0, np.log(np.maximum(full, 1e-3)), 0.0).astype(np.float32)
        Xs.append(features(shapes, cls)); Ts.append(T); Ms.append(mask); Ts_us.append(full)
    return np.concatenate(Xs), np.concatenate(Ts), np.concatenate(Ms), np.concatenate(Ts_us)


class Trainer:
    """Parameters and Adam state in device memory; every step runs the
    library's kernels (no autograd, no torch math on the training path)."""

    def __init__(self, seed: int = 0, out_bias: float = 0.0):
        import torch
        self.torch = torch
        rng = np.random.default_rng(seed)
        p = np.zeros(NPARAM, np.float32)
        i = 0
        for (fin, fout) in ((F, H), (H, H), (H, O)):
            p[i: i + fin * fout] = rng.normal(0.0, 1.0 / np.sqrt(fin), fin * fout)
            i += fin * fout
            if fout == O:
                p[i: i + fout] = out_bias
            i += fout
        self.params = torch.from_numpy(p).cuda()
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step_no = 0

    def _ptr(self, t):
        return t.data_ptr()

    def fit(self, X, T, mask, steps: int = 3000, lr: float = 3e-3, log_every: int = 0) -> list[float]:
        torch = self.torch
        B = X.shape[0]
        dX = torch.from_numpy(X).cuda(); dT = torch.from_numpy(T).cuda(); dM = torch.from_numpy(mask).cuda()
        Z1 = torch.empty(B * H, device="cuda"); H1 = torch.empty_like(Z1)
        Z2 = torch.empty_like(Z1); H2 = torch.empty_like(Z1)
        Y = torch.empty(B * O, device="cuda")
        work = torch.empty(B * (O + 2 * H), device="cuda")
        rowloss = torch.empty(B, device="cuda")
        count = float(mask.sum())
        L = lib()
        s = torch.cuda.current_stream().cuda_stream
        losses = []
        for it in range(steps):
            lr_t = lr * (0.05 + 0.95 * 0.5 * (1 + np.cos(np.pi * it / steps)))
            check(L.maxmulsk_mlp_forward_dev(self.params.data_ptr(), dX.data_ptr(), B, Z1.data_ptr(), H1.data_ptr(),
                                             Z2.data_ptr(), H2.data_ptr(), Y.data_ptr(), s), "forward")
            check(L.maxmulsk_mlp_backward_dev(self.params.data_ptr(), dX.data_ptr(), Z1.data_ptr(), H1.data_ptr(),
                                              Z2.data_ptr(), H2.data_ptr(), Y.data_ptr(), dT.data_ptr(),
                                              dM.data_ptr(), B, count, self.grads.data_ptr(), work.data_ptr(),
                                              rowloss.data_ptr(), s), "backward")
            self.step_no += 1
            check(L.maxmulsk_mlp_adam_dev(self.params.data_ptr(), self.grads.data_ptr(), self.m.data_ptr(),
                                          self.v.data_ptr(), lr_t, 0.9, 0.999, 1e-8, self.step_no, s), "adam")
            if log_every and (it % log_every == 0 or it == steps - 1):
                losses.append(float(rowloss.sum().item()) / count)
        return losses

    def predict(self, X, mask) -> tuple[np.ndarray, np.ndarray]:
        torch = self.torch
        B = X.shape[0]
        dX = torch.from_numpy(X).cuda(); dM = torch.from_numpy(mask).cuda()
        Y = torch.empty(B * O, device="cuda"); work = torch.empty(2 * B * H, device="cuda")
        best = torch.empty(B, dtype=torch.int32, device="cuda")
        check(lib().maxmulsk_mlp_predict_dev(self.params.data_ptr(), dX.data_ptr(), dM.data_ptr(), B,
                                             work.data_ptr(), Y.data_ptr(), best.data_ptr(),
                                             torch.cuda.current_stream().cuda_stream), "predict")
        return Y.cpu().numpy().reshape(B, O), best.cpu().numpy()

    def save(self, path: str) -> None:
        save_params(path, self.params.cpu().numpy())


def save_params(path: str, p: np.ndarray) -> None:
    with open(path, "wb") as f:
        f.write(b"MMSKMLP1")
        f.write(struct.pack("<4i", F, H, O, NPARAM))
        f.write(np.ascontiguousarray(p, np.float32).tobytes())


def regret(times_us: np.ndarray, picks: np.ndarray) -> dict:
    """Regret of picks against the best measured candidate per row."""
    best = np.min(times_us, axis=1)
    ok = np.isfinite(best) & (picks >= 0)
    t = times_us[np.arange(len(picks)), np.maximum(picks, 0)]
    r = t[ok] / best[ok] - 1.0
    return {"rows": int(ok.sum()), "mean": float(r.mean()), "median": float(np.median(r)),
            "p90": float(np.quantile(r, 0.9)), "geomean": float(np.exp(np.log1p(r).mean()) - 1.0),
            "within_5pct": float((r <= 0.05).mean()),
            "total_time": float(t[ok].sum() / best[ok].sum() - 1.0)}


def _padded(t: np.ndarray) -> np.ndarray:
    full = np.full((t.shape[0], O), np.inf, np.float32)
    full[:, : t.shape[1]] = t
    return full


def rule_regret(d: dict, rows) -> dict:
    times = np.concatenate([_padded(d["t_fp32"][rows]), _padded(d["t_split"][rows])], axis=0)
    rule = np.concatenate([d["t_rule_fp32"][rows], d["t_rule_split"][rows]])
    best = np.min(times, axis=1)
    ok = np.isfinite(best) & np.isfinite(rule)
    r = rule[ok] / best[ok] - 1.0
    return {"rows": int(ok.sum()), "mean": float(r.mean()), "median": float(np.median(r)),
            "p90": float(np.quantile(r, 0.9)), "geomean": float(np.exp(np.log1p(r).mean()) - 1.0),
            "within_5pct": float((r <= 0.05).mean()), "total_time": float(rule[ok].sum() / best[ok].sum() - 1.0)}


def _fit_and_score(d: dict, fit_rows, eval_rows, seed: int, steps: int, lr: float):
    X, T, M, _ = dataset(d, fit_rows)
    mean_t = float((T * M).sum() / M.sum())
    trainer = Trainer(seed=seed, out_bias=mean_t)
    losses = trainer.fit(X, T, M, steps=steps, lr=lr, log_every=max(1, steps // 10))
    Xe, _, Me, Ue = dataset(d, eval_rows)
    _, best = trainer.predict(Xe, Me)
    return trainer, losses, regret(Ue, best)


def train_and_evaluate(d: dict, steps: int = 5000, lr: float = 1e-2, seeds=(0, 1, 2, 3), n_val: int = 400):
    """Model selection on the training shapes only: each seed is trained on
    the first n_train - n_val of them and scored (total-time + geometric-mean
    regret) on the last n_val; the best seed is retrained on all training
    shapes and evaluated once on the held-out shapes, beside the rule."""
    n_train = int(d["n_train"])
    fit_rows, val_rows = np.arange(n_train - n_val), np.arange(n_train - n_val, n_train)
    test_rows = np.arange(n_train, len(d["shapes"]))
    scores = []
    for seed in seeds:
        _, _, r_val = _fit_and_score(d, fit_rows, val_rows, seed, steps, lr)
        scores.append(r_val["total_time"] + r_val["geomean"])
    seed = int(seeds[int(np.argmin(scores))])
    trainer, losses, r_mlp = _fit_and_score(d, np.arange(n_train), test_rows, seed, steps, lr)
    r_mlp["seed"] = seed
    r_mlp["validation_scores"] = [float(x) for x in scores]
    return trainer, losses, r_mlp, rule_regret(d, test_rows)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--data", required=True)
    ap.add_argument("--out", required=True)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--lr", type=float, default=1e-2)
    a = ap.parse_args()
    d = dict(np.load(a.data))
    trainer, losses, r_mlp, r_rule = train_and_evaluate(d, steps=a.steps, lr=a.lr)
    trainer.save(a.out)
    print("loss", [round(x, 4) for x in losses])
    print("held-out regret, MLP :", r_mlp)
    print("held-out regret, rule:", r_rule)


if __name__ == "__main__":
    main()
