"""Trains the learned schedule cost model on timings from collect.py.

A 3-layer MLP (hidden 128, fp32, ReLU) maps the features of features.py to
log10 of the measured device time of a candidate schedule.  Patterns are split
70/30 (seeded) into train and test sets; candidates that ran out of the
collection budget count at the budget (their true time is larger).  The
selection a model makes for a (pattern, graph) is the candidate with the
smallest predicted time; its regret is time(chosen) / time(fastest measured)
- 1.  The report compares that regret with the analytic model's own choice
(the valid candidate of smallest analytic cost).

    python -m graphindor_b200.schedule_cost.train runs.json [more_runs.json ...] --out weights.bin
        [--report report.json] [--device gpu]

weights.bin: magic "GIMLP1\\0\\0", int32 dims (in, hidden), then float32
feature means and scales (in each), W1 (hidden x in), b1, W2 (hidden x
hidden), b2, w3 (hidden), b3, row-major.  The engine reads it with
gi_cost_model_load (include/gi.h).
"""
from __future__ import annotations

import argparse
import json
import random
import struct

import numpy as np

from .features import DIM, plan_features

HIDDEN = 128


def merge_runs(paths):
    """One runs record from several collections (rows concatenated, graphs
    united; a row timed out at its own collection's budget)."""
    out = {"budget_ms": None, "graphs": {}, "rows": []}
    for p in paths:
        r = json.load(open(p))
        out["graphs"].update(r["graphs"])
        for row in r["rows"]:
            row = dict(row)
            if row["ms"] is None:
                row.setdefault("censored_at_ms", r["budget_ms"])
            out["rows"].append(row)
        out["budget_ms"] = r["budget_ms"] if out["budget_ms"] is None else max(out["budget_ms"], r["budget_ms"])
    return out


def load_rows(path):
    runs = merge_runs(path if isinstance(path, (list, tuple)) else [path])
    budget = runs["budget_ms"]
    gfeat = {k: np.asarray(v["features"], dtype=np.float32) for k, v in runs["graphs"].items()}
    X, y, keys, censored = [], [], [], []
    for r in runs["rows"]:
        f = np.concatenate([plan_features(r["n"], r["adj"], r["order"], r["restricts"], r["model_cost"],
                                          r["iep_k"]), gfeat[r["graph"]]])
        ms = r["ms"] if r["ms"] is not None else r.get("censored_at_ms", budget)
        X.append(f)
        y.append(np.log10(max(ms, 1e-3)))
        keys.append((r["graph"], r["adj"]))
        censored.append(r["ms"] is None)
    return np.stack(X), np.asarray(y, dtype=np.float32), keys, np.asarray(censored), runs


class MLP:
    def __init__(self, d_in: int, hidden: int, seed: int = 0):
        rng = np.random.default_rng(seed)
        self.W1 = (rng.standard_normal((hidden, d_in)) * np.sqrt(2.0 / d_in)).astype(np.float32)
        self.b1 = np.zeros(hidden, np.float32)
        self.W2 = (rng.standard_normal((hidden, hidden)) * np.sqrt(2.0 / hidden)).astype(np.float32)
        self.b2 = np.zeros(hidden, np.float32)
        self.w3 = (rng.standard_normal(hidden) * np.sqrt(1.0 / hidden)).astype(np.float32)
        self.b3 = np.float32(0.0)

    def params(self):
        return [self.W1, self.b1, self.W2, self.b2, self.w3]

    def pack(self) -> np.ndarray:
        """All parameters as one float32 array, in the model file's order."""
        return np.concatenate([self.W1.ravel(), self.b1, self.W2.ravel(), self.b2, self.w3,
                               np.asarray([self.b3], np.float32)]).astype(np.float32)

    def unpack(self, p: np.ndarray) -> None:
        H, I = self.W1.shape
        o = 0
        for name, shape in (("W1", (H, I)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("w3", (H,))):
            n = int(np.prod(shape))
            setattr(self, name, p[o:o + n].reshape(shape).astype(np.float32).copy())
            o += n
        self.b3 = np.float32(p[o])

    def grads(self, X, y) -> np.ndarray:
        """Gradient of the mean squared error over the rows of X, packed like
        pack() (the host oracle of the GPU kernels)."""
        pred, (x0, h1, h2) = self.forward(X)
        g = 2.0 * (pred - y) / len(X)
        gh2 = np.outer(g, self.w3) * (h2 > 0)
        gh1 = (gh2 @ self.W2) * (h1 > 0)
        return np.concatenate([(gh1.T @ x0).ravel(), gh1.sum(0), (gh2.T @ h1).ravel(), gh2.sum(0), h2.T @ g,
                               [g.sum()]]).astype(np.float32)

    def forward(self, X):
        h1 = np.maximum(X @ self.W1.T + self.b1, 0)
        h2 = np.maximum(h1 @ self.W2.T + self.b2, 0)
        return h2 @ self.w3 + self.b3, (X, h1, h2)

    def fit(self, X, y, epochs=400, lr=2e-3, batch=128, wd=1e-4, seed=0):
        rng = np.random.default_rng(seed)
        m = [np.zeros_like(p) for p in self.params()] + [0.0]
        v = [np.zeros_like(p) for p in self.params()] + [0.0]
        t = 0
        for _ in range(epochs):
            perm = rng.permutation(len(X))
            for s in range(0, len(X), batch):
                idx = perm[s:s + batch]
                pred, (x0, h1, h2) = self.forward(X[idx])
                g = 2.0 * (pred - y[idx]) / len(idx)
                gw3 = h2.T @ g
                gb3 = g.sum()
                gh2 = np.outer(g, self.w3) * (h2 > 0)
                gW2 = gh2.T @ h1
                gb2 = gh2.sum(0)
                gh1 = (gh2 @ self.W2) * (h1 > 0)
                gW1 = gh1.T @ x0
                gb1 = gh1.sum(0)
                grads = [gW1 + wd * self.W1, gb1, gW2 + wd * self.W2, gb2, gw3 + wd * self.w3, gb3]
                t += 1
                ps = self.params()
                for i, gr in enumerate(grads):
                    m[i] = 0.9 * m[i] + 0.1 * gr
                    v[i] = 0.999 * v[i] + 0.001 * gr * gr
                    mh = m[i] / (1 - 0.9 ** t)
                    vh = v[i] / (1 - 0.999 ** t)
                    step = lr * mh / (np.sqrt(vh) + 1e-8)
                    if i < 5:
                        ps[i] -= step.astype(np.float32)
                    else:
                        self.b3 = np.float32(self.b3 - step)


def train_gpu(mlp: MLP, X, y, epochs=400, lr=2e-3, batch=128, wd=1e-4, seed=0) -> float:
    """Trains `mlp` in place with gi_mlp_train (the engine's kernels);
    returns the final training loss."""
    import ctypes as C

    from .. import _native as N
    X = np.ascontiguousarray(X, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    p = mlp.pack()
    loss = C.c_float()
    N.check(N.lib().gi_mlp_train(X.ctypes.data, y.ctypes.data, len(X), X.shape[1], mlp.W1.shape[0], epochs, batch,
                                 lr, wd, seed, p.ctypes.data, C.byref(loss)), "gi_mlp_train")
    mlp.unpack(p)
    return loss.value


def selection_report(keys, y_true_ms, pred, model_cost, test_keys):
    """Regret of the learned choice and of the analytic choice per test
    (graph, pattern), and the total time of each selection."""
    by = {}
    for i, k in enumerate(keys):
        if k in test_keys:
            by.setdefault(k, []).append(i)
    reg_l, reg_a, tot_l, tot_a, tot_b = [], [], 0.0, 0.0, 0.0
    for k, idx in by.items():
        if len(idx) < 2:
            continue  # nothing to choose between
        t = np.asarray([y_true_ms[i] for i in idx])
        best = t.min()
        li = idx[int(np.argmin([pred[i] for i in idx]))]
        ai = idx[int(np.argmin([model_cost[i] for i in idx]))]
        reg_l.append(y_true_ms[li] / best - 1)
        reg_a.append(y_true_ms[ai] / best - 1)
        tot_l += float(y_true_ms[li])
        tot_a += float(y_true_ms[ai])
        tot_b += float(best)
    return {"cases": len(reg_l), "learned_regret_mean": float(np.mean(reg_l)), "learned_regret_median":
            float(np.median(reg_l)), "analytic_regret_mean": float(np.mean(reg_a)), "analytic_regret_median":
            float(np.median(reg_a)), "learned_total_ms": tot_l, "analytic_total_ms": tot_a, "best_total_ms": tot_b}


def save(path: str, mlp: MLP, mu: np.ndarray, sd: np.ndarray) -> None:
    with open(path, "wb") as f:
        f.write(b"GIMLP1\0\0")
        f.write(struct.pack("<ii", mu.size, HIDDEN))
        for a in (mu, sd, mlp.W1, mlp.b1, mlp.W2, mlp.b2, mlp.w3, np.asarray([mlp.b3], np.float32)):
            f.write(np.ascontiguousarray(a, dtype="<f4").tobytes())


def load(path: str):
    """(MLP, feature means, feature scales) from a file written by save()."""
    raw = open(path, "rb").read()
    assert raw[:8] == b"GIMLP1\0\0", "not a schedule cost model file"
    d_in, hidden = struct.unpack_from("<ii", raw, 8)
    a = np.frombuffer(raw, dtype="<f4", offset=16)
    sizes = [d_in, d_in, hidden * d_in, hidden, hidden * hidden, hidden, hidden, 1]
    parts, o = [], 0
    for n in sizes:
        parts.append(a[o:o + n].copy())
        o += n
    m = MLP(d_in, hidden)
    m.W1, m.b1 = parts[2].reshape(hidden, d_in), parts[3]
    m.W2, m.b2 = parts[4].reshape(hidden, hidden), parts[5]
    m.w3, m.b3 = parts[6], np.float32(parts[7][0])
    return m, parts[0], parts[1]


def split(keys, seed: int = 0):
    """The seeded 70/30 split by pattern used for training."""
    pats = sorted({k[1] for k in keys})
    random.Random(seed).shuffle(pats)
    return set(pats[: int(round(0.3 * len(pats)))])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("runs", nargs="+", help="one or more collect.py outputs")
    ap.add_argument("--out", required=True)
    ap.add_argument("--report")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--device", choices=["host", "gpu"], default="host",
                    help="gpu: train with the engine's CUDA kernels (gi_mlp_train)")
    a = ap.parse_args()
    X, y, keys, censored, runs = load_rows(a.runs)
    assert X.shape[1] == DIM
    test_p = split(keys, a.seed)
    train = np.asarray([k[1] not in test_p for k in keys])
    mu = X[train].mean(0)
    sd = X[train].std(0) + 1e-6
    Xn = (X - mu) / sd
    mlp = MLP(DIM, HIDDEN, a.seed)
    if a.device == "gpu":
        train_gpu(mlp, Xn[train], y[train], seed=a.seed)
    else:
        mlp.fit(Xn[train], y[train], seed=a.seed)
    pred, _ = mlp.forward(Xn)
    ms = 10.0 ** y
    cost = [r["model_cost"] for r in runs["rows"]]
    test_keys = {k for k in keys if k[1] in test_p}
    train_keys = {k for k in keys if k[1] not in test_p}
    rep = {"rows": int(len(y)), "train_rows": int(train.sum()), "test_rows": int((~train).sum()),
           "censored_rows": int(censored.sum()),
           "test_rmse_log10": float(np.sqrt(np.mean((pred[~train] - y[~train]) ** 2))),
           "train_rmse_log10": float(np.sqrt(np.mean((pred[train] - y[train]) ** 2))),
           "test": selection_report(keys, ms, pred, cost, test_keys),
           "train": selection_report(keys, ms, pred, cost, train_keys)}
    save(a.out, mlp, mu, sd)
    print(json.dumps(rep, indent=1))
    if a.report:
        json.dump(rep, open(a.report, "w"), indent=1)


if __name__ == "__main__":
    main()
