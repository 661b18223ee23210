"""The learned schedule cost model on the CPU: the engine's features and MLP
forward pass (csrc/schedule_cost.cpp) agree with the Python definitions used
for training (graphindor_b200/schedule_cost), and a learned plan is one of
the pattern's valid candidates, so its count is exact."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import graphindor_b200 as gi
from graphindor_b200 import _native as N
from graphindor_b200 import gen
from graphindor_b200.schedule_cost.features import DIM, graph_features, plan_features
from graphindor_b200.schedule_cost.train import HIDDEN, MLP, save


def test_graph_features_match(native):
    for g, tri in ((gen.rmat(12, 8.0, 3), 12345), (gen.erdos_renyi(3000, 20000, 4), 0)):
        f = (C.c_float * N.GI_GRAPH_FEATURES)()
        N.check(gi.lib().gi_graph_features_host(g.vertex.ctypes.data, g.v_cnt, tri, f, N.GI_GRAPH_FEATURES), "f")
        assert np.allclose(np.array(f[:]), graph_features(g.vertex, tri), atol=1e-6)


@pytest.mark.parametrize("seed", [1, 2])
def test_learned_choice_is_the_python_argmin(tmp_path, native, seed):
    mlp = MLP(DIM, HIDDEN, seed)
    rng = np.random.default_rng(seed)
    mu = rng.standard_normal(DIM).astype(np.float32) * 0.1
    sd = (1.0 + rng.random(DIM)).astype(np.float32)
    path = tmp_path / "w.bin"
    save(str(path), mlp, mu, sd)
    gi.load_cost_model(str(path))
    g = gen.rmat(11, 8.0, 5)
    gf = graph_features(g.vertex, 777)
    feats = (C.c_float * N.GI_GRAPH_FEATURES)(*gf.tolist())
    for n, adj in [(5, "0101110101010101010011000"), (6, "011100101010110001100011010101001110"),
                   (4, "0110100110010110")]:
        p = gi.Pattern(n, adj)
        valid = [c for c in gi.Schedule_IEP.candidates(p, g.v_cnt, g.e_cnt, 777) if c[3] > 0]
        # The model re-ranks the analytic model's best GI_LEARNED_CANDIDATES, kept in enumeration order.
        top = sorted(sorted(range(len(valid)), key=lambda i: valid[i][2])[:N.GI_LEARNED_CANDIDATES])
        cands = [valid[i] for i in top]
        k = gi.Schedule_IEP(p, order=cands[0][0], restricts=cands[0][1]).export()["in_exclusion_optimize_num"]
        X = np.stack([np.concatenate([plan_features(n, adj, o, r, cost, k), gf]) for o, r, cost, _ in cands])
        pred, _ = mlp.forward((X - mu) / sd)
        want = cands[int(np.argmin(pred))]
        h = C.c_void_p()
        ms = C.c_double()
        N.check(gi.lib().gi_plan_create_learned(n, adj.encode(), g.v_cnt, g.e_cnt, 777, feats, 1, C.byref(h),
                                                C.byref(ms)), "learned")
        s = gi.Schedule_IEP.__new__(gi.Schedule_IEP)
        s._h, s.pattern = h, p
        e = s.export()
        assert e["order"] == list(want[0]) and e["exact"] == 1
        assert ms.value == pytest.approx(10.0 ** float(pred.min()), rel=1e-3)
    gi.load_cost_model()  # back to the shipped model (if present) for later tests


def test_missing_model_file_is_an_error(native):
    assert gi.lib().gi_cost_model_load(b"/nonexistent/w.bin") == N.GI_EIO


def test_shipped_model_against_the_analytic_choice_on_held_out_patterns():
    """What the trained network gains over the analytic model on the patterns
    it was not trained on (the committed B200 timings, seeded 70/30 split by
    pattern), recomputed from the committed timings and weights: it must
    equal the figures recorded in report.json, and the learned picks must
    take less time in total than the analytic model's picks.  The recorded
    figures (weights trained on the B200 by the engine's own kernels,
    gi_mlp_train): 22 held-out (pattern, graph) cases; learned picks 1,024.1 ms
    in total against 1,032.3 ms for the analytic picks (0.8 % less; the
    fastest measured candidate of each case, 983.3 ms); median regret 1.3 %
    against 2.8 %, mean regret 6.4 % against 6.2 %."""
    import json
    from pathlib import Path
    from graphindor_b200.schedule_cost import train
    here = Path(gi.__file__).resolve().parent / "schedule_cost"
    X, y, keys, censored, runs = train.load_rows(str(here / "runs_b200.json"))
    mlp, mu, sd = train.load(str(here / "weights.bin"))
    pred, _ = mlp.forward((X - mu) / sd)
    test_p = train.split(keys, 0)
    rep = train.selection_report(keys, 10.0 ** y, pred, [r["model_cost"] for r in runs["rows"]],
                                 {k for k in keys if k[1] in test_p})
    recorded = json.loads((here / "report.json").read_text())["test"]
    for k, v in recorded.items():
        assert rep[k] == pytest.approx(v, rel=1e-5), k
    assert rep["cases"] >= 20
    assert rep["learned_total_ms"] < rep["analytic_total_ms"]


def test_host_gradient_oracle_matches_finite_differences():
    """The host trainer's gradient (the oracle of the GPU training kernels)
    against central differences in float64."""
    from graphindor_b200.schedule_cost.train import MLP as M
    rng = np.random.default_rng(0)
    m = M(5, 8, 1)
    X = rng.standard_normal((7, 5))
    y = np.arange(7, dtype=np.float64)
    p = m.pack().astype(np.float64)

    def split64(q):  # float64 views in pack() order
        out, o = [], 0
        for shape in ((8, 5), (8,), (8, 8), (8,), (8,)):
            n = int(np.prod(shape))
            out.append(q[o:o + n].reshape(shape))
            o += n
        return out + [float(q[o])]

    def loss(q):
        W1, b1, W2, b2, w3, b3 = split64(q)
        h = np.maximum(np.maximum(X @ W1.T + b1, 0) @ W2.T + b2, 0)
        return float(np.mean((h @ w3 + b3 - y) ** 2))

    m64 = M(5, 8, 0)
    m64.W1, m64.b1, m64.W2, m64.b2, m64.w3, m64.b3 = split64(p)
    pr, (x0, h1, h2) = m64.forward(X)
    g = 2.0 * (pr - y) / len(X)
    gh2 = np.outer(g, m64.w3) * (h2 > 0)
    gh1 = (gh2 @ m64.W2) * (h1 > 0)
    grad = np.concatenate([(gh1.T @ x0).ravel(), gh1.sum(0), (gh2.T @ h1).ravel(), gh2.sum(0), h2.T @ g, [g.sum()]])
    eye = np.eye(len(p))
    num = np.array([(loss(p + 1e-6 * eye[i]) - loss(p - 1e-6 * eye[i])) / 2e-6 for i in range(len(p))])
    assert np.max(np.abs(num - grad)) <= 1e-6 * np.max(np.abs(grad))
    assert np.allclose(m64.grads(X, y), grad, rtol=1e-5, atol=1e-6)
