"""GPU training kernels of the learned schedule cost model (csrc/mlp.cu):
the gradient against the host trainer's (the oracle), and a training run on
the committed B200 timings that fits as well as the host trainer."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import pytest

import graphindor_b200 as gi
from graphindor_b200 import _native as N
from graphindor_b200.schedule_cost import train
from graphindor_b200.schedule_cost.features import DIM

pytestmark = pytest.mark.gpu


def test_gpu_gradient_matches_the_host_oracle():
    rng = np.random.default_rng(3)
    X = rng.standard_normal((300, DIM)).astype(np.float32)
    y = rng.standard_normal(300).astype(np.float32)
    m = train.MLP(DIM, train.HIDDEN, 5)
    p = m.pack()
    g = np.zeros_like(p)
    loss = C.c_float()
    N.check(gi.lib().gi_mlp_grad(X.ctypes.data, y.ctypes.data, len(X), DIM, train.HIDDEN, p.ctypes.data,
                                 g.ctypes.data, C.byref(loss)), "gi_mlp_grad")
    want = m.grads(X, y)
    assert np.max(np.abs(g - want)) <= 1e-4 * np.max(np.abs(want))
    pred, _ = m.forward(X)
    assert loss.value == pytest.approx(float(np.mean((pred - y) ** 2)), rel=1e-4)


def test_gpu_training_fits_like_the_host_trainer():
    here = Path(gi.__file__).resolve().parent / "schedule_cost"
    X, y, keys, _, _ = train.load_rows(str(here / "runs_b200.json"))
    mu, sd = X.mean(0), X.std(0) + 1e-6
    Xn = ((X - mu) / sd).astype(np.float32)
    host = train.MLP(DIM, train.HIDDEN, 0)
    host.fit(Xn, y, epochs=100)
    gpu = train.MLP(DIM, train.HIDDEN, 0)
    start, _ = gpu.forward(Xn)
    loss0 = float(np.mean((start - y) ** 2))
    final = train.train_gpu(gpu, Xn, y, epochs=100)
    pred, _ = gpu.forward(Xn)
    assert final == pytest.approx(float(np.mean((pred - y) ** 2)), rel=1e-3)
    hp, _ = host.forward(Xn)
    host_loss = float(np.mean((hp - y) ** 2))
    assert final < 0.25 * loss0
    assert final < 2.0 * host_loss + 1e-3


def test_gpu_inference_matches_the_host_forward():
    """The shipped model's predictions on the committed feature rows, GPU
    against host."""
    here = Path(gi.__file__).resolve().parent / "schedule_cost"
    X, _, _, _, _ = train.load_rows(str(here / "runs_b200.json"))
    mlp, mu, sd = train.load(str(here / "weights.bin"))
    Xn = np.ascontiguousarray((X - mu) / sd, dtype=np.float32)
    p = mlp.pack()
    out = np.zeros(len(Xn), dtype=np.float32)
    N.check(gi.lib().gi_mlp_predict(Xn.ctypes.data, len(Xn), DIM, train.HIDDEN, p.ctypes.data, out.ctypes.data),
            "gi_mlp_predict")
    want, _ = mlp.forward(Xn)
    assert np.allclose(out, want, rtol=1e-4, atol=1e-4)
