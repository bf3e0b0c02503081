"""The learned variant picker: the GPU forward/backward kernels against the
float64 CPU oracle (oracle/mlp_ref.py), training convergence, and what the
trained network gains over the methods without it (the autotuner's single
configuration and the measured table's nearest class) on 20 held-out seeded
request mixes whose every variant was measured on the B200."""
import json
import os

import numpy as np
import pytest

from nvshmem_b200 import picker as P
from oracle import mlp_ref as R

pytestmark = pytest.mark.gpu


def _data(seed, n):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, 6)).astype(np.float32) * 3 + 5
    Y = rng.normal(size=(n, 12)).astype(np.float32)
    M = (rng.random((n, 12)) > 0.15).astype(np.float32)
    return X, Y, M


@pytest.mark.parametrize("n", [1, 31, 32, 100, 257])
def test_gradients_match_cpu_oracle(n):
    X, Y, M = _data(n, n)
    M[0, 0] = 1.0
    mean, std = X.mean(0), np.maximum(X.std(0), 1e-3)
    net = P.MLP(seed=3)
    net.set_normalization(mean, std)
    p = net.params().astype(np.float64)
    loss, g = net.loss_grad(X, Y, M)
    ref_loss, ref_g = R.loss_grad(p, X, Y, M, mean, std)
    assert abs(loss - ref_loss) <= 1e-4 * max(1.0, abs(ref_loss))
    # float32 GPU sums vs float64 oracle: relative to the gradient's scale
    scale = np.abs(ref_g).max()
    assert np.max(np.abs(g - ref_g)) <= 2e-4 * scale + 1e-7
    fw = net.forward(X)
    ref_o, _ = R.forward(p, X, mean, std)
    assert np.allclose(fw, ref_o, rtol=1e-4, atol=1e-4)


def test_training_reduces_loss():
    rng = np.random.default_rng(7)
    X = rng.uniform(0, 10, size=(2048, 6)).astype(np.float32)
    # a smooth target per variant, like log-times that grow with size
    W = rng.normal(size=(6, 12)).astype(np.float32) * 0.3
    Y = (np.tanh(X / 5 - 1) @ W + 0.1 * np.sin(X[:, :1])).astype(np.float32)
    M = np.ones_like(Y)
    net = P.MLP(seed=1)
    net.set_normalization(X.mean(0), X.std(0))
    curve = net.train(X, Y, M, epochs=60, batch=128, lr=2e-3, seed=2)
    assert curve[-1] < 0.1 * curve[0]
    loss, _ = net.loss_grad(X, Y, M)
    assert loss < 0.05


def test_variant_table():
    from ctypes import byref, c_int
    from nvshmem_b200 import _lib as L
    for v in range(12):
        mode, cfg = c_int(), L.BatchConfig()
        assert L.lib.nvshmemx_variant_describe(v, byref(mode), byref(cfg)) == 0
        assert (mode.value >= 0) == (v < 4)


@pytest.mark.skipif(not os.path.exists(P.DATA), reason="variant timings not measured yet")
def test_picker_beats_the_methods_without_it():
    summary, res, pk = P.evaluate(P.DATA, epochs=400)
    print(json.dumps(summary))
    mlp = res["mlp"].mean()
    # the network must beat the single autotuned configuration and the
    # per-call path, and must not be worse than the table it falls back to
    assert mlp < res["default_variant"].mean()
    assert mlp < res["percall_thread"].mean()
    assert mlp <= res["table"].mean() + 0.02
    # on the classes the network decides itself, it beats the table
    nd = summary["network_decided"]
    assert nd["classes"] > 0.5 * summary["held_out_classes"]
    assert nd["network_regret_pct"] < nd["table_regret_pct"]
    assert summary["train_loss_first_last"][1] < 0.5 * summary["train_loss_first_last"][0]
