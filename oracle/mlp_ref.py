"""CPU oracle of the learned picker's network (TEST INFRASTRUCTURE ONLY).

Forward and backward of the 6 -> 64 -> 64 -> 64 -> 12 ReLU MLP in float64
numpy, with the parameter layout of include/nvshmemx_picker.h (W1[64][6] b1
W2[64][64] b2 W3[64][64] b3 W4[12][64] b4, row-major, concatenated), the
input standardisation (x - mean) / std, and the masked mean squared error
L = sum(M * (O - Y)^2) / sum(M).  The GPU kernels' gradients are checked
against this.  The reference has no learned component; this restates the
mathematics only.
"""
from __future__ import annotations

import numpy as np

NI, NH, NO = 6, 64, 12
SHAPES = [("W1", (NH, NI)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)),
          ("W3", (NH, NH)), ("b3", (NH,)), ("W4", (NO, NH)), ("b4", (NO,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(p: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([d[name].reshape(-1) for name, _ in SHAPES])


def forward(p, X, mean=None, std=None):
    w = unpack(p)
    X = np.asarray(X, np.float64)
    if mean is not None:
        X = (X - mean) / np.where(std > 1e-12, std, 1.0)
    z1 = X @ w["W1"].T + w["b1"]
    a1 = np.maximum(z1, 0)
    z2 = a1 @ w["W2"].T + w["b2"]
    a2 = np.maximum(z2, 0)
    z3 = a2 @ w["W3"].T + w["b3"]
    a3 = np.maximum(z3, 0)
    o = a3 @ w["W4"].T + w["b4"]
    return o, (X, a1, a2, a3)


def loss_grad(p, X, Y, M, mean=None, std=None):
    w = unpack(p)
    o, (x, a1, a2, a3) = forward(p, X, mean, std)
    cnt = float(np.sum(M))
    diff = o - Y
    loss = float(np.sum(M * diff * diff) / cnt)
    do = 2.0 * M * diff / cnt
    g = {"W4": do.T @ a3, "b4": do.sum(0)}
    dz3 = (do @ w["W4"]) * (a3 > 0)
    g["W3"], g["b3"] = dz3.T @ a2, dz3.sum(0)
    dz2 = (dz3 @ w["W3"]) * (a2 > 0)
    g["W2"], g["b2"] = dz2.T @ a1, dz2.sum(0)
    dz1 = (dz2 @ w["W2"]) * (a1 > 0)
    g["W1"], g["b1"] = dz1.T @ x, dz1.sum(0)
    return loss, pack(g)
