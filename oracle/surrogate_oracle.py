"""CPU oracle of the learned audit surrogate (test infrastructure only).

FP64 restatement of the library's 48 -> 128 -> 128 -> 2 MLP forward and
backward passes, rounding to BF16 exactly where the tensor-core kernels do:
the normalised inputs, both hidden activations, and the three backward
operands (output gradient, both hidden-layer gradients). Accumulation is FP64
here and FP32 on the GPU, so parity is a relative tolerance, not bit equality.

The surrogate has no reference counterpart (the reference's learned policies
are FP32 networks over other features, src/neural/inference.cu:75-108,
src/neural/fused.cu:95-120); this oracle pins the library's own kernels.
The loss mirrors the train step: mean over rows of
BCE(logit, accepted) + Huber_1(predicted - error ratio).
"""
from __future__ import annotations

import numpy as np

FEATURES = 48
OFF = {"w1": (0, (128, 64)), "b1": (8192, (128,)), "w2": (8320, (128, 128)), "b2": (24704, (128,)),
       "w3": (24832, (16, 128)), "b3": (26880, (16,))}
PARAMS = 26896


def bf16(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even to BF16, returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    out = ((u + r) & 0xFFFF0000).astype(np.uint32).view(np.float32)
    return out.astype(np.float64)


def unpack(params: np.ndarray) -> dict:
    return {k: np.asarray(params[o:o + int(np.prod(s))], np.float64).reshape(s) for k, (o, s) in OFF.items()}


def pack(parts: dict) -> np.ndarray:
    out = np.zeros(PARAMS, np.float64)
    for k, (o, s) in OFF.items():
        out[o:o + int(np.prod(s))] = parts[k].reshape(-1)
    return out


def _identity(x):
    return np.asarray(x, np.float64)


def inputs(features: np.ndarray, mean: np.ndarray, inv_std: np.ndarray, rnd=bf16) -> np.ndarray:
    if rnd is bf16:
        f = np.asarray(features, np.float32)
        x = ((f - np.asarray(mean, np.float32)) * np.asarray(inv_std, np.float32)).astype(np.float32)
    else:
        x = (np.asarray(features, np.float64) - mean) * inv_std
    out = np.zeros((x.shape[0], 64), np.float64)
    out[:, :FEATURES] = rnd(x)
    return out


def forward(features, params, mean, inv_std, rounding: bool = True):
    """Returns (outputs n x 2, cache). rounding=False is the plain FP64
    network (used to check the backward algebra by finite differences)."""
    rnd = bf16 if rounding else _identity
    p = unpack(params)
    w1, w2, w3 = rnd(p["w1"]), rnd(p["w2"]), rnd(p["w3"])
    x = inputs(features, mean, inv_std, rnd)
    h1 = rnd(np.maximum(x @ w1.T + p["b1"], 0))
    h2 = rnd(np.maximum(h1 @ w2.T + p["b2"], 0))
    o = h2 @ w3.T + p["b3"]
    return o[:, :2], {"x": x, "h1": h1, "h2": h2, "w1": w1, "w2": w2, "w3": w3, "rnd": rnd}


def loss_of(features, labels, params, mean, inv_std, rounding: bool = True) -> float:
    out, _ = forward(features, params, mean, inv_std, rounding)
    y, target = labels[:, 0].astype(np.float64), labels[:, 1].astype(np.float64)
    z, d = out[:, 0], out[:, 1] - target
    loss = (np.maximum(z, 0) + np.log1p(np.exp(-np.abs(z))) - y * z) + np.where(np.abs(d) <= 1, 0.5 * d * d,
                                                                              np.abs(d) - 0.5)
    return float(loss.mean())


def gradients(features, labels, params, mean, inv_std, rounding: bool = True):
    """Gradient vector (parameter layout) and mean loss of one batch."""
    out, c = forward(features, params, mean, inv_std, rounding)
    bf = c["rnd"]
    n = out.shape[0]
    y, target = labels[:, 0].astype(np.float64), labels[:, 1].astype(np.float64)
    z, pred = out[:, 0], out[:, 1]
    d = pred - target
    loss = (np.maximum(z, 0) + np.log1p(np.exp(-np.abs(z))) - y * z) + np.where(np.abs(d) <= 1, 0.5 * d * d,
                                                                              np.abs(d) - 0.5)
    g3 = np.zeros((n, 16))
    g3[:, 0] = bf((1 / (1 + np.exp(-z)) - y) / n)
    g3[:, 1] = bf(np.clip(d, -1, 1) / n)
    gw3 = g3.T @ c["h2"]
    gb3 = g3.sum(0)
    dh2 = g3 @ c["w3"]
    g2 = bf(dh2 * (c["h2"] > 0))
    gw2 = g2.T @ c["h1"]
    gb2 = g2.sum(0)
    dh1 = g2 @ c["w2"]
    g1 = bf(dh1 * (c["h1"] > 0))
    gw1 = g1.T @ c["x"]
    gb1 = g1.sum(0)
    gw3[2:] = 0
    gb3[2:] = 0
    gw1[:, FEATURES:] = 0
    return pack({"w1": gw1, "b1": gb1, "w2": gw2, "b2": gb2, "w3": gw3, "b3": gb3}), float(loss.mean())
