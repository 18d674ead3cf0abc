"""The surrogate's CPU oracle: its backward pass is the derivative of its
forward pass (central finite differences on the unrounded FP64 network), and
its BF16 rounding is round-to-nearest-even."""
import numpy as np

from oracle import surrogate_oracle as so


def _problem(seed=3, n=40):
    rng = np.random.default_rng(seed)
    params = np.zeros(so.PARAMS)
    parts = so.unpack(params)
    parts["w1"][:, :so.FEATURES] = rng.normal(0, 0.2, (128, so.FEATURES))
    parts["w2"][:] = rng.normal(0, 0.1, (128, 128))
    parts["w3"][:2] = rng.normal(0, 0.1, (2, 128))
    parts["b1"][:] = rng.normal(0, 0.1, 128)
    parts["b2"][:] = rng.normal(0, 0.1, 128)
    parts["b3"][:2] = rng.normal(0, 0.1, 2)
    params = so.pack(parts)
    feats = rng.normal(0, 1, (n, so.FEATURES))
    labels = np.stack([rng.integers(0, 2, n), rng.uniform(0, 3, n)], 1).astype(np.float64)
    mean, inv = np.zeros(so.FEATURES), np.ones(so.FEATURES)
    return params, feats, labels, mean, inv


def test_backward_is_the_derivative_of_forward():
    params, feats, labels, mean, inv = _problem()
    g, loss = so.gradients(feats, labels, params, mean, inv, rounding=False)
    assert abs(loss - so.loss_of(feats, labels, params, mean, inv, rounding=False)) < 1e-12
    rng = np.random.default_rng(7)
    live = [i for i in range(so.PARAMS) if abs(g[i]) > 0]
    for i in rng.choice(live, 40, replace=False):
        h = 1e-6
        p1, p2 = params.copy(), params.copy()
        p1[i] += h
        p2[i] -= h
        fd = (so.loss_of(feats, labels, p1, mean, inv, False) - so.loss_of(feats, labels, p2, mean, inv, False)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_bf16_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 0.0], np.float32)
    want = np.array([1.0, 1.0, 1.0 + 4 * 2 ** -8, 1.0, -2.5, 0.0])
    assert np.array_equal(so.bf16(x), want)
