"""Pins the CPU reference of the warm-start MLP (oracle/mlp_ref.py) on the
CPU: float64 gradients against central finite differences, and the bf16
rounding helper against known bit patterns."""
import numpy as np

import mlp_ref


def _small_problem(seed=0, n=8, in_raw=5, nout=3):
    rng = np.random.default_rng(seed)
    in_pad = 64
    shapes = mlp_ref.layer_shapes(in_pad)
    layers = []
    for r, c in shapes:
        W = rng.normal(scale=0.3, size=(r, c))
        W[:, in_raw:] = 0 if c == in_pad else W[:, in_raw:]
        layers.append((W, rng.normal(scale=0.1, size=r)))
    params = mlp_ref.pack(layers)
    x = rng.normal(size=(n, in_raw))
    t = rng.normal(size=(n, nout))
    return params, x, t, in_pad, nout


def test_gradients_match_finite_differences():
    params, x, t, in_pad, nout = _small_problem()
    mean, std = np.zeros(x.shape[1]), np.ones(x.shape[1])
    om, os_ = np.zeros(nout), np.ones(nout)
    loss, g = mlp_ref.loss_and_grads(params, x, t, mean, std, om, os_, in_pad, nout, bf16=False)
    rng = np.random.default_rng(1)
    nz = np.flatnonzero(g)
    for i in rng.choice(nz, 40, replace=False):
        h = 1e-6
        p1, p2 = params.copy(), params.copy()
        p1[i] += h
        p2[i] -= h
        l1, _ = mlp_ref.loss_and_grads(p1, x, t, mean, std, om, os_, in_pad, nout, bf16=False)
        l2, _ = mlp_ref.loss_and_grads(p2, x, t, mean, std, om, os_, in_pad, nout, bf16=False)
        fd = (l1 - l2) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_round_known_values():
    v = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.1415926], np.float32)
    r = mlp_ref.bf16_round(v)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: rounds to even (1.0)
    assert list(r[:4]) == [1.0, 1.0, 1.0078125, -2.5]
    assert r[4] == 3.140625
