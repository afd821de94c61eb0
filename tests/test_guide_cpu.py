"""CPU tests of the path-guiding oracle and host helpers (no GPU).

The oracle of the guiding network (oracle/guide_oracle.py) is pinned by finite differences of its
own loss; the mixture head is checked to be a normalised density on the sphere; the figure-of-merit
helpers are checked against direct formulas.
"""
import numpy as np
import pytest

import guide_oracle as go
from skgpu import guiding


def _batch(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, go.N_IN))
    k = rng.normal(size=(n, 3))
    k /= np.linalg.norm(k, axis=1, keepdims=True)
    w = rng.uniform(0.1, 1.0, n)
    return x, k, w


def test_oracle_gradient_matches_finite_differences():
    p = go.random_params(3)
    x, k, w = _batch(9, 1)
    _, g = go.loss_grad(p, x, k, w)
    rng = np.random.default_rng(2)
    eps = 1e-6
    for i in rng.choice(len(p), 60, replace=False):
        q = p.copy()
        q[i] += eps
        lp, _ = go.loss_grad(q, x, k, w)
        q[i] -= 2 * eps
        lm, _ = go.loss_grad(q, x, k, w)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-5 * max(1e-3, abs(fd) + abs(g[i]))


def test_mixture_is_a_normalised_density():
    p = go.random_params(5)
    x, _, _ = _batch(3, 4)
    out, _ = go.forward(p, x)
    # Fibonacci-sphere quadrature: mean density times 4 pi
    m = 200000
    i = np.arange(m) + 0.5
    z = 1 - 2 * i / m
    phi = np.pi * (1 + 5 ** 0.5) * i
    r = np.sqrt(1 - z * z)
    dirs = np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)
    for b in range(len(out)):
        logq = go.log_density(np.repeat(out[b:b + 1], m, axis=0), dirs)
        assert np.exp(logq).mean() * 4 * np.pi == pytest.approx(1.0, rel=2e-3)


def test_bf16_rounding():
    a = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -9, -2.5, 0.0], np.float32)
    r = go.bf16(a)
    # bf16 keeps 8 significant bits: 1 + 2^-8 is a tie and rounds to even (1.0); 1 + 3*2^-9 rounds up
    assert r[1] == 1.0 and r[2] == 1.0 and r[3] == 1.0 + 2 ** -7 and r[4] == -2.5 and r[5] == 0.0


def test_relative_error_and_fom():
    rng = np.random.default_rng(0)
    n = 1000
    w = rng.exponential(size=(n, 4)) * (rng.random((n, 4)) < 0.3)
    stats = np.stack([np.sum(w ** k, axis=0) for k in range(5)])
    r = guiding.relative_error(stats, n)
    direct = np.sqrt(np.sum(w ** 2, axis=0) / np.sum(w, axis=0) ** 2 - 1.0 / n)
    assert np.allclose(r, direct)
    assert guiding.figure_of_merit(stats, n, 2.0) == pytest.approx(1.0 / (np.median(direct) ** 2 * 2.0))


def test_importance_weights():
    img = np.array([0.0, 1.0, 2.0, 4.0, 1e-6])
    w = guiding.importance_from_image(img, floor_quantile=0.0, cap=1e9)
    assert w[0] == 0 and np.isclose(w[1:].mean(), 1.0)
    assert w[1] / w[2] == pytest.approx(2.0) and w[2] / w[3] == pytest.approx(2.0)
    capped = guiding.importance_from_image(img, floor_quantile=0.0, cap=3.0)
    assert capped.max() <= 3.0
