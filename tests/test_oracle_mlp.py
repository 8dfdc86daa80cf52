"""The warm-start network's CPU oracle, pinned: its gradient against central
finite differences, its bf16 rounding against known values, and the
product's initialization and rounding helpers against it (no GPU)."""

import numpy as np

from microsimulator_b200 import learned
from oracle import mlp_oracle as mo


def test_bf16_rounding_known_values():
    x = np.array([1.0, 1.0 + 2**-8, 1.0 + 3 * 2**-8, -2.5, 1e-40, 65504.0, 3.0e38], dtype=np.float32)
    r = mo.bf16_round(x)
    assert r[0] == 1.0
    assert r[1] == 1.0  # a tie rounds to the even neighbour
    assert r[2] == np.float32(1.0 + 4 * 2**-8)
    assert r[3] == -2.5
    assert np.array_equal(mo.bf16_bits(x), learned.to_bf16_bits(x))


def test_product_initialization_matches_oracle():
    assert np.array_equal(learned.initial_parameters(3), mo.init(3))
    assert learned.PARAMETERS == mo.PARAMETERS and learned.WEIGHTS == mo.WEIGHTS


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    params = mo.init(1).astype(np.float64)
    params[mo.WEIGHTS:] = rng.normal(0, 0.1, mo.PARAMETERS - mo.WEIGHTS)
    x = rng.normal(0, 1, (7, mo.INPUT))
    x[:, mo.FEATURES:] = 0
    t = rng.normal(0, 1, (7, mo.OUTPUTS))

    def loss(p):
        y, _ = mo.forward(p, x)
        return mo.mse(y, t)[0]

    y, cache = mo.forward(params, x)
    _, dy = mo.mse(y, t)
    g = mo.backward(cache, dy)
    live = np.flatnonzero(np.abs(g) > 1e-6)
    for i in rng.choice(live, size=40, replace=False):
        h = 1e-6
        p1, p2 = params.copy(), params.copy()
        p1[i] += h
        p2[i] -= h
        fd = (loss(p1) - loss(p2)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(g[i]), (i, fd, g[i])


def test_oracle_adam_step():
    p = np.ones(4)
    g = np.array([1.0, -1.0, 0.5, 0.0])
    p2, m, v = mo.adam(p, g, np.zeros(4), np.zeros(4), 1, lr=0.1)
    # The first bias-corrected step moves each parameter by lr * sign(g).
    assert np.allclose(p2, [0.9, 1.1, 0.9, 1.0], atol=1e-6)
