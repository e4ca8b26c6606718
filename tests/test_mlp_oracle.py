"""The FP64 oracle of the surrogate MLP: analytic gradients against central differences (CPU)."""

import numpy as np

import mlp_oracle as MO


def test_oracle_gradients_match_central_differences():
    rng = np.random.default_rng(0)
    dims = (6, 5, 4, 3)
    params = [(rng.normal(0, 0.5, (dims[i + 1], dims[i])), rng.normal(0, 0.1, dims[i + 1])) for i in range(3)]
    X = rng.normal(0, 1, (7, dims[0]))
    Y = rng.poisson(1.5, (7, dims[-1])).astype(np.float64)
    L, grads = MO.loss_and_grads(params, X, Y)
    assert np.isclose(L, MO.loss(params, X, Y))
    for li in range(3):
        for which in (0, 1):
            g = grads[li][which]
            for idx in [tuple(rng.integers(0, s) for s in g.shape) for _ in range(4)]:
                num = MO.numeric_grad(params, X, Y, li, which, idx)
                assert abs(num - g[idx]) <= 1e-6 * max(1.0, abs(num)), (li, which, idx, num, g[idx])


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.01171875, -3.3e-3, 65504.0], np.float32)
    r = MO.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.015625      # ties to even, then up
    assert np.all(np.abs(r - x) <= np.abs(x) * 2.0 ** -8)
