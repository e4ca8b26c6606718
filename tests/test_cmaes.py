"""CMA-ES restatement (host logic, CPU): converges on box-bounded quadratics, also when told only
a subset of each generation (the surrogate's fallback mode)."""

import numpy as np

from flyzero_b200.cmaes import CMAES


def _ellipsoid(X, opt):
    s = 10.0 ** np.linspace(0, 2, X.shape[1])
    return np.sum(s * (X - opt) ** 2, axis=1)


def test_cmaes_finds_the_box_optimum():
    opt = np.linspace(0.15, 0.85, 12)
    es = CMAES(np.full(12, 0.5), 0.3, popsize=32, seed=1)
    for _ in range(150):
        X = es.ask()
        es.tell(X, _ellipsoid(X, opt))
    assert np.abs(es.mean - opt).max() < 2e-3


def test_cmaes_respects_bounds_and_subset_tells():
    opt = np.r_[np.zeros(6), np.ones(6)]           # on the box's corner
    es = CMAES(np.full(12, 0.5), 0.3, popsize=256, seed=2)
    for _ in range(60):
        X = es.ask()
        assert X.min() >= 0.0 and X.max() <= 1.0
        f = _ellipsoid(X, opt)
        top = np.argsort(f)[:16]
        es.tell(X[top], f[top])                    # only 16 of 256 evaluated
    assert np.abs(np.clip(es.mean, 0, 1) - opt).max() < 0.05
