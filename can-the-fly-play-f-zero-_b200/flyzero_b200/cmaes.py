"""CMA-ES for the interface calibration (the reference uses pycma, flyzero/tune.py:140-166;
pycma is not available here, so this is a restatement of the published algorithm: Hansen, "The
CMA Evolution Strategy: A Tutorial", arXiv:1604.00772, with rank-one and rank-mu covariance
updates, cumulative step-size adaptation and box bounds [0, 1] by clipping the evaluated points).

Minimises. ``tell`` accepts any number (>= 2) of evaluated points, so a generation may be told
only the candidates that were evaluated exactly (the surrogate's fallback mode).
"""

from __future__ import annotations

import numpy as np


class CMAES:
    def __init__(self, x0, sigma: float, popsize: int, seed: int = 0, lower: float = 0.0, upper: float = 1.0):
        self.mean = np.array(x0, dtype=np.float64)
        self.n = n = len(self.mean)
        self.sigma = float(sigma)
        self.lam = int(popsize)
        self.lower, self.upper = lower, upper
        self.rng = np.random.default_rng(seed)
        self.C = np.eye(n)
        self.B = np.eye(n)
        self.D = np.ones(n)
        self.pc = np.zeros(n)
        self.ps = np.zeros(n)
        self.gen = 0
        self.chiN = np.sqrt(n) * (1 - 1 / (4 * n) + 1 / (21 * n * n))

    def ask(self) -> np.ndarray:
        """`popsize` candidates (rows), clipped into the box."""
        z = self.rng.standard_normal((self.lam, self.n))
        x = self.mean + self.sigma * (z * self.D) @ self.B.T
        return np.clip(x, self.lower, self.upper)

    def tell(self, X, f):
        X = np.asarray(X, np.float64)
        f = np.asarray(f, np.float64)
        lam, n = len(f), self.n
        if lam < 2:
            raise ValueError("tell needs at least two evaluated points")
        mu = lam // 2
        w = np.log(mu + 0.5) - np.log(np.arange(1, mu + 1))
        w /= w.sum()
        mueff = 1.0 / np.sum(w * w)
        cc = (4 + mueff / n) / (n + 4 + 2 * mueff / n)
        cs = (mueff + 2) / (n + mueff + 5)
        c1 = 2 / ((n + 1.3) ** 2 + mueff)
        cmu = min(1 - c1, 2 * (mueff - 2 + 1 / mueff) / ((n + 2) ** 2 + mueff))
        damps = 1 + 2 * max(0.0, np.sqrt((mueff - 1) / (n + 1)) - 1) + cs
        sel = X[np.argsort(f, kind="stable")[:mu]]
        old = self.mean.copy()
        self.mean = w @ sel
        step = (self.mean - old) / self.sigma
        inv_sqrt_c = self.B @ np.diag(1 / self.D) @ self.B.T
        self.ps = (1 - cs) * self.ps + np.sqrt(cs * (2 - cs) * mueff) * (inv_sqrt_c @ step)
        hsig = (np.linalg.norm(self.ps) / np.sqrt(1 - (1 - cs) ** (2 * (self.gen + 1))) / self.chiN
                < 1.4 + 2 / (n + 1))
        self.pc = (1 - cc) * self.pc + hsig * np.sqrt(cc * (2 - cc) * mueff) * step
        art = (sel - old) / self.sigma
        self.C = ((1 - c1 - cmu) * self.C + c1 * (np.outer(self.pc, self.pc) + (1 - hsig) * cc * (2 - cc) * self.C)
                  + cmu * (art.T * w) @ art)
        self.sigma *= np.exp((cs / damps) * (np.linalg.norm(self.ps) / self.chiN - 1))
        self.C = (self.C + self.C.T) / 2
        evals, self.B = np.linalg.eigh(self.C)
        self.D = np.sqrt(np.maximum(evals, 1e-20))
        self.gen += 1
