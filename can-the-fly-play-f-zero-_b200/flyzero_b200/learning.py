"""Reward learning on the plastic synapses onto descending neurons, run on the B200 engine.

Drop-in for ``flyzero.learning.RewardPlasticity`` (flyzero/learning.py:89-142): the exploratory-
Hebbian rule of Hoerzer, Legenstein & Maass (2014),

    E_ij <- lambda * E_ij + pre_i * (post_j - <post_j>)        w_ij <- w_ij + eta * (R - <R>) * E_ij

with Dale's law and caps (w keeps its sign, |w| <= cap * max(|w0|, w_syn)). The per-synapse update is
one fused CUDA kernel (fb_reward_step); it is bit-exact to the reference's NumPy arithmetic (float64
traces and weights rounded to float32). The new weights land in the engine's per-instance plastic
weights and, as in the reference, in ``brain.data[pos]``.

``targets`` may be given directly; otherwise they are found by cell type through ``conn.find`` as
the reference does (learning.py:94), which needs a connectome with cell-type annotations.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib


@dataclass
class LearnParams:
    eta: float = 2e-4             # mV per unit of (reward x eligibility)
    tau_elig_ms: float = 500.0
    tau_post_ms: float = 500.0
    tau_reward_ms: float = 1000.0
    cap: float = 3.0              # |w| <= cap * max(|w0|, one synapse)
    noise_hz: float = 20.0        # exploratory drive to the targets (OU-modulated Poisson)
    noise_tau_ms: float = 300.0
    targets: tuple = ("DNa02", "DNa01", "DNg02*", "DNp09", "MDN")
    hurt_hz: float = 200.0
    hurt_ms: float = 150.0
    w_speed: float = 0.2
    w_progress: float = 20.0
    w_reverse: float = 60.0
    w_crash: float = 100.0
    w_rank: float = 0.0


def find_targets(conn, types) -> np.ndarray:
    return np.unique(np.concatenate([conn.find(t) for t in types])).astype(np.int64)


def _dev(torch, x, dtype, device):
    return torch.as_tensor(np.ascontiguousarray(x), dtype=dtype, device=device)


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


class RewardPlasticity:
    """One instance (a ``Brain``) learning from a scalar reward per frame."""

    def __init__(self, brain, conn=None, params: LearnParams | None = None, seed: int = 0, targets=None):
        import torch

        self.p = p = params or LearnParams()
        self.brain = brain
        self.rng = np.random.default_rng(seed)
        targets = find_targets(conn, p.targets) if targets is None else np.unique(np.asarray(targets, np.int64))
        self.targets = targets
        is_target = np.zeros(brain.n, bool)
        is_target[targets] = True
        self.pos = np.flatnonzero(is_target[brain.indices])            # plastic entries in CSR data
        rows = np.repeat(np.arange(brain.n), np.diff(brain.indptr))
        self.pre = rows[self.pos]
        self.post = brain.indices[self.pos]
        self.w0 = brain.data[self.pos].copy()
        self.sign = np.sign(self.w0)
        self.wmax = p.cap * np.maximum(np.abs(self.w0), brain.p.w_syn)
        self.post_mean = np.zeros(brain.n, np.float32)
        self.r_mean = 0.0
        self.noise = np.zeros(len(targets))
        # the engine holds these entries as per-instance plastic weights
        eng = brain._eng
        if not np.isin(self.pos, eng.plastic_pos).all():
            eng.make_plastic(self.pos)
        self._k = np.searchsorted(eng.plastic_pos, self.pos)
        dev = eng.device
        mask = np.zeros(len(eng.plastic_pos), np.uint8)
        mask[self._k] = 1
        self._mask = _dev(torch, mask, torch.uint8, dev)
        self._elig = torch.zeros((1, len(eng.plastic_pos)), dtype=torch.float64, device=dev)
        n_ppost = len(np.unique(eng.pl_post))
        self._post_mean = torch.zeros((1, n_ppost), dtype=torch.float32, device=dev)
        self._coef = torch.zeros(1, dtype=torch.float64, device=dev)
        self._fly_ptr = _dev(torch, [0, 1], torch.int32, dev)
        self._fly_slots = _dev(torch, [0], torch.int32, dev)
        self._fly_w = _dev(torch, [1.0], torch.float32, dev)

    @property
    def elig(self) -> np.ndarray:
        return self._elig[0, self._k].cpu().numpy()

    def exploration(self, window_ms: float):
        """Extra Poisson drive to the target neurons (indices, Hz) for the next window."""
        a = window_ms / self.p.noise_tau_ms
        self.noise += -a * self.noise + np.sqrt(2 * a) * self.rng.standard_normal(len(self.noise))
        return self.targets, np.maximum(self.p.noise_hz * self.noise, 0.0)

    def step(self, counts: np.ndarray, reward: float, window_ms: float):
        import torch

        p = self.p
        ae = np.exp(-window_ms / p.tau_elig_ms)
        ap = 1 - np.exp(-window_ms / p.tau_post_ms)
        ar = 1 - np.exp(-window_ms / p.tau_reward_ms)
        self.brain._push_data()                  # weights written to brain.data since the last run
        c_dev = self.brain.device_counts(counts)
        adv = reward - self.r_mean
        self.r_mean += ar * adv
        self._coef.fill_(float(p.eta * adv))
        eng = self.brain._eng
        _lib.check(eng._L.fb_reward_step(eng._h, _ptr(c_dev), _ptr(self._elig), _ptr(self._post_mean),
                                         _ptr(self._coef), _ptr(self._fly_ptr), _ptr(self._fly_slots),
                                         _ptr(self._fly_w), 1, _ptr(self._mask), float(ae), float(ap),
                                         float(np.float32(p.cap)), 1,
                                         C.c_void_p(torch.cuda.current_stream(eng.device).cuda_stream)))
        # the reference's own record of the targets' mean counts (learning.py:124)
        c = np.asarray(counts).astype(np.float32)
        t = self.targets
        self.post_mean[t] += ap * (c[t] - self.post_mean[t])
        w = eng.pw[0, torch.as_tensor(self._k, device=eng.device)].cpu().numpy()
        self.brain.data[self.pos] = w
        self.brain._data_synced[self.pos] = w
        return adv

    def state(self) -> dict:
        return {"pos": self.pos, "data": self.brain.data[self.pos].copy(), "w0": self.w0}

    def load(self, st: dict):
        assert np.array_equal(st["pos"], self.pos)
        self.brain.data[self.pos] = st["data"]

    def drift(self) -> float:
        """Mean relative change of plastic weights from the connectome."""
        return float(np.mean(np.abs(self.brain.data[self.pos] - self.w0) / self.wmax))
