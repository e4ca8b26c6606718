"""One whole-brain LIF instance with the reference's CPU-engine API, run on the B200 engine.

Drop-in for ``flyzero.brain.Brain`` (flyzero/brain.py:79-172): same constructor, ``reset``,
``set_bias``, ``set_input``, ``run(duration_ms) -> np.ndarray[int32]`` and the attributes callers
use (``n, p, v, g, ref, t, spike_count, indptr, indices, data, n_delay, n_ref, decay_m, decay_syn,
kick``). Host arrays stay host arrays: ``v``, ``g`` and ``ref`` are NumPy copies of the device
state, and writes to them (``b.v[:40] = -40``) or to ``data`` (learning rules write
``brain.data[pos]``, flyzero/learning.py:130) are carried to the device before the next ``run``.

Poisson input follows the reference stream by default (``rng="reference"``): every ``run`` draws
``seed_k = rng.integers(2**31)`` (brain.py:144) and the kicks are exactly those of
``np.random.seed(seed_k); np.random.random() < p_in`` per input per step (brain.py:34, :46-48),
precomputed on the host and handed to the engine as a bit raster. ``rng="device"`` uses the
engine's counter hash instead (faster; same distribution, different draws).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp


@dataclass
class LIFParams:
    v_rest: float = -52.0   # mV
    v_reset: float = -52.0  # mV
    v_th: float = -45.0     # mV
    tau_m: float = 20.0     # ms, membrane time constant
    tau_syn: float = 5.0    # ms, synaptic time constant
    t_ref: float = 2.2      # ms, refractory period
    delay: float = 1.8      # ms, synaptic delay
    w_syn: float = 0.275    # mV per synapse
    f_poisson: float = 250.0  # Poisson input weight = f_poisson * w_syn
    dt: float = 0.1         # ms


def pack_kicks(mask: np.ndarray) -> np.ndarray:
    """(..., k) bool -> (..., ceil(k/32)) uint32; bit j%32 of word j//32."""
    mask = np.asarray(mask, bool)
    k = mask.shape[-1]
    words = max(1, (k + 31) // 32)
    pad = np.zeros(mask.shape[:-1] + (words * 32,), bool)
    pad[..., :k] = mask
    return np.packbits(pad, axis=-1, bitorder="little").view(np.uint32).reshape(mask.shape[:-1] + (words,))


class Brain:
    def __init__(self, weights: sp.csr_matrix, params: LIFParams | None = None, seed: int = 0,
                 backend: str = "auto", *, rng: str = "reference", plastic_pos=None, device=None):
        from .gpu import BatchBrain

        self.p = p = params or LIFParams()
        self.backend = "b200"      # the reference's "numba"/"numpy" choice has no meaning here
        if rng not in ("reference", "device"):
            raise ValueError("rng must be 'reference' or 'device'")
        self.rng_mode = rng
        self._eng = BatchBrain(weights, p, 1, seed, plastic_pos, device=device)
        e = self._eng
        self.n = e.n
        self.indptr, self.indices = e.indptr, e.indices
        self.data = e.data                       # host float32 (count * w_syn), writable
        self._data_synced = self.data.copy()
        self.rng = np.random.default_rng(seed)
        self.n_delay, self.n_ref = e.n_delay, e.n_ref
        self.decay_m, self.decay_syn, self.kick = e.decay_m, e.decay_syn, e.kick
        self.input_idx = np.zeros(0, np.int64)
        self.input_rate = np.zeros(0, np.float32)
        self.bias = np.zeros(self.n, np.float32)
        self._cache = {}
        self.t = 0
        self.spike_count = np.zeros(self.n, np.int32)

    # ---- state views ----------------------------------------------------------------------------
    def _host(self, name):
        if name not in self._cache:
            a = getattr(self._eng, name)[0].cpu().numpy()
            self._cache[name] = (a, a.copy())
        return self._cache[name][0]

    v = property(lambda self: self._host("v"))
    g = property(lambda self: self._host("g"))
    ref = property(lambda self: self._host("ref"))

    def _push_host_state(self):
        import torch

        for name, (a, snap) in self._cache.items():
            if not np.array_equal(a, snap):
                getattr(self._eng, name)[0].copy_(torch.as_tensor(a))
        self._cache = {}

    def _push_data(self):
        """Carry writes to ``data`` to the engine: changed entries become plastic (their weight is
        then per instance and takes effect for spikes after this point, as in the reference)."""
        import torch

        changed = np.flatnonzero(self.data != self._data_synced)
        if len(changed) == 0:
            return
        e = self._eng
        if not np.isin(changed, e.plastic_pos).all():
            e.make_plastic(changed)
        k = np.searchsorted(e.plastic_pos, changed)
        e.pw[0, torch.as_tensor(k, device=e.device)] = torch.as_tensor(self.data[changed], device=e.device)
        self._data_synced[changed] = self.data[changed]

    # ---- the reference API (flyzero/brain.py:104-172) ---------------------------------------------
    def reset(self):
        self._eng.reset()
        self._cache = {}
        self.t = 0
        self.spike_count = np.zeros(self.n, np.int32)

    def set_bias(self, idx: np.ndarray, mv):
        """Steady depolarising current (in mV of steady-state shift) for the given neurons."""
        self.bias[:] = 0.0
        self.bias[np.asarray(idx, np.int64)] = mv

    def set_input(self, idx: np.ndarray, rate_hz):
        """Poisson drive (Hz) for the given neurons, replacing previous input."""
        self.input_idx = np.asarray(idx, np.int64)
        self.input_rate = np.broadcast_to(np.asarray(rate_hz, np.float32), self.input_idx.shape).copy()

    def run(self, duration_ms: float) -> np.ndarray:
        """Advance the simulation; returns per-neuron spike counts for this window."""
        import torch

        e = self._eng
        steps = max(1, int(round(duration_ms / self.p.dt)))
        self._push_host_state()
        self._push_data()
        bias_idx = np.flatnonzero(self.bias)
        if len(self.input_idx) or len(bias_idx):
            e.slots(np.r_[self.input_idx, bias_idx])
        if e.bias_ext.shape[1]:
            e.bias_ext.zero_()
            if len(bias_idx):
                e.bias_ext[0, torch.as_tensor(e._slot[bias_idx], device=e.device)] = torch.as_tensor(
                    self.bias[bias_idx], device=e.device)
        p_in = self.input_rate * np.float32(self.p.dt / 1000.0)
        kicks = None
        if self.rng_mode == "reference":
            seed_k = int(self.rng.integers(2 ** 31))
            if len(self.input_idx):
                if len(np.unique(self.input_idx)) != len(self.input_idx):
                    raise ValueError("duplicate input neurons are not supported with rng='reference'")
                draws = np.random.RandomState(seed_k).random_sample((steps, len(p_in))) < p_in.astype(np.float64)
                raster = np.zeros((steps, 1, e.p_ext.shape[1]), bool)
                raster[:, 0, e._slot[self.input_idx]] = draws
                kicks = torch.as_tensor(pack_kicks(raster).view(np.int32), device=e.device)
        else:
            e.p_ext.zero_()
            if len(self.input_idx):
                e.p_ext[0, torch.as_tensor(e._slot[self.input_idx], device=e.device)] = torch.as_tensor(
                    p_in, device=e.device)
        dev_counts = e.run_steps(steps, kicks)
        counts = dev_counts[0].cpu().numpy()
        self._last = (counts, dev_counts)
        self.t += steps
        self.spike_count += counts
        return counts

    def device_counts(self, counts: np.ndarray):
        """(1, n) int32 device tensor of ``counts``: the engine's own copy if ``counts`` is what the
        last ``run`` returned, else an upload."""
        import torch

        last = getattr(self, "_last", None)
        if last is not None and last[0] is counts:
            return last[1]
        return torch.as_tensor(np.asarray(counts, np.int32).reshape(1, -1), device=self._eng.device)
