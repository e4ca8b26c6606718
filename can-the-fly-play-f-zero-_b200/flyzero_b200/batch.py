"""Learning rules for a ``BatchBrain`` (many instances at once): the drop-in for the reward rule and
the plastic bookkeeping of ``flyzero.batch`` (flyzero/batch.py:141-223, 454-495).

Several slots (instances running different races) can belong to one fly (``fly_of_slot``): their
weight changes are averaged over the fly's learning slots and applied to every slot of the fly,
the sequential rule with a larger batch. ``BatchReward.step`` runs as one fused CUDA kernel pair
(fb_reward_step); ``_Plastic.apply`` takes any ``dw`` through the engine's fused per-fly delta
kernel (fb_delta_apply).

Arithmetic follows NumPy's promotion rules, as the CPU rule (flyzero/learning.py) computes them:
float64 eligibility traces, float32 running means, float32 weights.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .learning import LearnParams, find_targets

PLASTIC_TYPES = ("DNa02", "DNa01", "DNg02*", "DNp09", "MDN", "DNp01")


def plastic_positions(conn, types=PLASTIC_TYPES) -> np.ndarray:
    """CSR positions (``Brain.data`` layout) of every synapse onto the given cell types."""
    import scipy.sparse as sp

    targets = find_targets(conn, types)
    is_t = np.zeros(conn.n, bool)
    is_t[targets] = True
    w = sp.csr_matrix(conn.weights, dtype=np.float32)
    w.sort_indices()
    return np.flatnonzero(is_t[w.indices])


def save_state(path, st: dict):
    """Plastic weights of one fly as the reference stores them: an npz with ``pos`` (CSR
    positions), ``data`` (weights, mV), ``w0`` and, with intrinsic plasticity, ``bias_idx`` /
    ``bias`` (flyzero/batch.py:195-219)."""
    np.savez(path, **{k: np.asarray(v) for k, v in st.items()})


def load_state(path) -> dict:
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


class _Plastic:
    """Per-slot plastic weights of a ``BatchBrain`` grouped into flies, kept on the device.

    The engine stores slot b's weights as row b of ``brain.pw``. Slots that belong to one fly
    (``fly_of_slot``) share learning: a weight change is the mean over the fly's learning slots and
    lands on all of its slots. Flies are kept as a CSR over slots (``_fly_ptr``, ``_fly_slots``),
    the form the engine's fused kernels (fb_reward_step, fb_delta_apply) take; ``sign`` and
    ``wmax`` bound every weight to [0, wmax] on its connectome sign (the cap of
    flyzero/batch.py:141-156)."""

    def __init__(self, brain, cap: float, fly_of_slot=None):
        import torch

        self.brain = brain
        self.B = brain.B
        dev = brain.device
        self.pre = torch.as_tensor(brain.pl_pre, device=dev)
        self.post = torch.as_tensor(brain.pl_post, device=dev)
        w0 = np.asarray(brain.w0, np.float32)
        self.w0 = torch.as_tensor(w0, device=dev)
        self.sign = torch.as_tensor(np.sign(w0).astype(np.float32), device=dev)
        cap_w = np.float32(cap) * np.maximum(np.abs(w0), np.float32(brain.p.w_syn))
        self.wmax = torch.as_tensor(cap_w.astype(np.float32), device=dev)
        fos = np.arange(self.B) if fly_of_slot is None else np.asarray(fly_of_slot)
        self.fly_of_slot = fos
        self.n_flies = int(fos.max()) + 1
        self._fos = torch.as_tensor(fos, device=dev)
        per_fly = np.bincount(fos, minlength=self.n_flies)
        self._fly_ptr = torch.as_tensor(np.concatenate([[0], np.cumsum(per_fly)]).astype(np.int32), device=dev)
        self._fly_slots = torch.as_tensor(np.argsort(fos, kind="stable").astype(np.int32), device=dev)
        self._slow = None

    def _fly_weights(self, learn: np.ndarray) -> np.ndarray:
        """Per slot: f32(1 / number of learning slots of its fly) if it learns, else 0."""
        on = np.asarray(learn).astype(np.float32)
        count = np.bincount(self.fly_of_slot, weights=on, minlength=self.n_flies).astype(np.float32)
        return (on / np.maximum(count[self.fly_of_slot], np.float32(1.0))).astype(np.float32)

    def apply(self, dw, active: np.ndarray, sel=None):
        """Add to every slot the mean of ``dw`` (slots, n_pl, float32) over its fly's ``active``
        slots, then clip on the sign; with ``sel`` (plastic indices) ``dw`` is (slots, len(sel)) and
        only those weights change. One fb_delta_apply launch: ``dw`` enters as the trace, the
        per-slot mean weight as the coefficient and a unit error, so the kernel's per-fly sum is the
        average (summed in slot order)."""
        import torch

        b = self.brain
        dev = b.device
        d = torch.as_tensor(dw, device=dev).to(torch.float32).contiguous()
        idx = (torch.arange(d.shape[1], dtype=torch.int32, device=dev) if sel is None
               else torch.as_tensor(np.asarray(sel), device=dev).to(torch.int32).contiguous())
        if sel is None and d.shape[1] != b.pw.shape[1]:
            raise ValueError(f"dw has {d.shape[1]} columns, the brain {b.pw.shape[1]} plastic synapses")
        col = torch.arange(d.shape[1], dtype=torch.int32, device=dev)
        unit = torch.ones((self.B, 1), dtype=torch.float32, device=dev)
        zero = torch.zeros(d.shape[1], dtype=torch.int32, device=dev)
        coef = torch.as_tensor(self._fly_weights(active), device=dev)
        st = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        _lib.check(b._L.fb_delta_apply(b._h, _ptr(idx), _ptr(col), _ptr(zero), d.shape[1], _ptr(d), d.shape[1],
                                       _ptr(unit), 1, _ptr(coef), _ptr(self._fly_ptr), _ptr(self._fly_slots),
                                       self.n_flies, _ptr(self.sign), _ptr(self.wmax), st))

    # Consolidation: a slow copy of the plastic weights and of the biases trails the fast ones as an
    # exponential moving average (the fast/slow synapse pair of flyzero/batch.py:174-193).
    def consolidate(self, rate: float):
        fast = (self.brain.pw, self.brain.bias_ext)
        if self._slow is None:
            self._slow = tuple(t.clone() for t in fast)
        r = np.float32(rate)
        for slow, cur in zip(self._slow, fast):
            slow.add_((cur - slow) * r)

    def swap_slow(self):
        """Exchange the fast and the consolidated weights (call again to swap back)."""
        if self._slow is not None:
            held = tuple(t.clone() for t in (self.brain.pw, self.brain.bias_ext))
            self.brain.pw.copy_(self._slow[0])
            self.brain.bias_ext.copy_(self._slow[1])
            self._slow = held

    def state(self, fly: int) -> dict:
        """The fly's weights in the reference's npz layout {pos, data, w0}."""
        first = int(np.argmax(self.fly_of_slot == fly))
        return {"pos": self.brain.plastic_pos.astype(np.int32), "data": self.brain.pw[first].cpu().numpy(),
                "w0": self.w0.cpu().numpy()}

    def load(self, st: dict, flies=None):
        """Weights saved by this class or by the single-instance rules, matched by CSR position;
        plastic synapses the file does not name start from their connectome weight."""
        import torch

        mine = np.asarray(self.brain.plastic_pos, np.int64)
        _, at_mine, at_file = np.intersect1d(mine, np.asarray(st["pos"], np.int64), assume_unique=True,
                                             return_indices=True)
        row = self.w0.cpu().numpy().copy()
        row[at_mine] = np.asarray(st["data"], np.float32)[at_file]
        slots = np.arange(self.B) if flies is None else np.flatnonzero(np.isin(self.fly_of_slot, flies))
        dev = self.brain.device
        self.brain.pw.index_copy_(0, torch.as_tensor(slots, device=dev),
                                  torch.as_tensor(row, device=dev).expand(len(slots), -1).contiguous())

    def drift(self) -> np.ndarray:
        """Per slot: mean over the plastic synapses of |w - w0| / wmax."""
        import torch

        return torch.mean(torch.abs(self.brain.pw - self.w0) / self.wmax, dim=1).cpu().numpy()


class BatchReward(_Plastic):
    """Exploratory-Hebbian reward learning for every slot (flyzero/batch.py:454-495)."""

    def __init__(self, brain, conn=None, params: LearnParams | None = None, fly_of_slot=None, seed=0, targets=None):
        import torch

        self.p = p = params or LearnParams()
        super().__init__(brain, p.cap, fly_of_slot)
        self.rng = np.random.default_rng(seed)
        self.targets = find_targets(conn, p.targets) if targets is None else np.unique(np.asarray(targets, np.int64))
        self.upre, pre_inv = np.unique(brain.pl_pre, return_inverse=True)
        self.upost, post_inv = np.unique(brain.pl_post, return_inverse=True)
        dev = brain.device
        self.pre_k, self.post_k = torch.as_tensor(pre_inv, device=dev), torch.as_tensor(post_inv, device=dev)
        self.elig = torch.zeros((self.B, len(brain.plastic_pos)), dtype=torch.float64, device=dev)
        self.post_mean = torch.zeros((self.B, len(self.upost)), dtype=torch.float32, device=dev)
        self.r_mean = np.zeros(self.B, np.float32)
        self.noise = np.zeros((self.B, len(self.targets)))
        self._coef = torch.zeros(self.B, dtype=torch.float64, device=dev)
        self._fw = torch.zeros(self.B, dtype=torch.float32, device=dev)
        # the per-window scalars reach the device through pinned buffers: a step never blocks the host
        self._coef_in = _lib.HostStage(self.B, torch.float64)
        self._fw_in = _lib.HostStage(self.B, torch.float32)

    def reset(self, slots):
        s = np.atleast_1d(slots)
        self.elig[self._idx(s)] = 0
        self.noise[s] = 0

    def _idx(self, s):
        import torch

        return torch.as_tensor(np.asarray(s), device=self.brain.device)

    def exploration(self, window_ms: float) -> np.ndarray:
        """Extra Poisson rates (slots, len(self.targets)) for the target neurons: one Euler step of
        an Ornstein-Uhlenbeck process per window (time constant noise_tau_ms, unit stationary
        variance), rectified and scaled by noise_hz. The float64 operations and the generator's
        draws are those of flyzero/batch.py:476-480, so equal seeds give the reference's drive."""
        h = window_ms / self.p.noise_tau_ms
        shock = np.sqrt(2 * h) * self.rng.standard_normal(self.noise.shape)
        self.noise += shock - h * self.noise
        return np.maximum(self.p.noise_hz * self.noise, 0.0)

    def _run(self, counts, coef, learn, window_ms):
        import torch

        p = self.p
        ae = np.exp(-window_ms / p.tau_elig_ms)
        ap = 1 - np.exp(-window_ms / p.tau_post_ms)
        apply = bool(np.asarray(learn).any())
        b = self.brain
        stream = torch.cuda.current_stream(b.device)
        self._coef_in.put(self._coef, np.asarray(coef, np.float64))
        self._fw_in.put(self._fw, self._fly_weights(learn))
        _lib.check(b._L.fb_reward_step(b._h, _ptr(counts), _ptr(self.elig), _ptr(self.post_mean), _ptr(self._coef),
                                       _ptr(self._fly_ptr), _ptr(self._fly_slots), _ptr(self._fw), self.n_flies, None,
                                       float(ae), float(ap), float(np.float32(p.cap)), int(apply),
                                       C.c_void_p(stream.cuda_stream)))

    def step(self, counts, reward: np.ndarray, learn: np.ndarray, window_ms: float):
        """``counts``: device (slots, n) int32 of the window just run; ``reward``: (slots,);
        ``learn``: bool per slot. Returns the advantage per slot (batch.py:482-495)."""
        p = self.p
        ar = 1 - np.exp(-window_ms / p.tau_reward_ms)
        adv = np.asarray(reward, np.float64) - self.r_mean
        self.r_mean += ar * adv
        coef = (np.float32(p.eta) * adv.astype(np.float32)).astype(np.float64)   # eta * f32(adv), in f32
        self._run(counts, coef, learn, window_ms)
        return adv

    def step_scaled(self, counts, reward: np.ndarray, learn: np.ndarray, window_ms: float, eta_slot):
        """``step`` with a per-slot learning rate (flyzero/school.py:289-304)."""
        p = self.p
        ar = 1 - np.exp(-window_ms / p.tau_reward_ms)
        adv = np.asarray(reward, np.float64) - self.r_mean
        self.r_mean += ar * adv
        coef = (np.asarray(eta_slot) * adv).astype(np.float32).astype(np.float64)
        self._run(counts, coef, learn, window_ms)
        return adv
