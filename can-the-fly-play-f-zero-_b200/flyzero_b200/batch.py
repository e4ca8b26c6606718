"""Learning rules for a ``BatchBrain`` (many instances at once): the drop-in for the reward rule and
the plastic bookkeeping of ``flyzero.batch`` (flyzero/batch.py:141-223, 454-495).

Several slots (instances running different races) can belong to one fly (``fly_of_slot``): their
weight changes are averaged over the fly's learning slots and applied to every slot of the fly,
the sequential rule with a larger batch. ``BatchReward.step`` runs as one fused CUDA kernel pair
(fb_reward_step); ``_Plastic.apply`` keeps the reference's generic form (any ``dw``) in torch for
other rules.

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
    """Shared bookkeeping: the brain's plastic synapses, their caps and slot -> fly grouping."""

    def __init__(self, brain, cap: float, fly_of_slot=None):
        import torch

        self.brain = brain
        self.B = brain.B
        dev = brain.device
        self.pre = torch.as_tensor(brain.pl_pre, device=dev)
        self.post = torch.as_tensor(brain.pl_post, device=dev)
        self.w0 = torch.as_tensor(brain.w0, device=dev)
        self.sign = torch.sign(self.w0)
        self.wmax = np.float32(cap) * torch.maximum(torch.abs(self.w0), torch.tensor(np.float32(brain.p.w_syn), device=dev))
        fos = np.arange(self.B) if fly_of_slot is None else np.asarray(fly_of_slot)
        self.fly_of_slot = fos
        self.n_flies = int(fos.max()) + 1
        self._fos = torch.as_tensor(fos, device=dev)
        order = np.argsort(fos, kind="stable")
        self._fly_ptr = torch.as_tensor(np.r_[0, np.cumsum(np.bincount(fos, minlength=self.n_flies))].astype(np.int32),
                                        device=dev)
        self._fly_slots = torch.as_tensor(order.astype(np.int32), device=dev)

    def _fly_weights(self, learn: np.ndarray) -> np.ndarray:
        """f32(1 / learning slots of the fly) per learning slot, 0 elsewhere (the onehot / n GEMM
        operand, batch.py:161-165)."""
        act = np.asarray(learn).astype(np.float32)
        n = np.bincount(self.fly_of_slot, weights=act, minlength=self.n_flies).astype(np.float32)
        return (act / np.maximum(n[self.fly_of_slot], np.float32(1.0))).astype(np.float32)

    def apply(self, dw, active: np.ndarray, sel=None):
        """Average ``dw`` (slots, n_pl) over each fly's active slots; update every slot of the fly.
        With ``sel`` (plastic indices), ``dw`` is (slots, len(sel)) and only those change."""
        import torch

        dev = self.brain.device
        onehot = torch.zeros((self.n_flies, self.B), dtype=torch.float32, device=dev)
        onehot[self._fos, torch.arange(self.B, device=dev)] = torch.as_tensor(np.asarray(active, np.float32), device=dev)
        n = onehot.sum(1, keepdim=True)
        dw = torch.as_tensor(dw, device=dev)
        per_fly = (onehot / torch.clamp(n, min=1.0)).to(dw.dtype) @ dw
        pw = self.brain.pw
        if sel is None:
            w = pw.to(per_fly.dtype) + per_fly[self._fos]
            pw[...] = (self.sign * torch.minimum(torch.clamp(self.sign * w, min=0.0), self.wmax)).to(pw.dtype)
        else:
            sel = torch.as_tensor(sel, device=dev)
            sign, wmax = self.sign[sel], self.wmax[sel]
            w = pw[:, sel].to(per_fly.dtype) + per_fly[self._fos]
            pw[:, sel] = (sign * torch.minimum(torch.clamp(sign * w, min=0.0), wmax)).to(pw.dtype)

    # consolidation: a slow copy of every plastic synapse (and of the bias) follows the fast one
    def consolidate(self, rate: float):
        if getattr(self, "_slow", None) is None:
            self._slow = (self.brain.pw.clone(), self.brain.bias_ext.clone())
        self._slow[0].add_(np.float32(rate) * (self.brain.pw - self._slow[0]))
        self._slow[1].add_(np.float32(rate) * (self.brain.bias_ext - self._slow[1]))

    def swap_slow(self):
        """Exchange the fast and the consolidated weights (call again to swap back)."""
        if getattr(self, "_slow", None) is None:
            return
        pw, bias = self._slow
        fast = (self.brain.pw.clone(), self.brain.bias_ext.clone())
        self.brain.pw.copy_(pw)
        self.brain.bias_ext.copy_(bias)
        self._slow = fast

    def state(self, fly: int) -> dict:
        slot = int(np.flatnonzero(self.fly_of_slot == fly)[0])
        return {"pos": self.brain.plastic_pos.astype(np.int32), "data": self.brain.pw[slot].cpu().numpy(),
                "w0": self.w0.cpu().numpy()}

    def load(self, st: dict, flies=None):
        """Load weights saved by this class or by the single-instance rules (entries matched by CSR
        position; positions not in the file keep their connectome values), batch.py:203-212."""
        import torch

        pos = self.brain.plastic_pos
        vals = self.w0.cpu().numpy().copy()
        where = np.searchsorted(pos, st["pos"])
        ok = (where < len(pos)) & (pos[np.minimum(where, len(pos) - 1)] == st["pos"])
        vals[where[ok]] = np.asarray(st["data"])[ok]
        slots = np.arange(self.B) if flies is None else np.flatnonzero(np.isin(self.fly_of_slot, flies))
        self.brain.pw[torch.as_tensor(slots, device=self.brain.device)] = torch.as_tensor(vals, device=self.brain.device)

    def drift(self) -> np.ndarray:
        """Mean relative change from the connectome, per slot."""
        return (self.brain.pw - self.w0).abs().div(self.wmax).mean(1).cpu().numpy()


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

    def reset(self, slots):
        s = np.atleast_1d(slots)
        self.elig[self._idx(s)] = 0
        self.noise[s] = 0

    def _idx(self, s):
        import torch

        return torch.as_tensor(np.asarray(s), device=self.brain.device)

    def exploration(self, window_ms: float) -> np.ndarray:
        """Extra Poisson rates (slots, len(self.targets)) for the target neurons."""
        a = window_ms / self.p.noise_tau_ms
        self.noise += -a * self.noise + np.sqrt(2 * a) * self.rng.standard_normal(self.noise.shape)
        return np.maximum(self.p.noise_hz * self.noise, 0.0)

    def _run(self, counts, coef, learn, window_ms):
        import torch

        p = self.p
        ae = np.exp(-window_ms / p.tau_elig_ms)
        ap = 1 - np.exp(-window_ms / p.tau_post_ms)
        apply = bool(np.asarray(learn).any())
        self._coef.copy_(torch.as_tensor(coef, dtype=torch.float64))
        self._fw.copy_(torch.as_tensor(self._fly_weights(learn)))
        b = self.brain
        _lib.check(b._L.fb_reward_step(b._h, _ptr(counts), _ptr(self.elig), _ptr(self.post_mean), _ptr(self._coef),
                                       _ptr(self._fly_ptr), _ptr(self._fly_slots), _ptr(self._fw), self.n_flies, None,
                                       float(ae), float(ap), float(np.float32(p.cap)), int(apply),
                                       C.c_void_p(torch.cuda.current_stream(b.device).cuda_stream)))

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
