"""Instructed plasticity for a ``BatchBrain``: the delta rule towards a teacher's target rates on
the synapses onto the motor descending neurons (DNs), and its deep versions that pass the DN error
back through the fly's own synapses one or two layers (flyzero/batch.py:226-451).

Every per-synapse operation runs as the library's CUDA kernels (include/flybrain.h:
fb_trace_rates, fb_backprop, fb_delta_apply); torch only holds the buffers. Groups are neuron
index arrays in ``GROUPS`` order (the reference resolves them by cell type and side through
``conn.find``; ``groups_from_connectome`` does that for a connectome with types).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp

from . import _lib

# name: (cell type, side); the batched rules also instruct the giant fiber (flyzero/batch.py:22)
GROUPS = {"a02L": ("DNa02", "left"), "a02R": ("DNa02", "right"), "g02L": ("DNg02*", "left"),
          "g02R": ("DNg02*", "right"), "a01L": ("DNa01", "left"), "a01R": ("DNa01", "right"),
          "gas": ("DNp09", None), "brake": ("MDN", None), "gf": ("DNp01", None)}


@dataclass
class InstructParams:
    eta: float = 2e-4
    tau_pre_ms: float = 50.0
    tau_rate_ms: float = 80.0
    high_hz: float = 80.0
    low_hz: float = 0.0
    rest_hz: float = 20.0
    cap: float = 3.0


def targets(x, p: InstructParams) -> list:
    """Target rates in ``GROUPS`` order for an intent vector (steer, lean, gas, brake, boost)
    (flyzero/instruct.py:69-79 with the giant fiber of flyzero/batch.py:67-72)."""
    steer, lean, gas, brake = (float(v) for v in x[:4])
    hi, lo, rest = p.high_hz, p.low_hz, p.rest_hz

    def pair(v):
        return (rest + (hi - rest) * max(-v, 0) - (rest - lo) * max(v, 0),
                rest + (hi - rest) * max(v, 0) - (rest - lo) * max(-v, 0))

    a02L, a02R = pair(steer)
    t = {"a02L": a02L, "a02R": a02R, "g02L": a02R, "g02R": a02L,
         "a01L": lo + (hi - lo) * max(-lean, 0), "a01R": lo + (hi - lo) * max(lean, 0),
         "gas": lo + (hi - lo) * gas, "brake": lo + (hi - lo) * brake,
         "gf": lo + (hi - lo) * float(x[4])}
    return [t[g] for g in GROUPS]


def groups_from_connectome(conn) -> dict:
    return {g: np.asarray(conn.find(t, s), np.int64) for g, (t, s) in GROUPS.items()}


def _csr_rows(weights):
    w = sp.csr_matrix(weights, dtype=np.float32)
    w.sort_indices()
    return w, np.repeat(np.arange(w.shape[0]), np.diff(w.indptr))


def deep_positions(weights, dn_pos) -> np.ndarray:
    """CSR positions of every synapse onto the DNs' presynaptic partners (L1)."""
    w, rows = _csr_rows(weights)
    is_l1 = np.zeros(w.shape[0], bool)
    is_l1[np.unique(rows[dn_pos])] = True
    return np.flatnonzero(is_l1[w.indices])


def deep2_positions(weights, dn_pos) -> np.ndarray:
    """CSR positions of every synapse onto L2 (the inputs of L1), leaving out L1 and the DNs."""
    w, rows = _csr_rows(weights)
    l1 = np.unique(rows[dn_pos])
    is_l1 = np.zeros(w.shape[0], bool)
    is_l1[l1] = True
    l2 = np.unique(rows[is_l1[w.indices]])
    is_l2 = np.zeros(w.shape[0], bool)
    is_l2[l2] = True
    is_l2[l1] = False
    is_l2[w.indices[dn_pos]] = False
    return np.flatnonzero(is_l2[w.indices])


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


class BatchInstruct:
    """Delta rule towards the teacher's target rates, every slot (flyzero/batch.py:226-315)."""

    def __init__(self, brain, groups: dict, params: InstructParams | None = None, fly_of_slot=None,
                 eta_bias: float = 0.0, bias_limit: float = 8.0):
        import torch

        self.p = p = params or InstructParams()
        self.brain = brain
        self.B = B = brain.B
        self.dev = dev = brain.device
        self.names = list(GROUPS)
        fos = np.arange(B) if fly_of_slot is None else np.asarray(fly_of_slot)
        self.fly_of_slot = fos
        self.n_flies = int(fos.max()) + 1
        order = np.argsort(fos, kind="stable")
        self._fly_ptr = torch.as_tensor(np.r_[0, np.cumsum(np.bincount(fos, minlength=self.n_flies))].astype(np.int32),
                                        device=dev)
        self._fly_slots = torch.as_tensor(order.astype(np.int32), device=dev)
        self.w0 = brain.w0.astype(np.float32)
        self.sign_h = np.sign(self.w0).astype(np.float32)
        self.wmax_h = (np.float32(p.cap) * np.maximum(np.abs(self.w0), np.float32(brain.p.w_syn))).astype(np.float32)
        self.sign = torch.as_tensor(self.sign_h, device=dev)
        self.wmax = torch.as_tensor(self.wmax_h, device=dev)
        self.eta_bias, self.bias_limit = eta_bias, bias_limit
        group_of = np.full(brain.n, -1, np.int32)
        for k, g in enumerate(self.names):
            group_of[np.asarray(groups.get(g, []), np.int64)] = k
        self.group_of = group_of
        pg = group_of[brain.pl_post]
        self.mask_h = pg >= 0
        self.post_group_h = np.maximum(pg, 0)
        self.upre, self.pre_k_h = np.unique(brain.pl_pre, return_inverse=True)
        self.upost, self.post_k_h = np.unique(brain.pl_post, return_inverse=True)
        i32 = lambda a: torch.as_tensor(np.asarray(a, np.int32), device=dev)
        self.d_upre, self.d_upost = i32(self.upre), i32(self.upost)
        self.trace = torch.zeros((B, len(self.upre)), dtype=torch.float32, device=dev)
        self.rate = torch.zeros((B, len(self.upost)), dtype=torch.float32, device=dev)
        self.upost_group = torch.as_tensor(group_of[self.upost].astype(np.int64), device=dev)
        self.group_members = [np.flatnonzero(group_of[self.upost] == k) for k in range(len(self.names))]
        self.dn_sel_h = np.flatnonzero(self.mask_h)                      # synapses onto the DNs
        self.dn_sel, self.dn_pre_k, self.dn_post_k = (i32(self.dn_sel_h), i32(self.pre_k_h[self.dn_sel_h]),
                                                      i32(self.post_k_h[self.dn_sel_h]))
        self.dn = np.flatnonzero(group_of >= 0)
        self.ib = None
        if eta_bias > 0:
            self.dn_group = torch.as_tensor(group_of[self.dn].astype(np.int64), device=dev)
            self.dn_rate_k = torch.as_tensor(np.searchsorted(self.upost, self.dn), device=dev)
            self.dn_slots = brain.slots(self.dn).long()
            self.ib = torch.zeros((B, len(self.dn)), dtype=torch.float32, device=dev)
        self._coef = torch.zeros(B, dtype=torch.float32, device=dev)
        self._err = torch.zeros((B, len(self.upost)), dtype=torch.float32, device=dev)

    def _stream(self):
        import torch

        return C.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)

    def reset(self, slots):
        s = list(np.atleast_1d(slots))
        self.trace[s] = 0
        self.rate[s] = 0

    def _coefs(self, learn, eta, scale=1.0):
        """Per-slot coefficient: eta_b * scale / learning slots of its fly, 0 if not learning."""
        learn = np.asarray(learn, bool)
        eta_b = np.broadcast_to(np.asarray(eta, np.float32).ravel(), (self.B,)) * scale
        n_act = np.bincount(self.fly_of_slot, weights=learn, minlength=self.n_flies)
        return np.where(learn, eta_b / np.maximum(n_act[self.fly_of_slot], 1), 0.0).astype(np.float32)

    def _apply(self, sel, pre_k, post_x, x, coef):
        b = self.brain
        self._coef.copy_(self._torch().as_tensor(coef))
        _lib.check(b._L.fb_delta_apply(b._h, _p(sel), _p(pre_k), _p(post_x), len(sel), _p(self.trace),
                                       self.trace.shape[1], _p(x), x.shape[1], _p(self._coef), _p(self._fly_ptr),
                                       _p(self._fly_slots), self.n_flies, _p(self.sign), _p(self.wmax), self._stream()))

    @staticmethod
    def _torch():
        import torch

        return torch

    def step(self, counts, targets, learn, window_ms: float, eta=None):
        """``counts``: device (slots, n) int32; ``targets``: (slots, len(GROUPS)) Hz or None;
        ``learn``: bool per slot; ``eta`` scalar or per slot. Returns the mean |target - rate| per
        slot (0 where not learning), as batch.py:268-309."""
        torch = self._torch()
        p = self.p
        a_pre = 1 - np.exp(-window_ms / p.tau_pre_ms)
        a_rate = 1 - np.exp(-window_ms / p.tau_rate_ms)
        hz = 1000.0 / window_ms
        b = self.brain
        _lib.check(b._L.fb_trace_rates(b._h, _p(counts), _p(self.d_upre), len(self.upre), _p(self.trace), float(a_pre),
                                       float(np.float32(hz) * np.float32(p.tau_pre_ms / 1000.0)), _p(self.d_upost),
                                       len(self.upost), _p(self.rate), float(a_rate), float(hz), self._stream()))
        learn = np.asarray(learn, bool)
        if targets is None or not learn.any():
            return np.zeros(self.B)
        tgt = torch.as_tensor(np.asarray(targets, np.float32), device=self.dev)
        eta = p.eta if eta is None else eta
        self._learn(tgt, learn, eta)
        if self.ib is not None:
            err = tgt[:, self.dn_group] - self.rate[:, self.dn_rate_k]
            act = torch.as_tensor(learn.astype(np.float32), device=self.dev)
            onehot = torch.zeros((self.n_flies, self.B), dtype=torch.float32, device=self.dev)
            onehot[torch.as_tensor(self.fly_of_slot, device=self.dev), torch.arange(self.B, device=self.dev)] = act
            per_fly = (onehot / torch.clamp(onehot.sum(1, keepdim=True), min=1.0)) @ err
            scale = torch.as_tensor(np.asarray(eta, np.float32) / p.eta, device=self.dev).reshape(-1, 1)
            step = self.eta_bias * per_fly[torch.as_tensor(self.fly_of_slot, device=self.dev)] * scale
            new = torch.clamp(self.ib + step, -self.bias_limit, self.bias_limit)
            self.brain.bias_ext[:, self.dn_slots] += new - self.ib
            self.ib = new
        rate = self.rate.cpu().numpy()
        out = np.zeros(self.B)
        for k, mem in enumerate(self.group_members):
            if len(mem):
                out += np.abs(np.asarray(targets)[:, k] - rate[:, mem].mean(1))
        return np.where(learn, out / len(self.names), 0.0)

    def state(self, fly: int) -> dict:
        """One fly's plastic weights (and learned intrinsic biases), batch.py:195-201."""
        slot = int(np.flatnonzero(self.fly_of_slot == fly)[0])
        st = {"pos": self.brain.plastic_pos.astype(np.int32), "data": self.brain.pw[slot].cpu().numpy(), "w0": self.w0}
        if self.ib is not None:
            st["bias_idx"], st["bias"] = self.dn, self.ib[slot].cpu().numpy()
        return st

    def load(self, st: dict, flies=None):
        """Weights saved by any of the rules (matched by CSR position; positions not in the file
        keep their connectome values) and saved intrinsic biases (batch.py:203-219)."""
        torch = self._torch()
        pos = self.brain.plastic_pos
        vals = self.w0.copy()
        where = np.searchsorted(pos, st["pos"])
        ok = (where < len(pos)) & (pos[np.minimum(where, len(pos) - 1)] == st["pos"])
        vals[where[ok]] = np.asarray(st["data"])[ok]
        slots = np.arange(self.B) if flies is None else np.flatnonzero(np.isin(self.fly_of_slot, flies))
        s = torch.as_tensor(slots, device=self.dev)
        self.brain.pw[s] = torch.as_tensor(vals, device=self.dev)
        if "bias" in st:
            assert np.isin(st["bias_idx"], self.dn).all(), "saved intrinsic biases are for other neurons"
            j = self.brain.slots(np.asarray(st["bias_idx"])).long()
            k = torch.as_tensor(np.searchsorted(self.dn, st["bias_idx"]), device=self.dev)
            bias = torch.as_tensor(np.asarray(st["bias"], np.float32), device=self.dev)
            base = self.brain.bias_ext[:, j]
            if self.ib is not None:
                base = base - self.ib[:, k]
                self.ib[s[:, None], k[None, :]] = bias
            self.brain.bias_ext[s[:, None], j[None, :]] = base[s] + bias

    def _dn_error(self, tgt):
        """err[b][k] = target of the group of upost_k - rate[b][k] (0 for non-DN targets)."""
        torch = self._torch()
        g = self.upost_group
        e = tgt[:, torch.clamp(g, min=0)] - self.rate
        self._err.copy_(torch.where(g[None, :] >= 0, e, torch.zeros_like(e)))
        return self._err

    def _learn(self, tgt, learn, eta):
        err = self._dn_error(tgt)
        self._apply(self.dn_sel, self.dn_pre_k, self.dn_post_k, err, self._coefs(learn, eta))


class BatchInstructDeep(BatchInstruct):
    """The delta rule one layer deeper (flyzero/batch.py:331-409): L1 neuron i's error is
    delta_i = sum_j (w_ij / w_syn) * err_j over its synapses onto the DNs (before their update),
    and synapses onto L1 learn dw_ki = eta_deep * trace_k * delta_i."""

    def __init__(self, brain, groups: dict, params: InstructParams | None = None, fly_of_slot=None,
                 eta_deep: float = 1e-6, deep_scale=None, eta_bias: float = 0.0):
        torch = self._torch()
        super().__init__(brain, groups, params, fly_of_slot, eta_bias=eta_bias)
        self.eta_deep = eta_deep
        self.deep_scale = np.ones(self.B) if deep_scale is None else np.asarray(deep_scale, float)
        post, pre = brain.pl_post, brain.pl_pre
        is_dn = self.group_of >= 0
        self.l1 = np.unique(pre[self.dn_sel_h])
        l1_index = np.full(brain.n, -1, np.int64)
        l1_index[self.l1] = np.arange(len(self.l1))
        self.l1_index = l1_index
        i32 = lambda a: torch.as_tensor(np.asarray(a, np.int32), device=self.dev)
        self.dn_pre_l1 = i32(l1_index[pre[self.dn_sel_h]])
        deep = (l1_index[post] >= 0) & ~is_dn[post]
        self.deep_sel_h = np.flatnonzero(deep)
        self.deep_sel = i32(self.deep_sel_h)
        self.deep_pre_k = i32(self.pre_k_h[self.deep_sel_h])
        self.deep_post_l1 = i32(l1_index[post[self.deep_sel_h]])
        self.n_deep = int(deep.sum())
        self.delta = torch.zeros((self.B, max(1, len(self.l1))), dtype=torch.float32, device=self.dev)

    def _learn(self, tgt, learn, eta):
        b = self.brain
        err = self._dn_error(tgt)
        # the retrograde error uses the DN synapses before their own update
        self.delta.zero_()
        _lib.check(b._L.fb_backprop(b._h, _p(self.dn_sel), _p(self.dn_pre_l1), _p(self.dn_post_k), len(self.dn_sel_h),
                                    _p(err), err.shape[1], _p(self.delta), self.delta.shape[1], self._stream()))
        self._apply(self.dn_sel, self.dn_pre_k, self.dn_post_k, err, self._coefs(learn, eta))
        coef = self._coefs(learn, eta, (self.eta_deep / self.p.eta) * self.deep_scale)
        self._apply(self.deep_sel, self.deep_pre_k, self.deep_post_l1, self.delta, coef)
        self._deeper(self.delta, learn, eta)

    def _deeper(self, delta, learn, eta):
        """Hook for a further layer (``BatchInstructDeep2``)."""


class BatchInstructDeep2(BatchInstructDeep):
    """One more layer (flyzero/batch.py:430-451): delta2_k = sum_i (w_ki / w_syn) * delta1_i over
    L2 -> L1 synapses (after their own update), dw_jk = eta_deep2 * trace_j * delta2_k."""

    def __init__(self, brain, groups: dict, params: InstructParams | None = None, fly_of_slot=None,
                 eta_deep: float = 1e-6, deep_scale=None, eta_bias: float = 0.0, eta_deep2: float = 1e-8):
        torch = self._torch()
        super().__init__(brain, groups, params, fly_of_slot, eta_deep, deep_scale, eta_bias)
        self.eta_deep2 = eta_deep2
        post, pre = brain.pl_post, brain.pl_pre
        deep_sel = self.deep_sel_h
        self.l2 = np.unique(pre[deep_sel])
        l2_index = np.full(brain.n, -1, np.int64)
        l2_index[self.l2] = np.arange(len(self.l2))
        i32 = lambda a: torch.as_tensor(np.asarray(a, np.int32), device=self.dev)
        self.d2_back_h = deep_sel
        self.d2_back = i32(deep_sel)
        self.d2_back_pre = i32(l2_index[pre[deep_sel]])
        self.d2_back_post = i32(self.l1_index[post[deep_sel]])
        is_sel = np.zeros(len(post), bool)
        is_sel[self.dn_sel_h] = True
        is_sel[deep_sel] = True
        sel2 = np.flatnonzero((l2_index[post] >= 0) & ~is_sel)
        self.n_deep2 = len(sel2)
        self.k2_sel_h = sel2
        self.k2_sel = i32(sel2)
        self.k2_pre = i32(self.pre_k_h[sel2])
        self.k2_post = i32(l2_index[post[sel2]])
        self.delta2 = torch.zeros((self.B, max(1, len(self.l2))), dtype=torch.float32, device=self.dev)

    def _deeper(self, delta1, learn, eta):
        b = self.brain
        self.delta2.zero_()
        _lib.check(b._L.fb_backprop(b._h, _p(self.d2_back), _p(self.d2_back_pre), _p(self.d2_back_post),
                                    len(self.d2_back_h), _p(delta1), delta1.shape[1], _p(self.delta2),
                                    self.delta2.shape[1], self._stream()))
        coef = self._coefs(learn, eta, (self.eta_deep2 / self.p.eta) * self.deep_scale)
        self._apply(self.k2_sel, self.k2_pre, self.k2_post, self.delta2, coef)
