"""Frame-end readout and closed-loop clamp of neuron groups, fused on the device.

``BatchMotor`` is the drop-in for ``flyzero.batch.BatchMotor`` (flyzero/batch.py:77-138): the
smoothed rates of the readout groups come from one kernel over the frame's device counts
(fb_group_rates) instead of a gather + GEMM + host copy; only the (slots, 9) rates cross to the
host for the button logic. ``Clamp`` is the drop-in for ``flyzero.implant.Clamp``
(flyzero/implant.py:69-104): rate filter, controller and bias writes in one kernel (fb_clamp).

Groups are given as neuron index arrays (the reference resolves them by cell type and side
through ``conn.find``; ``groups_from_connectome`` does that for a connectome that has types).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib

BUTTONS = ("B", "Y", "A", "X", "L", "R", "LEFT", "RIGHT", "UP", "DOWN", "SELECT", "START")
READOUT = ["steer_left", "steer_right", "lean_left", "lean_right", "wing_left", "wing_right",
           "accelerate", "brake", "boost"]


@dataclass
class MotorParams:
    tau_ms: float = 80.0
    steer_threshold: float = 10.0
    steer_bias: float = 0.0
    lean_threshold: float = 10.0
    accel_threshold: float = 5.0
    brake_threshold: float = 15.0
    boost_threshold: float = 1.0
    taps: bool = False
    steer_span: float = 150.0
    lean_span: float = 70.0
    groups: dict = field(default_factory=lambda: {
        "steer_left": ("DNa02", "left"), "steer_right": ("DNa02", "right"),
        "lean_left": ("DNa01", "left"), "lean_right": ("DNa01", "right"),
        "wing_left": ("DNg02*", "left"), "wing_right": ("DNg02*", "right"),
        "accelerate": ("DNp09", None), "brake": ("MDN", None), "boost": ("DNp01", None)})


def groups_from_connectome(conn, params: MotorParams | None = None) -> dict:
    p = params or MotorParams()
    return {name: np.asarray(conn.find(t, side), np.int64) for name, (t, side) in p.groups.items()}


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream(dev):
    import torch

    return C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


class _Groups:
    def __init__(self, brain, groups):
        import torch

        self.brain = brain
        idx = [np.asarray(g, np.int64).ravel() for g in groups]
        self.size = np.array([len(g) for g in idx], np.int64)
        self.idx_h = np.concatenate(idx) if idx else np.zeros(0, np.int64)
        dev = brain.device
        self.idx = torch.as_tensor(self.idx_h.astype(np.int32), device=dev)
        self.ptr = torch.as_tensor(np.r_[0, np.cumsum(self.size)].astype(np.int32), device=dev)
        self.n_groups = len(idx)


class BatchMotor:
    """``MotorReadout`` for every slot: smoothed DN rates -> button dicts."""

    def __init__(self, brain, groups: dict, params: MotorParams | None = None):
        import torch

        self.p = params or MotorParams()
        self.brain = brain
        self.B = brain.B
        self.g = _Groups(brain, [groups[name] for name in READOUT])
        self.w = torch.as_tensor((1.0 / np.maximum(self.g.size, 1)).astype(np.float32), device=brain.device)
        self.rates_dev = torch.zeros((self.B, len(READOUT)), dtype=torch.float32, device=brain.device)
        self.acc = np.zeros((self.B, 2))          # sigma-delta accumulators for taps (steer, lean)

    @property
    def rates(self) -> np.ndarray:
        return self.rates_dev.cpu().numpy()

    def reset(self, slots=None):
        if slots is None:
            self.rates_dev.zero_()
            self.acc[:] = 0
        else:
            s = np.atleast_1d(slots)
            self.rates_dev[list(s)] = 0
            self.acc[s] = 0

    def update(self, counts, window_ms: float) -> list:
        """``counts``: the frame's device (slots, n) int32. Returns one button dict per slot."""
        a = np.float32(1.0 - np.exp(-window_ms / self.p.tau_ms))
        hz = np.float32(1000.0 / window_ms)
        b = self.brain
        _lib.check(b._L.fb_group_rates(b._h, _p(counts), _p(self.g.idx), _p(self.g.ptr), self.g.n_groups, _p(self.w),
                                       float(a), float(hz), _p(self.rates_dev), _stream(b.device)))
        rates = self.rates
        return [self.buttons(r, k) for k, r in enumerate(rates)]

    def _tap(self, k, j, x, threshold, span):
        """Pulse-density modulation of a steering command: a first-order sigma-delta quantiser.
        The command's duty, clip((|x| - threshold) / span, 0, 1) with the sign of x, is integrated
        per (slot k, axis j); a frame emits +1 or -1 when the integral reaches +-0.5 and subtracts
        it, else 0. The button timing must equal flyzero/batch.py:113-119 frame for frame."""
        level = self.acc[k, j] + np.clip((abs(x) - threshold) / span, 0.0, 1.0) * np.sign(x)
        tap = int(level >= 0.5) - int(level <= -0.5)
        self.acc[k, j] = level - tap
        return tap

    def buttons(self, r, k: int = 0) -> dict:
        """Buttons of one slot from its smoothed rates (batch.py:121-138)."""
        p = self.p
        steer = (r[0] - r[1]) + (r[5] - r[4]) + p.steer_bias
        lean = r[2] - r[3]
        b = {name: False for name in BUTTONS}
        if p.taps:
            s = self._tap(k, 0, steer, p.steer_threshold, p.steer_span)
            le = self._tap(k, 1, lean, p.lean_threshold, p.lean_span)
            b["LEFT"], b["RIGHT"], b["L"], b["R"] = s > 0, s < 0, le > 0, le < 0
        else:
            b["LEFT"] = bool(steer > p.steer_threshold)
            b["RIGHT"] = bool(steer < -p.steer_threshold)
            b["L"] = bool(lean > p.lean_threshold)
            b["R"] = bool(lean < -p.lean_threshold)
        b["B"] = bool(r[6] > p.accel_threshold)
        b["Y"] = bool(r[7] > p.brake_threshold)
        b["A"] = bool(r[8] > p.boost_threshold)
        return b


class Clamp:
    """Closed-loop current injection into neuron groups, per slot (implant.py:69-104)."""

    def __init__(self, brain, groups: list, gain: float = 0.02, limit: float = 20.0, tau_ms: float = 80.0):
        import torch

        self.brain, self.gain, self.limit, self.tau_ms = brain, gain, limit, tau_ms
        self.g = _Groups(brain, groups)
        dev = brain.device
        slots = brain.slots(self.g.idx_h)
        self.slot = slots.to(torch.int32)
        self.base = brain.bias_ext[:, slots.long()].clone().contiguous()
        B, G = brain.B, self.g.n_groups
        self.u = torch.zeros((B, G), dtype=torch.float32, device=dev)
        self.rate = torch.zeros((B, G), dtype=torch.float32, device=dev)

    def reset(self, slots):
        s = list(np.atleast_1d(slots))
        self.u[s] = 0
        self.rate[s] = 0

    def step(self, counts, targets, active, window_ms: float, gate=None):
        """``targets``: (slots, groups) Hz; ``active``: bool per slot; ``gate``: (slots, groups)
        0/1 or None (all open)."""
        import torch

        b = self.brain
        dev = b.device
        tgt = torch.as_tensor(np.asarray(targets, np.float32), device=dev)
        act = torch.as_tensor(np.asarray(active, np.uint8), device=dev)
        gt = None if gate is None else torch.as_tensor(np.asarray(gate, np.float32), device=dev)
        a = 1.0 - np.exp(-window_ms / self.tau_ms)
        _lib.check(b._L.fb_clamp(b._h, _p(counts), _p(self.g.idx), _p(self.g.ptr), self.g.n_groups, _p(self.slot),
                                 _p(self.base), float(a), 1000.0 / window_ms, float(self.gain), float(self.limit),
                                 _p(self.rate), _p(self.u), _p(tgt), _p(act), _p(gt), _stream(dev)))
