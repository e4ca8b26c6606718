"""Motion-vision front end on the device: game frames -> T4/T5 (and columnar) Poisson drive.

``BatchMotionEye`` is the batched drop-in for ``flyzero.vision.MotionEye`` (flyzero/vision.py:
64-191): one eye per instance, the same neurons in the same order (``idx``, ``px``, ``py``,
``side``), the same float32 filter state per instance, and ``see`` computes every instance's rates
from a device batch of frames in one kernel launch (fb_motion_eye), writing them straight into
the brain's Poisson probabilities (``p_ext``) — the reference computes one eye per fly on the host
and hands the rates to ``set_input``.

The layout (which neurons, where on the screen, which channel) is host setup run once:
``retinotopy`` restates flyzero/eyes.py:37-87 and the channel assignment vision.py:67-124.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib


@dataclass
class MotionParams:
    """As flyzero/vision.py:34-50."""

    max_rate: float = 150.0
    gain: float = 1000.0
    cell: int = 4
    tau_hp: float = 4.0
    tau_delay: float = 2.0
    shift: int = 1
    overlap: float = 0.1
    y_min: float = 0.0
    transient_gain: float = 0.0
    sustained_gain: float = 0.0
    surround: int = 3
    chromatic_gain: float = 0.0


# T4/T5 subtype -> preferred direction in eye coordinates (vision.py:53)
SUBTYPES = {"a": "front_to_back", "b": "back_to_front", "c": "up", "d": "down"}
# medulla columnar types -> the feature that drives them (vision.py:57-61)
COLUMNAR = {
    "Mi1": "on_transient", "Tm3": "on_transient",
    "Tm1": "off_transient", "Tm2": "off_transient", "Tm4": "off_transient",
    "Mi4": "on_sustained", "Mi9": "off_sustained", "Tm9": "off_sustained",
}
# channel codes of fb_motion_eye
SCREEN = {"right": 0, "left": 1, "down": 2, "up": 3}
FEATURE = {"on_transient": 8, "off_transient": 9, "on_sustained": 10, "off_sustained": 11, "blue": 12, "green": 13}


def _field(pos: np.ndarray, mid: float) -> np.ndarray:
    """Visual-field coordinates (u lateral, v ventral; both 0..1) of one eye's neurons from the two
    main axes of their positions (flyzero/eyes.py:72-87)."""
    c = pos - pos.mean(0)
    _, _, vt = np.linalg.svd(c, full_matrices=False)
    uv = c @ vt[:2].T
    vert = int(np.argmax([abs(np.corrcoef(uv[:, k], pos[:, 1])[0, 1]) for k in range(2)]))
    u, v = uv[:, 1 - vert], uv[:, vert]
    if np.corrcoef(v, pos[:, 1])[0, 1] < 0:
        v = -v
    if np.corrcoef(u, np.abs(pos[:, 0] - mid))[0, 1] < 0:
        u = -u

    def unit(a):
        return (a - a.min()) / max(np.ptp(a), 1e-9)

    return np.c_[unit(u), unit(v)]


def retinotopy(conn, cells: np.ndarray, w: int, h: int, overlap: float = 0.1):
    """Screen pixel ``px, py``, eye ``side`` and placeable mask ``keep`` of ``cells``
    (flyzero/eyes.py:37-69): per eye the positions' main axes, the left eye on [0, 0.5 + o] of the
    screen, the right eye on [0.5 - o, 1], lateral at the outer edge."""
    nrn = conn.neurons.iloc[cells]
    pos = nrn[["pos_x", "pos_y", "pos_z"]].to_numpy(float)
    side = nrn["side"].fillna("").to_numpy().astype(object)
    ok = np.isfinite(pos).all(1)
    mid = np.nanmedian(conn.neurons["pos_x"].to_numpy(float))
    unknown = ~np.isin(side, ["left", "right"])
    side = np.where(unknown, np.where(pos[:, 0] > mid, "left", "right"), side)
    xy = np.full((len(cells), 2), np.nan)
    for s in ("left", "right"):
        m = (side == s) & ok
        if m.sum() >= 3:
            xy[m] = _field(pos[m], mid)
    keep = np.isfinite(xy).all(1)
    xy = np.nan_to_num(xy)
    o = overlap / 2
    left = side == "left"
    sx = np.where(left, (1 - xy[:, 0]) * (0.5 + o), 0.5 - o + xy[:, 0] * (0.5 + o))
    px = np.clip((sx * w).astype(int), 0, w - 1)
    py = np.clip((xy[:, 1] * h).astype(int), 0, h - 1)
    return px, py, side.astype(str), keep


@dataclass
class EyeLayout:
    """The eye's neurons in the reference's order and the channel each reads."""

    idx: np.ndarray       # neuron indices
    px: np.ndarray        # screen column (pixels)
    py: np.ndarray        # screen row (pixels)
    side: np.ndarray      # "left" / "right"
    chan: np.ndarray      # fb_motion_eye channel code per neuron
    gx: np.ndarray        # grid column
    gy: np.ndarray        # grid row
    visible: np.ndarray   # False above y_min


def layout(conn, frame_shape, p: MotionParams) -> EyeLayout:
    """Which neurons the eye drives and from which channel (vision.py:67-124)."""
    h, w = frame_shape
    gh, gw = h // p.cell, w // p.cell
    idx, xs, ys, sides, names = [], [], [], [], []

    def add(cells, name):
        if len(cells) == 0:
            return
        px, py, side, keep = retinotopy(conn, cells, w, h, p.overlap)
        idx.append(cells[keep]); xs.append(px[keep]); ys.append(py[keep]); sides.append(side[keep])
        names.append(np.array([name] * int(keep.sum()), dtype=object))

    for kind, pol in (("T4", "on"), ("T5", "off")):
        for sub, direction in SUBTYPES.items():
            add(conn.find(kind + sub), f"{pol}:{direction}")
    if not idx:
        raise ValueError("connectome has no T4/T5 neurons")
    if p.chromatic_gain > 0:
        for cell_type, feature in (("R7", "blue"), ("R8", "green")):
            add(conn.find(cell_type), f"col:{feature}")
    if p.transient_gain > 0 or p.sustained_gain > 0:
        for cell_type, feature in COLUMNAR.items():
            add(conn.find(cell_type), f"col:{feature}")
    idx_a, px, py, side = np.concatenate(idx), np.concatenate(xs), np.concatenate(ys), np.concatenate(sides)
    name = np.concatenate(names)
    chan = np.zeros(len(idx_a), np.uint8)
    for k, (nm, s) in enumerate(zip(name, side)):
        pol, what = nm.split(":")
        if pol == "col":
            chan[k] = FEATURE[what]
            continue
        if what == "front_to_back":          # front-to-back is leftwards for the left eye
            screen = "left" if s == "left" else "right"
        elif what == "back_to_front":
            screen = "right" if s == "left" else "left"
        else:
            screen = what
        chan[k] = (0 if pol == "on" else 4) + SCREEN[screen]
    gx = np.clip(px // p.cell, 0, gw - 1)
    gy = np.clip(py // p.cell, 0, gh - 1)
    visible = ~(py < p.y_min * h)
    return EyeLayout(idx_a, px, py, side, chan, gx, gy, visible)


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


class BatchMotionEye:
    """One ``MotionEye`` per instance of ``brain``; ``see`` drives the eye neurons' Poisson input.
    ``kernels``: "fused" runs each instance's eye in one thread block with its grid in shared
    memory (one launch), "split" runs four grid-wide kernels, "auto" the first when it fits."""

    def __init__(self, brain, conn, frame_shape, params: MotionParams | None = None, eye_layout: EyeLayout | None = None,
                 kernels: str = "auto"):
        import torch

        self.p = p = params or MotionParams()
        self.brain = brain
        self.h, self.w = frame_shape
        self.gh, self.gw = self.h // p.cell, self.w // p.cell
        self.layout = lo = eye_layout if eye_layout is not None else layout(conn, frame_shape, p)
        self.idx, self.px, self.py, self.side = lo.idx, lo.px, lo.py, lo.side
        dev = brain.device
        self.slot = brain.slots(lo.idx).to(torch.int32).contiguous()
        self.gx = torch.as_tensor(lo.gx.astype(np.int32), device=dev)
        self.gy = torch.as_tensor(lo.gy.astype(np.int32), device=dev)
        self.chan = torch.as_tensor(lo.chan, device=dev)
        self.visible = torch.as_tensor(lo.visible.astype(np.uint8), device=dev)
        L = brain._L
        n = int(L.fb_eye_state_floats(brain.B, self.h, self.w, p.cell))
        if n < 0:
            raise ValueError(f"frame {frame_shape} smaller than one {p.cell}-pixel cell")
        self.state = torch.zeros(n, dtype=torch.float32, device=dev)
        self.restart = torch.ones(brain.B, dtype=torch.uint8, device=dev)
        self.rates_dev = torch.zeros((brain.B, len(lo.idx)), dtype=torch.float32, device=dev)
        self.params = _lib.EyeParams(cell=p.cell, shift=p.shift, surround=p.surround,
                                     kernels={"auto": 0, "fused": 1, "split": 2}[kernels],
                                     a_hp=float(np.float32(1.0 / p.tau_hp)), a_d=float(np.float32(1.0 / p.tau_delay)),
                                     p_scale=float(np.float32(brain.p.dt / 1000.0)), gain=float(p.gain),
                                     max_rate=float(p.max_rate), transient_gain=float(p.transient_gain),
                                     sustained_gain=float(p.sustained_gain), chromatic_gain=float(p.chromatic_gain))

    def describe(self) -> str:
        n_col = int((self.layout.chan >= FEATURE["on_transient"]).sum())
        return (f"{len(self.idx) - n_col} T4/T5 motion detectors + {n_col} photoreceptor/medulla cells "
                f"({(self.side == 'left').sum()} left, {(self.side == 'right').sum()} right)")

    def reset(self, slots=None):
        """The next frame of these instances (all when None) restarts their filters."""
        if slots is None:
            self.restart.fill_(1)
        else:
            self.restart[list(np.atleast_1d(slots))] = 1

    @property
    def last_rates(self):
        """(batch, neurons) rates in Hz of the last frame, on the device."""
        return self.rates_dev

    def see(self, frames, flip=None):
        """``frames``: (batch, H, W, 3) uint8 (a device tensor, or host memory copied over);
        ``flip``: per-instance bool, mirror that frame left-right (flyzero/pool.py:44), or None.
        Writes the eye neurons' Poisson probabilities into the brain's input."""
        import torch

        b = self.brain
        dev = b.device
        fr = torch.as_tensor(frames, device=dev)
        if fr.dtype != torch.uint8 or tuple(fr.shape[1:]) != (self.h, self.w, 3) or fr.shape[0] != b.B:
            raise ValueError(f"frames must be uint8 ({b.B}, {self.h}, {self.w}, 3), got {tuple(fr.shape)} {fr.dtype}")
        fr = fr.contiguous()
        fl = None
        if flip is not None:
            fl = np.asarray(flip, np.uint8).ravel()
            if len(fl) != b.B:
                raise ValueError(f"flip needs one flag per instance ({b.B}), got {len(fl)}")
            fl = torch.as_tensor(fl, device=dev)
        st = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        _lib.check(b._L.fb_motion_eye(b._h, _p(fr), self.h, self.w, C.byref(self.params), _p(self.state),
                                      _p(self.restart), _p(fl), len(self.idx), _p(self.gx), _p(self.gy),
                                      _p(self.chan), _p(self.visible), _p(self.slot), _p(self.rates_dev), st))
        return self.rates_dev
