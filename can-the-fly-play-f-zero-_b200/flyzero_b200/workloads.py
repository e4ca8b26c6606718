"""Seeded synthetic inputs for the benchmark workloads.

The reference drives its brain with T4/T5 motion-detector Poisson rates computed from game
frames (flyzero/vision.py:142-191) and a tonic walking drive to DNp09 (flyzero/tune.py:104-106).
No emulator or ROM exists here, so the frames are replaced by a drifting sinusoidal grating seen
by retinotopically placed stand-in T4/T5 neurons:

    rate_j(t) = 100 Hz * (1 + c * sin(2 pi (k <x_j, d> - f t)))      in [0, 200] Hz

with x_j uniform in [0, 1]^2, k = 4 cycles per field, f = 2 Hz, contrast c and a direction d
drawn per 166-step frame. Rates are constant within a frame, as in ``Fleet.think``
(flyzero/fleet.py:74-81), which rewrites ``p_ext`` once per frame.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

FRAME_MS = 1000.0 / 60.0988          # one SNES frame (flyzero/fleet.py:68)


def frame_steps(dt: float) -> int:
    return max(1, int(round(FRAME_MS / dt)))


@dataclass
class Drive:
    """Which neurons take outside input and how they are split."""
    inputs: np.ndarray        # T4/T5 stand-ins (or generic inputs)
    xy: np.ndarray            # (n_inputs, 2) retinotopic positions in [0, 1]^2
    tonic: np.ndarray         # DNp09 stand-in(s)
    readout: np.ndarray       # descending neurons whose counts are read every frame


def grating_drive(n: int, seed: int = 0, n_inputs: int = 12_246, exclude=()) -> Drive:
    """12,246 seeded T4/T5 stand-ins, one DNp09 stand-in, 10 readout DNs (the ``exclude`` set,
    typically the plastic motor neurons, first, then the DNp09 stand-in, then seeded others)."""
    rng = np.random.default_rng(seed + 7919)
    exclude = np.asarray(exclude, np.int64)
    pool = np.setdiff1d(np.arange(n, dtype=np.int64), exclude)
    pick = rng.choice(pool, n_inputs + 2, replace=False)
    inputs = np.sort(pick[:n_inputs])
    dnp09 = pick[n_inputs:n_inputs + 1]
    extra = pick[n_inputs + 1:]
    readout = np.r_[exclude[:8], dnp09, extra][:10].astype(np.int64)
    xy = rng.random((n_inputs, 2))
    return Drive(inputs, xy, dnp09.astype(np.int64), readout)


def grating_rates(drive: Drive, t_ms: float, direction: float, contrast: float = 1.0,
                  k: float = 4.0, f_hz: float = 2.0) -> np.ndarray:
    d = np.array([np.cos(direction), np.sin(direction)])
    phase = k * (drive.xy @ d) - f_hz * (t_ms / 1000.0)
    return (100.0 * (1.0 + contrast * np.sin(2 * np.pi * phase))).astype(np.float32)


def config1_inputs(n: int, seed: int = 0):
    """20 'drive' neurons at 60 Hz and 512 'input' neurons at 100 Hz (seeded, disjoint)."""
    rng = np.random.default_rng(seed + 104729)
    pick = rng.choice(n, 532, replace=False).astype(np.int64)
    idx = np.r_[pick[:20], pick[20:]]
    rate = np.r_[np.full(20, 60.0), np.full(512, 100.0)].astype(np.float32)
    return idx, rate


@dataclass
class BatchedWorkload:
    """Per-instance parameters of the batched workload: seed, contrast U[0.2, 1], tonic drive
    U[20, 100] Hz, run length U{0.5, 1, 2, 3} s; a grating direction per instance per frame."""
    seeds: np.ndarray
    contrast: np.ndarray
    tonic_hz: np.ndarray
    run_ms: np.ndarray
    rng: np.random.Generator

    @classmethod
    def make(cls, batch: int, seed: int = 0):
        rng = np.random.default_rng(seed + 15485863)
        return cls(rng.integers(0, 2 ** 31, batch), rng.uniform(0.2, 1.0, batch), rng.uniform(20, 100, batch),
                   rng.choice([500.0, 1000.0, 2000.0, 3000.0], batch), rng)

    def directions(self) -> np.ndarray:
        return self.rng.uniform(0, 2 * np.pi, len(self.seeds))

    def rates(self, drive: Drive, t_ms: float, dirs: np.ndarray) -> np.ndarray:
        """(B, n_inputs + 1) rates: grating per instance, then the tonic DNp09 drive."""
        out = np.empty((len(self.seeds), len(drive.inputs) + len(drive.tonic)), np.float32)
        for b in range(len(self.seeds)):
            out[b, :len(drive.inputs)] = grating_rates(drive, t_ms, dirs[b], self.contrast[b])
            out[b, len(drive.inputs):] = self.tonic_hz[b]
        return out


def high_activity_inputs(n: int, seed: int = 0, frac: float = 0.05, rate_hz: float = 210.0):
    """5% of neurons Poisson-driven at 210 Hz (the precision / high-activity workload). On the
    seeded 138,639-neuron synthetic graph this is the strongest drive of 5% whose activity stays
    put: ~15 Hz mean over 1 s (~210 spikes per step per instance); 150 Hz gives 8 Hz, and from
    ~220 Hz (or 7.8% at 150 Hz) the network ignites within 0.4 s to ~196 Hz, every neuron firing
    as fast as its refractory period allows (measured with the CPU restatement, 10,000 steps)."""
    rng = np.random.default_rng(seed + 32452843)
    idx = np.sort(rng.choice(n, int(round(frac * n)), replace=False)).astype(np.int64)
    return idx, np.full(len(idx), rate_hz, np.float32)


def game_frames(batch: int, n: int, shape=(224, 256), seed: int = 0) -> np.ndarray:
    """Seeded synthetic game frames (n, batch, H, W, 3) uint8 in the SNES frame shape: per instance
    a drifting grating of its own direction and speed, two moving blocks, a sky band and pixel
    noise (stand-ins for the emulator's frames, which are not available here)."""
    h, w = shape
    rng = np.random.default_rng(seed + 31337)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float32)
    out = np.empty((n, batch, h, w, 3), np.uint8)
    ang = rng.uniform(0, 2 * np.pi, batch)
    speed = rng.uniform(1, 6, batch)
    blocks = rng.integers(0, [h, w], (batch, 2, 2))
    vel = rng.integers(-5, 6, (batch, 2, 2))
    for t in range(n):
        for b in range(batch):
            ph = (np.cos(ang[b]) * xx + np.sin(ang[b]) * yy + speed[b] * t) / 19.0
            g = 0.5 + 0.5 * np.sin(2 * np.pi * ph)
            img = np.stack([g * 180, g * 120 + 40, 255 - g * 200], -1)
            for k in range(2):
                y, x = (blocks[b, k] + vel[b, k] * t) % [h, w]
                img[y:y + h // 6, x:x + w // 7] = (250, 30, 30) if k == 0 else (20, 220, 90)
            img[: h // 8] = (90, 140, 250)
            img += rng.integers(-12, 13, img.shape)
            out[t, b] = np.clip(img, 0, 255).astype(np.uint8)
    return out


def eye_layout(drive: Drive, shape=(224, 256), cell: int = 4, y_min: float = 0.2, seed: int = 0):
    """A motion-eye layout for the synthetic connectome (which has no cell types or positions):
    the drive's T4/T5 stand-ins at their screen points, each on one of the 14 eye channels."""
    from .vision import EyeLayout

    h, w = shape
    rng = np.random.default_rng(seed + 271828)
    px = np.minimum((drive.xy[:, 0] * w).astype(np.int64), w - 1)
    py = np.minimum((drive.xy[:, 1] * h).astype(np.int64), h - 1)
    side = np.where(px < w // 2, "left", "right")
    chan = rng.integers(0, 14, len(px)).astype(np.uint8)
    gx = np.clip(px // cell, 0, w // cell - 1)
    gy = np.clip(py // cell, 0, h // cell - 1)
    return EyeLayout(drive.inputs, px, py, side, chan, gx, gy, ~(py < y_min * h))
