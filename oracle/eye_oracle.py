"""CPU oracle of the motion-vision front end (test infrastructure: the checker, never the product).

Restates ``MotionEye.see`` (flyzero/vision.py:136-191) for one instance in NumPy, in the same
float32 / float64 operations the reference evaluates, so the GPU eye (fb_motion_eye) can be
compared bit for bit. The eye's neurons come as arrays: grid column ``gx``, row ``gy``, channel
code ``chan`` (0-7 motion: polarity ON 0 / OFF 4 plus screen direction right 0, left 1, down 2,
up 3; 8/9 ON/OFF transient, 10/11 ON/OFF sustained, 12 blue, 13 green) and ``visible`` (False
above y_min). Pinned against the reference's own ``MotionEye`` outputs in tests/golden/eye.npz.
"""

from __future__ import annotations

import numpy as np


class EyeOracle:
    """One eye: ``see(frame) -> rates`` (float32 Hz per neuron), keeping the filter state."""

    def __init__(self, frame_shape, gx, gy, chan, visible, *, max_rate=150.0, gain=1000.0, cell=4, tau_hp=4.0,
                 tau_delay=2.0, shift=1, transient_gain=0.0, sustained_gain=0.0, surround=3, chromatic_gain=0.0):
        self.h, self.w = frame_shape
        self.cell = cell
        self.gh, self.gw = self.h // cell, self.w // cell
        self.gx, self.gy = np.asarray(gx, np.int64), np.asarray(gy, np.int64)
        self.chan, self.visible = np.asarray(chan, np.int64), np.asarray(visible, bool)
        self.max_rate, self.gain, self.tau_hp, self.tau_delay, self.shift = max_rate, gain, tau_hp, tau_delay, shift
        self.transient_gain, self.sustained_gain, self.surround = transient_gain, sustained_gain, surround
        self.chromatic_gain = chromatic_gain
        self.lp = None
        self.delayed = None

    def grid(self, frame, channel=None):
        """vision.py:136-140: per-cell mean of the pixel luminance (or one channel) / 255."""
        c = self.cell
        img = frame[: self.gh * c, : self.gw * c].astype(np.float32)
        lum = (img.mean(2) if channel is None else img[..., channel]) / 255.0
        return lum.reshape(self.gh, c, self.gw, c).mean((1, 3))

    def see(self, frame):
        lum = self.grid(frame)
        if self.lp is None:                                    # vision.py:145-147
            self.lp = lum.copy()
            self.delayed = [np.zeros_like(lum), np.zeros_like(lum)]
        self.lp += (1.0 / self.tau_hp) * (lum - self.lp)       # vision.py:148-151
        hp = lum - self.lp
        k = self.shift
        motion = np.zeros((8,) + lum.shape, np.float32)
        for pol, sig in enumerate((np.maximum(hp, 0), np.maximum(-hp, 0))):
            d = self.delayed[pol]
            right = np.zeros_like(sig)                         # vision.py:154-162
            down = np.zeros_like(sig)
            right[:, :-k] = d[:, :-k] * sig[:, k:] - sig[:, :-k] * d[:, k:]
            down[:-k] = d[:-k] * sig[k:] - sig[:-k] * d[k:]
            motion[4 * pol + 0] = np.maximum(right, 0)
            motion[4 * pol + 1] = np.maximum(-right, 0)
            motion[4 * pol + 2] = np.maximum(down, 0)
            motion[4 * pol + 3] = np.maximum(-down, 0)
            d += (1.0 / self.tau_delay) * (sig - d)
        feats = {}
        if self.transient_gain > 0:                            # vision.py:164-166
            feats[8] = self.transient_gain * np.maximum(hp, 0)
            feats[9] = self.transient_gain * np.maximum(-hp, 0)
        if self.sustained_gain > 0:                            # vision.py:167-176 (float64 after the box sum)
            r = self.surround
            ii = np.pad(lum, ((1, 0), (1, 0))).cumsum(0).cumsum(1)
            yy, xx = np.mgrid[0:self.gh, 0:self.gw]
            y0, y1 = np.clip(yy - r, 0, self.gh), np.clip(yy + r + 1, 0, self.gh)
            x0, x1 = np.clip(xx - r, 0, self.gw), np.clip(xx + r + 1, 0, self.gw)
            sur = (ii[y1, x1] - ii[y0, x1] - ii[y1, x0] + ii[y0, x0]) / ((y1 - y0) * (x1 - x0))
            con = lum - sur
            feats[10] = self.sustained_gain * np.maximum(con, 0)
            feats[11] = self.sustained_gain * np.maximum(-con, 0)
        if self.chromatic_gain > 0:                            # vision.py:177-179
            feats[12] = self.chromatic_gain * self.grid(frame, 2)
            feats[13] = self.chromatic_gain * self.grid(frame, 1)
        rates = np.zeros(len(self.chan), np.float32)
        for c in np.unique(self.chan):                         # vision.py:180-186
            sel = np.flatnonzero(self.chan == c)
            if c < 8:
                rates[sel] = motion[c][self.gy[sel], self.gx[sel]]
            elif c in feats:
                rates[sel] = feats[c][self.gy[sel], self.gx[sel]] / self.gain
        rates[~self.visible] = 0.0                             # vision.py:187-189
        return (self.max_rate * np.clip(self.gain * rates, 0, 1)).astype(np.float32)
