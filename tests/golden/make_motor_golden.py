"""Generate tests/golden/motor.npz from the reference's own ``MotorReadout.update``
(flyzero/motor.py:78-95): the smoothed rates of the nine readout groups and the buttons, frame by
frame, for several independent slots (one reference readout per slot).

Run where the reference project is importable (default: /root/reference):

    python tests/golden/make_motor_golden.py [--reference PATH]

A seeded network of 600 neurons; the readout groups are seeded disjoint neuron sets (one group is
empty, as a cell type missing from a connectome would be); per slot and frame, Poisson spike counts
whose group means drift so that every button turns on and off over the run.
"""

from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
READOUT = ["steer_left", "steer_right", "lean_left", "lean_right", "wing_left", "wing_right",
           "accelerate", "brake", "boost"]
BUTTONS = ["B", "Y", "A", "L", "R", "LEFT", "RIGHT"]
N, SLOTS, FRAMES = 600, 4, 48
WINDOW = 1000.0 / 60.0988


def groups(seed=5):
    rng = np.random.default_rng(seed)
    perm = rng.permutation(N)
    out, at = {}, 0
    for k, name in enumerate(READOUT):
        size = 0 if name == "wing_right" else int(rng.integers(1, 7))
        out[name] = np.sort(perm[at:at + size]).astype(np.int64)
        at += size
    return out


def counts(grp, seed=6):
    """(FRAMES, SLOTS, N) int32: neuron rates that wander between silence and ~90 Hz; the boost
    group (threshold 1 Hz) falls silent for a stretch of frames so that its button turns off."""
    rng = np.random.default_rng(seed)
    lam = np.zeros((FRAMES, SLOTS, N))
    phase = rng.uniform(0, 2 * np.pi, (SLOTS, N))
    speed = rng.uniform(0.05, 0.4, (SLOTS, N))
    for f in range(FRAMES):
        lam[f] = 1.5 * np.maximum(np.sin(phase + speed * f), 0.0) ** 2
    quiet = np.arange(FRAMES)[:, None] % 40 >= 12 + 2 * np.arange(SLOTS)[None, :]
    lam[:, :, grp["boost"]] *= np.where(quiet, 0.0, 1.0)[:, :, None]
    return rng.poisson(lam).astype(np.int32)


class _Conn:
    """Enough of flyzero.connectome.Connectome for MotorReadout: find(type, side) -> indices."""

    def __init__(self, grp, params):
        self.by = {params.groups[name]: grp[name] for name in READOUT}

    def find(self, t, side=None):
        return self.by[(t, side)]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    args = ap.parse_args()
    sys.path.insert(0, args.reference)
    from flyzero.motor import MotorParams, MotorReadout

    grp = groups()
    cnt = counts(grp)
    rates = np.zeros((FRAMES, SLOTS, len(READOUT)))
    buttons = np.zeros((FRAMES, SLOTS, len(BUTTONS)), bool)
    for s in range(SLOTS):
        m = MotorReadout(_Conn(grp, MotorParams()), MotorParams())
        for f in range(FRAMES):
            b = m.update(cnt[f, s], WINDOW)
            rates[f, s] = [m.rates[name] for name in READOUT]
            buttons[f, s] = [b[k] for k in BUTTONS]
    assert buttons.any(axis=(0, 1)).all() and (~buttons).any(axis=(0, 1)).all(), "every button must toggle"
    np.savez_compressed(os.path.join(HERE, "motor.npz"), counts=cnt, rates=rates, buttons=buttons,
                        window=np.array(WINDOW), button_names=np.array(BUTTONS),
                        **{f"group_{name}": grp[name] for name in READOUT})
    print("motor.npz:", FRAMES, "frames x", SLOTS, "slots; buttons on:", buttons.mean(axis=(0, 1)).round(2))


if __name__ == "__main__":
    main()
