"""Generate tests/golden/eye.npz from the reference's own ``MotionEye`` (flyzero/vision.py).

Run where the reference project is importable (default: /root/reference):

    python tests/golden/make_eye_golden.py [--reference PATH]

A synthetic neuron table with T4/T5 subtypes, R7/R8 and the medulla columnar types (two optic
lobes as point clouds; some neurons without a side label, a few without a position) stands in for
FlyWire's; frames are seeded synthetic game frames (moving gratings and blocks, plus noise). Per
case the file holds the eye's layout (idx, px, py, side) and the rates of every frame, as the
reference computes them, and the SHA-256 of the frames (the tests regenerate them with
``frames`` and check the digest).
"""

from __future__ import annotations

import argparse
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

TYPES = ([f"T4{s}" for s in "abcd"] + [f"T5{s}" for s in "abcd"] + ["R7", "R8", "Mi1", "Tm3", "Tm1", "Tm2", "Tm4",
                                                                      "Mi4", "Mi9", "Tm9", "LPLC2", "DNa02"])

# (name, frame shape, frames, MotionParams overrides)
CASES = [
    ("default", (48, 64), 6, {}),
    ("train", (224, 256), 4, dict(gain=10 ** 2.7, y_min=0.2, transient_gain=4.0, sustained_gain=4.0,
                                  chromatic_gain=1.0)),
    ("odd", (50, 61), 5, dict(cell=3, shift=2, tau_hp=3.0, tau_delay=3.0, gain=300.0, surround=2,
                              sustained_gain=2.0, transient_gain=0.5, y_min=0.1, overlap=0.3)),
    ("wide_cell", (72, 90), 4, dict(cell=9, gain=50.0, sustained_gain=1.5, surround=1, chromatic_gain=0.7)),
]


def neuron_table(seed: int = 7):
    import pandas as pd

    rng = np.random.default_rng(seed)
    rows = []
    for t in TYPES:
        for lobe, cx in (("left", 300.0), ("right", -300.0)):
            m = int(rng.integers(12, 40))
            # an elongated sheet: main axis ~ y (dorsal-ventral), second ~ z
            pos = np.c_[cx + rng.normal(0, 15, m), rng.normal(0, 120, m), rng.normal(0, 70, m)]
            for k in range(m):
                side = lobe if rng.random() > 0.1 else None
                p = pos[k].copy()
                if rng.random() < 0.03:
                    p[0] = np.nan
                rows.append(dict(cell_type=t, hemibrain_type=None, side=side, pos_x=p[0], pos_y=p[1], pos_z=p[2],
                                 super_class="optic"))
    perm = rng.permutation(len(rows))
    df = pd.DataFrame([rows[i] for i in perm])
    df.insert(0, "root_id", np.arange(len(df), dtype=np.int64) + 720575940600000000)
    return df


def frames(shape, n, seed):
    """Seeded synthetic game frames: a drifting grating, two moving blocks, a sky band, noise."""
    h, w = shape
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    out = np.zeros((n, h, w, 3), np.uint8)
    for t in range(n):
        g = 0.5 + 0.5 * np.sin(2 * np.pi * (xx + 3 * t) / 23.0 + 0.3 * yy / 7.0)
        img = np.stack([g * 180, g * 120 + 40, 255 - g * 200], -1)
        for (y0, x0, vy, vx, col) in ((h // 3, w // 5, 1, 4, (250, 30, 30)), (h // 2, w // 2, -2, -3, (20, 220, 90))):
            y, x = y0 + vy * t, x0 + vx * t
            img[max(y, 0):max(y + h // 6, 0), max(x, 0):max(x + w // 7, 0)] = col
        img[: h // 8] = (90, 140, 250)
        img = img + rng.integers(-12, 13, img.shape)
        out[t] = np.clip(img, 0, 255).astype(np.uint8)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    args = ap.parse_args()
    sys.path.insert(0, args.reference)
    import scipy.sparse as sp
    from flyzero.connectome import Connectome
    from flyzero.vision import MotionEye, MotionParams

    df = neuron_table()
    conn = Connectome(sp.csr_matrix((len(df), len(df)), dtype=np.float32), df, name="eye-fixture")
    out = {"n_neurons": np.int64(len(df)), "types": np.array(TYPES)}
    for col in ("pos_x", "pos_y", "pos_z"):
        out[f"table_{col}"] = df[col].to_numpy(float)
    out["table_type"] = df["cell_type"].to_numpy().astype(str)
    out["table_side"] = df["side"].fillna("").to_numpy().astype(str)
    for k, (name, shape, n, kw) in enumerate(CASES):
        eye = MotionEye(conn, shape, MotionParams(**kw))
        fr = frames(shape, n, seed=100 + k)
        rates = np.stack([eye.see(f) for f in fr])
        out[f"{name}_frames_sha256"] = np.array(hashlib.sha256(fr.tobytes()).hexdigest())
        out[f"{name}_rates"] = rates
        out[f"{name}_idx"] = eye.idx.astype(np.int64)
        out[f"{name}_px"] = eye.px.astype(np.int64)
        out[f"{name}_py"] = eye.py.astype(np.int64)
        out[f"{name}_side"] = eye.side.astype(str)
        print(f"{name}: {len(eye.idx)} neurons, {eye.describe()}, mean rate {rates.mean():.3f} Hz, "
              f"nonzero {np.count_nonzero(rates)} of {rates.size}")
    np.savez_compressed(os.path.join(HERE, "eye.npz"), **out)


if __name__ == "__main__":
    main()
