"""Shared setup of the motion-eye tests: the fixture's neuron table as a Connectome, its cases'
parameters and frames (regenerated and checked against the fixture's digests)."""

import hashlib
import os
import sys

import numpy as np
import scipy.sparse as sp

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import make_eye_golden as G  # noqa: E402


def connectome(z):
    import pandas as pd

    from flyzero_b200.connectome import Connectome

    side = z["table_side"].astype(object)
    side[side == ""] = None
    df = pd.DataFrame(dict(cell_type=z["table_type"].astype(object), side=side, pos_x=z["table_pos_x"],
                           pos_y=z["table_pos_y"], pos_z=z["table_pos_z"]))
    n = len(df)
    return Connectome(sp.csr_matrix((n, n), dtype=np.float32), df, name="eye-fixture")


def cases():
    return [(k, name, shape, n, kw) for k, (name, shape, n, kw) in enumerate(G.CASES)]


def frames(z, k, name, shape, n):
    fr = G.frames(shape, n, seed=100 + k)
    assert hashlib.sha256(fr.tobytes()).hexdigest() == str(z[f"{name}_frames_sha256"]), "frame generator changed"
    return fr


def oracle_params(p):
    return dict(max_rate=p.max_rate, gain=p.gain, cell=p.cell, tau_hp=p.tau_hp, tau_delay=p.tau_delay, shift=p.shift,
                transient_gain=p.transient_gain, sustained_gain=p.sustained_gain, surround=p.surround,
                chromatic_gain=p.chromatic_gain)
