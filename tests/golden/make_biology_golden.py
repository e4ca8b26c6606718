"""Generate tests/golden/biology.npz from the reference's own ``biology.corrected``
(flyzero/biology.py:38-55).

Run where the reference project is importable (default: /root/reference):

    python tests/golden/make_biology_golden.py [--reference PATH]

A seeded random connectome of 400 neurons (some Kenyon cells, every transmitter label, missing
labels) and, per set of fixes, the corrected CSR (indptr, indices, data).
"""

from __future__ import annotations

import argparse
import os
import sys

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
FIXES = {"all": ("modulatory", "kenyon_cholinergic"), "modulatory": ("modulatory",),
         "kenyon": ("kenyon_cholinergic",), "none": ()}
TRANSMITTERS = np.array(["acetylcholine", "gaba", "glutamate", "dopamine", "serotonin", "octopamine", ""])


def table(n=400, seed=3):
    rng = np.random.default_rng(seed)
    w = sp.random(n, n, density=0.03, random_state=seed, format="csr", dtype=np.float32)
    w.data = np.rint(rng.normal(0, 6, w.nnz)).astype(np.float32)
    w.data[w.data == 0] = 2
    nt = TRANSMITTERS[rng.integers(0, len(TRANSMITTERS), n)]
    cls = np.where(rng.random(n) < 0.15, "Kenyon_Cell", np.where(rng.random(n) < 0.1, "", "other"))
    return w, nt, cls


def neurons(nt, cls):
    import pandas as pd

    df = pd.DataFrame({"root_id": np.arange(len(nt), dtype=np.int64)})
    df["top_nt"] = pd.array([None if s == "" else s for s in nt], dtype="string")
    df["cell_class"] = pd.array([None if s == "" else s for s in cls], dtype="string")
    return df


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    args = ap.parse_args()
    sys.path.insert(0, args.reference)
    from flyzero.biology import corrected
    from flyzero.connectome import Connectome

    w, nt, cls = table()
    out = {"w_indptr": w.indptr, "w_indices": w.indices, "w_data": w.data, "nt": nt, "cls": cls}
    for name, fixes in FIXES.items():
        c = corrected(Connectome(w, neurons(nt, cls)), fixes).weights.tocsr()
        out[f"{name}_indptr"], out[f"{name}_indices"], out[f"{name}_data"] = c.indptr, c.indices, c.data
        print(name, c.nnz, "synapses,", int((c.data < 0).sum()), "inhibitory")
    np.savez_compressed(os.path.join(HERE, "biology.npz"), **out)


if __name__ == "__main__":
    main()
