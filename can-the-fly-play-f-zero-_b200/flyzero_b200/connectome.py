"""Seeded synthetic connectomes with the shape of FlyWire v783, and their CSR layout.

The engine consumes exactly what the reference engine consumes: a pre x post CSR matrix of
signed synapse counts stored as float32 (flyzero/connectome.py:68-82, built at :140-146).
FlyWire itself cannot be downloaded here, so every benchmark and most tests run on a
stand-in generated from a seed:

* out-degree ~ lognormal with mean 109 (sigma 1, mu = ln 109 - sigma^2 / 2), rounded;
* targets uniform over the other n - 1 neurons (no self-loops); duplicate (pre, post)
  draws are merged by adding their counts;
* synapse count per edge ~ geometric(p = 0.28) on {1, 2, ...} (mean 3.57), capped at 255
  after merging;
* a seeded 25% of presynaptic neurons are inhibitory (every outgoing count negative).

``motor > 0`` designates that many seeded "motor" neurons and wires extra inputs onto them
until together they receive ``motor_in`` synapses (CSR entries). Real descending neurons
have thousands of inputs, which uniform random wiring (in-degree ~ 109) cannot give; the
batched workload makes exactly those entries plastic.
"""

from __future__ import annotations

import functools
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

FLYWIRE_N = 138_639
MEAN_DEGREE = 109.0


@dataclass
class SyntheticConnectome:
    weights: sp.csr_matrix                 # (n, n) float32 signed synapse counts
    seed: int
    motor: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    inhibitory: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))

    @property
    def n(self) -> int:
        return self.weights.shape[0]

    @property
    def nnz(self) -> int:
        return self.weights.nnz

    def synapses(self) -> int:
        return int(np.abs(self.weights.data).sum())

    def summary(self) -> str:
        return (f"synthetic connectome (seed {self.seed}): {self.n:,} neurons, {self.nnz:,} connections, "
                f"{self.synapses():,} synapses")


def _merge(pre: np.ndarray, post: np.ndarray, cnt: np.ndarray, n: int):
    """Sort edges by (pre, post) and add the counts of duplicates."""
    key = pre.astype(np.int64) * n + post.astype(np.int64)
    order = np.argsort(key, kind="stable")
    key = key[order]
    cnt = cnt[order]
    if len(key) == 0:
        return key, cnt
    first = np.r_[True, key[1:] != key[:-1]]
    starts = np.flatnonzero(first)
    return key[starts], np.add.reduceat(cnt, starts)


def synthetic(n: int = FLYWIRE_N, seed: int = 0, mean_degree: float = MEAN_DEGREE, sigma: float = 1.0,
              p_count: float = 0.28, cap: int = 255, inhibitory: float = 0.25, motor: int = 0,
              motor_in: int = 0) -> SyntheticConnectome:
    rng = np.random.default_rng(seed)
    mu = np.log(mean_degree) - 0.5 * sigma * sigma
    deg = np.clip(np.rint(rng.lognormal(mu, sigma, n)), 0, n - 1).astype(np.int64)
    e = int(deg.sum())
    pre = np.repeat(np.arange(n, dtype=np.int64), deg)
    post = rng.integers(0, n - 1, e, dtype=np.int64)
    post += post >= pre                                    # skip the diagonal: uniform over the others
    cnt = rng.geometric(p_count, e).astype(np.int64)
    key, cnt = _merge(pre, post, cnt, n)

    motor_idx = np.zeros(0, np.int64)
    if motor > 0:
        motor_idx = np.sort(rng.choice(n, motor, replace=False)).astype(np.int64)
        post_all = key % n
        have = np.isin(post_all, motor_idx)
        need = max(0, motor_in - int(have.sum()))
        per = np.full(motor, need // motor, np.int64)
        per[: need % motor] += 1
        extra_pre, extra_post = [], []
        for m, k in zip(motor_idx, per):
            existing = key[have & (post_all == m)] // n
            cand = np.setdiff1d(np.arange(n, dtype=np.int64), np.r_[existing, m])
            extra_pre.append(rng.choice(cand, int(k), replace=False))
            extra_post.append(np.full(int(k), m, np.int64))
        if need:
            ep, eq = np.concatenate(extra_pre), np.concatenate(extra_post)
            ec = rng.geometric(p_count, len(ep)).astype(np.int64)
            key, cnt = _merge(np.r_[key // n, ep], np.r_[key % n, eq], np.r_[cnt, ec], n)

    cnt = np.minimum(cnt, cap)
    n_inh = int(round(inhibitory * n))
    inh = np.sort(rng.choice(n, n_inh, replace=False)).astype(np.int64)
    sign = np.ones(n, np.int64)
    sign[inh] = -1
    rows = key // n
    cols = (key % n).astype(np.int32)
    data = (cnt * sign[rows]).astype(np.float32)
    indptr = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(rows, minlength=n), out=indptr[1:])
    w = sp.csr_matrix((data, cols, indptr), shape=(n, n))
    return SyntheticConnectome(w, seed, motor_idx, inh)


@functools.lru_cache(maxsize=4)
def flywire_scale(seed: int = 0, motor: int = 8, motor_in: int = 7300) -> SyntheticConnectome:
    """The 138,639-neuron stand-in shared by the full-scale workloads (cached per process)."""
    return synthetic(FLYWIRE_N, seed=seed, motor=motor, motor_in=motor_in)


def csr_checksum(w: sp.csr_matrix) -> str:
    """sha256 over indptr, indices and data: pins that two machines built the same graph."""
    import hashlib

    h = hashlib.sha256()
    for a in (np.asarray(w.indptr, np.int64), np.asarray(w.indices, np.int32), np.asarray(w.data, np.float32)):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


# ---- FlyWire v783 files (flyzero/connectome.py:123-165 reads the same three) ----------------
FLYWIRE_FILES = ("Completeness_783.csv", "Connectivity_783.parquet", "neuron_annotations.tsv")
_ANNOT_COLUMNS = ("super_class", "cell_class", "cell_type", "hemibrain_type", "side", "top_nt",
                  "pos_x", "pos_y", "pos_z")


@dataclass
class Connectome:
    """A connectome with its neuron table: ``weights`` (pre x post CSR, float32 signed synapse
    counts) and ``neurons`` (one row per neuron in index order, with ``root_id``, ``cell_type``,
    ``hemibrain_type``, ``side`` ... as in flyzero/connectome.py:68-82)."""

    weights: sp.csr_matrix
    neurons: object                        # pandas.DataFrame
    name: str = "connectome"
    _type_cache: dict = field(default_factory=dict, repr=False)

    @property
    def n(self) -> int:
        return self.weights.shape[0]

    @property
    def nnz(self) -> int:
        return self.weights.nnz

    def find(self, cell_type: str, side: str | None = None) -> np.ndarray:
        """Neurons whose cell type (or hemibrain type) equals ``cell_type`` (case-insensitive); a
        trailing ``*`` matches a prefix (``DNg02*``). ``side`` filters by hemisphere."""
        key = cell_type.lower()
        if key not in self._type_cache:
            ct = self.neurons["cell_type"].astype("string").str.lower()
            if key.endswith("*"):
                m = ct.str.startswith(key[:-1])
            else:
                m = ct.eq(key)
                if "hemibrain_type" in self.neurons:
                    m = m | self.neurons["hemibrain_type"].astype("string").str.lower().eq(key)
            self._type_cache[key] = m.to_numpy(dtype=bool, na_value=False)
        m = self._type_cache[key]
        if side is not None:
            m = m & self.neurons["side"].astype("string").eq(side).to_numpy(dtype=bool, na_value=False)
        return np.flatnonzero(m)


def load_flywire(data_dir) -> Connectome:
    """The FlyWire v783 connectome from the files of Shiu et al. 2024 (neuron order of
    ``Completeness_783.csv``; ``Connectivity_783.parquet`` pairs with their signed synapse counts,
    duplicates added) and the FlyWire annotations (matched on the root-id column that covers the
    most of the 783 ids)."""
    import os

    import pandas as pd

    missing = [f for f in FLYWIRE_FILES if not os.path.exists(os.path.join(data_dir, f))]
    if missing:
        raise FileNotFoundError(f"missing {missing} in {data_dir}")
    comp = pd.read_csv(os.path.join(data_dir, FLYWIRE_FILES[0]), index_col=0)
    root_ids = comp.index.to_numpy(dtype=np.int64)
    n = len(root_ids)
    con = pd.read_parquet(os.path.join(data_dir, FLYWIRE_FILES[1]),
                          columns=["Presynaptic_Index", "Postsynaptic_Index", "Excitatory x Connectivity"])
    w = sp.coo_matrix((con["Excitatory x Connectivity"].to_numpy(np.float32),
                       (con["Presynaptic_Index"].to_numpy(np.int64), con["Postsynaptic_Index"].to_numpy(np.int64))),
                      shape=(n, n)).tocsr()
    w.sum_duplicates()
    w.sort_indices()
    ann = pd.read_csv(os.path.join(data_dir, FLYWIRE_FILES[2]), sep="\t", low_memory=False)
    id_cols = [c for c in ann.columns if c == "root_id" or c.startswith("root_")]
    best = max(id_cols, key=lambda c: int(pd.Index(ann[c]).isin(root_ids).sum()))
    ann = ann.drop_duplicates(best).set_index(best)
    neurons = pd.DataFrame({"root_id": root_ids})
    for col in _ANNOT_COLUMNS:
        neurons[col] = ann[col].reindex(root_ids).to_numpy() if col in ann else np.nan
    for col in ("super_class", "cell_class", "cell_type", "hemibrain_type", "side", "top_nt"):
        neurons[col] = neurons[col].astype("string")
    return Connectome(w, neurons, name="FlyWire v783")


# ---- biological sign corrections (flyzero/biology.py:38-55) --------------------------------------
MODULATORY = ("dopamine", "serotonin", "octopamine")
CORRECTIONS = ("modulatory", "kenyon_cholinergic")


def corrected(conn: Connectome, fixes=CORRECTIONS) -> Connectome:
    """The connectome with the reference's sign fixes (flyzero/biology.py:38-55): ``modulatory``
    zeroes the fast weight of synapses whose presynaptic neuron's predicted transmitter is
    dopamine, serotonin or octopamine (Kenyon cells excepted); ``kenyon_cholinergic`` makes Kenyon
    cell outputs excitatory, inhibitory onto other Kenyon cells (with ``modulatory`` alone their
    outputs are zeroed). Zeroed synapses are dropped from the CSR; the neuron table is shared."""
    if not fixes:
        return conn
    w = conn.weights.tocoo()
    val = w.data.copy()
    transmitter = conn.neurons["top_nt"].fillna("").to_numpy().astype(str)
    kenyon = conn.neurons["cell_class"].eq("Kenyon_Cell").to_numpy(dtype=bool, na_value=False)
    from_kc = kenyon[w.row]
    if "modulatory" in fixes:
        val[np.isin(transmitter[w.row], MODULATORY) & ~from_kc] = 0.0
    if "kenyon_cholinergic" in fixes:
        size = np.abs(val[from_kc])
        val[from_kc] = np.where(kenyon[w.col[from_kc]], -size, size)
    elif "modulatory" in fixes:
        val[from_kc] = 0.0
    out = sp.csr_matrix((val, (w.row, w.col)), shape=w.shape)
    out.eliminate_zeros()
    return Connectome(out, conn.neurons, name=conn.name + " + corrections(" + ",".join(fixes) + ")")
