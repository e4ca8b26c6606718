"""CPU oracle for the LIF hot path. TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use this
module, and only as the checker or as the timed CPU reference. The engine never imports it.

What it restates (file:line in the reference project):

* ``ref_run``: ``flyzero/brain.py:32-58`` (``_kernel``), float32 or float64 state, CSR entries
  summed one at a time in spike order; kicks from a precomputed raster over input entries.
* ``reference_kicks``: the reference's Poisson stream. ``Brain.run`` draws
  ``seed_k = default_rng(seed).integers(2**31)`` per call (brain.py:90, :144) and the kernel
  draws ``np.random.random()`` per input per step after ``np.random.seed(seed_k)``
  (brain.py:34, :46-48); numba's generator is NumPy's legacy MT19937, so the kick raster of a
  run is ``RandomState(seed_k).random_sample((steps, n_in)) < p_in``.
* ``EngineOracle``: the batched engine's semantics (``flyzero/gpu.py:33-118`` order of
  operations, exact INT32 / Q32.32 accumulation, ext slots, per-instance plastic weights
  entering as Q32.32 deltas over the connectome weight).
* ``reward_step`` / ``batch_reward_step``: ``flyzero/learning.py:116-131`` and
  ``flyzero/batch.py:158-172, 482-495`` in NumPy.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

i64p = C.POINTER(C.c_int64)
i32p = C.POINTER(C.c_int32)
i16p = C.POINTER(C.c_int16)
i8p = C.POINTER(C.c_int8)
u8p = C.POINTER(C.c_uint8)
u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
vp = C.c_void_p


class _Net(C.Structure):
    _fields_ = [("n", C.c_int64), ("nnz", C.c_int64), ("B", C.c_int64),
                ("n_delay", C.c_int32), ("n_ref", C.c_int32), ("acc_mode", C.c_int32), ("contract", C.c_int32),
                ("indptr", i64p), ("indices", i32p), ("cnt", i16p), ("wfx", i64p),
                ("n_pl", C.c_int64), ("pl_indptr", i64p), ("pl_post", i32p), ("pl_q0", i64p),
                ("is_ppost", u8p)] + \
               [(f"{k}_f32", C.c_float) for k in ("decay_syn", "decay_m", "kick", "w_syn", "v_rest", "v_th", "v_reset")] + \
               [(f"{k}_f64", C.c_double) for k in ("decay_syn", "decay_m", "kick", "w_syn", "v_rest", "v_th", "v_reset")]


def build() -> str:
    path = os.path.join(_HERE, "liblif_oracle.so")
    src = [os.path.join(_HERE, f) for f in ("lif_oracle.c", "lif_oracle_impl.h", "Makefile")]
    if not os.path.exists(path) or any(os.path.getmtime(s) > os.path.getmtime(path) for s in src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return path


def lib():
    global _LIB
    if _LIB is None:
        L = C.CDLL(build())
        for sfx, real, rp in (("f32", C.c_float, f32p), ("f64", C.c_double, f64p)):
            f = getattr(L, f"fbo_ref_run_{sfx}")
            f.restype = C.c_int64
            f.argtypes = [C.c_int64, C.c_int64, C.c_int32, C.c_int64, rp, rp, i16p, rp, i32p, i64p, i32p, rp,
                          i64p, C.c_int64, u32p, real, real, real, real, real, real, C.c_int16, rp, C.c_int32,
                          i32p, u64p]
            f = getattr(L, f"fbo_engine_run_{sfx}")
            f.restype = C.c_int64
            f.argtypes = [C.POINTER(_Net), C.c_int64, C.c_int64, C.c_uint32, rp, rp, i8p, vp, i64p, i32p, f32p,
                          i32p, C.c_int32, f32p, f32p, u32p, C.c_uint32, i64p, i32p, u64p]
        L.fbo_ref_pool_f32.restype = C.c_int64
        L.fbo_ref_pool_f32.argtypes = [C.c_int32, C.c_int64, C.c_int64, C.c_int32, C.c_int64, i64p, i32p, f32p,
                                       i64p, C.c_int64, u32p, C.c_float, C.c_float, C.c_float, C.c_float,
                                       C.c_float, C.c_float, C.c_int16, C.c_int32, i64p]
        L.fbo_spike_tag_export.restype = C.c_uint64
        L.fbo_spike_tag_export.argtypes = [C.c_uint64]
        L.fbo_mix32_export.restype = C.c_uint32
        L.fbo_mix32_export.argtypes = [C.c_uint32]
        L.fbo_q32_export.restype = C.c_int64
        L.fbo_q32_export.argtypes = [C.c_float]
        _LIB = L
    return _LIB


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


# ------------------------------------------------------------------------------------------
# Constants derived exactly as brain.py:92-96 derives them
# ------------------------------------------------------------------------------------------
@dataclass
class Params:
    v_rest: float = -52.0
    v_reset: float = -52.0
    v_th: float = -45.0
    tau_m: float = 20.0
    tau_syn: float = 5.0
    t_ref: float = 2.2
    delay: float = 1.8
    w_syn: float = 0.275
    f_poisson: float = 250.0
    dt: float = 0.1

    @property
    def n_delay(self):
        return max(1, int(round(self.delay / self.dt)))

    @property
    def n_ref(self):
        return int(round(self.t_ref / self.dt))

    def consts(self, real=np.float32):
        """(decay_syn, decay_m, kick): brain.py:94-96 for float32; the unrounded doubles for float64."""
        return (real(np.exp(-self.dt / self.tau_syn)), real(self.dt / self.tau_m),
                real(self.f_poisson * self.w_syn))


def pack_bits(mask: np.ndarray) -> np.ndarray:
    """(..., k) bool -> (..., ceil(k/32)) uint32, bit j%32 of word j//32 (little-endian)."""
    mask = np.asarray(mask, bool)
    k = mask.shape[-1]
    words = (k + 31) // 32
    pad = np.zeros(mask.shape[:-1] + (words * 32,), bool)
    pad[..., :k] = mask
    return np.packbits(pad, axis=-1, bitorder="little").view(np.uint32).reshape(mask.shape[:-1] + (words,))


def reference_kicks(seed_k: int, steps: int, p_in: np.ndarray) -> np.ndarray:
    """Kick raster (steps, n_in) bool of one reference ``Brain.run`` call with seed ``seed_k``."""
    p64 = np.asarray(p_in, np.float32).astype(np.float64)
    rs = np.random.RandomState(seed_k)
    return rs.random_sample((steps, len(p64))) < p64


def run_seeds(seed: int, calls: int) -> list:
    """``seed_k`` for the first ``calls`` ``Brain.run`` calls of a Brain built with ``seed`` (brain.py:90, :144)."""
    rng = np.random.default_rng(seed)
    return [int(rng.integers(2 ** 31)) for _ in range(calls)]


def spike_tag(i):
    L = lib()
    return np.array([L.fbo_spike_tag_export(int(x)) for x in np.atleast_1d(i)], np.uint64)


def digest_of(spiking: np.ndarray) -> np.uint64:
    """Raster fingerprint of one step from a boolean spike vector (wrapping sum of tags)."""
    idx = np.flatnonzero(spiking)
    with np.errstate(over="ignore"):
        return np.uint64(spike_tag(idx).sum(dtype=np.uint64)) if len(idx) else np.uint64(0)


# ------------------------------------------------------------------------------------------
# brain.py:32-58, restated
# ------------------------------------------------------------------------------------------
class RefBrain:
    """One instance with the reference's own state layout and float summation order."""

    def __init__(self, weights, params: Params | None = None, real=np.float32, contract: bool = True):
        import scipy.sparse as sp

        self.p = p = params or Params()
        self.real = real
        self.contract = contract
        w = sp.csr_matrix(weights, dtype=np.float32)
        w.sort_indices()
        self.n = w.shape[0]
        self.indptr = w.indptr.astype(np.int64)
        self.indices = w.indices.astype(np.int32)
        if real is np.float32:
            self.data = (w.data * p.w_syn).astype(np.float32)          # brain.py:89
        else:
            self.data = w.data.astype(np.float64) * p.w_syn
        self.n_delay, self.n_ref = p.n_delay, p.n_ref
        self.decay_syn, self.decay_m, self.kick = p.consts(real)
        self.reset()
        self.bias = np.zeros(self.n, real)

    def reset(self):
        self.v = np.full(self.n, self.p.v_rest, self.real)
        self.g = np.zeros(self.n, self.real)
        self.ref = np.zeros(self.n, np.int16)
        self.pending = np.zeros((self.n_delay, self.n), self.real)
        self.t = 0

    def run_steps(self, steps: int, input_idx=None, kicks=None, record=False):
        """Advance ``steps``; ``kicks`` (steps, n_in) bool. Returns counts (and per-step
        spike counts and digests if ``record``)."""
        L = lib()
        sfx = "f32" if self.real is np.float32 else "f64"
        rp = f32p if self.real is np.float32 else f64p
        counts = np.zeros(self.n, np.int32)
        idx = np.zeros(0, np.int64) if input_idx is None else np.asarray(input_idx, np.int64)
        packed = None if kicks is None else np.ascontiguousarray(pack_bits(kicks))
        sc = np.zeros(steps, np.int32) if record else None
        sd = np.zeros(steps, np.uint64) if record else None
        r = self.real
        self.t = getattr(L, f"fbo_ref_run_{sfx}")(
            steps, self.t, self.n_delay, self.n, _p(self.v, rp), _p(self.g, rp), _p(self.ref, i16p),
            _p(self.pending, rp), _p(counts, i32p), _p(self.indptr, i64p), _p(self.indices, i32p),
            _p(self.data, rp), _p(idx, i64p), len(idx), _p(packed, u32p), r(self.kick), r(self.decay_syn),
            r(self.decay_m), r(self.p.v_rest), r(self.p.v_th), r(self.p.v_reset), self.n_ref,
            _p(self.bias, rp), int(self.contract), _p(sc, i32p), _p(sd, u64p))
        return (counts, sc, sd) if record else counts


# ------------------------------------------------------------------------------------------
# The engine's semantics
# ------------------------------------------------------------------------------------------
def q32(w: np.ndarray) -> np.ndarray:
    """float32 weights -> Q32.32 int64, round half to even (exact scaling by 2^32)."""
    return np.rint(np.asarray(w, np.float32).astype(np.float64) * 2.0 ** 32).astype(np.int64)


def integral_counts(data: np.ndarray) -> bool:
    d = np.asarray(data, np.float32)
    return bool(np.all(d == np.rint(d)) and (len(d) == 0 or np.abs(d).max() <= 32767))


class EngineOracle:
    """B instances with the engine's exact-accumulation semantics (state layout (B, n))."""

    def __init__(self, weights, params: Params | None = None, batch: int = 1, plastic_pos=None,
                 real=np.float32, acc_mode: str = "auto", seed: int = 0, contract: bool = True):
        import scipy.sparse as sp

        self.p = p = params or Params()
        self.real = real
        self.contract = contract
        self.B = batch
        w = sp.csr_matrix(weights, dtype=np.float32)
        w.sort_indices()
        self.n = n = w.shape[0]
        self.indptr = w.indptr.astype(np.int64)
        self.indices = w.indices.astype(np.int32)
        raw = w.data.astype(np.float32)
        self.data = (raw * p.w_syn).astype(np.float32)
        pos = np.zeros(0, np.int64) if plastic_pos is None else np.sort(np.asarray(plastic_pos, np.int64))
        self.plastic_pos = pos
        if acc_mode == "auto":
            acc_mode = "count" if integral_counts(raw) else "fixed"
        self.acc_mode = acc_mode
        if acc_mode == "count":
            self.cnt, self.wfx = np.rint(raw).astype(np.int16), None
        else:
            self.cnt, self.wfx = None, q32(self.data)
        rows = np.repeat(np.arange(n), np.diff(self.indptr))
        self.pl_pre = rows[pos]
        self.pl_post = self.indices[pos].astype(np.int32)
        self.pl_indptr = np.searchsorted(self.pl_pre, np.arange(n + 1)).astype(np.int64)
        self.is_ppost = np.zeros(n, np.uint8)
        self.is_ppost[self.pl_post] = 1
        self.w0 = self.data[pos].copy()
        self.pl_q0 = q32(self.w0)
        self.pw = np.tile(self.w0, (batch, 1)).astype(np.float32)
        self.n_delay, self.n_ref = p.n_delay, p.n_ref
        self.seed = np.uint32(seed)
        self.step_no = 0
        self.ext_idx = np.full(n, -1, np.int32)
        self.n_ext = 0
        self.p_ext = np.zeros((batch, 0), np.float32)
        self.bias_ext = np.zeros((batch, 0), np.float32)
        self.reset()

    def _net(self):
        p = self.p
        ds32, dm32, k32 = p.consts(np.float32)
        ds64, dm64, k64 = p.consts(np.float64)
        net = _Net(n=self.n, nnz=len(self.indices), B=self.B, n_delay=self.n_delay, n_ref=self.n_ref,
                   acc_mode=0 if self.acc_mode == "count" else 1, contract=int(self.contract),
                   indptr=_p(self.indptr, i64p), indices=_p(self.indices, i32p), cnt=_p(self.cnt, i16p),
                   wfx=_p(self.wfx, i64p), n_pl=len(self.plastic_pos), pl_indptr=_p(self.pl_indptr, i64p),
                   pl_post=_p(self.pl_post, i32p), pl_q0=_p(self.pl_q0, i64p), is_ppost=_p(self.is_ppost, u8p),
                   decay_syn_f32=ds32, decay_m_f32=dm32, kick_f32=k32, w_syn_f32=np.float32(p.w_syn),
                   v_rest_f32=np.float32(p.v_rest), v_th_f32=np.float32(p.v_th), v_reset_f32=np.float32(p.v_reset),
                   decay_syn_f64=ds64, decay_m_f64=dm64, kick_f64=k64, w_syn_f64=float(p.w_syn),
                   v_rest_f64=float(p.v_rest), v_th_f64=float(p.v_th), v_reset_f64=float(p.v_reset))
        return net

    def reset(self):
        B, n = self.B, self.n
        self.v = np.full((B, n), self.p.v_rest, self.real)
        self.g = np.zeros((B, n), self.real)
        self.ref = np.zeros((B, n), np.int8)
        self.ring = np.zeros((self.n_delay, B, n), np.int32 if self.acc_mode == "count" else np.int64)
        self.pring = np.zeros((self.n_delay, B, n), np.int64) if len(self.plastic_pos) else None
        self.t = 0

    def reset_flies(self, flies):
        """BatchBrain.reset(flies) (gpu.py:195-199): rest state, no input in flight."""
        f = np.atleast_1d(np.asarray(flies, np.int64))
        self.v[f] = self.p.v_rest
        self.g[f] = 0
        self.ref[f] = 0
        self.ring[:, f] = 0
        if self.pring is not None:
            self.pring[:, f] = 0

    def slots(self, idx):
        idx = np.asarray(idx, np.int64).ravel()
        new = np.unique(idx[self.ext_idx[idx] < 0])
        if len(new):
            k = self.n_ext
            self.ext_idx[new] = np.arange(k, k + len(new), dtype=np.int32)
            self.n_ext += len(new)
            pad = np.zeros((self.B, len(new)), np.float32)
            self.p_ext = np.concatenate([self.p_ext, pad], 1)
            self.bias_ext = np.concatenate([self.bias_ext, pad], 1)
        return self.ext_idx[idx]

    def run_steps(self, steps: int, kicks=None, stop_tick=None, record=False):
        """``kicks``: (steps, B, n_ext) bool raster over ext slots, or None for the hash stream."""
        L = lib()
        sfx = "f32" if self.real is np.float32 else "f64"
        rp = f32p if self.real is np.float32 else f64p
        counts = np.zeros((self.B, self.n), np.int32)
        packed = None if kicks is None else np.ascontiguousarray(pack_bits(kicks))
        sc = np.zeros((steps, self.B), np.int32) if record else None
        sd = np.zeros((steps, self.B), np.uint64) if record else None
        st = None if stop_tick is None else np.ascontiguousarray(stop_tick, np.int64)
        net = self._net()
        p_ext = np.ascontiguousarray(self.p_ext, np.float32)
        bias_ext = np.ascontiguousarray(self.bias_ext, np.float32)
        pw = np.ascontiguousarray(self.pw, np.float32)
        self.t = getattr(L, f"fbo_engine_run_{sfx}")(
            C.byref(net), steps, self.t, self.step_no & 0xFFFFFFFF, _p(self.v, rp), _p(self.g, rp),
            _p(self.ref, i8p), self.ring.ctypes.data_as(vp), _p(self.pring, i64p), _p(counts, i32p),
            _p(pw, f32p), _p(self.ext_idx, i32p), self.n_ext, _p(p_ext, f32p), _p(bias_ext, f32p),
            _p(packed, u32p), int(self.seed), _p(st, i64p), _p(sc, i32p), _p(sd, u64p))
        self.step_no += steps
        return (counts, sc, sd) if record else counts


def ref_pool(threads: int, n_inst: int, brain: RefBrain, steps: int, input_idx, kicks) -> int:
    """Threaded CPU baseline: ``n_inst`` independent reference runs of ``steps`` steps, one
    instance per thread at a time (``kicks``: (n_inst, steps, n_in) bool, or (steps, n_in) shared
    by all instances). Returns the total spike count."""
    L = lib()
    idx = np.asarray(input_idx, np.int64)
    shared = kicks.ndim == 2
    packed = np.ascontiguousarray(pack_bits(kicks))
    total = np.zeros(1, np.int64)
    b = brain
    L.fbo_ref_pool_f32(threads, n_inst, steps, b.n_delay, b.n, _p(b.indptr, i64p), _p(b.indices, i32p),
                       _p(b.data, f32p), _p(idx, i64p), len(idx), _p(packed, u32p), b.kick, b.decay_syn,
                       b.decay_m, np.float32(b.p.v_rest), np.float32(b.p.v_th), np.float32(b.p.v_reset),
                       b.n_ref, int(shared), _p(total, i64p))
    return int(total[0])


# ------------------------------------------------------------------------------------------
# Learning rules (NumPy restatements)
# ------------------------------------------------------------------------------------------
@dataclass
class LearnParams:
    eta: float = 2e-4
    tau_elig_ms: float = 500.0
    tau_post_ms: float = 500.0
    tau_reward_ms: float = 1000.0
    cap: float = 3.0


def reward_step(st: dict, data: np.ndarray, counts: np.ndarray, reward: float, window_ms: float,
                p: LearnParams) -> float:
    """learning.py:116-131 on a state dict {pos, pre, post, targets, sign, wmax, elig, post_mean,
    r_mean}; writes ``data[pos]`` in place and returns the advantage."""
    ae = np.exp(-window_ms / p.tau_elig_ms)
    ap = 1 - np.exp(-window_ms / p.tau_post_ms)
    ar = 1 - np.exp(-window_ms / p.tau_reward_ms)
    c = counts.astype(np.float32)
    dev = c[st["post"]] - st["post_mean"][st["post"]]
    st["elig"] = ae * st["elig"] + c[st["pre"]] * dev
    t = st["targets"]
    st["post_mean"][t] += ap * (c[t] - st["post_mean"][t])
    adv = reward - st["r_mean"]
    st["r_mean"] += ar * adv
    w = data[st["pos"]] + p.eta * adv * st["elig"]
    w = st["sign"] * np.clip(st["sign"] * w, 0.0, st["wmax"])
    data[st["pos"]] = w.astype(np.float32)
    return adv


def batch_reward_step(st: dict, pw: np.ndarray, counts: np.ndarray, reward: np.ndarray, learn: np.ndarray,
                      window_ms: float, p: LearnParams, eta_slot=None) -> np.ndarray:
    """batch.py:482-495 (``eta_slot`` given: school.py:289-304) with ``_Plastic.apply``
    (batch.py:158-172), NumPy in place of CuPy. State dict {upre, upost, pre_k, post_k, elig,
    post_mean, r_mean, sign, wmax, fos, n_flies}."""
    ae = np.exp(-window_ms / p.tau_elig_ms)
    ap = 1 - np.exp(-window_ms / p.tau_post_ms)
    ar = 1 - np.exp(-window_ms / p.tau_reward_ms)
    c_post = counts[:, st["upost"]].astype(np.float32)
    dev = (c_post - st["post_mean"])[:, st["post_k"]]
    st["elig"] = ae * st["elig"] + counts[:, st["upre"]].astype(np.float32)[:, st["pre_k"]] * dev
    st["post_mean"] += ap * (c_post - st["post_mean"])
    adv = reward - st["r_mean"]
    st["r_mean"] += ar * adv
    if learn.any():
        if eta_slot is None:
            dw = p.eta * adv.astype(np.float32)[:, None] * st["elig"]
        else:
            dw = (eta_slot * adv).astype(np.float32)[:, None] * st["elig"]
        B = pw.shape[0]
        onehot = np.zeros((st["n_flies"], B), np.float32)
        onehot[st["fos"], np.arange(B)] = learn.astype(np.float32)
        nrm = onehot.sum(1, keepdims=True)
        per_fly = (onehot / np.maximum(nrm, 1.0)) @ dw
        w = pw + per_fly[st["fos"]]
        pw[...] = st["sign"] * np.clip(st["sign"] * w, 0.0, st["wmax"])
    return adv
