"""Many instances of the whole-brain LIF model on one B200: the drop-in for ``flyzero.gpu.BatchBrain``.

Same constructor, methods and mutable device attributes as the reference (flyzero/gpu.py:131-254):
``pw`` (B, n_plastic), ``p_ext`` / ``bias_ext`` (B, n_ext), ``v`` / ``g`` / ``ref`` (B, n) are
torch tensors on the engine's device that callers may read and write in place between runs; ``run``
returns a fresh (B, n) int32 tensor of spike counts without synchronising the host.

The engine underneath (libflybrain.so) is hand-written CUDA for sm_100a; it accumulates synaptic
input exactly (INT32 synapse counts, or Q32.32 fixed point for non-integer weights), so spike
rasters do not depend on the order of atomic adds, unlike the reference GPU engine (gpu.py:11-14).
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import scipy.sparse as sp

from . import _lib
from .brain import LIFParams

# Phase stamps of the persistent engine's trace (csrc/persist.cuh): 0 step start, 4 the next step's
# kicks drawn, 1 slice wait begins, 2 slice in shared memory, 3 neurons advanced, 8 listing warps
# done; at an epoch's first step 7 / 10 push warps start / done; at its last 5 / 6 grid-barrier
# arrival / exit.
TRACE_SLOTS = 11


def phase_summary(T, epoch: int, sm_mhz: float) -> dict:
    """Medians over steps and CTAs (microseconds at ``sm_mhz``) of a phase trace from
    ``BatchBrain.phase_trace``."""
    T = np.asarray(T, np.float64) / float(sm_mhz)
    K = int(epoch)
    med = lambda a: float(np.median(a)) if a.size else float("nan")
    return {
        "step": med(T[1:, :, 0] - T[:-1, :, 0]),
        "start_to_kicks_drawn": med(T[:, :, 4] - T[:, :, 0]),
        "kicks_to_wait": med(T[:, :, 1] - T[:, :, 4]),
        "slice_wait": med(T[:, :, 2] - T[:, :, 1]),
        "neuron_loop": med(T[:, :, 3] - T[:, :, 2]),
        "loop_end_to_next_step": med(T[1:, :, 0] - T[:-1, :, 3]),
        "listing": med(T[1:, :, 8] - T[1:, :, 0]),
        "push_per_epoch": med(T[::K, :, 10] - T[::K, :, 7]),
        "grid_barrier_wait": med(T[K - 1::K, :, 6] - T[K - 1::K, :, 5]),
        "neuron_loop_max_over_ctas": float(np.median((T[:, :, 3] - T[:, :, 2]).max(1))),
    }


def _stream(device):
    import torch

    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


class BatchBrain:
    """``batch`` instances with shared connectome weights and private plastic synapses.

    ``plastic_pos``: indices into the CSR ``data`` (as in ``Brain.data``) of synapses that may
    differ between instances; ``self.pw`` (batch, n_plastic) holds their current weights in mV,
    already multiplied by ``w_syn`` (flyzero/gpu.py:132-137).

    Extensions over the reference: ``fp64=True`` runs FP64 state (the oracle-mode step used for
    precision reports); ``run_steps`` takes a precomputed kick raster and can record per-step
    spike counts and raster fingerprints; ``set_schedule`` / ``autotune`` pick the engine.
    """

    def __init__(self, weights: sp.csr_matrix, params: LIFParams | None = None, batch: int = 1,
                 seed: int = 0, plastic_pos: np.ndarray | None = None, *, device=None, fp64: bool = False,
                 fixed_point: bool = False):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("BatchBrain needs a CUDA device (B200); there is no CPU fallback")
        self.p = p = params or LIFParams()
        self.B = int(batch)
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else torch.device(device).index or 0)
        w = sp.csr_matrix(weights, dtype=np.float32)
        w.sort_indices()
        self.n = n = w.shape[0]
        # host copies with the same layout as brain.Brain (plasticity code indexes into them)
        self.indptr = w.indptr.astype(np.int64)
        self.indices = w.indices.astype(np.int32)
        raw = np.ascontiguousarray(w.data, np.float32)
        self.data = (raw * p.w_syn).astype(np.float32)
        pos = np.zeros(0, np.int64) if plastic_pos is None else np.unique(np.asarray(plastic_pos, np.int64))
        self.plastic_pos = pos
        rows = np.repeat(np.arange(n), np.diff(self.indptr))
        self.pl_pre = rows[pos]
        self.pl_post = self.indices[pos]
        self.w0 = self.data[pos].copy()
        self.n_delay = max(1, int(round(p.delay / p.dt)))
        self.n_ref = int(round(p.t_ref / p.dt))
        self.seed = np.uint32(seed)
        self.ext = np.zeros(0, np.int64)
        self._slot = np.full(n, -1, np.int32)
        L = _lib.load()
        prm = _lib.Params(**{k: float(getattr(p, k)) for k, _ in _lib.Params._fields_})
        flags = (_lib.FB_FLAG_F64 if fp64 else 0) | (_lib.FB_FLAG_ACC_FIXED if fixed_point else 0)
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(L.fb_create(C.byref(prm), _lib.ptr(self.indptr, _lib.i64p), _lib.ptr(self.indices, _lib.i32p),
                                   _lib.ptr(raw, _lib.f32p), n, len(self.indices), self.B, int(self.seed),
                                   _lib.ptr(pos, _lib.i64p), len(pos), flags, self.device.index, C.byref(h)))
        self._h = h
        self._L = L
        info = self.info()
        self.fp64 = bool(info.f64)
        # FP64 decay factors computed on the device, rounded like brain.py:94-96
        self.decay_syn = np.float32(info.decay_syn)
        self.decay_m = np.float32(info.decay_m)
        self.kick = np.float32(info.kick)
        self._wrap()

    # ---- engine plumbing ------------------------------------------------------------------------
    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._L.fb_destroy(h)
            except Exception:
                pass
            self._h = None

    def info(self) -> _lib.Info:
        out = _lib.Info()
        _lib.check(self._L.fb_get_info(self._h, C.byref(out)))
        return out

    def _wrap(self):
        vw = _lib.Views()
        _lib.check(self._L.fb_get_views(self._h, C.byref(vw)))
        info = self.info()
        real = "float64" if info.f64 else "float32"
        dev, B, n = self.device, self.B, self.n
        self.v = _lib.device_tensor(vw.v, (B, n), real, dev, self)
        self.g = _lib.device_tensor(vw.g, (B, n), real, dev, self)
        self.ref = _lib.device_tensor(vw.ref, (B, n), "int8", dev, self)
        self.pw = _lib.device_tensor(vw.pw, (B, info.n_plastic), "float32", dev, self)
        self.d_ext_idx = _lib.device_tensor(vw.ext_idx, (n,), "int32", dev, self)
        self.p_ext = _lib.device_tensor(vw.p_ext, (B, info.n_ext), "float32", dev, self)
        self.bias_ext = _lib.device_tensor(vw.bias_ext, (B, info.n_ext), "float32", dev, self)
        self.stop_tick = _lib.device_tensor(vw.stop_tick, (B,), "int64", dev, self)

    @property
    def t(self) -> int:
        return int(self.info().t)

    @property
    def step_no(self) -> int:
        return int(self.info().step_no)

    @property
    def launches(self) -> int:
        return int(self.info().launches)

    def check(self):
        """Raise if the device flagged a work-list overflow or a barrier timeout (synchronises)."""
        _lib.check(self._L.fb_check(self._h, _stream(self.device)))

    # ---- the reference API (flyzero/gpu.py:186-254) ------------------------------------------------
    def reset(self, flies=None):
        """Back to rest (all instances, or the given ones). Plastic weights are kept."""
        if flies is None:
            _lib.check(self._L.fb_reset(self._h, None, -1, _stream(self.device)))
            return
        f = np.ascontiguousarray(np.atleast_1d(np.asarray(flies)).astype(np.int32))
        _lib.check(self._L.fb_reset(self._h, _lib.ptr(f, _lib.i32p), len(f), _stream(self.device)))

    def slots(self, idx):
        """Ext slots of neurons ``idx`` (adding any that don't have one yet)."""
        import torch

        idx = np.asarray(idx, np.int64).ravel()
        new = np.unique(idx[self._slot[idx] < 0])
        if len(new):
            k = len(self.ext)
            self.ext = np.r_[self.ext, new]
            self._slot[new] = np.arange(k, k + len(new), dtype=np.int32)
            torch.cuda.current_stream(self.device).synchronize()
            nn = np.ascontiguousarray(new)
            _lib.check(self._L.fb_set_ext(self._h, _lib.ptr(nn, _lib.i64p), len(nn)))
            self._wrap()
        return torch.as_tensor(self._slot[idx], device=self.device)

    def set_bias(self, idx, mv, flies=None):
        """Steady depolarisation (mV) for neurons ``idx``, as ``Brain.set_bias`` (replaces it)."""
        import torch

        j = self.slots(idx)
        sel = slice(None) if flies is None else torch.as_tensor(np.atleast_1d(flies), device=self.device)
        self.bias_ext[sel] = 0.0
        self.bias_ext[sel, j] = torch.as_tensor(mv, dtype=torch.float32, device=self.device)

    def set_input(self, idx, rate_hz):
        """Poisson drive (Hz): ``rate_hz`` (batch, len(idx)) or broadcastable, replacing earlier input."""
        import torch

        j = self.slots(idx)
        self.p_ext.fill_(0)
        scale = torch.tensor(np.float32(self.p.dt / 1000.0), device=self.device)
        self.p_ext[:, j] = torch.as_tensor(rate_hz, dtype=torch.float32, device=self.device) * scale

    def run(self, duration_ms: float):
        """Advance every instance; returns spike counts (batch, n) on the GPU for this window."""
        steps = max(1, int(round(duration_ms / self.p.dt)))
        return self.run_steps(steps)

    # ---- extensions ---------------------------------------------------------------------------
    def run_steps(self, steps: int, kicks=None, record: bool = False, counts=None):
        """Advance ``steps`` steps. ``kicks``: device uint32 raster (steps, B, ceil(n_ext/32)) of
        precomputed input spikes (parity mode) or None for the Poisson hash. ``record``: also return
        per-step spike counts (steps, B) and raster fingerprints (steps, B) uint64."""
        import torch

        if counts is None:
            counts = torch.empty((self.B, self.n), dtype=torch.int32, device=self.device)
        sc = sd = None
        if record:
            sc = torch.empty((steps, self.B), dtype=torch.int32, device=self.device)
            sd = torch.empty((steps, self.B), dtype=torch.int64, device=self.device)
        kp = None
        if kicks is not None:
            words = (self.info().n_ext + 31) // 32
            assert kicks.dtype in (torch.int32, torch.uint32) and kicks.is_cuda and kicks.is_contiguous()
            assert tuple(kicks.shape) == (steps, self.B, words), f"kick raster must be {(steps, self.B, words)}"
            kp = C.c_void_p(kicks.data_ptr())
        _lib.check(self._L.fb_run(self._h, int(steps), C.c_void_p(counts.data_ptr()), kp,
                                  None if sc is None else C.c_void_p(sc.data_ptr()),
                                  None if sd is None else C.c_void_p(sd.data_ptr()), _stream(self.device)))
        return (counts, sc, sd) if record else counts

    def phase_trace(self, steps: int, counts=None):
        """Advance ``steps`` steps on the persistent engine with its phase trace on (fb_set_trace, a
        diagnostic): returns the (steps, ctas, 11) int64 SM-clock stamps of each step's phases per
        CTA (the last instance group's launch when there are several) and the epoch length."""
        import torch

        info = self.info()
        if info.group <= 0:
            raise RuntimeError("the persistent engine is unavailable for this network")
        ctas = int(info.ctas)
        tr = torch.zeros(steps * ctas * TRACE_SLOTS, dtype=torch.int64, device=self.device)
        _lib.check(self._L.fb_set_trace(self._h, C.c_void_p(tr.data_ptr()), tr.numel()))
        try:
            self.run_steps(steps, counts=counts)
            torch.cuda.synchronize(self.device)
        finally:
            _lib.check(self._L.fb_set_trace(self._h, None, 0))
        return tr.cpu().numpy().reshape(steps, ctas, TRACE_SLOTS), int(info.epoch)

    def make_plastic(self, pos):
        """Add CSR positions to the plastic set (keeps state and input in flight)."""
        import torch

        pos = np.ascontiguousarray(np.unique(np.asarray(pos, np.int64)))
        torch.cuda.current_stream(self.device).synchronize()
        _lib.check(self._L.fb_set_plastic(self._h, _lib.ptr(pos, _lib.i64p), len(pos)))
        self.plastic_pos = np.union1d(self.plastic_pos, pos)
        rows = np.repeat(np.arange(self.n), np.diff(self.indptr))
        self.pl_pre = rows[self.plastic_pos]
        self.pl_post = self.indices[self.plastic_pos]
        self.w0 = self.data[self.plastic_pos].copy()
        self._wrap()

    def set_schedule(self, engine: str | None = None, propagation: str | None = None, lanes: int = 0):
        """engine: 'auto' | 'step' | 'persistent'; propagation: 'push' | 'pull' (pull runs on the step
        engine; its first n_delay steps after the switch still push); lanes: 8/16/32 per work item."""
        e = {None: 0, "auto": 0, "step": 1, "persistent": 2}[engine]
        pr = {None: -1, "push": 0, "pull": 1}[propagation]
        _lib.check(self._L.fb_set_schedule(self._h, e, pr, int(lanes)))

    def set_run_length(self, steps_per_instance):
        """Instance b advances only for its next ``steps_per_instance[b]`` steps (then it is frozen
        until ``reset([b])`` and ``set_run_length`` again); a negative entry means unlimited."""
        import torch

        s = np.asarray(steps_per_instance, np.int64)
        self.set_stop_tick(np.where(s < 0, np.iinfo(np.int64).max, self.t + s))

    def set_stop_tick(self, ticks):
        """Instance b advances until the engine's tick reaches ``ticks[b]`` (absolute ticks, as
        ``t`` counts them). Enqueued on the current stream through pinned staging: the host is
        not synchronised."""
        import torch

        if getattr(self, "_stop_in", None) is None:
            self._stop_in = _lib.HostStage(self.B, torch.int64)
        self._stop_in.put(self.stop_tick, np.asarray(ticks, np.int64))

    # ---- schedule autotuner -------------------------------------------------------------------
    def schedule_candidates(self):
        """Schedules worth timing for this engine: (engine, propagation, lanes)."""
        info = self.info()
        cands = []
        if info.group > 0 and not info.f64:
            cands += [("persistent", "push", lanes) for lanes in (8, 16, 32)]
        cands += [("step", "push", 8), ("step", "push", 32), ("step", "pull", 8)]
        return cands

    def autotune(self, steps: int = 166, candidates=None, apply: bool = True) -> dict:
        """Time each candidate schedule on the next ``steps`` steps of the simulation and keep the
        fastest. Every schedule computes bit-identical results, so the simulation simply continues
        through the trials: the call advances every instance by (len(candidates)) * (steps + warm-up)
        steps, best done right after a reset. Also reports the measured activity and the modelled
        bytes of push (16 + 14 * out-degree per spike) and pull (14 per connectome entry + masks)."""
        import torch

        cands = list(candidates) if candidates is not None else self.schedule_candidates()
        st = torch.cuda.current_stream(self.device)
        warm = self.info().n_delay + 2          # pull needs n_delay recorded steps before it gathers
        rowlen = torch.as_tensor(np.diff(self.indptr), device=self.device)
        times, spikes, edges = {}, 0, 0
        counts = torch.empty((self.B, self.n), dtype=torch.int32, device=self.device)
        for c in cands:
            self.set_schedule(c[0], c[1], c[2])
            self.run_steps(warm, counts=counts)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            self.run_steps(steps, counts=counts)
            b.record(st)
            b.synchronize()
            times[c] = a.elapsed_time(b) / steps
            per_neuron = counts.sum(0).to(torch.int64)
            spikes += int(per_neuron.sum())
            edges += int((per_neuron * rowlen).sum())
        self.check()
        best = choose_schedule(times)
        if apply:
            self.set_schedule(*best)
        trials = len(cands) * steps
        return {"best": best, "ms_per_step": {"/".join(map(str, k)): v for k, v in times.items()},
                "spikes_per_step": spikes / max(trials, 1),
                "push_bytes_per_step": (16 * spikes + 14 * edges) / max(trials, 1),
                "pull_bytes_per_step": 14.0 * len(self.indices) + 8.0 * self.n * ((self.B + 63) // 64)}


def choose_schedule(ms_per_step: dict):
    """The fastest schedule of a {schedule: ms per step} table (the first listed on ties)."""
    if not ms_per_step:
        raise ValueError("no schedule was timed")
    return min(ms_per_step, key=lambda k: (ms_per_step[k], list(ms_per_step).index(k)))
