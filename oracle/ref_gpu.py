"""The reference's own GPU method, driven from Python (test infrastructure: a comparison, never the
product).

``RefGpuBrain`` restates the host side of ``flyzero.gpu.BatchBrain`` (flyzero/gpu.py:139-254: the
CSR split into fixed and plastic weights, ext slots, the (n_delay, B, n) pending ring, the work-item
list, two launches per step) over torch device buffers, and launches the reference's own kernels
`update` and `propagate` (gpu.py:26-119) from oracle/_ref/libref_gpu.so (built by
oracle/make_ref_gpu.py from the reference checkout). CuPy, which the reference uses for the
buffers and the launches, is absent here; ctypes launches stand in for its RawKernel calls.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libref_gpu.so")
_L = None


def available() -> bool:
    return os.path.exists(LIB)


def _lib():
    global _L
    if _L is None:
        L = C.CDLL(LIB)
        vp, i32, u32, f32 = C.c_void_p, C.c_int32, C.c_uint32, C.c_float
        L.refgpu_update.restype = C.c_int
        L.refgpu_update.argtypes = [i32, vp, i32, i32, i32, u32, u32, vp, vp, vp, vp, vp, vp, i32, vp, vp, f32, f32, f32,
                                    f32, f32, f32, i32, vp, vp, vp, vp]
        L.refgpu_propagate.restype = C.c_int
        L.refgpu_propagate.argtypes = [i32, vp, i32, i32, i32, vp, vp, i32, vp, vp, vp, vp, vp, vp, i32, vp]
        _L = L
    return _L


def _p(t):
    return C.c_void_p(t.data_ptr())


class RefGpuBrain:
    """``batch`` instances on the reference's kernels; the API subset the comparisons use."""

    def __init__(self, weights, params, batch: int = 1, seed: int = 0, plastic_pos=None, device="cuda"):
        import scipy.sparse as sp
        import torch

        self.p = p = params
        self.B = batch
        self.dev = torch.device(device)
        w = sp.csr_matrix(weights, dtype=np.float32)
        w.sort_indices()
        self.n = n = w.shape[0]
        indptr = w.indptr.astype(np.int64)
        indices = w.indices.astype(np.int32)
        data = (w.data * np.float32(p.w_syn)).astype(np.float32)
        pos = np.zeros(0, np.int64) if plastic_pos is None else np.sort(np.asarray(plastic_pos, np.int64))
        rows = np.repeat(np.arange(n), np.diff(indptr))
        pl_pre, pl_post = rows[pos], indices[pos]
        fixed = data.copy()
        fixed[pos] = 0.0                                           # gpu.py:155-159
        T = lambda a: torch.as_tensor(a, device=self.dev)          # noqa: E731
        self.d_indptr, self.d_indices, self.d_data = T(indptr), T(indices), T(fixed)
        self.d_pl_indptr = T(np.searchsorted(pl_pre, np.arange(n + 1)).astype(np.int64))
        self.d_pl_post = T(pl_post.astype(np.int32))
        self.pw = T(np.tile(data[pos], (batch, 1)).astype(np.float32))
        self.n_delay = max(1, int(round(p.delay / p.dt)))
        self.n_ref = int(round(p.t_ref / p.dt))
        self.decay_m = float(np.float32(p.dt / p.tau_m))
        self.decay_syn = float(np.float32(np.exp(-p.dt / p.tau_syn)))
        self.kick = float(np.float32(p.f_poisson * p.w_syn))
        self.seed = int(np.uint32(seed))
        self.step_no = 0
        self.t = 0
        self._slot = np.full(n, -1, np.int32)
        self.ext = np.zeros(0, np.int64)
        self.d_ext_idx = T(self._slot)
        self.p_ext = torch.zeros((batch, 0), dtype=torch.float32, device=self.dev)
        self.bias_ext = torch.zeros((batch, 0), dtype=torch.float32, device=self.dev)
        self.spikes = torch.zeros(batch * (2 * n + 2 * (w.nnz // 256) + 2), dtype=torch.int32, device=self.dev)
        self.n_spikes = torch.zeros(2, dtype=torch.int32, device=self.dev)
        self.reset()

    def reset(self):
        import torch

        self.v = torch.full((self.B, self.n), float(self.p.v_rest), dtype=torch.float32, device=self.dev)
        self.g = torch.zeros((self.B, self.n), dtype=torch.float32, device=self.dev)
        self.ref = torch.zeros((self.B, self.n), dtype=torch.int8, device=self.dev)
        self.pending = torch.zeros((self.n_delay, self.B, self.n), dtype=torch.float32, device=self.dev)
        self.t = 0

    def slots(self, idx):
        import torch

        idx = np.asarray(idx, np.int64).ravel()
        new = np.unique(idx[self._slot[idx] < 0])
        if len(new):
            k = len(self.ext)
            self.ext = np.r_[self.ext, new]
            self._slot[new] = np.arange(k, k + len(new), dtype=np.int32)
            self.d_ext_idx = torch.as_tensor(self._slot, device=self.dev)
            pad = torch.zeros((self.B, len(new)), dtype=torch.float32, device=self.dev)
            self.p_ext = torch.cat([self.p_ext, pad], 1).contiguous()
            self.bias_ext = torch.cat([self.bias_ext, pad], 1).contiguous()
        return torch.as_tensor(self._slot[idx], device=self.dev).long()

    def set_input(self, idx, rate_hz):
        import torch

        j = self.slots(idx)
        self.p_ext.fill_(0)
        self.p_ext[:, j] = torch.as_tensor(rate_hz, dtype=torch.float32, device=self.dev) * float(
            np.float32(self.p.dt / 1000.0))

    def run_steps(self, steps: int):
        """gpu.py:228-254: per step `update` then `propagate`; returns (B, n) int32 counts."""
        import torch

        L = _lib()
        p = self.p
        counts = torch.zeros((self.B, self.n), dtype=torch.int32, device=self.dev)
        blocks = (self.B * self.n + 255) // 256
        n_pl = self.pw.shape[1]
        pl_w = self.pw if self.pw.numel() else torch.zeros(1, dtype=torch.float32, device=self.dev)
        n_ext = len(self.ext)
        one = torch.zeros(1, dtype=torch.float32, device=self.dev)
        p_ext = self.p_ext if n_ext else one
        bias_ext = self.bias_ext if n_ext else one
        st = C.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)
        ns = self.n_spikes.data_ptr()
        for _ in range(steps):
            slot = self.t % self.n_delay
            nxt = (self.step_no + 1) & 1
            rc = L.refgpu_update(blocks, st, self.B, self.n, slot, self.step_no & 0xFFFFFFFF, self.seed, _p(self.v),
                                 _p(self.g), _p(self.ref), _p(self.pending), _p(counts), _p(self.d_ext_idx), n_ext,
                                 _p(p_ext), _p(bias_ext), self.kick, self.decay_syn, self.decay_m, float(p.v_rest),
                                 float(p.v_th), float(p.v_reset), self.n_ref, _p(self.d_indptr), _p(self.d_pl_indptr),
                                 _p(self.spikes), C.c_void_p(ns + 4 * (1 - nxt)))
            if rc:
                raise RuntimeError(f"reference update launch failed ({rc})")
            rc = L.refgpu_propagate(240, st, self.B, self.n, slot, _p(self.spikes), _p(self.n_spikes), nxt,
                                    _p(self.d_indptr), _p(self.d_indices), _p(self.d_data), _p(self.d_pl_indptr),
                                    _p(self.d_pl_post), _p(pl_w), n_pl, _p(self.pending))
            if rc:
                raise RuntimeError(f"reference propagate launch failed ({rc})")
            self.t += 1
            self.step_no += 1
        return counts
