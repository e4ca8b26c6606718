"""Learned surrogate of the whole-brain simulator: a BF16 MLP trained on frames the engine
generates, used to pre-screen candidates of the interface calibration (flyzero/tune.py:26-166).

Network: 1280 -> 512 -> 512 -> 10, GELU, log-rate outputs, Poisson negative log-likelihood,
Adam. Inputs per frame: the frame's T4/T5 drive binned to 1,024 retinotopic patches (log1p of the
expected input spike counts) and a fixed 256-d projection of the previous frame's descending-
neuron (DN) counts; targets: the 10 DN spike counts of the frame.

Every GEMM, the loss, the bias gradients and the optimizer run as the library's own CUDA kernels
(include/flysurrogate.h): BF16 tensor-core MMAs with FP32 accumulation, FP32 master weights.
torch only allocates the buffers.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

DIMS = (1280, 512, 512, 10)
OUT_PAD = 16                 # the 10-wide output's gradients are stored with rows of 16 (GEMM operand stride)


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream(dev):
    import torch

    return C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


class MLP:
    """The surrogate network with its training state on one GPU."""

    def __init__(self, dims=DIMS, seed: int = 0, device=None, lr: float = 1e-3, betas=(0.9, 0.999), eps: float = 1e-8):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("the surrogate needs a CUDA device; there is no CPU fallback")
        self.dims = tuple(dims)
        self.dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.lr, self.betas, self.eps = lr, betas, eps
        self.t = 0
        self.L = _lib.load()
        g = np.random.default_rng(seed)
        self.W, self.b, self.Wb, self.WTb, self.m, self.v = [], [], [], [], [], []
        f32 = dict(dtype=torch.float32, device=self.dev)
        for li in range(len(dims) - 1):
            k, n = dims[li], dims[li + 1]
            bound = 1.0 / np.sqrt(k)            # torch.nn.Linear's default initialisation range
            W = torch.as_tensor(g.uniform(-bound, bound, (n, k)).astype(np.float32), device=self.dev)
            b = torch.as_tensor(g.uniform(-bound, bound, n).astype(np.float32), device=self.dev)
            self.W.append(W)
            self.b.append(b)
            self.m.append((torch.zeros_like(W), torch.zeros_like(b)))
            self.v.append((torch.zeros_like(W), torch.zeros_like(b)))
            self.Wb.append(torch.empty((n, k), dtype=torch.bfloat16, device=self.dev))
            ldt = max(8, -(-n // 8) * 8)
            self.WTb.append(torch.zeros((k, ldt), dtype=torch.bfloat16, device=self.dev))
            self._refresh_bf16(li)
        self._ws = {}
        self._loss = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self.grads = [(torch.zeros_like(W), torch.zeros_like(b)) for W, b in zip(self.W, self.b)]
        del f32

    def _refresh_bf16(self, li):
        W = self.W[li]
        n, k = W.shape
        _lib.check(self.L.fs_to_bf16(_p(W), W.numel(), _p(self.Wb[li]), _p(self.WTb[li]), n, k,
                                     self.WTb[li].shape[1], _stream(self.dev)))

    def _workspace(self, M):
        import torch

        if M in self._ws:
            return self._ws[M]
        d = self.dims
        bf = dict(dtype=torch.bfloat16, device=self.dev)
        f32 = dict(dtype=torch.float32, device=self.dev)
        ws = {"Z": [torch.empty((M, n), **f32) for n in d[1:]],
              "H": [torch.empty((M, n), **bf) for n in d[1:-1]],
              "HT": [torch.empty((n, M), **bf) for n in d[1:-1]],
              "dZ": [torch.empty((M, n), **bf) for n in d[1:-1]] + [torch.zeros((M, OUT_PAD), **bf)],
              "dZT": [torch.empty((n, M), **bf) for n in d[1:]],
              "Xb": torch.empty((M, d[0]), **bf), "XTb": torch.empty((d[0], M), **bf)}
        self._ws[M] = ws
        return ws

    def _gemm(self, A, B, M, N, K, lda, ldb, epi, bias=None, zin=None, out_f32=None, out_bf16=None, out_bf16_t=None,
              ldo=0, ldo_t=0):
        _lib.check(self.L.fs_gemm(_p(A), _p(B), M, N, K, lda, ldb, epi, _p(bias), _p(zin), _p(out_f32), _p(out_bf16),
                                  _p(out_bf16_t), ldo, ldo_t, _stream(self.dev)))

    def _load_inputs(self, X, transpose: bool):
        """X: (M, 1280) float32 device tensor -> bf16 copy (and its transpose for the weight grads)."""
        M = X.shape[0]
        ws = self._workspace(M)
        _lib.check(self.L.fs_to_bf16(_p(X), X.numel(), _p(ws["Xb"]), _p(ws["XTb"]) if transpose else None, M,
                                     self.dims[0], M, _stream(self.dev)))
        return ws

    def forward(self, X, training: bool = False):
        """Log-rates (M, 10) FP32 of the inputs X (M, 1280) FP32 (device tensors)."""
        M = X.shape[0]
        ws = self._load_inputs(X, transpose=training)
        d = self.dims
        h, ldh = ws["Xb"], d[0]
        nl = len(d) - 1
        for li in range(nl):
            n, k = d[li + 1], d[li]
            if li < nl - 1:
                self._gemm(h, self.Wb[li], M, n, k, ldh, k, 1, bias=self.b[li], out_f32=ws["Z"][li],
                           out_bf16=ws["H"][li], out_bf16_t=ws["HT"][li] if training else None, ldo=n, ldo_t=M)
                h, ldh = ws["H"][li], n
            else:
                self._gemm(h, self.Wb[li], M, n, k, ldh, k, 2, bias=self.b[li], out_f32=ws["Z"][li], ldo=n)
        return ws["Z"][-1]

    def backward(self, Y):
        """Gradients of the Poisson NLL (mean over the batch) after forward(X, training=True);
        Y: (M, 10) FP32 counts. Fills self.grads, returns the loss (a device scalar, FP64)."""
        M = Y.shape[0]
        ws = self._ws[M]
        d = self.dims
        nl = len(d) - 1
        self._loss.zero_()
        _lib.check(self.L.fs_poisson_nll(_p(ws["Z"][-1]), _p(Y), M, d[-1], _p(self._loss), _p(ws["dZ"][-1]), OUT_PAD,
                                         _p(ws["dZT"][-1]), _stream(self.dev)))
        for li in range(nl - 1, -1, -1):
            n, k = d[li + 1], d[li]
            A_in_T = ws["XTb"] if li == 0 else ws["HT"][li - 1]
            dW, db = self.grads[li]
            # dW = dZ^T X  (n x k): A = dZ^T (n x M), B = X^T (k x M)
            self._gemm(ws["dZT"][li], A_in_T, n, k, M, M, M, 0, out_f32=dW, ldo=k)
            ldz = OUT_PAD if li == nl - 1 else n
            _lib.check(self.L.fs_colsum(_p(ws["dZ"][li]), M, n, ldz, _p(db), _stream(self.dev)))
            if li > 0:
                # dZ_prev = (dZ W) * gelu'(Z_prev): A = dZ (M x n), B = W^T (k x n)
                self._gemm(ws["dZ"][li], self.WTb[li], M, k, n, ldz, self.WTb[li].shape[1], 3, zin=ws["Z"][li - 1],
                           out_bf16=ws["dZ"][li - 1], out_bf16_t=ws["dZT"][li - 1], ldo=k, ldo_t=M)
        return self._loss / M

    def step(self):
        """One Adam update from self.grads (then the bf16 copies follow)."""
        self.t += 1
        b1, b2 = self.betas
        for li in range(len(self.W)):
            W, b = self.W[li], self.b[li]
            gW, gb = self.grads[li]
            n, k = W.shape
            _lib.check(self.L.fs_adam(_p(W), _p(gW), _p(self.m[li][0]), _p(self.v[li][0]), W.numel(), self.lr, b1, b2,
                                      self.eps, self.t, _p(self.Wb[li]), _p(self.WTb[li]), n, k, self.WTb[li].shape[1],
                                      _stream(self.dev)))
            _lib.check(self.L.fs_adam(_p(b), _p(gb), _p(self.m[li][1]), _p(self.v[li][1]), b.numel(), self.lr, b1, b2,
                                      self.eps, self.t, None, None, 0, 0, 0, _stream(self.dev)))

    def train_step(self, X, Y):
        self.forward(X, training=True)
        loss = self.backward(Y)
        self.step()
        return loss

    def params_f64(self):
        """The current weights as float64 arrays [(W, b), ...] with W rounded to bf16 as the GEMMs see it."""
        out = []
        for li in range(len(self.W)):
            Wb = self.Wb[li].float().cpu().numpy().astype(np.float64)
            out.append((Wb, self.b[li].cpu().numpy().astype(np.float64)))
        return out

    def predict_counts(self, X):
        """Expected DN counts exp(log-rate) of inputs X (device FP32 (M, 1280))."""
        import torch

        return torch.exp(self.forward(X))


GEMM_SHAPES = ((4096, 512, 1280), (4096, 512, 512), (4096, 10, 512),      # forward, batch 4096
               (512, 1280, 4096), (512, 512, 4096), (10, 512, 4096),      # weight gradients
               (4096, 512, 512), (4096, 512, 16))                         # input gradients


def time_kernels(batch: int = 4096, reps: int = 50, warm: int = 5) -> dict:
    """Device times (CUDA events on the current stream, `reps` launches after `warm`) of fs_gemm on the
    training step's shapes (F32 epilogue, TMA kind) with and without the K split, and of a whole
    training step at `batch`. Returns {name: microseconds}."""
    import torch

    L = _lib.load()
    old_kind, old_split = L.fs_gemm_kind(2), L.fs_gemm_split(-1)
    st = _stream(torch.cuda.current_device())

    def timed(fn):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps * 1e3

    out = {}
    g = torch.Generator(device="cuda").manual_seed(0)
    try:
        for M, N, K in GEMM_SHAPES:
            A = torch.randn((M, K), device="cuda", generator=g).to(torch.bfloat16)
            B = torch.randn((N, K), device="cuda", generator=g).to(torch.bfloat16)
            C_ = torch.empty((M, N), device="cuda")
            for split in (1, old_split):
                L.fs_gemm_split(split)
                out[f"gemm {M}x{N}x{K} split<={split}"] = timed(lambda: _lib.check(
                    L.fs_gemm(_p(A), _p(B), M, N, K, K, K, 0, None, None, _p(C_), None, None, N, 0, st)))
        L.fs_gemm_split(old_split)
        net = MLP(seed=0)
        X = torch.randn((batch, DIMS[0]), device="cuda", generator=g)
        Y = torch.poisson(torch.ones((batch, DIMS[-1]), device="cuda"), generator=g)
        out[f"train_step batch={batch}"] = timed(lambda: net.train_step(X, Y))
    finally:
        L.fs_gemm_kind(old_kind)
        L.fs_gemm_split(old_split)
    return out


if __name__ == "__main__":
    import json

    print(json.dumps({k: round(v, 2) for k, v in time_kernels().items()}, indent=1))
