"""The surrogate's CUDA kernels: the BF16 tensor-core GEMM and its epilogues against a plain
PyTorch FP32 reference, the training step's gradients against the CPU FP64 oracle, and training."""

import ctypes as C

import numpy as np
import pytest

import mlp_oracle as MO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


@pytest.mark.parametrize("kind", [2, 1, 0], ids=["tcgen05_tma", "tcgen05", "mma_sync"])
@pytest.mark.parametrize("M,N,K", [(300, 70, 200), (128, 64, 32), (37, 10, 16), (4096, 512, 1280)])
def test_gemm_and_epilogues_match_torch_fp32(torch, M, N, K, kind):
    """Every GEMM kind: tcgen05 fed by TMA, tcgen05 fed by cp.async (accumulator in tensor memory), and
    the warp MMA."""
    from flyzero_b200 import _lib

    L = _lib.load()
    old = L.fs_gemm_kind(kind)
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn((M, K), device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn((N, K), device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    ref = A.float() @ B.float().T                               # FP32 reference of the same bf16 operands
    tol = dict(rtol=2e-5 * K, atol=2e-5 * K)
    out = torch.empty((M, N), device="cuda")
    _lib.check(L.fs_gemm(_p(A), _p(B), M, N, K, K, K, 0, None, None, _p(out), None, None, N, 0, None))
    torch.testing.assert_close(out, ref, **tol)
    # bias + GELU: pre-activation, bf16 activation and its transpose
    z = torch.empty((M, N), device="cuda")
    h = torch.empty((M, N), dtype=torch.bfloat16, device="cuda")
    ht = torch.empty((N, M), dtype=torch.bfloat16, device="cuda")
    _lib.check(L.fs_gemm(_p(A), _p(B), M, N, K, K, K, 1, _p(bias), None, _p(z), _p(h), _p(ht), N, M, None))
    torch.testing.assert_close(z, ref + bias, **tol)
    want = torch.nn.functional.gelu(z).to(torch.bfloat16)
    torch.testing.assert_close(h.float(), want.float(), rtol=1e-2, atol=1e-2)
    assert torch.equal(ht.T, h)
    # GELU gradient epilogue: d = C * gelu'(zin)
    zin = torch.randn((M, N), device="cuda", generator=g)
    d = torch.empty((M, N), dtype=torch.bfloat16, device="cuda")
    _lib.check(L.fs_gemm(_p(A), _p(B), M, N, K, K, K, 3, None, _p(zin), None, _p(d), None, N, 0, None))
    zz = zin.clone().requires_grad_(True)
    torch.nn.functional.gelu(zz).backward(ref)
    torch.testing.assert_close(d.float(), zz.grad, rtol=1e-2, atol=1e-2 * float(ref.abs().max()))
    L.fs_gemm_kind(old)


@pytest.mark.parametrize("M,N,K", [(512, 1280, 4096), (512, 512, 4096), (10, 512, 4096), (300, 70, 2048),
                                   (130, 16, 712)])
def test_split_k_matches_torch_fp32_and_is_deterministic(torch, M, N, K):
    """The weight-gradient shapes (few output tiles, K = the batch) split K over clusters of blocks:
    every epilogue against torch FP32, the same bits on every run, and close to the unsplit kernel."""
    from flyzero_b200 import _lib

    L = _lib.load()
    old_kind, old_split = L.fs_gemm_kind(2), L.fs_gemm_split(8)
    try:
        g = torch.Generator(device="cuda").manual_seed(M * 7 + N + K)
        A = torch.randn((M, K), device="cuda", generator=g).to(torch.bfloat16)
        B = torch.randn((N, K), device="cuda", generator=g).to(torch.bfloat16)
        bias = torch.randn(N, device="cuda", generator=g)
        ref = A.float() @ B.float().T
        tol = dict(rtol=2e-5 * K, atol=2e-5 * K)

        def f32(split):
            L.fs_gemm_split(split)
            out = torch.full((M, N), float("nan"), device="cuda")
            _lib.check(L.fs_gemm(_p(A), _p(B), M, N, K, K, K, 0, None, None, _p(out), None, None, N, 0, None))
            torch.cuda.synchronize()
            return out

        split = f32(8)
        torch.testing.assert_close(split, ref, **tol)
        assert torch.equal(split, f32(8))
        torch.testing.assert_close(split, f32(1), **tol)
        L.fs_gemm_split(8)
        z = torch.empty((M, N), device="cuda")
        h = torch.empty((M, N), dtype=torch.bfloat16, device="cuda")
        ht = torch.empty((N, M), dtype=torch.bfloat16, device="cuda")
        _lib.check(L.fs_gemm(_p(A), _p(B), M, N, K, K, K, 1, _p(bias), None, _p(z), _p(h), _p(ht), N, M, None))
        torch.testing.assert_close(z, ref + bias, **tol)
        torch.testing.assert_close(h.float(), torch.nn.functional.gelu(z).to(torch.bfloat16).float(), rtol=1e-2, atol=1e-2)
        assert torch.equal(ht.T, h)
        zin = torch.randn((M, N), device="cuda", generator=g)
        d = torch.empty((M, N), dtype=torch.bfloat16, device="cuda")
        _lib.check(L.fs_gemm(_p(A), _p(B), M, N, K, K, K, 3, None, _p(zin), None, _p(d), None, N, 0, None))
        zz = zin.clone().requires_grad_(True)
        torch.nn.functional.gelu(zz).backward(ref)
        torch.testing.assert_close(d.float(), zz.grad, rtol=1e-2, atol=1e-2 * float(ref.abs().max()))
        assert L.fs_gemm_split(0) == -_lib.FB_ERR_ARG and L.fs_gemm_split(9) == -_lib.FB_ERR_ARG
        assert L.fs_gemm_split(-1) == 8
    finally:
        L.fs_gemm_kind(old_kind)
        L.fs_gemm_split(old_split)


def test_training_gradients_match_fp64_oracle(torch):
    from flyzero_b200.surrogate import MLP

    net = MLP(seed=1)
    rng = np.random.default_rng(2)
    M = 256
    X = rng.normal(0, 1, (M, 1280)).astype(np.float32)
    Y = rng.poisson(2.0, (M, 10)).astype(np.float32)
    Xd, Yd = torch.as_tensor(X, device="cuda"), torch.as_tensor(Y, device="cuda")
    net.forward(Xd, training=True)
    loss = float(net.backward(Yd))
    params = net.params_f64()
    L, grads = MO.loss_and_grads(params, MO.bf16_round(X), Y.astype(np.float64))
    assert abs(loss - L) <= 2e-3 * abs(L)
    for li, ((gW, gb), (oW, ob)) in enumerate(zip(net.grads, grads)):
        for got, want in ((gW.cpu().numpy(), oW), (gb.cpu().numpy(), ob)):
            rel = np.linalg.norm(got - want) / np.linalg.norm(want)
            cos = float(np.sum(got * want) / (np.linalg.norm(got) * np.linalg.norm(want)))
            assert rel < 3e-2 and cos > 0.9995, (li, rel, cos)


def test_training_learns_a_poisson_teacher(torch):
    from flyzero_b200.surrogate import MLP

    rng = np.random.default_rng(3)
    Wt = rng.normal(0, 0.02, (10, 1280)).astype(np.float32)
    def batch(M):
        X = rng.normal(0, 1, (M, 1280)).astype(np.float32)
        Y = rng.poisson(np.exp(X @ Wt.T + 0.5)).astype(np.float32)
        return torch.as_tensor(X, device="cuda"), torch.as_tensor(Y, device="cuda")
    net = MLP(seed=4, lr=1e-3)
    Xv, Yv = batch(4096)
    net.forward(Xv, training=True)
    first = float(net.backward(Yv))
    for _ in range(150):
        net.train_step(*batch(1024))
    net.forward(Xv, training=True)
    last = float(net.backward(Yv))
    # the teacher's own NLL is the floor; training closes most of the gap from the start
    z = Xv.cpu().numpy() @ Wt.T + 0.5
    floor = float(np.mean(np.sum(np.exp(z) - Yv.cpu().numpy() * z, 1)))
    assert last < first and (last - floor) < 0.5 * (first - floor), (first, last, floor)


@pytest.mark.parametrize("seed", [0, 1])
def test_surrogate_screening_gains_over_plain_search(torch, seed):
    """End to end on a 16,384-neuron graph: 40,960 frames from the engine, training, then CMA-ES with
    the surrogate pre-screen (1,024 screened, 64 simulated per generation) against CMA-ES that
    simulates its 64 candidates directly - same number of full simulations. The screened search
    reaches the better interface, and in the last generation the calibrated surrogate's DN counts
    on the simulated survivors are within 5 % of the simulated ones."""
    from flyzero_b200 import tuning as T

    gens = 5
    rep = T.run(n=16384, frames=40960, epochs=6, generations=gens, episode=30, seed=seed)
    s, p = rep["surrogate_search"], rep["plain_search"]
    assert s["sims"] == p["sims"] == gens * 64
    assert all(g["screened"] / g["simulated"] >= 10 for g in s["log"])
    assert s["best"] >= p["best"], (s["best"], p["best"])
    assert s["log"][-1]["count_error"] <= 0.05, [g["count_error"] for g in s["log"]]
