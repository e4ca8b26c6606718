"""The reference's own GPU kernels (flyzero/gpu.py:26-119, compiled from the reference checkout
into oracle/_ref by oracle/make_ref_gpu.py) against the engine on the same device: both draw the
same counter-hash Poisson kicks, so the spike counts agree; the reference snaps g and v
(gpu.py:52, 61), compiles with fast math and adds float weights in atomic order, so the rasters may
drift apart after a while and the comparison is statistical. Skipped where the comparison library
was not built (no reference checkout)."""

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import ref_gpu

    if not ref_gpu.available():
        pytest.skip("the reference's GPU kernels were not built (oracle/make_ref_gpu.py)")
    return torch


def test_reference_kernels_agree_with_the_engine(torch):
    import ref_gpu
    from flyzero_b200.brain import LIFParams
    from flyzero_b200.gpu import BatchBrain

    n, B, steps = 3000, 4, 600
    rng = np.random.default_rng(11)
    w = sp.random(n, n, density=0.01, random_state=3, format="csr")
    w.data = np.rint(rng.normal(2.0, 4.0, w.nnz)).astype(np.float32)
    w.data[w.data == 0] = 1
    w = sp.csr_matrix(w)
    p = LIFParams(dt=0.1)
    idx = np.sort(rng.choice(n, 300, replace=False))
    rate = rng.uniform(20, 150, (B, len(idx))).astype(np.float32)
    ours = BatchBrain(w, p, batch=B, seed=9)
    ours.set_input(idx, rate)
    ref = ref_gpu.RefGpuBrain(w, p, batch=B, seed=9)
    ref.set_input(idx, rate)
    a = ours.run_steps(steps).cpu().numpy().astype(np.int64)
    b = ref.run_steps(steps).cpu().numpy().astype(np.int64)
    assert a.sum() > 5 * B * len(idx)                       # the network is driven
    # the inputs fire from the same hash draws: identical counts on the driven neurons' first steps
    a10 = ours.run_steps(10).cpu().numpy()
    b10 = ref.run_steps(10).cpu().numpy()
    assert abs(int(a10.sum()) - int(b10.sum())) <= 0.05 * max(1, int(a10.sum()))
    tot_a, tot_b = a.sum(1), b.sum(1)
    np.testing.assert_allclose(tot_a, tot_b, rtol=0.02)
    r = np.corrcoef(a.ravel(), b.ravel())[0, 1]
    assert r > 0.97, r
