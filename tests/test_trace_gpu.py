"""The persistent engine's phase trace (fb_set_trace, a diagnostic with no counterpart in the
reference): every step and CTA gets its stamps, in the documented order within a CTA."""

import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_phase_trace_stamps_in_step_order(torch):
    from flyzero_b200 import _lib
    from flyzero_b200.brain import LIFParams
    from flyzero_b200.gpu import BatchBrain

    n, B, steps = 4000, 4, 40
    rng = np.random.default_rng(4)
    w = sp.random(n, n, density=0.01, random_state=4, format="csr")
    w.data = np.rint(rng.normal(2.0, 4.0, w.nnz)).astype(np.float32)
    w.data[w.data == 0] = 1
    gb = BatchBrain(sp.csr_matrix(w), LIFParams(dt=0.1), batch=B, seed=3)
    gb.set_schedule("persistent")
    gb.set_input(np.arange(0, n, 7), 80.0)
    gb.run_steps(5)
    info = gb.info()
    assert info.group > 0 and int(info.ctas) > 0
    T, K = gb.phase_trace(steps)
    assert T.shape == (steps, int(info.ctas), 11) and K == int(info.epoch)
    for slot in (0, 1, 2, 3, 4, 8):
        assert np.all(T[:, :, slot] > 0), slot
    # within a CTA: 0 step start <= 4 kicks drawn <= 1 <= 2 slice staged <= 3 neurons advanced
    for a, b in ((0, 4), (4, 1), (1, 2), (2, 3)):
        assert np.all(T[:, :, b] >= T[:, :, a]), (a, b)
    assert np.all(T[1:, :, 0] > T[:-1, :, 3])                  # the next step starts after this one
    first, last = np.arange(0, steps, K), np.arange(K - 1, steps, K)
    assert np.all(T[first, :, 10] >= T[first, :, 7]) and np.all(T[last, :, 6] >= T[last, :, 5])
    # the medians are positive and the loop is part of the step
    from flyzero_b200.gpu import phase_summary

    ph = phase_summary(T, K, 1965.0)
    assert ph["neuron_loop"] > 0 and ph["step"] >= ph["neuron_loop"]
    # the trace is off again: a later run writes nothing into a buffer that was set and cleared
    tr = torch.zeros(4 * int(info.ctas) * 11, dtype=torch.int64, device="cuda")
    _lib.check(gb._L.fb_set_trace(gb._h, C.c_void_p(tr.data_ptr()), tr.numel()))
    _lib.check(gb._L.fb_set_trace(gb._h, None, 0))
    gb.run_steps(4)
    torch.cuda.synchronize()
    assert int(tr.abs().sum()) == 0
