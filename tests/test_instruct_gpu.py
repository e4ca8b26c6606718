"""Instructed plasticity (BatchInstruct, BatchInstructDeep, BatchInstructDeep2) on the device
against the plain formulas, as the reference pins them (tests/test_gpu.py:75-102, 186-219)."""

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


def _setup(B, deep2=False, seed=0):
    from flyzero_b200 import connectome as cx
    from flyzero_b200 import instruct as I
    from flyzero_b200.brain import LIFParams
    from flyzero_b200.gpu import BatchBrain

    conn = cx.synthetic(3000, seed=seed)
    rng = np.random.default_rng(seed + 1)
    dns = rng.choice(conn.n, 27, replace=False)
    groups = {g: dns[3 * k:3 * k + 3] for k, g in enumerate(I.GROUPS)}
    w = sp.csr_matrix(conn.weights, dtype=np.float32)
    w.sort_indices()
    is_dn = np.zeros(conn.n, bool)
    is_dn[dns] = True
    p1 = np.flatnonzero(is_dn[w.indices])
    pos = np.union1d(p1, I.deep_positions(w, p1))
    if deep2:
        pos = np.union1d(pos, I.deep2_positions(w, p1))
    gb = BatchBrain(w, LIFParams(dt=0.25), batch=B, plastic_pos=pos)
    return gb, groups, rng


def test_deep_update_matches_plain_formula(torch):
    from flyzero_b200.instruct import BatchInstructDeep

    gb, groups, rng = _setup(4)
    bi = BatchInstructDeep(gb, groups, fly_of_slot=[0, 0, 1, 1], eta_deep=1e-3)
    assert bi.n_deep > 0
    bi.trace[...] = torch.as_tensor(rng.uniform(0, 5, bi.trace.shape).astype(np.float32), device="cuda")
    bi.rate[...] = torch.as_tensor(rng.uniform(0, 60, bi.rate.shape).astype(np.float32), device="cuda")
    tgt = rng.uniform(0, 80, (4, len(bi.names))).astype(np.float32)
    learn = np.array([True, False, True, True])
    w0 = gb.pw.cpu().numpy().copy()
    sel, dsel = bi.dn_sel_h, bi.deep_sel_h
    trace, rate = bi.trace.cpu().numpy(), bi.rate.cpu().numpy()
    err = tgt[:, bi.post_group_h[sel]] - rate[:, bi.post_k_h[sel]]
    delta = np.zeros((4, len(bi.l1)), np.float32)
    np.add.at(delta.T, bi.dn_pre_l1.cpu().numpy(), (w0[:, sel] / gb.p.w_syn * err).T)
    change = bi.eta_deep * trace[:, bi.deep_pre_k.cpu().numpy()] * delta[:, bi.deep_post_l1.cpu().numpy()]
    per_fly = np.stack([change[0], change[2:].mean(0)])
    sign, wmax = bi.sign_h[dsel], bi.wmax_h[dsel]
    expected = sign * np.clip(sign * (w0[:, dsel] + per_fly[[0, 0, 1, 1]]), 0, wmax)
    # and the DN synapses: the delta rule, averaged over each fly's learning slots
    dch = bi.p.eta * trace[:, bi.pre_k_h[sel]] * err
    dfly = np.stack([dch[0], dch[2:].mean(0)])
    s1, m1 = bi.sign_h[sel], bi.wmax_h[sel]
    dn_expected = s1 * np.clip(s1 * (w0[:, sel] + dfly[[0, 0, 1, 1]]), 0, m1)
    bi._learn(torch.as_tensor(tgt, device="cuda"), learn, bi.p.eta)
    pw = gb.pw.cpu().numpy()
    np.testing.assert_allclose(pw[:, dsel], expected, rtol=1e-4, atol=1e-5)
    np.testing.assert_allclose(pw[:, sel], dn_expected, rtol=1e-4, atol=1e-5)
    assert np.abs(expected - w0[:, dsel]).max() > 1e-4


def test_second_layer_update_matches_plain_formula(torch):
    from flyzero_b200.instruct import BatchInstructDeep2

    gb, groups, rng = _setup(2, deep2=True, seed=1)
    bi = BatchInstructDeep2(gb, groups, fly_of_slot=[0, 1], eta_deep=1e-3, eta_deep2=1e-4)
    assert bi.n_deep2 > 0
    bi.trace[...] = torch.as_tensor(rng.uniform(0, 5, bi.trace.shape).astype(np.float32), device="cuda")
    bi.rate[...] = torch.as_tensor(rng.uniform(0, 60, bi.rate.shape).astype(np.float32), device="cuda")
    tgt = rng.uniform(0, 80, (2, len(bi.names))).astype(np.float32)
    w0 = gb.pw.cpu().numpy().copy()
    g = lambda t: t.cpu().numpy()
    trace, rate = g(bi.trace), g(bi.rate)
    sel = bi.dn_sel_h
    err = tgt[:, bi.post_group_h[sel]] - rate[:, bi.post_k_h[sel]]
    d1 = np.zeros((2, len(bi.l1)), np.float32)
    np.add.at(d1.T, g(bi.dn_pre_l1), (w0[:, sel] / gb.p.w_syn * err).T)
    w1 = w0.copy()                      # layer-1 synapses after their own update (used backwards)
    ch1 = bi.eta_deep * trace[:, g(bi.deep_pre_k)] * d1[:, g(bi.deep_post_l1)]
    dsel = bi.deep_sel_h
    s1, m1 = bi.sign_h[dsel], bi.wmax_h[dsel]
    w1[:, dsel] = s1 * np.clip(s1 * (w0[:, dsel] + ch1), 0, m1)
    d2 = np.zeros((2, len(bi.l2)), np.float32)
    np.add.at(d2.T, g(bi.d2_back_pre), (w1[:, bi.d2_back_h] / gb.p.w_syn * d1[:, g(bi.d2_back_post)]).T)
    s2 = bi.k2_sel_h
    ch2 = bi.eta_deep2 * trace[:, g(bi.k2_pre)] * d2[:, g(bi.k2_post)]
    sg, mx = bi.sign_h[s2], bi.wmax_h[s2]
    expected = sg * np.clip(sg * (w0[:, s2] + ch2), 0, mx)
    bi._learn(torch.as_tensor(tgt, device="cuda"), np.array([True, True]), bi.p.eta)
    np.testing.assert_allclose(g(gb.pw)[:, s2], expected, rtol=1e-4, atol=1e-5)
    assert np.abs(expected - w0[:, s2]).max() > 1e-5


def test_instruct_step_traces_rates_and_error(torch):
    """step(): presynaptic traces and postsynaptic rates from the frame's counts (batch.py:282-287),
    the update only for learning slots, and the mean |target - rate| report."""
    from flyzero_b200.instruct import BatchInstruct, targets

    gb, groups, rng = _setup(3, seed=2)
    bi = BatchInstruct(gb, groups, fly_of_slot=[0, 1, 2])
    trace = np.zeros((3, len(bi.upre)), np.float32)
    rate = np.zeros((3, len(bi.upost)), np.float32)
    window = 16.64
    p = bi.p
    for f in range(5):
        counts = rng.poisson(0.5, (3, gb.n)).astype(np.int32)
        tg = np.array([targets(rng.uniform(-1, 1, 5).clip(0) if k else rng.uniform(-1, 1, 5), p) for k in range(3)],
                      np.float32)
        learn = np.array([True, f % 2 == 0, False])
        w_before = gb.pw.cpu().numpy().copy()
        out = bi.step(torch.as_tensor(counts, device="cuda"), tg, learn, window)
        a_pre, a_rate, hz = 1 - np.exp(-window / p.tau_pre_ms), 1 - np.exp(-window / p.tau_rate_ms), 1000.0 / window
        trace += a_pre * (counts[:, bi.upre].astype(np.float32) * hz * (p.tau_pre_ms / 1000.0) - trace)
        rate += a_rate * (counts[:, bi.upost].astype(np.float32) * hz - rate)
        np.testing.assert_allclose(bi.trace.cpu().numpy(), trace, rtol=1e-5, atol=1e-5)
        np.testing.assert_allclose(bi.rate.cpu().numpy(), rate, rtol=1e-5, atol=1e-4)
        pw = gb.pw.cpu().numpy()
        np.testing.assert_array_equal(pw[2], w_before[2])             # not learning: unchanged
        assert out[2] == 0 and (out[0] > 0)
