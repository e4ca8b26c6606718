"""Frame-end group readout (BatchMotor) and clamp (Clamp) on the device against NumPy
restatements of flyzero/batch.py:105-138 and flyzero/implant.py:84-104."""

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


def _brain(B):
    from flyzero_b200.brain import LIFParams
    from flyzero_b200.gpu import BatchBrain

    w = sp.random(300, 300, density=0.05, random_state=1, format="csr")
    w.data = np.rint(np.random.default_rng(1).normal(3, 4, w.nnz)).astype(np.float32)
    w.data[w.data == 0] = 1
    return BatchBrain(sp.csr_matrix(w), LIFParams(dt=0.25), batch=B, seed=2)


def test_batch_motor_rates_and_buttons(torch):
    from flyzero_b200.motor import READOUT, BatchMotor, MotorParams

    B = 5
    gb = _brain(B)
    rng = np.random.default_rng(3)
    groups = {name: rng.choice(300, rng.integers(1, 6), replace=False) for name in READOUT}
    for taps in (False, True):
        m = BatchMotor(gb, groups, MotorParams(taps=taps, steer_threshold=5.0))
        idx = np.concatenate([groups[g] for g in READOUT])
        size = np.array([len(groups[g]) for g in READOUT])
        avg = np.zeros((len(idx), len(READOUT)), np.float32)
        avg[np.arange(len(idx)), np.repeat(np.arange(len(READOUT)), size)] = 1.0 / size[np.repeat(np.arange(len(READOUT)), size)]
        rates = np.zeros((B, len(READOUT)), np.float32)
        window = 16.64
        for _ in range(6):
            counts = rng.poisson(0.6, (B, 300)).astype(np.int32)
            btn = m.update(torch.as_tensor(counts, device="cuda"), window)
            a = 1.0 - np.exp(-window / m.p.tau_ms)
            inst = (counts[:, idx].astype(np.float32) @ avg) * (1000.0 / window)
            rates += a * (inst - rates)
            np.testing.assert_allclose(m.rates, rates, rtol=1e-6, atol=1e-4)
            assert len(btn) == B and all(set(b) >= {"LEFT", "RIGHT", "L", "R", "A", "B", "Y"} for b in btn)
            r = m.rates
            if not taps:
                steer = (r[:, 0] - r[:, 1]) + (r[:, 5] - r[:, 4])
                assert [b["LEFT"] for b in btn] == list(steer > 5.0)
                assert [b["B"] for b in btn] == list(r[:, 6] > m.p.accel_threshold)
        m.reset([1])
        assert np.all(m.rates[1] == 0)


def test_clamp_controller_and_bias(torch):
    from flyzero_b200.motor import Clamp

    B = 4
    gb = _brain(B)
    rng = np.random.default_rng(4)
    groups = [rng.choice(300, 3, replace=False), rng.choice(300, 2, replace=False)]
    idx = np.concatenate(groups)
    gb.set_bias(idx, rng.uniform(0, 2, (B, len(idx))).astype(np.float32))
    base = gb.bias_ext[:, gb.slots(idx).long()].cpu().numpy().copy()
    c = Clamp(gb, groups, gain=0.05, limit=3.0, tau_ms=80.0)
    rate = np.zeros((B, 2), np.float32)
    u = np.zeros((B, 2), np.float32)
    window = 16.64
    for f in range(8):
        counts = rng.poisson(1.0, (B, 300)).astype(np.int32)
        targets = rng.uniform(0, 100, (B, 2)).astype(np.float32)
        active = np.array([True, False, True, True])
        gate = (rng.random((B, 2)) < 0.7).astype(np.float32) if f % 2 else None
        c.step(torch.as_tensor(counts, device="cuda"), targets, active, window, gate)
        a = 1 - np.exp(-window / 80.0)
        inst = np.stack([counts[:, g].mean(1) for g in groups], 1) * (1000.0 / window)
        rate = (rate + a * (inst - rate)).astype(np.float32)
        on = active[:, None] * (1.0 if gate is None else gate)
        u = (u + np.float32(0.05) * (targets - rate) * on).astype(np.float32)
        u = (np.clip(u, -3.0, 3.0) * active[:, None]).astype(np.float32)
        applied = np.repeat(u * on, [len(g) for g in groups], axis=1)
        np.testing.assert_allclose(c.rate.cpu().numpy(), rate, rtol=1e-6, atol=1e-4)
        np.testing.assert_allclose(c.u.cpu().numpy(), u, rtol=1e-5, atol=1e-5)
        np.testing.assert_allclose(gb.bias_ext[:, gb.slots(idx).long()].cpu().numpy(), base + applied, rtol=1e-5, atol=1e-5)
    assert np.abs(u).max() > 0.1


def test_batch_motor_matches_the_reference_readout(torch, golden):
    """Every slot of BatchMotor against the reference's own MotorReadout.update
    (flyzero/motor.py:78-95, tests/golden/motor.npz from make_motor_golden.py): smoothed rates within
    float32 rounding of the reference's float64 (relative 1e-5), the buttons equal, frame by frame;
    one readout group is empty, as a cell type missing from the connectome would be."""
    from flyzero_b200.brain import LIFParams
    from flyzero_b200.gpu import BatchBrain
    from flyzero_b200.motor import READOUT, BatchMotor, MotorParams

    g = golden("motor.npz")
    cnt = g["counts"]
    frames, slots, n = cnt.shape
    groups = {name: g["group_" + name] for name in READOUT}
    assert min(len(v) for v in groups.values()) == 0
    gb = BatchBrain(sp.identity(n, dtype=np.float32, format="csr"), LIFParams(), batch=slots)
    m = BatchMotor(gb, groups, MotorParams())
    names = [str(x) for x in g["button_names"]]
    for f in range(frames):
        btn = m.update(torch.as_tensor(cnt[f], device="cuda"), float(g["window"]))
        np.testing.assert_allclose(m.rates, g["rates"][f], rtol=1e-5, atol=1e-4)
        got = np.array([[b[k] for k in names] for b in btn])
        np.testing.assert_array_equal(got, g["buttons"][f], err_msg=f"frame {f}")
