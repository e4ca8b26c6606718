"""The motion eye on the device (fb_motion_eye) against the reference's own outputs
(tests/golden/eye.npz) and the CPU oracle of MotionEye.see (flyzero/vision.py:136-191): every
instance its own frames, mirrored frames (flyzero/pool.py:44), a restart in mid-sequence, the
Poisson probabilities written into the brain's input; the one-block-per-instance kernel and the
four grid-wide kernels. Bit-exact."""

import numpy as np
import pytest
import scipy.sparse as sp

import eye_cases as E

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def z(golden):
    return golden("eye.npz")


def _brain(n, B):
    from flyzero_b200.brain import LIFParams
    from flyzero_b200.gpu import BatchBrain

    w = sp.random(n, n, density=0.02, random_state=1, format="csr")
    w.data = np.rint(np.random.default_rng(1).normal(3, 4, w.nnz)).astype(np.float32)
    w.data[w.data == 0] = 1
    return BatchBrain(sp.csr_matrix(w), LIFParams(dt=0.25), batch=B, seed=2)


def _bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("kernels", ["fused", "split"])
@pytest.mark.parametrize("case", E.cases(), ids=lambda c: c[1])
def test_eye_matches_reference_and_oracle(torch, z, case, kernels):
    from eye_oracle import EyeOracle
    from flyzero_b200.vision import BatchMotionEye, MotionParams, layout

    k, name, shape, n, kw = case
    p = MotionParams(**kw)
    conn = E.connectome(z)
    lo = layout(conn, shape, p)
    fr = E.frames(z, k, name, shape, n)
    other = E.G.frames(shape, n, seed=900 + k)
    B = 3
    gb = _brain(int(z["n_neurons"]), B)
    bystander = int(np.setdiff1d(np.arange(gb.n), lo.idx)[0])
    gb.set_input([bystander], 42.0)
    eye = BatchMotionEye(gb, conn, shape, p, kernels=kernels)
    np.testing.assert_array_equal(eye.idx, z[f"{name}_idx"])
    want = z[f"{name}_rates"]
    o_flip = EyeOracle(shape, lo.gx, lo.gy, lo.chan, lo.visible, **E.oracle_params(p))
    o_other = EyeOracle(shape, lo.gx, lo.gy, lo.chan, lo.visible, **E.oracle_params(p))
    scale = np.float32(gb.p.dt / 1000.0)
    slot = eye.slot.long()
    restart_at = n // 2
    for t in range(n):
        if t == restart_at:
            eye.reset([2])
            o_other = EyeOracle(shape, lo.gx, lo.gy, lo.chan, lo.visible, **E.oracle_params(p))
        batch = torch.as_tensor(np.stack([fr[t], fr[t], other[t]]), device=gb.device)
        got = eye.see(batch, flip=[False, True, False]).cpu().numpy()
        np.testing.assert_array_equal(_bits(got[0]), _bits(want[t]), err_msg=f"{name} frame {t} vs reference")
        r_flip = o_flip.see(np.ascontiguousarray(fr[t][:, ::-1]))
        np.testing.assert_array_equal(_bits(got[1]), _bits(r_flip), err_msg=f"{name} frame {t} mirrored")
        np.testing.assert_array_equal(_bits(got[2]), _bits(o_other.see(other[t])), err_msg=f"{name} frame {t} other")
        pe = gb.p_ext[:, slot].cpu().numpy()
        np.testing.assert_array_equal(_bits(pe), _bits(got * scale))
    j = int(gb.slots([bystander])[0])
    assert np.all(gb.p_ext[:, j].cpu().numpy() == np.float32(42.0) * scale)
    assert np.count_nonzero(want) > 0


def test_eye_drives_the_brain(torch, z):
    """Frames -> eye -> run: the eye neurons spike at about their Poisson rates."""
    from flyzero_b200.vision import BatchMotionEye, MotionParams

    conn = E.connectome(z)
    shape = (48, 64)
    p = MotionParams(gain=5000.0)
    B = 4
    gb = _brain(int(z["n_neurons"]), B)
    eye = BatchMotionEye(gb, conn, shape, p)
    fr = E.G.frames(shape, 8, seed=5)
    total = np.zeros(B)
    expect = np.zeros(B)
    for t in range(8):
        rates = eye.see(torch.as_tensor(np.stack([fr[t]] * B), device=gb.device)).cpu().numpy()
        counts = gb.run(20.0).cpu().numpy()
        total += counts[:, eye.idx].sum(1)
        expect += rates.sum(1) * 0.02
    assert expect.min() > 50
    assert np.all(np.abs(total - expect) < 6 * np.sqrt(expect) + 0.1 * expect)


def test_eye_kernels_switch_mid_sequence(torch, z):
    """Both kernel forms keep the same state: alternating them frame by frame changes nothing."""
    from flyzero_b200.vision import BatchMotionEye, MotionParams

    k, name, shape, n, kw = E.cases()[1]
    conn = E.connectome(z)
    fr = E.frames(z, k, name, shape, n)
    gb = _brain(int(z["n_neurons"]), 1)
    eyes = [BatchMotionEye(gb, conn, shape, MotionParams(**kw), kernels=m) for m in ("fused", "split")]
    eyes[1].state = eyes[0].state
    eyes[1].restart = eyes[0].restart
    for t in range(n):
        got = eyes[t % 2].see(torch.as_tensor(fr[t:t + 1], device=gb.device)).cpu().numpy()
        np.testing.assert_array_equal(_bits(got[0]), _bits(z[f"{name}_rates"][t]))


def test_eye_rejects_bad_frames(torch, z):
    from flyzero_b200.vision import BatchMotionEye, MotionParams

    gb = _brain(int(z["n_neurons"]), 2)
    eye = BatchMotionEye(gb, E.connectome(z), (48, 64), MotionParams())
    with pytest.raises(ValueError):
        eye.see(torch.zeros((2, 48, 63, 3), dtype=torch.uint8, device=gb.device))
    with pytest.raises(ValueError):
        eye.see(torch.zeros((3, 48, 64, 3), dtype=torch.uint8, device=gb.device))
