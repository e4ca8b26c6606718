"""The reward rule on the GPU (fb_reward_step): bit-exact to the reference's RewardPlasticity on its
own golden vectors, and to the NumPy restatement of BatchReward/_Plastic.apply for many slots."""

import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_reward_plasticity_matches_reference(torch, golden):
    """learning.py:116-131 on the reference's toy connectome: traces, running means, advantage and
    the weights written to brain.data, frame by frame, bit for bit."""
    from flyzero_b200.brain import Brain, LIFParams
    from flyzero_b200.learning import RewardPlasticity

    g = golden("learning.npz")
    n = len(g["indptr"]) - 1
    counts_w = np.rint(g["data0"] / np.float32(0.275)).astype(np.float32)
    w = sp.csr_matrix((counts_w, g["indices"], g["indptr"]), shape=(n, n))
    brain = Brain(w, LIFParams(dt=0.25))
    np.testing.assert_array_equal(brain.data, g["data0"])
    rp = RewardPlasticity(brain, targets=g["targets"])
    np.testing.assert_array_equal(rp.pos, g["pos"])
    np.testing.assert_array_equal(rp.wmax, g["wmax"])
    for f in range(len(g["reward"])):
        adv = rp.step(g["counts"][f], float(g["reward"][f]), float(g["window"]))
        assert adv == g["adv"][f]
        np.testing.assert_array_equal(brain.data[rp.pos], g["w"][f])
        np.testing.assert_array_equal(rp.elig, g["elig"][f])
        np.testing.assert_array_equal(rp.post_mean[rp.targets], g["post_mean"][f])
    assert np.abs(g["w"][-1] - g["data0"][g["pos"]]).max() > 0     # the weights did move


def test_learned_weights_drive_the_next_run(torch):
    """After a reward step the engine simulates with the new weights (Brain.data and pw agree)."""
    from flyzero_b200.brain import Brain, LIFParams
    from flyzero_b200.learning import RewardPlasticity

    rng = np.random.default_rng(5)
    w = sp.random(400, 400, density=0.05, random_state=5, format="csr")
    w.data = np.rint(rng.normal(8, 6, w.nnz)).astype(np.float32)
    brain = Brain(w, LIFParams(dt=0.25), rng="device")
    brain.set_input(np.arange(40), 150.0)
    rp = RewardPlasticity(brain, targets=np.arange(300, 330))
    for _ in range(5):
        c = brain.run(16.6)
        rp.step(c, float(rng.standard_normal()), 16.6)
    eng = brain._eng
    k = np.searchsorted(eng.plastic_pos, rp.pos)
    np.testing.assert_array_equal(eng.pw[0].cpu().numpy()[k], brain.data[rp.pos])


def _batch_setup(torch, B=6, fos=(0, 0, 1, 1, 1, 2), seed=3):
    from flyzero_b200.brain import LIFParams
    from flyzero_b200.gpu import BatchBrain

    rng = np.random.default_rng(seed)
    n = 500
    w = sp.random(n, n, density=0.04, random_state=seed, format="csr")
    w.data = np.rint(rng.normal(4, 5, w.nnz)).astype(np.float32)
    w.data[w.data == 0] = 1
    w = sp.csr_matrix(w)
    w.sort_indices()
    targets = np.arange(450, 470)
    pos = np.flatnonzero(np.isin(w.indices, targets))
    gb = BatchBrain(w, LIFParams(dt=0.25), batch=B, plastic_pos=pos)
    return gb, rng, targets, np.asarray(fos)


def _oracle_state(gb, fos, cap=3.0):
    upre, pre_k = np.unique(gb.pl_pre, return_inverse=True)
    upost, post_k = np.unique(gb.pl_post, return_inverse=True)
    w0 = gb.w0
    return {"upre": upre, "upost": upost, "pre_k": pre_k, "post_k": post_k,
            "elig": np.zeros((gb.B, len(gb.plastic_pos)), np.float32),
            "post_mean": np.zeros((gb.B, len(upost)), np.float32), "r_mean": np.zeros(gb.B, np.float32),
            "sign": np.sign(w0), "wmax": cap * np.maximum(np.abs(w0), gb.p.w_syn), "fos": fos,
            "n_flies": int(fos.max()) + 1}


@pytest.mark.parametrize("scaled", [False, True])
def test_batch_reward_matches_numpy_restatement(torch, scaled):
    """batch.py:482-495 with _Plastic.apply (school.py:289-304 when scaled): slots of one fly share
    the averaged change; traces and means are exact, weights within the GEMM's summation order."""
    from flyzero_b200.batch import BatchReward

    gb, rng, targets, fos = _batch_setup(torch)
    br = BatchReward(gb, fly_of_slot=fos, targets=targets)
    st = _oracle_state(gb, fos)
    pw = gb.pw.cpu().numpy().copy()
    p = O.LearnParams()
    window = 1000.0 / 60.0988
    for f in range(12):
        counts = rng.poisson(3.0, (gb.B, gb.n)).astype(np.int32)
        reward = rng.standard_normal(gb.B)
        learn = rng.random(gb.B) < 0.7 if f % 4 else np.zeros(gb.B, bool)
        dev = torch.as_tensor(counts, device=gb.device)
        if scaled:
            eta_slot = rng.uniform(1e-4, 5e-4, gb.B)
            adv = br.step_scaled(dev, reward, learn, window, eta_slot)
            want = O.batch_reward_step(st, pw, counts, reward, learn, window, p, eta_slot=eta_slot)
        else:
            adv = br.step(dev, reward, learn, window)
            want = O.batch_reward_step(st, pw, counts, reward, learn, window, p)
        np.testing.assert_array_equal(adv, want)
        np.testing.assert_array_equal(br.r_mean, st["r_mean"])
        np.testing.assert_array_equal(br.elig.cpu().numpy(), st["elig"])
        np.testing.assert_array_equal(br.post_mean.cpu().numpy(), st["post_mean"])
        np.testing.assert_allclose(gb.pw.cpu().numpy(), pw, rtol=1e-6, atol=1e-7)
    assert np.abs(pw - gb.w0).max() > 1e-4
    same_fly = fos == 1
    np.testing.assert_array_equal(gb.pw.cpu().numpy()[same_fly][0], gb.pw.cpu().numpy()[same_fly][1])


def test_plastic_state_round_trips_through_npz(torch, tmp_path):
    """state() -> npz -> load() into a brain with a different plastic set: entries are matched by
    CSR position, the others keep their connectome weights (batch.py:195-219)."""
    from flyzero_b200.batch import BatchReward, load_state, save_state
    from flyzero_b200.brain import LIFParams
    from flyzero_b200.gpu import BatchBrain

    gb, rng, targets, fos = _batch_setup(torch)
    br = BatchReward(gb, fly_of_slot=fos, targets=targets)
    gb.pw += torch.as_tensor(rng.normal(0, 0.1, gb.pw.shape).astype(np.float32), device=gb.device)
    st = br.state(1)
    save_state(tmp_path / "fly1.npz", st)
    back = load_state(tmp_path / "fly1.npz")
    assert set(back) == {"pos", "data", "w0"}
    np.testing.assert_array_equal(back["data"], gb.pw[int(np.flatnonzero(fos == 1)[0])].cpu().numpy())
    # a second brain whose plastic set is a superset of the saved one
    extra = np.setdiff1d(np.arange(0, gb.indices.size, 7), gb.plastic_pos)
    pos2 = np.union1d(gb.plastic_pos, extra)
    gb2 = BatchBrain(sp.csr_matrix((gb.data / np.float32(0.275), gb.indices, gb.indptr), shape=(gb.n, gb.n)),
                     LIFParams(dt=0.25), batch=2, plastic_pos=pos2)
    br2 = BatchReward(gb2, targets=targets)
    br2.load(back)
    got = gb2.pw.cpu().numpy()
    k = np.searchsorted(pos2, back["pos"])
    np.testing.assert_array_equal(got[:, k], np.tile(back["data"], (2, 1)))
    rest = np.setdiff1d(np.arange(len(pos2)), k)
    np.testing.assert_array_equal(got[:, rest], np.tile(gb2.w0[rest], (2, 1)))


@pytest.mark.parametrize("with_sel", [False, True])
def test_plastic_apply_averages_over_each_flys_active_slots(torch, with_sel):
    """_Plastic.apply (batch.py:158-172) for an arbitrary dw: every slot of a fly gets the mean of
    dw over the fly's active slots, clipped on the connectome sign to [0, wmax]; with ``sel`` only
    those synapses move. Compared with the plain NumPy formula (float32; the per-fly sum's order
    is the only freedom, hence the tolerance)."""
    from flyzero_b200.batch import BatchReward

    gb, rng, targets, fos = _batch_setup(torch)
    br = BatchReward(gb, fly_of_slot=fos, targets=targets)
    n_pl = gb.pw.shape[1]
    sel = np.sort(rng.choice(n_pl, n_pl // 3, replace=False)) if with_sel else None
    cols = n_pl if sel is None else len(sel)
    w = gb.pw.cpu().numpy().copy()
    sign = np.sign(gb.w0).astype(np.float32)
    wmax = (np.float32(3.0) * np.maximum(np.abs(gb.w0), np.float32(gb.p.w_syn))).astype(np.float32)
    for f in range(4):
        dw = (rng.standard_normal((gb.B, cols)) * 0.2).astype(np.float32)
        active = rng.random(gb.B) < 0.6
        br.apply(torch.as_tensor(dw, device=gb.device), active, sel)
        onehot = np.zeros((int(fos.max()) + 1, gb.B), np.float32)
        onehot[fos, np.arange(gb.B)] = active
        per_fly = (onehot / np.maximum(onehot.sum(1, keepdims=True), 1)) @ dw
        k = np.arange(n_pl) if sel is None else sel
        cand = w[:, k] + per_fly[fos]
        w[:, k] = sign[k] * np.clip(sign[k] * cand, 0.0, wmax[k])
        np.testing.assert_allclose(gb.pw.cpu().numpy(), w, rtol=1e-6, atol=1e-7)
    if sel is not None:
        rest = np.setdiff1d(np.arange(n_pl), sel)
        np.testing.assert_array_equal(gb.pw.cpu().numpy()[:, rest], np.tile(gb.w0[rest], (gb.B, 1)))
    before = br.drift()
    assert before.shape == (gb.B,) and before.max() > 0
    br.consolidate(0.5)
    br.swap_slow()
    br.swap_slow()
    np.testing.assert_array_equal(br.drift(), before)
