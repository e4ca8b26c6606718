"""The CPU oracle against the reference's own outputs (tests/golden, made by make_golden.py).

Pins: the oracle restates flyzero/brain.py:32-58 bit for bit (strict compile and the shipped
fastmath compile, whose only effect is FMA contraction), reproduces the reference's Poisson
stream, and the engine's exact-accumulation semantics keep the reference raster.
"""

import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O
from flyzero_b200 import connectome as cx
from flyzero_b200 import workloads as wl

V_TOL = 1e-5   # mV: voltage agreement required against the reference (raster must be identical)


def _small(seed_w, seed_d, mean, sd, n=300, density=0.05):
    rng = np.random.default_rng(seed_d)
    w = sp.random(n, n, density=density, random_state=seed_w, format="csr")
    w.data = rng.normal(mean, sd, w.nnz)
    return w


def _long_rows():
    rng = np.random.default_rng(4)
    w = sp.random(600, 600, density=0.6, random_state=4, format="csr")
    w.data = rng.normal(5.0, 3, w.nnz)
    return w


CASES = {"backends": (lambda: _small(2, 3, 20, 15), 0.1, 500),       # test_flyzero.py:104-114
         "gpu_nonoise": (lambda: _small(2, 2, 40, 30), 0.25, 200),   # test_gpu.py:39-47
         "long_rows": (_long_rows, 0.25, 120)}                       # test_gpu.py:168-183


@pytest.mark.parametrize("case", list(CASES))
def test_restatement_is_bit_exact_to_strict_reference(golden, case):
    g = golden("reference_tests.npz")
    make, dt, steps = CASES[case]
    b = O.RefBrain(make(), O.Params(dt=dt), contract=False)
    b.v[:40] = -40.0
    c, sc, sd = b.run_steps(steps, record=True)
    np.testing.assert_array_equal(c, g[f"{case}_strict_counts"])
    np.testing.assert_array_equal(b.v, g[f"{case}_strict_v"])
    np.testing.assert_array_equal(sc, g[f"{case}_step_counts"])
    np.testing.assert_array_equal(sd, g[f"{case}_step_digest"])


@pytest.mark.parametrize("case", list(CASES))
def test_restatement_with_contraction_is_bit_exact_to_shipped_kernel(golden, case):
    g = golden("reference_tests.npz")
    make, dt, steps = CASES[case]
    b = O.RefBrain(make(), O.Params(dt=dt), contract=True)
    b.v[:40] = -40.0
    c = b.run_steps(steps)
    np.testing.assert_array_equal(c, g[f"{case}_counts"])
    np.testing.assert_array_equal(b.v, g[f"{case}_v"])


@pytest.mark.parametrize("case", list(CASES))
def test_engine_semantics_keep_the_reference_raster(golden, case):
    """Exact (Q32.32 here: these weights are not integers) accumulation vs float summation."""
    g = golden("reference_tests.npz")
    make, dt, steps = CASES[case]
    e = O.EngineOracle(make(), O.Params(dt=dt), batch=2)
    assert e.acc_mode == "fixed"
    e.v[:, :40] = -40.0
    c = e.run_steps(steps)
    for b in range(2):
        np.testing.assert_array_equal(c[b], g[f"{case}_counts"])
        assert np.abs(e.v[b] - g[f"{case}_v"]).max() <= V_TOL


@pytest.mark.parametrize("name", ["driven", "driven_inh"])
def test_reference_poisson_stream_is_reproduced(golden, name):
    """test_flyzero.py:16-24 with the genuine Brain(seed=0).run(200) stream."""
    g = golden("reference_tests.npz")
    w = np.zeros((2, 2))
    w[0, 1] = 100 if name == "driven" else -100
    b = O.RefBrain(sp.csr_matrix(w))
    seed_k = O.run_seeds(0, 1)[0]
    p_in = np.float32(200.0) * np.float32(0.1 / 1000.0)
    kicks = O.reference_kicks(seed_k, 2000, np.array([p_in]))
    c = b.run_steps(2000, [0], kicks)
    np.testing.assert_array_equal(c, g[f"{name}_counts"])
    if name == "driven":
        assert c[0] > 10 and c[1] > 5
    else:
        assert c[1] == 0


def test_one_step_push_equals_dense_row_sum(golden):
    """test_flyzero.py:27-34: the spikes of one step land in the ring as the dense row sum."""
    g = golden("reference_tests.npz")
    w = sp.random(50, 50, density=0.2, random_state=1, format="csr") * 10
    b = O.RefBrain(w)
    spk = np.array([3, 7, 20, 49])
    b.v[spk] = -40.0
    b.run_steps(1)
    np.testing.assert_allclose(b.pending[0], g["propagate_out"], rtol=1e-5)
    expected = np.asarray(sp.csr_matrix(w)[spk].sum(0)).ravel() * 0.275
    np.testing.assert_allclose(b.pending[0], expected, rtol=1e-5)


def test_per_instance_plastic_weights(golden):
    """test_gpu.py:50-62: each instance carries its own copy of the plastic synapses."""
    g = golden("reference_tests.npz")
    w = _small(2, 2, 40, 30)
    pos = g["plastic_pos"]
    e = O.EngineOracle(w, O.Params(dt=0.25), batch=2, plastic_pos=pos)
    e.pw[1] = g["plastic_changed_data"]
    e.v[:, :40] = -40.0
    c = e.run_steps(200)
    np.testing.assert_array_equal(c[0], g["plastic_orig_counts"])
    np.testing.assert_array_equal(c[1], g["plastic_changed_counts"])


def test_long_plastic_rows(golden):
    """test_gpu.py:168-183: every synapse plastic, rows longer than one work chunk."""
    g = golden("reference_tests.npz")
    w = _long_rows()
    e = O.EngineOracle(w, O.Params(dt=0.25), batch=2, plastic_pos=np.arange(sp.csr_matrix(w).nnz))
    e.pw[1] *= 0.5
    e.v[:, :40] = -40.0
    c = e.run_steps(120)
    np.testing.assert_array_equal(c[0], g["long_rows_counts"])
    assert not np.array_equal(c[0], c[1])


def test_hash_stream_poisson_rate():
    """test_gpu.py:65-72: 100 Hz on 10 unconnected neurons for 1 s at dt 0.25."""
    w = sp.csr_matrix((10, 10), dtype=np.float32)
    e = O.EngineOracle(w, O.Params(dt=0.25), batch=2, seed=5)
    j = e.slots(np.arange(10))
    e.p_ext[:, j] = np.float32(100.0) * np.float32(0.25 / 1000.0)
    c = e.run_steps(4000)
    assert 70 < c.mean() < 105
    assert not np.array_equal(c[0], c[1])


def test_workload_n16384(golden):
    """Benchmark workload 1 (N=16,384, 10,000 steps): shipped kernel bit for bit, FP64 kernel bit
    for bit, and the engine's INT32 semantics raster-exact with |dv| <= 1e-5 mV."""
    g = golden("workload_n16384.npz")
    conn = cx.synthetic(16_384, seed=1)
    assert str(g["checksum"]) == cx.csr_checksum(conn.weights)
    idx, rate = wl.config1_inputs(conn.n, seed=1)
    np.testing.assert_array_equal(idx, g["input_idx"])
    kicks = O.reference_kicks(int(g["seed_k"]), 10_000, rate * np.float32(0.1 / 1000.0))
    b = O.RefBrain(conn.weights)
    c, sc, sd = b.run_steps(10_000, idx, kicks, record=True)
    np.testing.assert_array_equal(c, g["run_counts"])
    np.testing.assert_array_equal(sd, g["step_digest"])
    np.testing.assert_array_equal(b.v, g["v"])
    b = O.RefBrain(conn.weights, real=np.float64, contract=False)
    c, sc, sd = b.run_steps(10_000, idx, kicks, record=True)
    np.testing.assert_array_equal(sd, g["f64_step_digest"])
    np.testing.assert_array_equal(b.v, g["f64_v"])
    e = O.EngineOracle(conn.weights, O.Params(), batch=1)
    assert e.acc_mode == "count"
    e.slots(idx)
    kr = np.zeros((10_000, 1, e.n_ext), bool)
    kr[:, 0, e.ext_idx[idx]] = kicks
    c, sc, sd = e.run_steps(10_000, kr, record=True)
    np.testing.assert_array_equal(sd[:, 0], g["step_digest"])
    assert np.abs(e.v[0] - g["v"]).max() <= V_TOL


def test_workload_n138639(golden):
    """Benchmark workload 2 (N=138,639, grating input, 10,000 steps in 61 Brain.run calls)."""
    g = golden("workload_n138639.npz")
    conn = cx.flywire_scale()
    assert str(g["checksum"]) == cx.csr_checksum(conn.weights)
    drive = wl.grating_drive(conn.n, seed=0, exclude=conn.motor)
    idx = g["input_idx"]
    np.testing.assert_array_equal(idx, np.r_[drive.inputs, drive.tonic])
    e = O.EngineOracle(conn.weights, O.Params(), batch=1)
    e.slots(idx)
    t_ms, sds = 0.0, []
    for k, sk, d in zip(g["frames"], g["seeds"], g["dirs"]):
        rate = np.r_[wl.grating_rates(drive, t_ms, d, 1.0), np.float32(60.0)].astype(np.float32)
        kicks = O.reference_kicks(int(sk), int(k), rate * np.float32(0.1 / 1000.0))
        kr = np.zeros((k, 1, e.n_ext), bool)
        kr[:, 0, e.ext_idx[idx]] = kicks
        _, _, sd = e.run_steps(int(k), kr, record=True)
        sds.append(sd[:, 0])
        t_ms += k * 0.1
    np.testing.assert_array_equal(np.concatenate(sds), g["step_digest"])
    assert np.abs(e.v[0] - g["v"]).max() <= V_TOL


def test_reward_rule_restatement(golden):
    """learning.py:116-131 against the reference's own RewardPlasticity on its toy connectome."""
    g = golden("learning.npz")
    data = g["data0"].copy()
    st = {k: g[k].copy() for k in ("pos", "pre", "post", "targets", "sign", "wmax")}
    n = len(g["indptr"]) - 1
    st.update(elig=np.zeros(len(st["pos"]), np.float32), post_mean=np.zeros(n, np.float32), r_mean=0.0)
    for f in range(len(g["reward"])):
        adv = O.reward_step(st, data, g["counts"][f], float(g["reward"][f]), float(g["window"]), O.LearnParams())
        assert adv == g["adv"][f]
        np.testing.assert_array_equal(data[st["pos"]], g["w"][f])
        np.testing.assert_array_equal(st["elig"], g["elig"][f])
        np.testing.assert_array_equal(st["post_mean"][st["targets"]], g["post_mean"][f])
