"""Parity of the CUDA engine (through the C ABI, via BatchBrain / Brain) with the oracle and the
reference's golden outputs. Every test needs a B200."""

import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O
from flyzero_b200 import connectome as cx
from flyzero_b200 import workloads as wl

pytestmark = pytest.mark.gpu

V_TOL = 1e-5   # mV, against the reference (its raster must match exactly)
ENGINES = ["step", "persistent"]


@pytest.fixture(scope="module")
def torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _small(seed_w, seed_d, mean, sd, n=300, density=0.05):
    rng = np.random.default_rng(seed_d)
    w = sp.random(n, n, density=density, random_state=seed_w, format="csr")
    w.data = rng.normal(mean, sd, w.nnz)
    return w


def _raster(torch, kicks_bool, device):
    from flyzero_b200.brain import pack_kicks

    return torch.as_tensor(pack_kicks(kicks_bool).view(np.int32), device=device)


def _bb(w, params, batch, engine, **kw):
    from flyzero_b200.gpu import BatchBrain

    b = BatchBrain(w, params, batch=batch, **kw)
    if engine == "persistent" and b.info().group == 0:
        pytest.skip("persistent engine unavailable for this configuration")
    b.set_schedule(engine)
    return b


def _compare_state(torch, gb, eo):
    np.testing.assert_array_equal(gb.v.cpu().numpy(), eo.v)
    np.testing.assert_array_equal(gb.g.cpu().numpy(), eo.g)
    np.testing.assert_array_equal(gb.ref.cpu().numpy(), eo.ref)


@pytest.mark.parametrize("engine", ENGINES)
def test_gpu_matches_cpu_without_noise(torch, golden, engine):
    """tests/test_gpu.py:39-47 (float weights -> Q32.32 accumulation), bit-exact vs the oracle."""
    from flyzero_b200.brain import LIFParams

    g = golden("reference_tests.npz")
    w = _small(2, 2, 40, 30)
    gb = _bb(w, LIFParams(dt=0.25), 3, engine)
    gb.v[:, :40] = -40.0
    out = gb.run(50).cpu().numpy()
    assert g["gpu_nonoise_counts"].sum() > 50
    for k in range(3):
        np.testing.assert_array_equal(out[k], g["gpu_nonoise_counts"])
    eo = O.EngineOracle(w, O.Params(dt=0.25), batch=3)
    eo.v[:, :40] = -40.0
    eo.run_steps(200)
    _compare_state(torch, gb, eo)
    assert np.abs(gb.v.cpu().numpy()[0] - g["gpu_nonoise_v"]).max() <= V_TOL


@pytest.mark.parametrize("engine", ENGINES)
def test_each_fly_has_its_own_plastic_synapses(torch, golden, engine):
    """tests/test_gpu.py:50-62."""
    from flyzero_b200.brain import LIFParams

    g = golden("reference_tests.npz")
    w = _small(2, 2, 40, 30)
    pos = g["plastic_pos"]
    gb = _bb(w, LIFParams(dt=0.25), 2, engine, plastic_pos=pos)
    gb.pw[1] = torch.as_tensor(g["plastic_changed_data"], device=gb.device)
    gb.v[:, :40] = -40.0
    out = gb.run(50).cpu().numpy()
    np.testing.assert_array_equal(out[0], g["plastic_orig_counts"])
    np.testing.assert_array_equal(out[1], g["plastic_changed_counts"])
    assert not np.array_equal(out[0], out[1])
    eo = O.EngineOracle(w, O.Params(dt=0.25), batch=2, plastic_pos=pos)
    eo.pw[1] = g["plastic_changed_data"]
    eo.v[:, :40] = -40.0
    eo.run_steps(200)
    _compare_state(torch, gb, eo)


@pytest.mark.parametrize("engine", ENGINES)
def test_long_plastic_rows_are_split_into_chunks(torch, golden, engine):
    """tests/test_gpu.py:168-183: every synapse plastic, rows longer than a 256-entry work item."""
    from flyzero_b200.brain import LIFParams

    g = golden("reference_tests.npz")
    rng = np.random.default_rng(4)
    w = sp.random(600, 600, density=0.6, random_state=4, format="csr")
    w.data = rng.normal(5.0, 3, w.nnz)
    assert np.diff(sp.csr_matrix(w).indptr).max() > 300
    gb = _bb(w, LIFParams(dt=0.25), 2, engine, plastic_pos=np.arange(w.nnz))
    gb.pw[1] *= 0.5
    gb.v[:, :40] = -40.0
    out = gb.run(30).cpu().numpy()
    np.testing.assert_array_equal(out[0], g["long_rows_counts"])
    assert not np.array_equal(out[0], out[1])


@pytest.mark.parametrize("engine", ENGINES)
def test_poisson_input_rate(torch, engine):
    """tests/test_gpu.py:65-72, plus: the hash stream equals the oracle's draw for draw."""
    from flyzero_b200.brain import LIFParams

    w = sp.csr_matrix((10, 10), dtype=np.float32)
    gb = _bb(w, LIFParams(dt=0.25), 2, engine, seed=5)
    gb.set_input(np.arange(10), 100.0)
    c = gb.run(1000).cpu().numpy()
    assert 70 < c.mean() < 105
    assert not np.array_equal(c[0], c[1])
    eo = O.EngineOracle(w, O.Params(dt=0.25), batch=2, seed=5)
    j = eo.slots(np.arange(10))
    eo.p_ext[:, j] = np.float32(100.0) * np.float32(0.25 / 1000.0)
    np.testing.assert_array_equal(c, eo.run_steps(4000))


@pytest.mark.parametrize("name", ["driven", "driven_inh"])
def test_brain_reference_stream(torch, golden, name):
    """tests/test_flyzero.py:16-24 through the Brain API with the reference's own Poisson stream."""
    from flyzero_b200.brain import Brain

    g = golden("reference_tests.npz")
    w = np.zeros((2, 2))
    w[0, 1] = 100 if name == "driven" else -100
    b = Brain(sp.csr_matrix(w))
    b.set_input([0], 200.0)
    c = b.run(200)
    np.testing.assert_array_equal(c, g[f"{name}_counts"])


def test_brain_numba_case_and_host_state_writes(torch, golden):
    """tests/test_flyzero.py:104-114 through Brain, with ``b.v[:40] = -40`` written on the host."""
    from flyzero_b200.brain import Brain

    g = golden("reference_tests.npz")
    b = Brain(_small(2, 3, 20, 15))
    b.v[:40] = -40.0
    c = b.run(50)
    np.testing.assert_array_equal(c, g["backends_counts"])
    assert np.abs(b.v - g["backends_v"]).max() <= V_TOL


def test_brain_data_writes_act_at_spike_time(torch):
    """Learning writes Brain.data between runs (learning.py:130): the new weight applies to spikes
    after the write, input already in flight keeps the old one, exactly as the reference ring."""
    from flyzero_b200.brain import Brain, LIFParams

    w = _small(2, 2, 40, 30)
    b = Brain(w, LIFParams(dt=0.25))
    ref = O.RefBrain(w, O.Params(dt=0.25))
    b.v[:40] = -40.0
    ref.v[:40] = -40.0
    rng = np.random.default_rng(0)
    pos = np.flatnonzero(b.indices < 60)
    for k in range(6):
        c = b.run(5)
        cr = ref.run_steps(20)
        np.testing.assert_array_equal(c, cr)
        new = (b.data[pos] * rng.uniform(0.5, 2.0, len(pos))).astype(np.float32)
        b.data[pos] = new
        ref.data[pos] = new
    assert np.abs(b.v - ref.v).max() <= 1e-4


@pytest.mark.parametrize("engine", ENGINES)
def test_workload_n16384_raster_parity(torch, golden, engine):
    """Benchmark workload 1: the reference's raster for 10,000 steps, every step, and bit-exact
    agreement with the oracle's INT32 semantics."""
    from flyzero_b200.brain import LIFParams

    g = golden("workload_n16384.npz")
    conn = cx.synthetic(16_384, seed=1)
    idx, rate = wl.config1_inputs(conn.n, seed=1)
    kicks = O.reference_kicks(int(g["seed_k"]), 10_000, rate * np.float32(0.1 / 1000.0))
    gb = _bb(conn.weights, LIFParams(), 1, engine)
    gb.slots(idx)
    kr = np.zeros((10_000, 1, gb.p_ext.shape[1]), bool)
    kr[:, 0, gb._slot[idx]] = kicks
    counts, sc, sd = gb.run_steps(10_000, _raster(torch, kr, gb.device), record=True)
    sd = sd.cpu().numpy().view(np.uint64)[:, 0]
    np.testing.assert_array_equal(sd, g["step_digest"])
    np.testing.assert_array_equal(counts.cpu().numpy()[0], g["run_counts"])
    assert np.abs(gb.v.cpu().numpy()[0] - g["v"]).max() <= V_TOL
    eo = O.EngineOracle(conn.weights, O.Params(), batch=1)
    eo.slots(idx)
    eo.run_steps(10_000, kr)
    _compare_state(torch, gb, eo)


@pytest.mark.parametrize("engine", ENGINES)
def test_workload_n138639_raster_parity(torch, golden, engine):
    """Benchmark workload 2 at full scale: 10,000 steps in 61 runs, raster identical to the
    reference's at every step, |dv| <= 1e-5 mV at the end."""
    from flyzero_b200.brain import LIFParams

    g = golden("workload_n138639.npz")
    conn = cx.flywire_scale()
    drive = wl.grating_drive(conn.n, seed=0, exclude=conn.motor)
    idx = g["input_idx"]
    gb = _bb(conn.weights, LIFParams(), 1, engine)
    gb.slots(idx)
    t_ms, sds = 0.0, []
    for k, sk, d in zip(g["frames"], g["seeds"], g["dirs"]):
        rate = np.r_[wl.grating_rates(drive, t_ms, d, 1.0), np.float32(60.0)].astype(np.float32)
        kicks = O.reference_kicks(int(sk), int(k), rate * np.float32(0.1 / 1000.0))
        kr = np.zeros((k, 1, gb.p_ext.shape[1]), bool)
        kr[:, 0, gb._slot[idx]] = kicks
        _, _, sd = gb.run_steps(int(k), _raster(torch, kr, gb.device), record=True)
        sds.append(sd.cpu().numpy().view(np.uint64)[:, 0])
        t_ms += k * 0.1
    np.testing.assert_array_equal(np.concatenate(sds), g["step_digest"])
    assert np.abs(gb.v.cpu().numpy()[0] - g["v"]).max() <= V_TOL


def test_batched_full_scale_hash_noise_plastic_deltas(torch):
    """40 instances on the 138,639-neuron graph, Poisson hash noise, grating rates, per-instance
    plastic weight deltas on the 7,300 motor inputs: bit-exact state vs the oracle, and the step
    and persistent engines agree."""
    from flyzero_b200.brain import LIFParams

    conn = cx.flywire_scale()
    drive = wl.grating_drive(conn.n, seed=0, exclude=conn.motor)
    pos = np.flatnonzero(np.isin(conn.weights.indices, conn.motor))
    assert len(pos) == 7300
    B, steps = 40, 120          # 40 > one persistent group at this size: two groups
    work = wl.BatchedWorkload.make(B, seed=3)
    rates = work.rates(drive, 0.0, work.directions())
    dw = np.random.default_rng(9).standard_normal((B, len(pos))).astype(np.float32) * np.float32(0.3)
    outs = {}
    for engine in ENGINES:
        gb = _bb(conn.weights, LIFParams(), B, engine, plastic_pos=pos, seed=17)
        gb.set_input(np.r_[drive.inputs, drive.tonic], rates)
        gb.pw += torch.as_tensor(dw, device=gb.device)
        c = gb.run_steps(steps).cpu().numpy()
        outs[engine] = (c, gb.v.cpu().numpy(), gb.g.cpu().numpy())
        pw = gb.pw.cpu().numpy()
    np.testing.assert_array_equal(outs["step"][0], outs["persistent"][0])
    np.testing.assert_array_equal(outs["step"][1], outs["persistent"][1])
    eo = O.EngineOracle(conn.weights, O.Params(), batch=B, plastic_pos=pos, seed=17)
    j = eo.slots(np.r_[drive.inputs, drive.tonic])
    eo.p_ext[:, j] = rates * np.float32(0.1 / 1000.0)
    eo.pw[:] = pw
    c = eo.run_steps(steps)
    np.testing.assert_array_equal(outs["persistent"][0], c)
    np.testing.assert_array_equal(outs["persistent"][1], eo.v)
    np.testing.assert_array_equal(outs["persistent"][2], eo.g)
    assert c.sum() > 0


@pytest.mark.parametrize("engine", ENGINES)
def test_partial_reset_and_run_lengths(torch, engine):
    """BatchBrain.reset(flies) (gpu.py:186-199) and per-instance run lengths, vs the oracle."""
    from flyzero_b200.brain import LIFParams

    conn = cx.synthetic(4096, seed=5)
    B = 4
    gb = _bb(conn.weights, LIFParams(), B, engine, seed=2)
    idx, rate = wl.config1_inputs(conn.n, seed=5)
    gb.set_input(idx, rate * 3)
    eo = O.EngineOracle(conn.weights, O.Params(), batch=B, seed=2)
    j = eo.slots(idx)
    eo.p_ext[:, j] = (rate * 3) * np.float32(0.1 / 1000.0)
    c1 = gb.run_steps(50).cpu().numpy()
    np.testing.assert_array_equal(c1, eo.run_steps(50))
    gb.reset([1, 3])
    eo.reset_flies([1, 3])
    gb.set_run_length([30, -1, 10, 45])
    stop = np.array([eo.t + 30, 2 ** 62, eo.t + 10, eo.t + 45], np.int64)
    c2 = gb.run_steps(60).cpu().numpy()
    np.testing.assert_array_equal(c2, eo.run_steps(60, stop_tick=stop))
    _compare_state(torch, gb, eo)


@pytest.mark.parametrize("lanes", [8, 16, 32])
def test_lanes_per_item_agree(torch, lanes):
    from flyzero_b200.brain import LIFParams

    conn = cx.synthetic(8192, seed=2)
    idx, rate = wl.config1_inputs(conn.n, seed=2)
    gb = _bb(conn.weights, LIFParams(), 3, "persistent", seed=4)
    gb.set_schedule(lanes=lanes)
    gb.set_input(idx, rate * 2)
    c = gb.run_steps(300).cpu().numpy()
    eo = O.EngineOracle(conn.weights, O.Params(), batch=3, seed=4)
    j = eo.slots(idx)
    eo.p_ext[:, j] = (rate * 2) * np.float32(0.1 / 1000.0)
    np.testing.assert_array_equal(c, eo.run_steps(300))


def test_fp64_oracle_mode(torch, golden):
    """FP64 state on the GPU over the whole config-1 run (10,000 steps of the 16,384-neuron
    workload): bit-exact vs the oracle's FP64 engine semantics; raster-exact at every step, equal
    counts and final voltages within V_TOL vs the reference kernel re-jitted on float64
    (flyzero/brain.py:32-58)."""
    from flyzero_b200.brain import LIFParams

    g = golden("workload_n16384.npz")
    conn = cx.synthetic(16_384, seed=1)
    idx, rate = wl.config1_inputs(conn.n, seed=1)
    steps = 10_000
    kicks = O.reference_kicks(int(g["seed_k"]), 10_000, rate * np.float32(0.1 / 1000.0))[:steps]
    gb = _bb(conn.weights, LIFParams(), 1, "step", fp64=True)
    gb.slots(idx)
    kr = np.zeros((steps, 1, gb.p_ext.shape[1]), bool)
    kr[:, 0, gb._slot[idx]] = kicks
    c, _, sd = gb.run_steps(steps, _raster(torch, kr, gb.device), record=True)
    np.testing.assert_array_equal(sd.cpu().numpy().view(np.uint64)[:, 0], g["f64_step_digest"][:steps])
    np.testing.assert_array_equal(c.cpu().numpy()[0], g["f64_counts"])
    assert np.abs(gb.v.cpu().numpy()[0] - g["f64_v"]).max() <= V_TOL
    eo = O.EngineOracle(conn.weights, O.Params(), batch=1, real=np.float64)
    eo.slots(idx)
    eo.run_steps(steps, kr)
    _compare_state(torch, gb, eo)


def test_device_decay_factors_match_numpy(torch):
    from flyzero_b200.brain import LIFParams
    from flyzero_b200.gpu import BatchBrain

    for dt in (0.1, 0.25, 0.05):
        p = LIFParams(dt=dt)
        b = BatchBrain(sp.csr_matrix((4, 4), dtype=np.float32), p)
        assert b.decay_syn == np.float32(np.exp(-dt / p.tau_syn))
        assert b.decay_m == np.float32(dt / p.tau_m)
        assert b.kick == np.float32(p.f_poisson * p.w_syn)


@pytest.mark.parametrize("dt", [0.6, 0.45, 0.36])
def test_persistent_short_delays_bias_and_plastic(torch, dt):
    """The persistent engine at its shortest delays (n_delay 3, 4, 5: spikes listed one step late,
    pushed n_delay-1 steps later), with biased neurons and plastic targets on the out-of-line path,
    over chained launches: bit-exact vs the oracle."""
    from flyzero_b200.brain import LIFParams

    conn = cx.synthetic(4096, seed=7)
    B = 3
    rng = np.random.default_rng(11)
    pos = np.sort(rng.choice(conn.weights.nnz, 300, replace=False))
    gb = _bb(conn.weights, LIFParams(dt=dt), B, "persistent", plastic_pos=pos, seed=6)
    assert gb.info().n_delay == int(round(1.8 / dt))
    eo = O.EngineOracle(conn.weights, O.Params(dt=dt), batch=B, plastic_pos=pos, seed=6)
    idx, rate = wl.config1_inputs(conn.n, seed=7)
    gb.set_input(idx, rate * 3)
    j = eo.slots(idx)
    eo.p_ext[:, j] = (rate * 3) * np.float32(dt / 1000.0)
    bidx = rng.choice(conn.n, 50, replace=False)
    mv = rng.uniform(0, 8, (B, 50)).astype(np.float32)
    gb.set_bias(bidx, mv)
    jb = eo.slots(bidx)              # (grows the oracle's ext arrays)
    eo.bias_ext[:, jb] = mv
    scale = rng.uniform(0.5, 2.0, (B, len(pos))).astype(np.float32)
    gb.pw *= torch.as_tensor(scale, device=gb.device)
    eo.pw[:] = gb.pw.cpu().numpy()
    total = 0
    for steps in (40, 25, 60):
        c = gb.run_steps(steps).cpu().numpy()
        np.testing.assert_array_equal(c, eo.run_steps(steps))
        total += c.sum()
    _compare_state(torch, gb, eo)
    assert total > 0


def test_persistent_long_plastic_rows(torch):
    """Every synapse onto 150 target neurons plastic (about five plastic synapses per presynaptic
    neuron: the persistent engine batches their pushes), per-instance weights, hash noise, chained
    launches with a partial reset between them: bit-exact vs the oracle."""
    from flyzero_b200.brain import LIFParams

    conn = cx.synthetic(4096, seed=13)
    w = conn.weights
    rng = np.random.default_rng(13)
    targets = rng.choice(conn.n, 150, replace=False)
    pos = np.flatnonzero(np.isin(w.indices, targets))
    rows = np.repeat(np.arange(conn.n), np.diff(w.indptr))[pos]
    assert len(pos) >= 2 * len(np.unique(rows))          # long plastic rows on average
    B = 4
    gb = _bb(w, LIFParams(), B, "persistent", plastic_pos=pos, seed=8)
    eo = O.EngineOracle(w, O.Params(), batch=B, plastic_pos=pos, seed=8)
    idx, rate = wl.config1_inputs(conn.n, seed=13)
    gb.set_input(idx, rate * 4)
    j = eo.slots(idx)
    eo.p_ext[:, j] = (rate * 4) * np.float32(0.1 / 1000.0)
    scale = rng.uniform(0.5, 2.5, (B, len(pos))).astype(np.float32)
    gb.pw *= torch.as_tensor(scale, device=gb.device)
    eo.pw[:] = gb.pw.cpu().numpy()
    total = 0
    for k, steps in enumerate((60, 45, 80)):
        if k == 2:
            gb.reset([1])
            eo.reset_flies([1])
        c = gb.run_steps(steps).cpu().numpy()
        np.testing.assert_array_equal(c, eo.run_steps(steps))
        total += c.sum()
    gb.check()
    _compare_state(torch, gb, eo)
    assert total > 0


@pytest.mark.parametrize("B,float_weights", [(3, False), (70, False), (3, True)])
def test_pull_propagation_is_exact(torch, B, float_weights):
    """Pull (gather by postsynaptic neuron over spike masks, 64 instances per mask word) gives the
    same accumulators as push: bit-exact vs the oracle across a push -> pull switch, a partial reset
    and per-instance run lengths; integer counts (INT32) and float weights (Q32.32)."""
    from flyzero_b200.brain import LIFParams

    conn = cx.synthetic(4096, seed=9)
    w = conn.weights.copy()
    if float_weights:
        w.data = w.data * np.float32(0.75)
    idx, rate = wl.high_activity_inputs(conn.n, seed=9)
    gb = _bb(w, LIFParams(), B, "step", seed=3)
    gb.set_input(idx, rate)
    eo = O.EngineOracle(w, O.Params(), batch=B, seed=3)
    j = eo.slots(idx)
    eo.p_ext[:, j] = rate * np.float32(0.1 / 1000.0)
    np.testing.assert_array_equal(gb.run_steps(30).cpu().numpy(), eo.run_steps(30))     # push
    gb.set_schedule("step", "pull")
    assert gb.info().propagation == 1
    np.testing.assert_array_equal(gb.run_steps(60).cpu().numpy(), eo.run_steps(60))     # pull after n_delay
    flies = [1] if B < 64 else [1, 65]
    gb.reset(flies)
    eo.reset_flies(flies)
    lengths = np.full(B, -1)
    lengths[0] = 25
    gb.set_run_length(lengths)
    stop = np.full(B, 2 ** 62, np.int64)
    stop[0] = eo.t + 25
    np.testing.assert_array_equal(gb.run_steps(50).cpu().numpy(), eo.run_steps(50, stop_tick=stop))
    _compare_state(torch, gb, eo)


def test_persistent_then_pull_then_persistent(torch):
    """Switching engines mid-run: spike masks restart after persistent steps (push serves the gap)."""
    from flyzero_b200.brain import LIFParams

    conn = cx.synthetic(4096, seed=12)
    idx, rate = wl.high_activity_inputs(conn.n, seed=12)
    gb = _bb(conn.weights, LIFParams(), 2, "persistent", seed=8)
    gb.set_input(idx, rate)
    eo = O.EngineOracle(conn.weights, O.Params(), batch=2, seed=8)
    j = eo.slots(idx)
    eo.p_ext[:, j] = rate * np.float32(0.1 / 1000.0)
    for engine, prop, steps in (("persistent", "push", 40), ("step", "pull", 45), ("persistent", "push", 30),
                                ("step", "pull", 10), ("step", "pull", 35)):
        gb.set_schedule(engine, prop)
        np.testing.assert_array_equal(gb.run_steps(steps).cpu().numpy(), eo.run_steps(steps))
    _compare_state(torch, gb, eo)


def test_autotune_keeps_results_exact(torch):
    """The autotuner times every schedule on the running simulation and keeps the fastest; the
    simulation it advanced is still bit-exact."""
    from flyzero_b200.brain import LIFParams

    conn = cx.synthetic(8192, seed=4)
    idx, rate = wl.config1_inputs(conn.n, seed=4)
    gb = _bb(conn.weights, LIFParams(), 4, "auto", seed=2)
    gb.set_input(idx, rate * 3)
    eo = O.EngineOracle(conn.weights, O.Params(), batch=4, seed=2)
    j = eo.slots(idx)
    eo.p_ext[:, j] = (rate * 3) * np.float32(0.1 / 1000.0)
    rep = gb.autotune(steps=20)
    assert rep["best"] in gb.schedule_candidates()
    assert len(rep["ms_per_step"]) == len(gb.schedule_candidates())
    advanced = gb.t
    eo.run_steps(advanced)
    np.testing.assert_array_equal(gb.run_steps(50).cpu().numpy(), eo.run_steps(50))
    _compare_state(torch, gb, eo)
