"""Generate the golden fixtures from the reference's own LIF kernel.

Run in a checkout where the reference project is importable (default: /root/reference):

    NUMBA_CACHE_DIR=/tmp/numba python tests/golden/make_golden.py [--reference PATH]

It imports ``flyzero.brain`` (brain.py:32-172) and records, per case, what the shipped kernel
(numba, fastmath, as brain.py:61-62 compiles it) produces, plus the same kernel recompiled
without fastmath (bit-exact target for the strict CPU oracle) and, for the 16,384-neuron case,
the kernel re-jitted on float64 arrays (the FP64 reference).

Cases follow the reference's tests (tests/test_flyzero.py:16-34, :104-114;
tests/test_gpu.py:39-62, :168-183) and the two CPU-runnable benchmark workloads. Per-step
rasters are taken by calling ``_kernel`` one step at a time with the precomputed kick raster
fed through ``p_in`` (1.0 for a kick, 0.0 otherwise: ``np.random.random() < p`` is then exactly
the raster); the generator checks that this reproduces the single-call ``Brain.run`` counts.
"""

from __future__ import annotations

import argparse
import os
import sys

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "can-the-fly-play-f-zero-_b200"))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--skip-full", action="store_true", help="skip the 138,639-neuron case")
    ap.add_argument("--learning-only", action="store_true", help="only the reward-rule vectors")
    args = ap.parse_args()
    sys.path.insert(0, args.reference)
    learning_vectors()
    if args.learning_only:
        return
    import numba
    from flyzero import brain as RB

    import oracle as O
    from flyzero_b200 import connectome as cx
    from flyzero_b200 import workloads as wl

    strict32 = numba.njit(RB._kernel.py_func)
    strict64 = numba.njit(RB._kernel.py_func)

    def kernel_args(b, counts, p_in, idx, seed=0):
        p = b.p
        return (b.n_delay, b.v, b.g, b.ref, b.pending, counts, b.indptr, b.indices, b.data, idx, p_in,
                b.kick, b.decay_syn, b.decay_m, np.float32(p.v_rest), np.float32(p.v_th), np.float32(p.v_reset),
                np.int16(b.n_ref), seed, b.bias)

    def stepwise(b, kern, steps, idx=None, kicks=None, real=np.float32):
        """Run ``steps`` one kernel call at a time; returns (counts, per-step counts, digests)."""
        idx = np.zeros(0, np.int64) if idx is None else np.asarray(idx, np.int64)
        counts = np.zeros(b.n, np.int32)
        sc = np.zeros(steps, np.int32)
        sd = np.zeros(steps, np.uint64)
        for s in range(steps):
            before = counts.copy()
            p_in = np.zeros(len(idx)) if kicks is None else kicks[s].astype(np.float64)
            a = list(kernel_args(b, counts, p_in, idx))
            if real is np.float64:
                p = b.p
                a[11:17] = [b.kick, b.decay_syn, b.decay_m, float(p.v_rest), float(p.v_th), float(p.v_reset)]
            b.t = kern(1, b.t, *a)
            fired = counts != before
            sc[s] = fired.sum()
            sd[s] = O.digest_of(fired)
        return counts, sc, sd

    def as64(b):
        """Turn a reference Brain into the float64 variant (same constants, unrounded)."""
        p = b.p
        b.v = b.v.astype(np.float64)
        b.g = b.g.astype(np.float64)
        b.pending = b.pending.astype(np.float64)
        b.bias = b.bias.astype(np.float64)
        b.data = b.data_raw.astype(np.float64) * p.w_syn
        b.decay_syn = np.exp(-p.dt / p.tau_syn)
        b.decay_m = p.dt / p.tau_m
        b.kick = p.f_poisson * p.w_syn
        return b

    out = {}

    # --- tests/test_flyzero.py:16-24: driven neuron excites its target after the delay ---------
    w = np.zeros((2, 2)); w[0, 1] = 100
    for name, m in (("driven", w), ("driven_inh", -w)):
        b = RB.Brain(sp.csr_matrix(m), backend="numba")
        b.set_input([0], 200.0)
        out[f"{name}_counts"] = b.run(200)

    # --- tests/test_flyzero.py:27-34: push equals the dense row sum ------------------------------
    w = sp.random(50, 50, density=0.2, random_state=1, format="csr") * 10
    b = RB.Brain(w)
    spk = np.array([3, 7, 20, 49])
    o = np.zeros(50, np.float32)
    b._propagate(spk, o)
    out["propagate_out"] = o

    # --- tests/test_flyzero.py:104-114 (dt 0.1) and tests/test_gpu.py:39-47 (dt 0.25) -----------
    def small(seed_w, seed_d, mean, sd, n=300, density=0.05):
        rng = np.random.default_rng(seed_d)
        w = sp.random(n, n, density=density, random_state=seed_w, format="csr")
        w.data = rng.normal(mean, sd, w.nnz)
        return w

    cases = {"backends": (small(2, 3, 20, 15), 0.1, 50.0, None),
             "gpu_nonoise": (small(2, 2, 40, 30), 0.25, 50.0, None)}
    rng = np.random.default_rng(4)
    w_long = sp.random(600, 600, density=0.6, random_state=4, format="csr")
    w_long.data = rng.normal(5.0, 3, w_long.nnz)
    cases["long_rows"] = (w_long, 0.25, 30.0, None)
    for name, (w, dt, ms, _) in cases.items():
        b = RB.Brain(w, RB.LIFParams(dt=dt), backend="numba")
        b.v[:40] = -40.0
        out[f"{name}_counts"] = b.run(ms)
        out[f"{name}_v"] = b.v.copy()
        steps = max(1, int(round(ms / dt)))
        b2 = RB.Brain(w, RB.LIFParams(dt=dt), backend="numba")
        b2.v[:40] = -40.0
        c, sc, sd = stepwise(b2, strict32, steps)
        out[f"{name}_strict_counts"], out[f"{name}_strict_v"] = c, b2.v.copy()
        out[f"{name}_step_counts"], out[f"{name}_step_digest"] = sc, sd

    # --- tests/test_gpu.py:50-62: per-fly plastic synapses (CPU side of the comparison) ---------
    w = small(2, 2, 40, 30)
    cpu = RB.Brain(w, RB.LIFParams(dt=0.25))
    pos = np.flatnonzero(cpu.indices < 30)
    changed = cpu.data.copy()
    changed[pos] = np.abs(changed[pos]) * 3
    for name, data in (("plastic_orig", None), ("plastic_changed", changed)):
        b = RB.Brain(w, RB.LIFParams(dt=0.25), backend="numba")
        if data is not None:
            b.data[:] = data
        b.v[:40] = -40.0
        out[f"{name}_counts"] = b.run(50)
    out["plastic_pos"] = pos
    out["plastic_changed_data"] = changed[pos]
    np.savez_compressed(os.path.join(HERE, "reference_tests.npz"), **out)
    print("reference_tests.npz:", {k: v.shape for k, v in out.items()})

    # --- benchmark workload 1: N=16,384, 10,000 steps, 20 @ 60 Hz + 512 @ 100 Hz ---------------
    conn = cx.synthetic(16_384, seed=1)
    idx, rate = wl.config1_inputs(conn.n, seed=1)
    steps = 10_000
    b = RB.Brain(conn.weights, RB.LIFParams(dt=0.1), seed=0, backend="numba")
    b.set_input(idx, rate)
    whole = b.run(steps * 0.1)                           # genuine single call
    seed_k = O.run_seeds(0, 1)[0]
    p_in = (b.input_rate * np.float32(0.1 / 1000.0))
    kicks = O.reference_kicks(seed_k, steps, p_in)
    c1 = {"checksum": np.array(cx.csr_checksum(conn.weights)), "input_idx": idx, "input_rate": rate,
          "seed_k": np.array(seed_k), "run_counts": whole}
    b = RB.Brain(conn.weights, RB.LIFParams(dt=0.1), seed=0, backend="numba")
    c, sc, sd = stepwise(b, RB._kernel, steps, idx, kicks)
    assert np.array_equal(c, whole), "per-step replay of the kick raster must reproduce Brain.run"
    c1.update(counts=c, step_counts=sc, step_digest=sd, v=b.v.copy())
    b = RB.Brain(conn.weights, RB.LIFParams(dt=0.1), seed=0, backend="numba")
    c, sc, sd = stepwise(b, strict32, steps, idx, kicks)
    c1.update(strict_counts=c, strict_step_digest=sd, strict_v=b.v.copy(), strict_g=b.g.copy())
    b = RB.Brain(conn.weights, RB.LIFParams(dt=0.1), seed=0, backend="numba")
    b.data_raw = np.asarray(sp.csr_matrix(conn.weights, dtype=np.float32).data, np.float32)
    b = as64(b)
    c, sc, sd = stepwise(b, strict64, steps, idx, kicks, real=np.float64)
    c1.update(f64_counts=c, f64_step_counts=sc, f64_step_digest=sd, f64_v=b.v.copy())
    np.savez_compressed(os.path.join(HERE, "workload_n16384.npz"), **c1)
    print("workload_n16384.npz: spikes", int(c1["counts"].sum()), "f64 spikes", int(c1["f64_counts"].sum()))

    if args.skip_full:
        return
    # --- benchmark workload 2: N=138,639, 10,000 steps, grating T4/T5 + DNp09 at 60 Hz ----------
    conn = cx.flywire_scale()
    drive = wl.grating_drive(conn.n, seed=0, exclude=conn.motor)
    idx = np.r_[drive.inputs, drive.tonic]
    fs = wl.frame_steps(0.1)
    frames = [fs] * (steps // fs) + ([steps % fs] if steps % fs else [])
    seeds = O.run_seeds(0, len(frames))
    drng = np.random.default_rng(2024)
    dirs = drng.uniform(0, 2 * np.pi, len(frames))
    b = RB.Brain(conn.weights, RB.LIFParams(dt=0.1), seed=0, backend="numba")
    chk = RB.Brain(conn.weights, RB.LIFParams(dt=0.1), seed=0, backend="numba")
    allc = np.zeros(conn.n, np.int32)
    scs, sds = [], []
    t_ms = 0.0
    for f, (k, sk, d) in enumerate(zip(frames, seeds, dirs)):
        rate = np.r_[wl.grating_rates(drive, t_ms, d, 1.0), np.float32(60.0)].astype(np.float32)
        b.set_input(idx, rate)
        p_in = b.input_rate * np.float32(0.1 / 1000.0)
        kicks = O.reference_kicks(sk, k, p_in)
        if f == 0:
            chk.set_input(idx, rate)
            first = chk.run(k * 0.1)
        c, sc, sd = stepwise(b, RB._kernel, k, idx, kicks)
        if f == 0:
            assert np.array_equal(c, first), "full-scale kick raster must reproduce Brain.run"
        allc += c
        scs.append(sc)
        sds.append(sd)
        t_ms += k * 0.1
    c2 = {"checksum": np.array(cx.csr_checksum(conn.weights)), "input_idx": idx, "frames": np.array(frames),
          "seeds": np.array(seeds), "dirs": dirs, "counts": allc, "step_counts": np.concatenate(scs),
          "step_digest": np.concatenate(sds), "v": b.v.copy()}
    np.savez_compressed(os.path.join(HERE, "workload_n138639.npz"), **c2)
    print("workload_n138639.npz: spikes", int(allc.sum()), "mean rate Hz", allc.sum() / conn.n / (steps * 1e-4))


def learning_vectors():
    """learning.RewardPlasticity.step (learning.py:116-131) on the reference's own toy connectome
    (connectome.py:172-265), 20 frames of seeded spike counts and N(0, 1) rewards."""
    from flyzero import connectome as rcx
    from flyzero.brain import Brain, LIFParams
    from flyzero.learning import RewardPlasticity

    conn = rcx.synthetic()
    brain = Brain(conn.weights, LIFParams(dt=0.25))
    rp = RewardPlasticity(brain, conn, seed=0)
    rng = np.random.default_rng(11)
    frames, window = 20, 1000.0 / 60.0988
    counts = rng.poisson(1.5, (frames, brain.n)).astype(np.int32)
    reward = rng.standard_normal(frames)
    out = {"indptr": brain.indptr, "indices": brain.indices, "data0": brain.data.copy(), "targets": rp.targets,
           "pos": rp.pos, "pre": rp.pre, "post": rp.post, "w0": rp.w0, "sign": rp.sign, "wmax": rp.wmax,
           "counts": counts, "reward": reward, "window": np.array(window)}
    ws, el, pm, rm, adv = [], [], [], [], []
    for f in range(frames):
        adv.append(rp.step(counts[f], float(reward[f]), window))
        ws.append(brain.data[rp.pos].copy())
        el.append(np.asarray(rp.elig).copy())
        pm.append(rp.post_mean[rp.targets].copy())
        rm.append(rp.r_mean)
    out.update(w=np.array(ws), elig=np.array(el), post_mean=np.array(pm), r_mean=np.array(rm), adv=np.array(adv))
    np.savez_compressed(os.path.join(HERE, "learning.npz"), **out)
    print("learning.npz: elig dtype", out["elig"].dtype, "plastic", len(rp.pos))


if __name__ == "__main__":
    main()
