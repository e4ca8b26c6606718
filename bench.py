#!/usr/bin/env python
"""Benchmark: simulated neuron-steps/s of the batched LIF engine on one B200 per rank.

Workload (the batched configuration): 64 instances share the seeded 138,639-neuron synthetic
connectome (15.1M connections, 54.0M synapses); each has its own seed, grating direction per frame,
contrast U[0.2, 1], tonic DNp09 drive U[20, 100] Hz, run length U{0.5, 1, 2, 3} s and its own
plastic weights on the 7,300 inputs of 8 motor neurons. One bench step = one 166-step frame
(16.64 ms at dt = 0.1 ms) for every instance, i.e. BatchBrain.run(16.64) after the frame's rates
are written (flyzero/fleet.py:74-81). Inputs (per-frame rates) are resident in HBM before the
timed region; the working set (state 80 MB + accumulators 71 MB + CSR 94 MB) exceeds the 126 MB L2.

Also reported in the same line: the roofline of the dominant kernel, the plain single-instance
engine (B=1, two launches per step), the end-to-end path through the public API with host buffers,
and the CPU oracle port timed on this host. ``--impl reference`` times the CPU port of the
reference kernel (flyzero/brain.py:32-58) on all host cores, one instance per thread.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "can-the-fly-play-f-zero-_b200"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "sim neuron-steps/s (138k LIF, B=64 batched vs B=1 plain) at matched rates"
UNIT = "neuron-steps/s"
DT = 0.1
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
BYTES_PER_NEURON_STEP = 26        # v r/w 8 + g r/w 8 + ref r/w 2 + accumulator read+clear 8
BYTES_PER_SPIKE = 16              # row pointers 8 + count r/w 8
BYTES_PER_EDGE = 14               # column 4 + count 2 + accumulator read-modify-write 8


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60, help="timed frames (166 LIF steps each)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip plain/e2e legs (profiling runs)")
    ap.add_argument("--engine", default="auto", choices=["auto", "step", "persistent"])
    ap.add_argument("--lanes", type=int, default=0, help="lanes per spike work item (8/16/32; 0 = default)")
    ap.add_argument("--component", default="brain", choices=["brain", "eye", "fleet", "tune", "trace", "instruct"],
                    help="brain: the LIF engine (default); eye: the motion eye front end alone; fleet: the "
                         "whole frame loop (frames -> eye -> brain -> readout) through the public API; "
                         "tune: the surrogate-screened interface search at full scale (three searches); "
                         "trace: the persistent engine's phase trace on the headline workload (a diagnostic); "
                         "instruct: the frame loop with the deep instructed learning rule every frame")
    return ap.parse_args()


def peaks():
    try:
        d = json.load(open(PEAKS))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "50", "-i", str(self.index)], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        rows = [r.split(", ") for r in open(self.file.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[k] for r in rows if len(r) >= 9 for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def _reduce(x: float, world: int, op: str, device: str) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    """The slowest rank's time (replicas report the job's wall time as the max over ranks)."""
    return _reduce(x, world, "max", device)


def sum_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    return _reduce(x, world, "sum", device)


def replica_value(neuron_steps: float, elapsed_ms: float, world: int, device: str = "cuda") -> tuple:
    """Whole-job throughput of independent replicas: all ranks' neuron-steps over the slowest
    rank's device time. Returns (value, max_ms)."""
    total = sum_over_ranks(float(neuron_steps), world, device)
    max_ms = max_over_ranks(float(elapsed_ms), world, device)
    return total / (max_ms / 1000.0), max_ms


def workload(batch: int, seed: int):
    from flyzero_b200 import connectome as cx
    from flyzero_b200 import workloads as wl

    conn = cx.flywire_scale()
    drive = wl.grating_drive(conn.n, seed=0, exclude=conn.motor)
    pos = np.flatnonzero(np.isin(conn.weights.indices, conn.motor))
    work = wl.BatchedWorkload.make(batch, seed=seed)
    return conn, drive, pos, work


def cpu_model() -> str:
    """The host CPU's model name and logical CPU count, for the CPU timings' records."""
    name = "unknown CPU"
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    name = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return f"{name}, {os.cpu_count()} logical CPUs, {len(os.sched_getaffinity(0))} usable"


def cpu_baseline(conn, drive, seconds: float) -> dict:
    """The oracle's restatement of the reference kernel, one thread, on a bounded sample of the
    same workload (one instance, grating input, frames of 166 steps until ~`seconds` elapse)."""
    import oracle as O
    from flyzero_b200 import workloads as wl

    b = O.RefBrain(conn.weights)
    idx = np.r_[drive.inputs, drive.tonic]
    rng = np.random.default_rng(1)
    steps = done = 0
    busy = 0.0
    t_ms = 0.0
    while busy < seconds:
        rate = np.r_[wl.grating_rates(drive, t_ms, rng.uniform(0, 2 * np.pi)), np.float32(60.0)].astype(np.float32)
        kicks = O.reference_kicks(int(rng.integers(2 ** 31)), 166, rate * np.float32(DT / 1000.0))
        t0 = time.perf_counter()
        b.run_steps(166, idx, kicks)
        busy += time.perf_counter() - t0
        steps += 166
        done += 1
        t_ms += 166 * DT
    return {"value": steps * conn.n / busy, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"1 instance x {steps} steps ({done} frames) of the 138,639-neuron grating workload, "
                      f"{busy:.1f} s, C port of flyzero/brain.py:32-58 (gcc -O3, AVX2)", "cpu": cpu_model()}


def run_reference(args, world, rank):
    """CPU port of the reference kernel on all host cores: independent instances, one per thread
    (the reference's one-fly-per-process model, flyzero/train.py:117-126)."""
    import oracle as O
    from flyzero_b200 import connectome as cx
    from flyzero_b200 import workloads as wl

    if rank != 0:
        return
    conn = cx.flywire_scale()
    drive = wl.grating_drive(conn.n, seed=0, exclude=conn.motor)
    idx = np.r_[drive.inputs, drive.tonic]
    threads = len(os.sched_getaffinity(0))
    b = O.RefBrain(conn.weights)
    steps = 166
    rate = np.r_[wl.grating_rates(drive, 0.0, 0.7), np.float32(60.0)].astype(np.float32)
    kicks = O.reference_kicks(12345, steps, rate * np.float32(DT / 1000.0))
    times = []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        O.ref_pool(threads, threads, b, steps, idx, kicks)
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            times.append(dt)
    total = sum(times)
    value = args.steps * threads * steps * conn.n / total
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": {"workload": "one 166-step frame of the 138,639-neuron grating workload per "
                                                    "host thread, independent instances", "threads": threads},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{threads} instances x {steps} steps per bench step", "cpu": cpu_model()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    gpu = reference_gpu(conn, drive, idx)
    if gpu is not None:
        line["reference_gpu"] = gpu
    print(json.dumps(line), flush=True)


def reference_gpu(conn, drive, idx, frames: int = 3):
    """The reference's own CUDA kernels (flyzero/gpu.py:26-119, built into oracle/_ref by
    oracle/make_ref_gpu.py) with its host loop (two launches per step, gpu.py:228-254) on this
    device, at B=1 and B=64 on the same grating workload: the reference's GPU method, for comparison."""
    try:
        import torch
    except ImportError:
        return None
    import ref_gpu
    from flyzero_b200 import workloads as wl
    from flyzero_b200.brain import LIFParams

    if not (ref_gpu.available() and torch.cuda.is_available()):
        return None
    fs = wl.frame_steps(DT)
    out = {"kernels": "flyzero/gpu.py update + propagate, nvcc --use_fast_math, sm_100a, launched from Python"}
    for B in (1, 64):
        rb = ref_gpu.RefGpuBrain(conn.weights, LIFParams(dt=DT), batch=B, seed=5)
        rate = np.r_[wl.grating_rates(drive, 0.0, 0.7), np.float32(60.0)].astype(np.float32)
        rb.set_input(idx, np.broadcast_to(rate, (B, len(idx))))
        rb.run_steps(fs)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        spikes = 0
        for _ in range(frames):
            c = rb.run_steps(fs)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        spikes = int(c.sum())
        out[f"b{B}"] = {"value": B * fs * frames * conn.n / (ms / 1000.0), "unit": UNIT, "ms_per_frame": ms / frames,
                        "spikes_last_frame": spikes}
        del rb
        torch.cuda.empty_cache()
    return out


def spike_bytes(counts_list, rowlen_dev):
    """Algorithmic bytes of the spikes in the given count tensors: sum over spikes of 16 + 14 * deg."""
    import torch

    tot_spk = 0
    tot_edges = 0
    for c in counts_list:
        s = c.sum(0).to(torch.int64)
        tot_spk += int(s.sum())
        tot_edges += int((s * rowlen_dev).sum())
    return tot_spk, tot_edges


def dram_traffic_record():
    """DRAM bytes (read + write) of one persistent-kernel launch of this workload, read from the
    committed ncu summary of that kernel (its 'traffic per launch' line names the commit and the
    command it was measured at); None if the record is missing."""
    import re

    path = os.path.join(ROOT, "profiles", "k_persist_b64_138k.md")
    try:
        text = open(path).read()
    except OSError:
        return None, None
    m = re.search(r"traffic-per-launch-bytes:\s*([0-9_]+)\s+\(commit ([0-9a-f]+)", text)
    if not m:
        return None, None
    return int(m.group(1).replace("_", "")), f"profiles/k_persist_b64_138k.md, commit {m.group(2)}"


class Episodes:
    """Per-instance runs of the batched workload. Instance b runs for a length drawn from
    U{0.5, 1, 2, 3} s (5,000 - 30,000 steps), then it is reset (state, synaptic input in flight,
    eligibility traces) and starts a new run of a fresh length, as the reference's fleet restarts a
    fly's race. When the loop starts every instance is at a seeded random point of its first run,
    so runs end inside any window of frames: an instance whose run ends inside a frame is frozen
    by the engine for the rest of that frame (its run length) and restarted at the next frame."""

    LENGTHS = np.array([5000, 10000, 20000, 30000], np.int64)

    def __init__(self, work, seed: int, t0: int = 0):
        self.rng = np.random.default_rng(seed)
        first = (work.run_ms / DT).astype(np.int64)
        self.stop = t0 + first - self.rng.integers(0, first)

    def frame(self, t: int):
        """Instances whose run ended by tick t (to reset now); draws their next run lengths."""
        ended = np.flatnonzero(self.stop <= t)
        self.stop[ended] = t + self.rng.choice(self.LENGTHS, len(ended))
        return ended

    def active(self, t: int, fs: int) -> np.ndarray:
        """Steps each instance advances in the frame starting at tick t."""
        return np.clip(self.stop - t, 0, fs)


class FrameLoop:
    """One bench step of the batched workload, the reference's frame (flyzero/fleet.py:74-81 with
    the reward rule of flyzero/batch.py:482-495 / school.py:289-304): restart the instances whose
    run ended, write the frame's rates into p_ext, run 166 steps, then the reward-modulated update
    of every instance's plastic deltas with reward ~ N(0, 1), for the instances that ran."""

    def __init__(self, gb, conn, work, rank: int, frames: int, t0: int = 0):
        from flyzero_b200.batch import BatchReward

        self.gb = gb
        self.br = BatchReward(gb, targets=conn.motor, seed=rank)
        self.rewards = np.random.default_rng(11 + rank).standard_normal((frames, gb.B))
        self.ep = Episodes(work, seed=23 + rank, t0=t0)
        self.fs = 166
        self.t = t0
        self.resets = 0
        self.reset_instances = 0
        self.public = False           # True: BatchBrain.run(ms), the reference's call
        self.run_launches = 0         # the engine's launches inside the runs alone
        gb.set_stop_tick(self.ep.stop)

    def __call__(self, f: int, write_rates, counts=None, events=None):
        """One frame; ``events`` (start, end) CUDA events are recorded around the engine's run."""
        gb = self.gb
        ended = self.ep.frame(self.t)
        if len(ended):
            gb.reset(ended)
            self.br.reset(ended)
            gb.set_stop_tick(self.ep.stop)
            self.resets += 1
            self.reset_instances += len(ended)
        act = self.ep.active(self.t, self.fs)
        write_rates(f)
        if events:
            events[0].record()
        l0 = gb.launches
        c = gb.run(self.fs * DT) if self.public else gb.run_steps(self.fs, counts=counts)
        self.run_launches += gb.launches - l0
        if events:
            events[1].record()
        self.br.step(c, self.rewards[f], act > 0, self.fs * DT)
        self.t += self.fs
        return c, int(act.sum())


def run_ours(args, world, rank, local):
    import torch

    from flyzero_b200 import workloads as wl
    from flyzero_b200.brain import LIFParams
    from flyzero_b200.gpu import BatchBrain

    dev = torch.device("cuda", local)
    conn, drive, pos, work = workload(args.batch, seed=rank)
    B, n = args.batch, conn.n
    fs = wl.frame_steps(DT)
    assert fs == 166
    frames = args.warmup + args.steps
    gb = BatchBrain(conn.weights, LIFParams(dt=DT), batch=B, seed=1000 + rank, plastic_pos=pos)
    gb.set_schedule(args.engine, lanes=args.lanes)
    idx_in = np.r_[drive.inputs, drive.tonic]
    j = gb.slots(idx_in).cpu().numpy()
    assert np.array_equal(np.sort(j), np.arange(len(idx_in))), "inputs own the first ext slots"
    inv = np.empty_like(j)
    inv[j] = np.arange(len(j))
    # every frame's rates, resident on the device, already in ext-slot order and scaled to p
    t_ms = 0.0
    host_rates = np.empty((frames, B, len(idx_in)), np.float32)
    for f in range(frames):
        host_rates[f] = work.rates(drive, t_ms, work.directions())[:, inv]
        t_ms += fs * DT
    scale = np.float32(DT / 1000.0)
    p_dev = torch.as_tensor(host_rates, device=dev) * torch.tensor(scale, device=dev)
    counts = [torch.empty((B, n), dtype=torch.int32, device=dev) for _ in range(frames)]
    rowlen = torch.as_tensor(np.diff(conn.weights.indptr), device=dev)
    n_in = len(idx_in)
    st = torch.cuda.current_stream(dev)
    loop = FrameLoop(gb, conn, work, rank, frames)

    def rates(f):
        gb.p_ext[:, :n_in].copy_(p_dev[f])

    for f in range(args.warmup):
        loop(f, rates, counts[f])
    gb.check()
    torch.cuda.synchronize(dev)
    barrier(world)
    torch.cuda.synchronize(dev)
    launches0 = gb.launches
    resets0, reset_inst0 = loop.resets, loop.reset_instances
    clocks = Clocks(local)
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    e_all0, e_all1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    active = 0
    l_run0 = loop.run_launches
    e_all0.record(st)
    for k in range(args.steps):
        f = args.warmup + k
        _, a = loop(f, rates, counts[f], events=ev[k])     # events around the run's launches
        active += a
    e_all1.record(st)
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    barrier(world)
    gb.check()
    elapsed_ms = e_all0.elapsed_time(e_all1)
    run_ms = sum(a.elapsed_time(b) for a, b in ev)     # the engine's runs alone (persistent launches)
    # per frame: the engine's launches (runs, resets, reward steps) + one p_ext copy kernel
    launches = gb.launches - launches0 + args.steps
    neuron_steps = active * n
    value, max_ms = replica_value(neuron_steps, elapsed_ms, world)
    spk, edges = spike_bytes(counts[args.warmup:], rowlen)
    alg_bytes = BYTES_PER_NEURON_STEP * neuron_steps + BYTES_PER_SPIKE * spk + BYTES_PER_EDGE * edges
    info = gb.info()
    peak, peak_kind = peaks()
    n_kern = max(1, loop.run_launches - l_run0)   # the runs' launches: one per instance group per frame
    achieved = (alg_bytes / n_kern) / (run_ms / 1000.0 / n_kern) / 1e9
    traffic, traffic_src = dram_traffic_record()
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+i32", "data": "synthetic",
        "config": {"workload": "batched: 64 instances x 138,639-neuron synthetic connectome, 1 frame = 166 steps "
                               "at dt 0.1 ms per bench step, grating + tonic Poisson input, 7,300 plastic synapses "
                               "onto 8 motor neurons updated every frame by the reward rule (reward ~ N(0,1))",
                   "neurons": n, "connections": int(conn.nnz), "synapses": conn.synapses(), "batch": B,
                   "steps_per_frame": fs, "active_instance_steps": active, "parallelism": f"replicas x{world}",
                   "engine": "persistent" if info.group else "step", "group": int(info.group),
                   "in_timed_loop": "per frame: restart of ended runs (fb_reset of those instances + stop ticks), "
                                    "p_ext write, run(166 steps) with per-instance run-length masking, "
                                    "BatchReward.step on the frame's counts",
                   "run_lengths": "U{0.5,1,2,3} s per run, each instance starting at a seeded random point of its "
                                  "first run; ended runs are reset and restarted at the next frame",
                   "runs_restarted_in_timed_loop": loop.reset_instances - reset_inst0,
                   "frames_with_restarts": loop.resets - resets0,
                   "l2": "no flush: working set (state 80 MB + accumulators 71 MB + CSR 94 MB) exceeds the 126 MB L2",
                   "spikes": spk, "mean_rate_hz": spk / max(1, active) / (DT / 1000.0) / n * 1.0},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": traffic if info.group else None, "peak_kind": peak_kind,
                     "traffic_source": traffic_src,
                     "kernel_ms_per_launch": run_ms / n_kern, "kernel_launches": n_kern,
                     "kernel_timing": "CUDA events on the launching stream around each frame's run (its "
                                      "persistent launches) inside the timed loop",
                     "model": "26 B per instance-neuron-step + 16 B per spike + 14 B per edge pushed, per launch of the "
                              "persistent kernel (one per instance group per frame)"},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if not args.no_extras:
        out["plain_b1"] = plain_b1(conn, drive, dev)
        out["persistent_b1"] = persistent_b1(conn, drive, dev)
        out["e2e"] = e2e(conn, work, drive, host_rates, args, fs, n_in, inv, dev, rank, pos)
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(conn, drive, args.cpu_seconds)
    if rank == 0:
        print(json.dumps(out), flush=True)


def persistent_b1(conn, drive, dev, frames: int = 6):
    """One instance on the persistent engine (the drop-in for the game loop's Brain.run,
    flyzero/brain.py:133-172): B=1, one cooperative launch per 166-step frame."""
    import torch

    from flyzero_b200 import workloads as wl
    from flyzero_b200.brain import LIFParams
    from flyzero_b200.gpu import BatchBrain

    gb = BatchBrain(conn.weights, LIFParams(dt=DT), batch=1, seed=5)
    if gb.info().group == 0:
        return None
    gb.set_schedule("persistent")
    gb.set_input(np.r_[drive.inputs, drive.tonic], np.r_[wl.grating_rates(drive, 0.0, 0.4), 60.0])
    fs = wl.frame_steps(DT)
    for _ in range(2):
        gb.run_steps(fs)
    torch.cuda.synchronize(dev)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st = torch.cuda.current_stream(dev)
    a.record(st)
    for _ in range(frames):
        c = gb.run_steps(fs)
    b.record(st)
    torch.cuda.synchronize(dev)
    ms = a.elapsed_time(b)
    return {"value": frames * fs * conn.n / (ms / 1000.0), "unit": UNIT, "engine": "persistent, B=1, 1 launch/frame",
            "ms_per_frame": ms / frames, "spikes_last_frame": int(c.sum())}


def plain_b1(conn, drive, dev, frames: int = 6):
    """The plain single-instance engine: B=1, two launches per step, no persistence, no graph."""
    import torch

    from flyzero_b200 import workloads as wl
    from flyzero_b200.brain import LIFParams
    from flyzero_b200.gpu import BatchBrain

    gb = BatchBrain(conn.weights, LIFParams(dt=DT), batch=1, seed=5)
    gb.set_schedule("step")
    gb.set_input(np.r_[drive.inputs, drive.tonic], np.r_[wl.grating_rates(drive, 0.0, 0.4), 60.0])
    fs = wl.frame_steps(DT)
    for _ in range(2):
        gb.run_steps(fs)
    torch.cuda.synchronize(dev)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st = torch.cuda.current_stream(dev)
    a.record(st)
    for _ in range(frames):
        c = gb.run_steps(fs)
    b.record(st)
    torch.cuda.synchronize(dev)
    ms = a.elapsed_time(b)
    return {"value": frames * fs * conn.n / (ms / 1000.0), "unit": UNIT, "engine": "step, B=1, 2 launches/step",
            "ms_per_frame": ms / frames, "spikes_last_frame": int(c.sum())}


def e2e(conn, work, drive, host_rates, args, fs, n_in, inv, dev, rank, pos):
    """End to end through the public API with host buffers, on a fresh engine: per frame, the
    restart of ended runs (BatchBrain.reset of those instances + stop ticks), H2D of the frame's
    rates from pinned memory and the p_ext write (Fleet.think, flyzero/fleet.py:76-77),
    BatchBrain.run(16.64 ms), BatchReward.step with the frame's rewards (batch.py:482-495) and a
    D2H read of the readout DNs' counts (BatchMotor.update reads DN counts, flyzero/batch.py:109)."""
    import torch

    from flyzero_b200.brain import LIFParams
    from flyzero_b200.gpu import BatchBrain

    B = args.batch
    gb = BatchBrain(conn.weights, LIFParams(dt=DT), batch=B, seed=2000 + rank, plastic_pos=pos)
    gb.set_schedule(args.engine, lanes=args.lanes)
    gb.slots(np.r_[drive.inputs, drive.tonic])
    frames = args.warmup + args.steps
    pinned = torch.as_tensor(host_rates).pin_memory()
    readout = torch.as_tensor(drive.readout, device=dev)
    out_h = torch.empty((args.steps, B, len(drive.readout)), dtype=torch.int32).pin_memory()
    stage = torch.empty((B, n_in), dtype=torch.float32, device=dev)
    scale = torch.tensor(np.float32(DT / 1000.0), device=dev)
    st = torch.cuda.current_stream(dev)
    loop = FrameLoop(gb, conn, work, rank, frames)
    loop.public = True

    def rates(f):
        stage.copy_(pinned[f], non_blocking=True)
        torch.mul(stage, scale, out=gb.p_ext[:, :n_in])

    for f in range(args.warmup):              # the same calls as a timed frame, readout included
        c, _ = loop(f, rates)
        out_h[0].copy_(c.index_select(1, readout), non_blocking=True)
    torch.cuda.synchronize(dev)
    r0 = loop.resets
    active = 0
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for k in range(args.steps):
        c, act = loop(args.warmup + k, rates)
        out_h[k].copy_(c.index_select(1, readout), non_blocking=True)
        active += act
    b.record(st)
    torch.cuda.synchronize(dev)
    gb.check()
    ms = a.elapsed_time(b)
    restarts = loop.resets - r0
    # rates + reward coefficients (f64) and fly weights (f32) every frame; stop ticks (i64) and the
    # reset list (one byte per instance) on frames that restart runs
    h2d = B * n_in * 4 + B * (8 + 4) + (B * (8 + 1) * restarts) // max(1, args.steps)
    return {"value": active * gb.n / (ms / 1000.0), "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": B * len(drive.readout) * 4, "ms_per_step": ms / args.steps,
            "frames_with_restarts": restarts}


EYE_METRIC = "motion-eye instance-frames/s (224x256 frames, training channels, B=64)"
EYE_SHAPE = (224, 256)


def eye_params():
    from flyzero_b200.vision import MotionParams

    return MotionParams(gain=10 ** 2.7, y_min=0.2, transient_gain=4.0, sustained_gain=4.0, chromatic_gain=1.0)


def eye_oracle(lo, p):
    from eye_oracle import EyeOracle

    return EyeOracle(EYE_SHAPE, lo.gx, lo.gy, lo.chan, lo.visible, max_rate=p.max_rate, gain=p.gain, cell=p.cell,
                     tau_hp=p.tau_hp, tau_delay=p.tau_delay, shift=p.shift, transient_gain=p.transient_gain,
                     sustained_gain=p.sustained_gain, surround=p.surround, chromatic_gain=p.chromatic_gain)


def eye_cpu_baseline(lo, frames, p, seconds: float) -> dict:
    """The oracle's restatement of MotionEye.see (flyzero/vision.py:136-191), NumPy, one thread,
    one instance, on the same frames until ~`seconds` elapse."""
    o = eye_oracle(lo, p)
    done, busy = 0, 0.0
    while busy < seconds:
        fr = frames[done % len(frames), 0]
        t0 = time.perf_counter()
        o.see(fr)
        busy += time.perf_counter() - t0
        done += 1
    return {"value": done / busy, "unit": "instance-frames/s", "cores": 1, "kind": "port",
            "sample": f"1 instance x {done} frames of 224x256, {busy:.1f} s, NumPy restatement of "
                      f"flyzero/vision.py:136-191 (the reference's own operations)"}


_EYE_CACHE: dict = {}


def _eye_worker(job):
    """One host process of the eye's reference arm: its own instance over its own frames; returns
    (frames, seconds spent in see)."""
    seed, n_frames = job
    from flyzero_b200 import workloads as wl

    if "layout" not in _EYE_CACHE:
        from flyzero_b200 import connectome as cx

        conn = cx.flywire_scale()
        _EYE_CACHE["layout"] = wl.eye_layout(wl.grating_drive(conn.n, seed=0, exclude=conn.motor), EYE_SHAPE, 4, 0.2)
    o = eye_oracle(_EYE_CACHE["layout"], eye_params())
    frames = wl.game_frames(1, n_frames, EYE_SHAPE, seed=seed)
    t0 = time.perf_counter()
    for f in frames:
        o.see(f[0])
    return n_frames, time.perf_counter() - t0


def run_eye_reference(args, world, rank):
    """The eye's CPU path (flyzero/vision.py:136-191 restated in NumPy) on all host cores: one
    instance per process, as the reference's pool runs one eye per worker (flyzero/pool.py:44)."""
    import multiprocessing as mp

    if rank != 0:
        return
    procs = len(os.sched_getaffinity(0))
    per = 12
    with mp.get_context("spawn").Pool(procs) as pool:
        pool.map(_eye_worker, [(k, 1) for k in range(procs)], chunksize=1)     # build each worker's layout
        times = []
        for s in range(args.warmup + args.steps):
            busy = pool.map(_eye_worker, [(1000 * s + k, per) for k in range(procs)], chunksize=1)
            if s >= args.warmup:
                times.append(max(t for _, t in busy))         # the processes run side by side
    total = sum(times)
    value = args.steps * procs * per / total
    print(json.dumps({
        "metric": EYE_METRIC, "value": value, "unit": "instance-frames/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8->f32", "data": "synthetic",
        "config": {"workload": f"{per} 224x256 frames per host process per bench step, training parameters",
                   "processes": procs},
        "cpu_baseline": {"value": value, "unit": "instance-frames/s", "cores": procs, "kind": "port",
                         "sample": f"{procs} instances x {per} frames per bench step; per step the slowest "
                                   "process's time over its frames (frame generation and setup untimed)"},
        "e2e": {"value": value, "unit": "instance-frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
        flush=True)


def run_eye(args, world, rank, local):
    """The motion eye alone: per bench step one frame for every instance -> fb_motion_eye -> p_ext."""
    import torch

    from flyzero_b200 import connectome as cx
    from flyzero_b200 import workloads as wl
    from flyzero_b200.brain import LIFParams
    from flyzero_b200.gpu import BatchBrain
    from flyzero_b200.vision import BatchMotionEye

    dev = torch.device("cuda", local)
    conn = cx.flywire_scale()
    drive = wl.grating_drive(conn.n, seed=0, exclude=conn.motor)
    B, shape, p = args.batch, EYE_SHAPE, eye_params()
    lo = wl.eye_layout(drive, shape, p.cell, p.y_min)
    frames = args.warmup + args.steps
    host = wl.game_frames(B, frames, shape, seed=rank)
    gb = BatchBrain(conn.weights, LIFParams(dt=DT), batch=B, seed=1000 + rank)
    eye = BatchMotionEye(gb, None, shape, p, eye_layout=lo)
    fr_dev = torch.as_tensor(host, device=dev)
    st = torch.cuda.current_stream(dev)
    for f in range(args.warmup):
        eye.see(fr_dev[f])
    torch.cuda.synchronize(dev)
    barrier(world)
    torch.cuda.synchronize(dev)
    clocks = Clocks(local)
    clocks.start()
    l0 = gb.launches
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for k in range(args.steps):
        eye.see(fr_dev[args.warmup + k])
    b.record(st)
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    barrier(world)
    ms = a.elapsed_time(b)
    launches = gb.launches - l0
    value, max_ms = replica_value(B * args.steps, ms, world)
    cells = (shape[0] // p.cell) * (shape[1] // p.cell)
    n_cells = len(lo.idx)
    # frame read + high-pass state r/w + two delay arms r/w + one p_ext write per eye neuron
    alg = B * (shape[0] * shape[1] * 3 + cells * (8 + 16) + n_cells * 4)
    peak, peak_kind = peaks()
    achieved = alg / (ms / 1000.0 / args.steps) / 1e9
    # end to end: frames from pinned host memory every step, then the eye; the rates stay on the device
    pinned = torch.as_tensor(host).pin_memory()
    stage = torch.empty_like(fr_dev[0])
    eye.reset()
    for f in range(args.warmup):
        stage.copy_(pinned[f], non_blocking=True)
        eye.see(stage)
    torch.cuda.synchronize(dev)
    a.record(st)
    for k in range(args.steps):
        stage.copy_(pinned[args.warmup + k], non_blocking=True)
        eye.see(stage)
    b.record(st)
    torch.cuda.synchronize(dev)
    e2e_ms = a.elapsed_time(b)
    out = {
        "metric": EYE_METRIC, "value": value, "unit": "instance-frames/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8->f32", "data": "synthetic",
        "config": {"workload": f"motion eye: {B} instances x one 224x256 RGB frame per step, cell 4 (56x64 grid), "
                               f"{n_cells} eye neurons on 14 channels (8 motion, 6 columnar), training parameters "
                               "(gain 10^2.7, y_min 0.2, transient 4, sustained 4, chromatic 1)",
                   "batch": B, "eye_neurons": n_cells, "parallelism": f"replicas x{world}",
                   "l2": "no flush: frames of all steps (%d MB) exceed the 126 MB L2" % (host.nbytes // 2 ** 20)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": peak_kind,
                     "model": "per instance: frame 224*256*3 B + 24 B per grid cell (high-pass and delay state "
                              "read and written) + 4 B per eye neuron (p_ext), per call"},
        "gpu_launches": launches,
        "clocks": clk,
        "e2e": {"value": B * args.steps / (e2e_ms / 1000.0), "unit": "instance-frames/s",
                "h2d_bytes_per_step": int(stage.numel()), "d2h_bytes_per_step": 0,
                "note": "frames copied from pinned host memory each step; the rates stay on the device in p_ext"},
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = eye_cpu_baseline(lo, host, p, min(args.cpu_seconds, 5.0))
    if rank == 0:
        print(json.dumps(out), flush=True)


FLEET_METRIC = "fleet frame loop: sim neuron-steps/s with the eye and the readout on the device (138k LIF, B=64)"


def run_fleet(args, world, rank, local):
    """The frame loop of flyzero/fleet.py:74-81 and batch.py:107-111 through the public API, every
    frame: the instances' game frames from pinned host memory, the motion eye into p_ext
    (BatchMotionEye.see), one frame of brain time (BatchBrain.run), the readout DNs' smoothed rates
    (BatchMotor.update: device gather + EMA, the (B, 9) rates read back, the buttons on the host)."""
    import torch

    from flyzero_b200 import connectome as cx
    from flyzero_b200 import workloads as wl
    from flyzero_b200.brain import LIFParams
    from flyzero_b200.gpu import BatchBrain
    from flyzero_b200.motor import READOUT, BatchMotor
    from flyzero_b200.vision import BatchMotionEye

    dev = torch.device("cuda", local)
    conn = cx.flywire_scale()
    drive = wl.grating_drive(conn.n, seed=0, exclude=conn.motor)
    pos = np.flatnonzero(np.isin(conn.weights.indices, conn.motor))
    B, shape, p = args.batch, EYE_SHAPE, eye_params()
    fs = wl.frame_steps(DT)
    frames = args.warmup + args.steps
    host = wl.game_frames(B, frames, shape, seed=rank)
    gb = BatchBrain(conn.weights, LIFParams(dt=DT), batch=B, seed=1000 + rank, plastic_pos=pos)
    gb.set_input(drive.tonic, 60.0)                       # the tonic DNp09 drive; the eye writes its own slots
    eye = BatchMotionEye(gb, None, shape, p, eye_layout=wl.eye_layout(drive, shape, p.cell, p.y_min))
    motor = BatchMotor(gb, {name: drive.readout[k:k + 1] for k, name in enumerate(READOUT)})
    pinned = torch.as_tensor(host).pin_memory()
    stage = torch.empty(host.shape[1:], dtype=torch.uint8, device=dev)
    window = fs * DT
    st = torch.cuda.current_stream(dev)

    def frame(f):
        stage.copy_(pinned[f], non_blocking=True)
        eye.see(stage)
        counts = gb.run(window)
        return motor.update(counts, window)

    for f in range(args.warmup):
        frame(f)
    gb.check()
    torch.cuda.synchronize(dev)
    barrier(world)
    torch.cuda.synchronize(dev)
    clocks = Clocks(local)
    clocks.start()
    l0 = gb.launches
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    pressed = 0
    for k in range(args.steps):
        buttons = frame(args.warmup + k)
        pressed += sum(v for bt in buttons for v in bt.values())
    b.record(st)
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    barrier(world)
    gb.check()
    ms = a.elapsed_time(b)
    value, max_ms = replica_value(B * args.steps * fs * conn.n, ms, world)
    out = {
        "metric": FLEET_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+i32", "data": "synthetic",
        "config": {"workload": f"fleet frame loop: {B} instances x 138,639-neuron synthetic connectome, per bench step "
                               "one 224x256 game frame per instance -> motion eye (training channels, 12,246 eye "
                               f"neurons) -> {fs} LIF steps at dt 0.1 ms -> readout of 9 DN groups -> buttons",
                   "batch": B, "steps_per_frame": fs, "parallelism": f"replicas x{world}",
                   "frames_per_s": B * args.steps / (max_ms / 1000.0), "buttons_pressed": int(pressed),
                   "l2": "no flush: the brain's working set (state 80 MB + accumulators 71 MB + CSR 94 MB) "
                         "exceeds the 126 MB L2"},
        "gpu_launches": gb.launches - l0,
        "clocks": clk,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": int(stage.numel()),
                "d2h_bytes_per_step": B * len(READOUT) * 4,
                "note": "the whole loop is end to end: frames from pinned host memory in, readout rates out"},
    }
    if rank == 0:
        print(json.dumps(out), flush=True)


TUNE_METRIC = ("surrogate DN-count error on the simulated survivors, last CMA-ES generation, median of three "
               "searches (138k LIF, 1,024 screened / 64 simulated)")
TUNE_SEEDS = (0, 1, 2)


def run_tune(args, world, rank, local):
    """The learned surrogate at full scale (config 5), three independent searches (seeds 0-2, each
    on rank * 3 + seed): 200,000 frames from the B=64 engine, the BF16 MLP trained on the device,
    then CMA-ES over the 12-parameter interface with 1,024 candidates screened and 64 re-simulated
    per generation, beside CMA-ES simulating its 64 directly. `value` is the median over the searches
    of the last generation's error; every search's per-generation errors are in the line. The whole
    search is the unit; --steps and --warmup are not used."""
    import torch

    from flyzero_b200 import tuning as T

    torch.cuda.set_device(local)
    t0 = time.perf_counter()
    runs = [T.run(n=138_639, frames=200_000, epochs=12, generations=8, episode=30, seed=rank * len(TUNE_SEEDS) + s)
            for s in TUNE_SEEDS]
    secs = (time.perf_counter() - t0) / len(runs)
    if rank == 0:
        last = [r["surrogate_search"]["log"][-1] for r in runs]
        print(json.dumps({
            "metric": TUNE_METRIC, "value": float(statistics.median([g["count_error"] for g in last])), "unit": "relative",
            "n_gpus": world, "steps": 1, "warmup": 0, "ms_per_step": 1000 * secs, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16 (surrogate) / f32+i32 (LIF)", "data": "synthetic",
            "config": {"workload": "config 5: 200,000 frames, MLP 1280-512-512-10, 8 generations of 1,024 "
                                   "candidates, 64 simulated at B=64, 30-frame episodes; three searches (seeds 0-2); "
                                   "ms_per_step = one whole search"},
            "screened_per_simulated": last[0]["screened"] / last[0]["simulated"],
            "searches": [{
                "seed": rank * len(TUNE_SEEDS) + s,
                "count_error_per_generation": [g["count_error"] for g in r["surrogate_search"]["log"]],
                "count_error_uncalibrated_per_generation": [g["count_error_uncalibrated"]
                                                            for g in r["surrogate_search"]["log"]],
                "best_fitness": {"surrogate": r["surrogate_search"]["best"], "plain": r["plain_search"]["best"]},
                "full_simulations": {"surrogate": r["surrogate_search"]["sims"], "plain": r["plain_search"]["sims"],
                                     "candidates_judged_by_surrogate": sum(g["screened"]
                                                                           for g in r["surrogate_search"]["log"])},
                "train": {k: r["train"][k] for k in ("epochs", "steps", "seconds", "tflops", "val_nll",
                                                     "val_total_count_error")},
                "frames_per_s": r["frames_per_s"]} for s, r in zip(TUNE_SEEDS, runs)]}), flush=True)


INSTRUCT_METRIC = ("instructed-learning frame loop: sim neuron-steps/s with the deep delta rule every frame "
                   "(138k LIF, B=64)")


def run_instruct(args, world, rank, local):
    """The reference's instructed training path (flyzero/batch.py:331-409, BatchInstructDeep): per
    frame the grating drive, one 166-step run, then the deep delta rule towards per-slot target
    rates (traces and rates, the DN error, its retrograde pass to the DNs' presynaptic partners L1,
    the per-fly averaged updates of the synapses onto the DNs and onto L1), all on the device; the
    rule's per-slot error summary is read back every frame as the reference's step returns it.
    The 9 DN groups are the connectome's 8 motor neurons and one readout neuron; every synapse onto
    them or onto their presynaptic partners is plastic."""
    import torch

    from flyzero_b200 import instruct as I
    from flyzero_b200 import workloads as wl
    from flyzero_b200.brain import LIFParams
    from flyzero_b200.gpu import BatchBrain

    dev = torch.device("cuda", local)
    conn, drive, _, work = workload(args.batch, seed=rank)
    B, n, fs = args.batch, conn.n, wl.frame_steps(DT)
    dn = [np.array([m], np.int64) for m in conn.motor[:8]] + [np.array([drive.readout[9]], np.int64)]
    groups = dict(zip(I.GROUPS, dn))
    w = conn.weights
    dn_all = np.concatenate(dn)
    dn_pos = np.flatnonzero(np.isin(w.indices, dn_all))
    pos = np.union1d(dn_pos, I.deep_positions(w, dn_pos))
    gb = BatchBrain(w, LIFParams(dt=DT), batch=B, seed=1000 + rank, plastic_pos=pos)
    rule = I.BatchInstructDeep(gb, groups, fly_of_slot=np.arange(B) // 2)
    idx_in = np.r_[drive.inputs, drive.tonic]
    j = gb.slots(idx_in).cpu().numpy()
    inv = np.empty_like(j)
    inv[j] = np.arange(len(j))
    frames = args.warmup + args.steps
    t_ms, host_rates = 0.0, np.empty((frames, B, len(idx_in)), np.float32)
    for f in range(frames):
        host_rates[f] = work.rates(drive, t_ms, work.directions())[:, inv]
        t_ms += fs * DT
    p_dev = torch.as_tensor(host_rates, device=dev) * torch.tensor(np.float32(DT / 1000.0), device=dev)
    rng = np.random.default_rng(77 + rank)
    intents = rng.uniform(-1, 1, (frames, B, 5)) * np.array([1, 1, 0.5, 0.5, 0.5]) + np.array([0, 0, 0.5, 0.5, 0.5])
    tgts = np.array([[I.targets(intents[f, b], rule.p) for b in range(B)] for f in range(frames)], np.float32)
    counts = torch.empty((B, n), dtype=torch.int32, device=dev)
    st = torch.cuda.current_stream(dev)
    run_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    err = 0.0

    def frame(f, ev=None):
        gb.p_ext[:, :len(idx_in)].copy_(p_dev[f])
        if ev is not None:
            ev[0].record(st)
        gb.run_steps(fs, counts=counts)
        if ev is not None:
            ev[1].record(st)
        return rule.step(counts, tgts[f], np.ones(B, bool), fs * DT)

    for f in range(args.warmup):
        frame(f)
    gb.check()
    torch.cuda.synchronize(dev)
    barrier(world)
    clocks = Clocks(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for k in range(args.steps):
        err = float(np.mean(frame(args.warmup + k, run_ev[k])))
    e1.record(st)
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    gb.check()
    ms = e0.elapsed_time(e1)
    run_ms = sum(a.elapsed_time(b) for a, b in run_ev)
    value, max_ms = replica_value(float(B) * n * fs * args.steps, ms, world)
    if rank == 0:
        print(json.dumps({
            "metric": INSTRUCT_METRIC, "value": value, "unit": "neuron-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+i32 (LIF), f32/Q32.32 (plastic)", "data": "synthetic",
            "config": {"workload": f"{B} instances (2 slots per fly) x 138,639-neuron synthetic connectome, per bench step "
                                   "grating drive, one 166-step frame, BatchInstructDeep.step towards seeded per-slot "
                                   "targets with every slot learning", "plastic_synapses": int(len(pos)),
                       "onto_dns": int(len(rule.dn_sel_h)), "onto_l1": int(rule.n_deep), "l1_neurons": int(len(rule.l1)),
                       "parallelism": f"replicas x{world}"},
            "brain_ms_per_frame": run_ms / args.steps, "learning_and_io_ms_per_frame": (ms - run_ms) / args.steps,
            "mean_rate_error_hz_last_frame": err, "clocks": clk}), flush=True)


def run_trace(args, world, rank, local):
    """Phase trace of the persistent engine on the headline workload (a diagnostic): after
    --warmup frames, one frame with fb_set_trace on, then untraced frames until a second has passed;
    medians over the last instance group's CTAs and steps, in microseconds at the median SM clock
    sampled over those frames."""
    import torch

    from flyzero_b200 import workloads as wl
    from flyzero_b200.brain import LIFParams
    from flyzero_b200.gpu import BatchBrain, phase_summary

    dev = torch.device("cuda", local)
    conn, drive, pos, work = workload(args.batch, seed=rank)
    gb = BatchBrain(conn.weights, LIFParams(dt=DT), batch=args.batch, seed=1000 + rank, plastic_pos=pos)
    gb.set_schedule("persistent", lanes=args.lanes)
    idx_in = np.r_[drive.inputs, drive.tonic]
    j = gb.slots(idx_in).cpu().numpy()
    inv = np.empty_like(j)
    inv[j] = np.arange(len(j))
    fs, t_ms = wl.frame_steps(DT), 0.0
    counts = torch.empty((gb.B, gb.n), dtype=torch.int32, device=dev)
    clocks = Clocks(local)
    clocks.start()                        # sampled over the warm-up, traced and following frames (>= 1 s)
    t0, f = time.perf_counter(), 0
    while f <= args.warmup or time.perf_counter() - t0 < 1.0:
        rates = torch.as_tensor(work.rates(drive, t_ms, work.directions())[:, inv], device=dev)
        gb.p_ext[:, :len(idx_in)].copy_(rates * torch.tensor(np.float32(DT / 1000.0), device=dev))
        if f == args.warmup:
            T, K = gb.phase_trace(fs, counts=counts)
        else:
            gb.run_steps(fs, counts=counts)
            torch.cuda.synchronize(dev)
        t_ms += fs * DT
        f += 1
    clk = clocks.stop()
    gb.check()
    mhz = clk["sm_mhz"] or 1965.0
    ph = phase_summary(T, K, mhz)
    if rank == 0:
        print(json.dumps({
            "metric": "persistent-engine step time (median over CTAs and steps, phase trace)", "value": ph["step"],
            "unit": "us", "n_gpus": world, "steps": 1, "warmup": args.warmup, "ms_per_step": None,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32+i32",
            "data": "synthetic",
            "config": {"workload": f"headline workload, {args.batch} instances x 138,639 neurons, one traced frame of "
                                   f"{fs} steps; the last instance group's launch", "epoch_steps": K,
                       "ctas": int(T.shape[1]), "clock_mhz_used": mhz},
            "phases_us": {k: round(v, 3) for k, v in ph.items()}, "clocks": clk}), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        if args.component == "tune":
            if rank == 0:
                print(json.dumps({"impl": "reference", "component": "tune",
                                  "unavailable": "the reference's search (flyzero/tune.py:139-166) races every "
                                                 "candidate on its emulator, which is out of scope"}))
            return
        if args.component == "instruct":
            if rank == 0:
                print(json.dumps({"impl": "reference", "component": "instruct",
                                  "unavailable": "the reference's instructed rule (flyzero/batch.py:331-409) runs on "
                                                 "CuPy, which is not installed here"}))
            return
        if args.component == "trace":
            if rank == 0:
                print(json.dumps({"impl": "reference", "component": "trace",
                                  "unavailable": "a diagnostic of this engine's persistent kernel; the reference "
                                                 "has no counterpart"}))
            return
        if args.component == "fleet":
            if rank == 0:
                print(json.dumps({"impl": "reference", "component": "fleet",
                                  "unavailable": "the reference's frame loop needs its emulator pool and CuPy; "
                                                 "see --component brain and --component eye for its two halves"}))
            return
        (run_eye_reference if args.component == "eye" else run_reference)(args, world, rank)
        return
    world, rank, local = dist_setup(args)
    try:
        {"eye": run_eye, "fleet": run_fleet, "tune": run_tune, "trace": run_trace,
         "instruct": run_instruct}.get(args.component, run_ours)(
            args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
