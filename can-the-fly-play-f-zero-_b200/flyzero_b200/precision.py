"""Precision report of the engine: exact INT32 synaptic accumulation with FP32 neuron state,
against the same engine in FP64 oracle mode (FP64 state, same accumulation, same Poisson draws).

For every instance it reports the per-step maximum |v32 - v64| (mV), the step of the first raster
mismatch (the horizon over which the FP32 raster equals the FP64 one), and the per-neuron rate
error over the run. Both engines step together one step at a time; all comparisons stay on the
device until the end.

Run as a script for the high-activity workload (5 % of neurons at 210 Hz Poisson, B=16); it also
reports which schedule (engine, push or pull propagation) the autotuner picks at that activity:

    python -m flyzero_b200.precision --n 138639 --batch 16 --steps 10000
"""

from __future__ import annotations

import argparse
import json

import numpy as np


def precision_report(weights, params=None, batch: int = 16, inputs=None, rate_hz=None, steps: int = 10_000,
                     seed: int = 0, engine32: str = "auto") -> dict:
    """Step an FP32 engine and an FP64 engine side by side and compare them (see module doc)."""
    import torch

    from .brain import LIFParams
    from .gpu import BatchBrain

    params = params or LIFParams()
    b32 = BatchBrain(weights, params, batch=batch, seed=seed)
    b64 = BatchBrain(weights, params, batch=batch, seed=seed, fp64=True)
    b32.set_schedule(engine32)
    for b in (b32, b64):
        if inputs is not None:
            b.set_input(inputs, rate_hz)
    dev = b32.device
    n = b32.n
    maxdv = torch.zeros((steps, batch), dtype=torch.float64, device=dev)
    first = torch.full((batch,), -1, dtype=torch.int64, device=dev)
    spikes = torch.zeros((steps, batch), dtype=torch.int64, device=dev)
    c32 = torch.zeros((batch, n), dtype=torch.int64, device=dev)
    c64 = torch.zeros((batch, n), dtype=torch.int64, device=dev)
    a = torch.empty((batch, n), dtype=torch.int32, device=dev)
    b = torch.empty((batch, n), dtype=torch.int32, device=dev)
    for s in range(steps):
        _, sc32, sd32 = b32.run_steps(1, record=True, counts=a)
        _, sc64, sd64 = b64.run_steps(1, record=True, counts=b)
        c32 += a
        c64 += b
        spikes[s] = sc64[0]
        maxdv[s] = (b32.v.double() - b64.v).abs().amax(1)
        bad = (sc32[0] != sc64[0]) | (sd32[0] != sd64[0])
        first = torch.where((first < 0) & bad, torch.full_like(first, s), first)
    b32.check()
    b64.check()
    maxdv_h = maxdv.cpu().numpy()
    first_h = first.cpu().numpy()
    c32_h = c32.cpu().numpy().astype(np.float64)
    c64_h = c64.cpu().numpy().astype(np.float64)
    secs = steps * params.dt / 1000.0
    out = {"steps": steps, "batch": batch, "n": n, "dt_ms": params.dt, "seconds": secs,
           "spikes_per_step_fp64": float(spikes.double().mean()), "instances": []}
    for k in range(batch):
        h = int(first_h[k]) if first_h[k] >= 0 else steps
        r32, r64 = c32_h[k] / secs, c64_h[k] / secs
        active = r64 > 0
        rel = np.abs(r32[active] - r64[active]) / r64[active] if active.any() else np.zeros(1)
        out["instances"].append({
            "horizon_steps": h,
            "raster_identical": bool(first_h[k] < 0),
            "max_dv_mv_before_horizon": float(maxdv_h[:h, k].max()) if h > 0 else 0.0,
            "max_dv_mv": float(maxdv_h[:, k].max()),
            "mean_rate_hz_fp32": float(r32.mean()), "mean_rate_hz_fp64": float(r64.mean()),
            "rate_error_l1_rel": float(np.abs(r32 - r64).sum() / max(r64.sum(), 1e-30)),
            "rate_error_per_neuron_mean_rel": float(rel.mean()),
            "rate_error_per_neuron_p99_rel": float(np.percentile(rel, 99)),
            "mean_rate_error_rel": float(abs(r32.mean() - r64.mean()) / max(r64.mean(), 1e-30)),
        })
    hs = [x["horizon_steps"] for x in out["instances"]]
    out["summary"] = {"horizon_min": int(min(hs)), "horizon_median": float(np.median(hs)),
                      "max_dv_mv_before_horizon": max(x["max_dv_mv_before_horizon"] for x in out["instances"]),
                      "rate_error_l1_rel_max": max(x["rate_error_l1_rel"] for x in out["instances"]),
                      "mean_rate_error_rel_max": max(x["mean_rate_error_rel"] for x in out["instances"])}
    return out


def main(argv=None):
    from . import connectome as cx
    from . import workloads as wl
    from .brain import LIFParams

    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--n", type=int, default=138_639)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--steps", type=int, default=10_000)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args(argv)
    conn = cx.flywire_scale() if args.n == 138_639 else cx.synthetic(args.n, seed=args.seed)
    idx, rate = wl.high_activity_inputs(conn.n, seed=args.seed)
    rep = precision_report(conn.weights, LIFParams(dt=0.1), args.batch, idx, rate, args.steps, seed=args.seed)
    rep["schedule"] = schedule_at_activity(conn.weights, LIFParams(dt=0.1), args.batch, idx, rate, seed=args.seed)
    print(json.dumps(rep))


def schedule_at_activity(weights, params, batch, inputs, rate_hz, seed: int = 0, warm: int = 1000,
                         steps: int = 166) -> dict:
    """The autotuner's choice on this workload once its activity has settled: every schedule
    (persistent, step engine with push, step engine with pull) timed on the running simulation."""
    from .gpu import BatchBrain

    b = BatchBrain(weights, params, batch=batch, seed=seed)
    b.set_input(inputs, rate_hz)
    b.run_steps(warm)
    rep = b.autotune(steps=steps)
    rep["best"] = "/".join(map(str, rep["best"]))
    return rep


if __name__ == "__main__":
    main()
