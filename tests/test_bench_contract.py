"""bench.py's reference arm on CPU: one JSON line with the contract's keys (the driver parses it)."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                         timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    return json.loads(lines[0])


def test_reference_arm_json_line():
    d = _run("--impl", "reference", "--steps", "1", "--warmup", "1")
    for k in ("metric", "value", "unit", "impl", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["unit"] == d["unit"]
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0


def test_fleet_reference_arm_is_marked_unavailable():
    d = _run("--impl", "reference", "--component", "fleet", "--steps", "1", "--warmup", "1")
    assert d["impl"] == "reference" and "unavailable" in d


def test_episode_bookkeeping_restarts_runs_inside_the_window():
    """The batched workload's runs: staggered starts make runs end inside a 30-frame window, ended
    instances are restarted with a new U{0.5,1,2,3} s length, and the active steps per frame are the
    ones the engine's run-length masking lets through."""
    import numpy as np

    sys.path.insert(0, ROOT)
    import bench
    from flyzero_b200 import workloads as wl

    work = wl.BatchedWorkload.make(64, seed=0)
    ep = bench.Episodes(work, seed=23)
    first = (work.run_ms / bench.DT).astype(np.int64)
    assert np.all(ep.stop >= 1) and np.all(ep.stop <= first)
    t, restarted, partial = 0, 0, 0
    for _ in range(33):
        ended = ep.frame(t)
        assert np.all(ep.stop[ended] - t >= 5000)
        assert np.all(np.isin(ep.stop[ended] - t, bench.Episodes.LENGTHS))
        act = ep.active(t, 166)
        assert np.all((act >= 0) & (act <= 166))
        partial += int(np.sum((act > 0) & (act < 166)))
        restarted += len(ended)
        t += 166
    assert restarted > 0 and partial > 0


def test_dram_traffic_comes_from_the_committed_profile():
    sys.path.insert(0, ROOT)
    import bench

    traffic, src = bench.dram_traffic_record()
    assert traffic and traffic > 1e8 and "commit" in src
