"""Replicas with the engine under them: two spawned ranks (gloo process group for the host-side
barrier and the max/sum of bench.py's replica arithmetic) each run their own seeded instances on
the one GPU of this machine with the step engine (ordinary launches: no kernel waits on another
rank's), and each rank's counts equal those of the same replica run alone in this process. The
job's value is all ranks' neuron-steps over the slowest rank's device time."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

N, B, STEPS = 4096, 4, 300


@pytest.fixture(scope="module")
def torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _replica(rank):
    """One replica's run: (counts (B, N) int64, device ms)."""
    import torch

    from flyzero_b200 import connectome as cx
    from flyzero_b200 import workloads as wl
    from flyzero_b200.brain import LIFParams
    from flyzero_b200.gpu import BatchBrain

    conn = cx.synthetic(N, seed=5)
    idx, rate = wl.config1_inputs(conn.n, seed=5)
    gb = BatchBrain(conn.weights, LIFParams(), batch=B, seed=1000 + rank)
    gb.set_schedule("step")
    gb.set_input(idx, rate * (2 + rank))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    counts = gb.run_steps(STEPS)
    e1.record()
    torch.cuda.synchronize()
    gb.check()
    return counts.cpu().numpy().astype(np.int64), e0.elapsed_time(e1)


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        counts, ms = _replica(rank)
        value, max_ms = bench.replica_value(float(B * N * STEPS), ms, world, device="cpu")
        out[rank] = (counts, ms, value, max_ms)
    finally:
        dist.destroy_process_group()


def test_two_engine_replicas_over_gloo(torch):
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    assert set(out.keys()) == {0, 1}
    ms = [out[r][1] for r in range(world)]
    for r in range(world):
        counts, _, value, max_ms = out[r]
        assert counts.sum() > 0
        assert max_ms == pytest.approx(max(ms))                        # the slowest rank sets the job time
        assert value == pytest.approx(world * B * N * STEPS / (max(ms) / 1000.0), rel=1e-6)
        alone, _ = _replica(r)                                          # the same replica, run alone
        np.testing.assert_array_equal(counts, alone)
    assert not np.array_equal(out[0][0], out[1][0])                     # independent replicas
