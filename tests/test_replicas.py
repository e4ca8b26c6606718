"""The multi-GPU path of bench.py is replicas only (instances are independent; the neuron
dimension does not shard): each rank runs its own B=64 workload with its own seed and the job's
throughput is all ranks' neuron-steps over the slowest rank's time. The rank plumbing is checked
here with world_size 2 on the gloo backend (CPU)."""

import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        steps = [1000.0, 3000.0][rank]
        ms = [5.0, 8.0][rank]
        value, max_ms = bench.replica_value(steps, ms, world, device="cpu")
        bench.barrier(world)
        # each rank draws its own instance workload (seeded by rank), as run_ours does
        from flyzero_b200 import workloads as wl

        w = wl.BatchedWorkload.make(4, seed=rank)
        out[rank] = (value, max_ms, float(w.contrast[0]))
    finally:
        dist.destroy_process_group()


def test_replica_throughput_over_two_gloo_ranks():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    assert set(out.keys()) == {0, 1}
    for r in range(world):
        value, max_ms, _ = out[r]
        assert max_ms == 8.0                                  # the slowest rank sets the job time
        assert np.isclose(value, (1000.0 + 3000.0) / 0.008)   # all ranks' work over it
    assert out[0][2] != out[1][2]                             # independent replicas, own seeds
