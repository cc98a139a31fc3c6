"""The multi-GPU path of the benchmark is replicas only (the solve does not
shard): every rank solves its own copy and the job's throughput is world x DOF
over the slowest rank's time.  Two gloo ranks on the CPU check that reduction
and that every rank builds the same workload.
"""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        per_step, value = bench.aggregate_replicas([0.25, 0.5][rank], 1_000_000, world, dist, "cpu")
        _, inp = bench.workload(32, 4, "shell")
        digest = float(np.asarray(inp.density.data).sum())
        q.put((rank, per_step, value, digest, int(inp.density.base.shape[0])))
    finally:
        dist.destroy_process_group()


def test_replica_throughput_uses_the_slowest_rank():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, per_step, value, _, _ in out:
        assert per_step == 0.5
        assert value == pytest.approx(2 * 1_000_000 / 0.5 / 1e6)
    assert out[0][3:] == out[1][3:]    # the same seeded workload on every replica
