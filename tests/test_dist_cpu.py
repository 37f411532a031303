"""The multi-rank helpers of bench.py (replicas, no data-path collective) on two gloo ranks on
the CPU: the timing reduction takes the slowest rank, and the whole-job value counts every
rank's units over that time."""
import os
import socket

import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    secs = [1.5, 4.0][rank]
    m = bench.max_over_ranks(secs, world)
    v = bench.replica_value(1000, world, secs)
    bench.barrier(world)
    out[rank] = (m, v)
    dist.destroy_process_group()


def test_max_over_ranks_and_replica_value_gloo():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert out[0] == out[1] == (4.0, 2 * 1000 / 4.0)
