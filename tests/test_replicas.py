"""CPU test of the multi-GPU replica path of bench.py with two gloo ranks:
every rank takes part in the same reductions, the slowest rank's time is
used, and the whole-job value is world * steps / max time."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    local_ms = 100.0 + 50.0 * rank  # rank 1 is the slow one
    m = bench.max_over_ranks(local_ms, dist, device="cpu")
    out[rank] = (m, bench.replica_rate(200, m, world))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas_use_the_slowest_rank():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == out[1]
    m, rate = out[0]
    assert m == 150.0
    assert rate == pytest.approx(2 * 200 / 0.150)
