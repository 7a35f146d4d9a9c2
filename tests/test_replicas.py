"""The multi-GPU path of bench.py: independent replicas, one per rank, whose
throughput is the units of all ranks over the slowest rank's device time.

The per-rank numbers here are made up (no GPU is needed): two gloo ranks on
the CPU report different times and unit counts, and every rank must agree on
the whole-job figure.  Rendezvous is on 127.0.0.1.
"""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    # rank r processed 1000 * (r + 1) units in 10 * (r + 1) ms
    value, t_ms = bench.job_throughput(1000.0 * (rank + 1), 10.0 * (rank + 1), dist)
    peak = bench.max_over_ranks(float(rank), dist)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, value, t_ms, peak))


def test_job_throughput_over_two_gloo_ranks():
    import torch.multiprocessing as mp

    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # units 1000 + 2000 over the slowest rank's 20 ms
    for rank, value, t_ms, peak in out:
        assert t_ms == pytest.approx(20.0)
        assert value == pytest.approx(3000.0 / 0.020)
        assert peak == pytest.approx(1.0)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench

    value, t_ms = bench.job_throughput(500.0, 5.0, None)
    assert t_ms == 5.0 and value == pytest.approx(500.0 / 0.005)
