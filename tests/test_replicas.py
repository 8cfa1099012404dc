"""The multi-GPU path of bench.py (replicas, no data-path collective) on CPU: two gloo ranks
reduce their step times to the slowest, and the job's throughput counts every rank's bar."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    from vpd.replicas import job_throughput, max_over_ranks
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = [12.5, 20.0][rank]                         # this rank's device time for K increments
    slowest = max_over_ranks(ms)
    out[rank] = (slowest, job_throughput(1_000_000, 100, slowest, world))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_reduce_to_the_slowest_rank():
    import torch.multiprocessing as mp
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1]
    slowest, value = res[0]
    assert slowest == 20.0
    assert value == pytest.approx(2 * 1_000_000 * 100 / 0.020)


def test_single_process_needs_no_group():
    from vpd.replicas import job_throughput, max_over_ranks
    assert max_over_ranks(3.5) == 3.5
    assert job_throughput(4000, 10, 1.0, 1) == pytest.approx(4.0e7)
