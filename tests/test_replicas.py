"""The multi-GPU path is replicas only: each rank renders the same job on its own
GPU and the ranks exchange nothing but the timing.  These CPU tests run that
host logic with two gloo ranks: the whole-job figures take the slowest rank's
device time and the samples of all ranks, and the rank environment is read as
torchrun sets it."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime

    import bench
    r, w, local = bench.dist_env()
    dist.init_process_group("gloo", rank=r, world_size=w, timeout=datetime.timedelta(seconds=60))
    dev_ms = [120.0, 150.0][rank]
    samples = [1000, 3000][rank]
    out[rank] = (r, w, local) + bench.aggregate(dist, dev_ms, samples)
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_aggregate_over_gloo():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    for rank in (0, 1):
        r, w, local, ms, samples = res[rank]
        assert (r, w, local) == (rank, 2, rank)
        assert ms == 150.0 and samples == 4000.0  # max of the device times, sum of the samples


def test_single_process_needs_no_group():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.aggregate(None, 42.0, 7) == (42.0, 7.0)
