"""The multi-GPU form of bench.py is N independent replicas (one TOD per rank, no data-path
collective).  Its only cross-rank step is the timing reduction: the job's time is the slowest
rank's, and the throughput counts every rank's samples.  Checked here with two gloo ranks on CPU."""

import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms, gs = bench.replica_throughput(10.0 + 5.0 * rank, 1_000_000, world, "cpu")
    out[rank] = (ms, gs)
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    world = 2
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        ms, gs = res[r]
        assert ms == pytest.approx(15.0)
        assert gs == pytest.approx(2 * 1_000_000 / 15e-3 / 1e9)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    ms, gs = bench.replica_throughput(4.0, 2 ** 20, 1, "cpu")
    assert ms == 4.0 and gs == pytest.approx(2 ** 20 / 4e-3 / 1e9)
