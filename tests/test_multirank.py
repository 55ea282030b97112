"""bench.py's replica aggregation on two gloo ranks (CPU; the GPU run uses NCCL).

One solve never shards, so N GPUs run N independent replicas; the whole-job
time is the slowest rank's device time and the whole-job s/iter divides it by
all iterations of all ranks.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    import bench
    per_rank_ms = [120.0, 150.0][rank]
    out[rank] = (bench.allmax(per_rank_ms, world), bench.job_seconds_per_iter(per_rank_ms, world, 10))
    bench.barrier(world)
    dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    for r in (0, 1):
        mx, spi = out[r]
        assert mx == 150.0
        assert spi == pytest.approx(150.0 / 1e3 / 20)
