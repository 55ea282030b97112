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


def _batch_worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    from ccq_b200 import batch

    def fake_solve(specs, **kw):
        # stands in for the device solve: one result per spec, tagged by its size
        return [dict(e_cor=-float(s.norb), iterations=s.norb, failed=False, device_ms=1.0) for s in specs], \
            {'setup_s': 0.0, 'solve_s': float(len(specs))}

    batch.solve_batch = fake_solve

    def gather(obj):
        objs = [None] * world
        dist.all_gather_object(objs, obj)
        return objs

    specs = batch.c3_specs()
    res, tims = batch.solve_sharded(specs, rank, world, gather)
    out[rank] = ([r['iterations'] for r in res], [t['solve_s'] for t in tims])
    dist.destroy_process_group()


def test_batched_instances_shard_and_gather():
    """64 instances over two ranks: each solved once, every rank sees every result in order."""
    from ccq_b200 import batch
    specs = batch.c3_specs()
    parts = batch.shard(specs, 2)
    assert sorted(parts[0] + parts[1]) == list(range(len(specs)))
    loads = [sum(batch.cost(specs[i]) for i in p) for p in parts]
    assert max(loads) / min(loads) < 1.1
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_batch_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    for r in (0, 1):
        its, times = out[r]
        assert its == [s.norb for s in specs]
        assert sum(times) == len(specs)
