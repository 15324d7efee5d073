"""Multi-rank host logic on CPU: two gloo ranks reduce their timings the way
bench.py does on N GPUs, and the job sharding is a balanced, deterministic
partition."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from peridyn_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        t, w = replicas.reduce_timing(1.0 + rank, 10.0 * (rank + 1), dist)
        out.put((rank, t, w))
    finally:
        dist.destroy_process_group()


def test_reduce_timing_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == [(0, 2.0, 30.0), (1, 2.0, 30.0)]


def test_reduce_timing_single_process():
    assert replicas.reduce_timing(1.5, 7, None) == (1.5, 7.0)


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_by_footprint_partition_and_balance(world):
    from peridyn_b200 import configs

    jobs, _ = configs.serving_jobs(48)
    sizes = [w["materials"][0].general.n for w in jobs]
    parts = replicas.shard_by_footprint(sizes, world)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(sizes)))
    assert parts == replicas.shard_by_footprint(sizes, world)
    loads = [sum(sizes[i] for i in p) for p in parts]
    # greedy largest-first: no rank exceeds the mean by more than the largest item
    assert max(loads) - sum(loads) / world <= max(sizes)
