"""The N>1 bench path on CPU: two gloo ranks, replicas, time = max over ranks.

The MD path does not shard (one MD system per GPU), so N ranks run N
independent replicas; the only cross-rank steps are the barrier and the
max-reduction of the timed region, which this test runs with world_size 2.
"""

import os

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, torch.device("cpu"))
    dist.barrier()
    v = bench.job_value(1000, world, 4, ms)
    q.put((rank, ms, v))
    dist.destroy_process_group()


def test_two_rank_replicas_take_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 2000)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    assert [o[1] for o in out] == [15.0, 15.0]
    # 2 replicas x 1000 atoms x 4 steps / 15 ms
    assert out[0][2] == pytest.approx(2 * 1000 * 4 / 0.015)
