"""The multi-rank plumbing of bench.py (one replica of the case per GPU, no
data-path collective) on two gloo ranks on the host: the barrier, the
maximum of the per-rank times and the whole-job rate."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import datetime
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        ms = 10.0 + 5.0 * rank            # rank 1 is the slower replica
        ms_max = bench.max_over_ranks(ms, world)
        out.put((rank, ms_max, bench.replica_rate(world, 1000, 4, ms_max)))
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_time_by_the_slowest():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]
    # 2 replicas x 1000 cells x 4 steps in 15 ms
    assert res[0][2] == pytest.approx(2 * 1000 * 4 / 0.015 / 1e6)
