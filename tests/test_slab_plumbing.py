"""Host side of the z-slab decomposition, on the CPU: the partition of the
planes, the slab grids, and (world size 2, gloo) the broadcast of rank 0's
128-byte NCCL unique id that every rank's transport is created from."""
import os

import numpy as np
import pytest

from falm_b200 import cases
from falm_b200 import slab as SL


@pytest.mark.parametrize("nz,n", [(24, 2), (24, 3), (25, 4), (256, 8), (4, 2)])
def test_partition_covers_the_planes(nz, n):
    parts = SL.partition(nz, n)
    assert [p[0] for p in parts] == list(np.cumsum([0] + [p[1] for p in parts[:-1]]))
    assert sum(p[1] for p in parts) == nz
    assert max(p[1] for p in parts) - min(p[1] for p in parts) <= 1
    assert min(p[1] for p in parts) >= 2
    with pytest.raises(ValueError):
        SL.partition(2 * n - 1, n)


def test_slab_grids_carry_the_neighbours_planes():
    case = cases.small_channel(32, 20, 24)
    g = case.grid
    for z0, nzl in SL.partition(24, 3):
        s = SL.slab_grid(g, z0, nzl)
        assert s.sz == nzl + 2 * g.gc and (s.sx, s.sy) == (g.sx, g.sy)
        np.testing.assert_array_equal(s.z, g.z[z0:z0 + nzl + 2 * g.gc])
        np.testing.assert_array_equal(s.hz, g.hz[z0:z0 + nzl + 2 * g.gc])
    c = SL.slab_case(case, 8, 8)
    assert c.alm is case.alm and c.grid.sz == 12


def _broadcast_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = bytes(range(rank, rank + 128)) if rank == 0 else bytes(128)
        got = SL.broadcast_id(mine, 0)
        parts = SL.partition(24, world)
        q.put((rank, got, parts[rank]))
    finally:
        dist.destroy_process_group()


def test_unique_id_broadcast_two_ranks_gloo():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_broadcast_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = bytes(range(0, 128))
    assert out[0][1] == want and out[1][1] == want
    assert out[0][2] == (0, 12) and out[1][2] == (12, 12)
