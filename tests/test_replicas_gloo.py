"""The multi-GPU mode of the benchmark is replicas only: every rank runs an
independent copy and the time is the maximum over ranks.  That reduction runs
here on CPU ranks of a gloo process group (world size 2)."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ws, r, local = bench.dist_env()
    val = bench.max_over_ranks(10.0 + 3.0 * rank, device="cpu")
    out.put((rank, ws, r, local, val))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [x[0] for x in res] == [0, 1]
    assert all(x[1] == 2 and x[2] == x[0] and x[3] == x[0] for x in res)
    assert all(x[4] == 13.0 for x in res)


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(4.5, device="cpu") == 4.5
