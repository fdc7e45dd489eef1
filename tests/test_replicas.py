"""The N > 1 path of bench.py: independent replicas whose step time is the
maximum over ranks (world size 2, gloo on the CPU)."""
import os
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = 10.0 + 5.0 * rank  # this rank's timed total (ms)
        tmax = bench.reduce_over_ranks(t, "max", "cpu")
        tmin = bench.reduce_over_ranks(t, "min", "cpu")
        out.put((rank, tmax, tmin))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29611
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert res == [(0, 15.0, 10.0), (1, 15.0, 10.0)]
