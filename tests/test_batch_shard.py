"""System-level sharding of the batched form over ranks (bench.py shard):
every system goes to exactly one rank, with no exchange between them.  Runs
as two gloo ranks on the CPU, gathering each rank's share."""
import os
import sys

import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, ws, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    mine = bench.shard(list(range(64)), rank, ws)
    got = [None] * ws
    dist.all_gather_object(got, mine)
    if rank == 0:
        out.put(got)
    dist.destroy_process_group()


def test_two_ranks_partition_the_systems():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, 29511, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    allsys = sorted(got[0] + got[1])
    assert allsys == list(range(64))
    assert not set(got[0]) & set(got[1])
    assert abs(len(got[0]) - len(got[1])) <= 1
