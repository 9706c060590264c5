"""Rank body of the multi-process CPU tests (gloo): each rank propagates its object shard with the
CPU oracle, the ranks gather the rows and reduce a time by max, as bench.py does over NCCL."""
import datetime
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))


def run(rank, world, port, out_path, n, steps, fail_rank):
    import torch.distributed as dist
    import oracle_api as O
    from opengpop_b200 import orbits, sharding
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        if rank == fail_rank:
            raise RuntimeError("rank %d fails before its first collective" % rank)
        r0, v0 = orbits.leo(n, seed=5)
        s, e = sharding.object_shards(n, world)[rank]
        data = O.Data(degree=8)
        rf, vf = O.propagate(data, "gravity", (2024, 1, 1, 0, 0, 0.0), 60.0, steps, r0[s:e], v0[s:e],
                             threads=1)
        r_all = sharding.gather_rows(rf, n)
        v_all = sharding.gather_rows(vf, n)
        t_max = sharding.max_over_ranks(1.0 + rank)
        if rank == 0:
            np.savez(out_path, r=r_all, v=v_all, t_max=t_max)
    finally:
        dist.destroy_process_group()
