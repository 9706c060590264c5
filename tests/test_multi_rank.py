"""Multi-GPU logic on CPU ranks (gloo, world size 2): object sharding with no exchange on the
data path, gathering the shards, the max-over-ranks timing reduction, LPT partitioning of uneven
requests, and a rank that fails before its first collective ending the job with an error on the
host (no GPU involved)."""
import os
import socket
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _spawn(tmp_path, n=12, steps=30, fail_rank=-1):
    import torch.multiprocessing as mp
    import multi_rank_worker as W
    out = str(tmp_path / "ranks.npz")
    mp.spawn(W.run, args=(2, _port(), out, n, steps, fail_rank), nprocs=2, join=True)
    return out


def test_sharded_propagation_equals_single_process(tmp_path, oracle_data):
    import oracle_api as O
    from opengpop_b200 import orbits
    n, steps = 12, 30
    out = np.load(_spawn(tmp_path, n, steps))
    r0, v0 = orbits.leo(n, seed=5)
    rf, vf = O.propagate(O.Data(degree=8), "gravity", (2024, 1, 1, 0, 0, 0.0), 60.0, steps, r0, v0,
                         threads=1)
    # objects are independent: the shards reproduce the single-process result bit for bit
    assert np.array_equal(out["r"], rf) and np.array_equal(out["v"], vf)
    assert float(out["t_max"]) == 2.0  # max over ranks of 1 + rank


def test_failing_rank_ends_the_job(tmp_path):
    with pytest.raises(Exception):
        _spawn(tmp_path, fail_rank=1)


def test_object_shards_cover_once():
    from opengpop_b200 import sharding
    for n, world in ((10, 3), (65536, 8), (7, 8), (0, 2)):
        sh = sharding.object_shards(n, world)
        assert sh[0][0] == 0 and sh[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(sh, sh[1:]))
        sizes = [e - s for s, e in sh]
        assert max(sizes) - min(sizes) <= 1


def test_lpt_partition_of_uneven_requests():
    from opengpop_b200 import orbits, sharding
    reqs = orbits.batch_requests(256, seed=3, max_days=0.1)
    costs = [sharding.request_cost(q["r"].shape[0], q["steps"], q["degree"]) for q in reqs]
    for world in (2, 4, 8):
        bins = sharding.lpt_partition(costs, world)
        assert sorted(i for b in bins for i in b) == list(range(len(reqs)))
        loads = [sum(costs[i] for i in b) for b in bins]
        # Graham: LPT makespan <= 4/3 OPT, and OPT >= max(mean load, largest request)
        assert max(loads) <= 4.0 / 3.0 * max(sum(costs) / world, max(costs)) * (1 + 1e-12)
