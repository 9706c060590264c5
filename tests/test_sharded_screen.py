"""Sharded closest-approach screen (sharding.closest_approach_sharded): each rank propagates its
object shard, the ranks all-gather the trajectory in windows, and each screens and refines the
pairs of its block of rows. CPU tests check the row blocks against a brute-force pair count, the
window exchange (gloo, world size 2) and the phase loop with stand-in propagator and
closest-approach objects. GPU tests check that row-restricted objects reproduce the full screen,
and that the sharded job on one rank and on two ranks sharing the GPU (gloo) gives the records of
the fused gpop_ca_propagate path."""
import os
import socket

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _set_layouts():
    rng = np.random.default_rng(7)
    yield np.concatenate([np.arange(200), np.full(1800, 200)])  # the screen benchmark's layout
    yield np.repeat(np.arange(3), [100, 50, 30])
    yield np.sort(rng.integers(0, 40, 700))  # ragged sets
    yield np.array([0, 1])


def _dense(ids):
    # set ids that start at 0 and grow by at most 1 (the partition's rule)
    _, inv = np.unique(ids, return_inverse=True)
    return inv.astype(np.uint32)


def test_pairs_per_row_brute_force():
    from opengpop_b200 import sharding
    for ids in _set_layouts():
        ids = _dense(ids)
        brute = np.array([(ids[a + 1:] > ids[a]).sum() for a in range(len(ids))])
        assert np.array_equal(sharding.pairs_per_row(ids), brute)


def test_row_pair_ranges_follow_the_partition_map():
    # the first pair index of every row (the start of a row block's pair range) is the oracle's
    # PartitionParameters map of (a, first b of a later set)
    import oracle_api as O
    from opengpop_b200 import sharding
    for ids in _set_layouts():
        ids = _dense(ids)
        p = O.partition(ids)
        cum = np.concatenate([[0], np.cumsum(sharding.pairs_per_row(ids))])
        assert cum[-1] == p["num_pairs"]
        for s in range(p["num_sets"] - 1):
            a0, a1 = int(p["set_offsets"][s]), int(p["set_offsets"][s + 1])
            for a in range(a0, a1):
                assert cum[a] == int(p["map_offsets"][s]) + (a - a0) * int(p["num_higher"][s])


def test_screen_rows_cover_tiles_and_balance():
    from opengpop_b200 import sharding
    for ids in _set_layouts():
        ids = _dense(ids)
        n = len(ids)
        per_row = sharding.pairs_per_row(ids)
        tile_max = max(int(per_row[i:i + 64].sum()) for i in range(0, n, 64))
        for world in (1, 2, 3, 8):
            rows = sharding.screen_rows(ids, world)
            assert len(rows) == world and rows[0][0] == 0 and rows[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(rows, rows[1:]))
            for b, e in rows:
                assert b <= e and (b % 64 == 0 or b == n) and (e % 64 == 0 or e == n)
            share = [int(per_row[b:e].sum()) for b, e in rows]
            assert sum(share) == int(per_row.sum())
            # each cut sits within one tile's pairs of the equal share
            cum = np.cumsum([0] + share)
            for k in range(1, world):
                assert abs(cum[k] - per_row.sum() * k / world) <= tile_max


def test_gather_window_single_rank():
    import torch
    from opengpop_b200 import sharding
    k, n = 3, 5
    soa = torch.arange(3 * k * 3 * n, dtype=torch.float64)
    out = sharding.gather_window(soa, k, n)
    for i in range(3):
        want = soa[i * k * 3 * n:(i + 1) * k * 3 * n].view(k, 3, n).permute(0, 2, 1)
        assert torch.equal(out[i], want) and out[i].is_contiguous()


def _spawn_fake(tmp_path, n, ids, phases, window, world=2):
    import torch.multiprocessing as mp
    import sharded_screen_worker as W
    out = str(tmp_path / "fake.npy")
    mp.spawn(W.run_fake, args=(world, _port(), out, n, ids, phases, window), nprocs=world, join=True)
    logs = [np.load(out.replace(".npy", "_log%d.npy" % r), allow_pickle=True) for r in range(world)]
    return np.load(out), logs


@pytest.mark.parametrize("n,phases,window", [(7, [5], 2), (130, [4, 3], 3), (3, [2, 2, 1], 8)])
def test_fake_job_two_ranks_equals_one(tmp_path, n, phases, window):
    import sharded_screen_worker as W
    from opengpop_b200 import sharding
    ids = _dense(np.minimum(np.arange(n) // 2, 3))
    recs1, log1 = W.fake_job(n, ids, phases, window)
    recs2, logs = _spawn_fake(tmp_path, n, ids, phases, window)
    one = np.array([(a, b, d, t) for a, b, d, t, _, _ in recs1])
    # every pair once, in (i, j) order, with the same checksum over all appended steps
    assert np.array_equal(one, recs2)
    assert len(one) == int(sharding.pairs_per_row(ids).sum())
    assert np.all(one[:, 3] == sum(phases))
    # each rank starts a phase per phase, on its own shard, at the phase's first global step
    for rank, log in enumerate(logs):
        s, e = sharding.object_shards(n, 2)[rank]
        starts = np.cumsum([0] + phases[:-1])
        want = [("phase", int(f), int(p), e - s) for f, p in zip(starts, phases)] if e > s else []
        assert [tuple(x) for x in log] == want


def test_fake_job_three_ranks_uneven_shards(tmp_path):
    # 5 objects over 3 ranks: shards of 2, 2 and 1 objects; every pair once, the same checksums
    import sharded_screen_worker as W
    n, phases = 5, [3, 4]
    ids = _dense(np.array([0, 0, 1, 2, 2]))
    recs1, _ = W.fake_job(n, ids, phases, 2)
    recs3, logs = _spawn_fake(tmp_path, n, ids, phases, 2, world=3)
    assert np.array_equal(np.array([(a, b, d, t) for a, b, d, t, _, _ in recs1]), recs3)
    assert [len(log) for log in logs] == [2, 2, 2]


def test_fake_job_rank_without_objects(tmp_path):
    # more ranks than objects: the empty rank still takes part in every exchange
    import sharded_screen_worker as W
    n, phases = 2, [3]
    ids = _dense(np.array([0, 1]))
    recs1, _ = W.fake_job(n, ids, phases, 2)
    recs3, logs = _spawn_fake(tmp_path, n, ids, phases, 2, world=3)
    assert np.array_equal(np.array([(a, b, d, t) for a, b, d, t, _, _ in recs1]), recs3)
    assert [len(log) for log in logs] == [1, 1, 0]


def test_fake_job_checksums_the_trajectory():
    import sharded_screen_worker as W
    n, phases = 6, [3, 2]
    ids = _dense(np.array([0, 0, 1, 1, 2, 2]))
    recs, _ = W.fake_job(n, ids, phases, 2)
    steps = sum(phases)
    w = np.arange(1, steps + 1)
    for a, b, d, _, _, _ in recs:
        want = 0.0
        for part in range(3):
            t = np.array([[[W.traj_value(part, s, c, o) for c in range(3)] for o in (a, b)]
                          for s in range(1, steps + 1)])
            want += float(np.sum(w[:, None] * (t[:, 0] - t[:, 1]) ** 2))
        assert d == pytest.approx(want, rel=1e-12)


def test_sharded_job_rejects_bad_phases():
    import sharded_screen_worker as W
    ids = _dense(np.array([0, 0, 1, 1]))
    for phases in ([], [3, 0], [-1]):
        with pytest.raises(ValueError):
            W.fake_job(4, ids, phases, 2)
    with pytest.raises(ValueError):
        W.fake_job(4, ids[:3], [2], 2)


# ---- GPU ----

def _fused(n, seed, phases, threshold):
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    r, v = orbits.leo(n, seed)
    ids = np.concatenate([np.arange(n // 10), np.full(n - n // 10, n // 10)]).astype(np.uint32)
    ctx = G.Context(gravity_degree=20)
    ca = ctx.closest_approach((2024, 1, 1, 0, 0, 0.0), 30.0, r, v, ids)
    for p in phases:
        ca.propagate(p)
    recs = ca.find(threshold)
    out = np.array([(x.object_index1, x.object_index2, x.distance, x.time) + tuple(x.position_a)
                    + tuple(x.position_b) for x in recs])
    pairs = ca.pairs()
    ca.close()
    ctx.close()
    return out, pairs, r, v, ids


@pytest.mark.gpu
def test_row_blocks_reproduce_the_full_screen():
    import opengpop_b200 as G
    from opengpop_b200 import sharding
    n, phases = 700, [90, 50]
    full, pairs, r, v, ids = _fused(n, 11, phases, -1.0)
    ctx = G.Context(gravity_degree=20)
    P = len(pairs["distance"])
    got = {k: np.full_like(a, np.nan, dtype=np.float64) for k, a in pairs.items()}
    recs = []
    for b, e in ((0, 64), (64, 64), (64, 128), (128, n)):
        ca = ctx.closest_approach((2024, 1, 1, 0, 0, 0.0), 30.0, r, v, ids)
        ca.set_rows(b, e)
        lo, hi = ca.pair_range
        per_row = sharding.pairs_per_row(ids)
        assert (lo, hi) == (int(per_row[:b].sum()), int(per_row[:e].sum()))
        for p in phases:
            ca.propagate(p)
        part = ca.pairs()
        for key in got:
            got[key][lo:hi] = part[key][lo:hi]
        recs += [(x.object_index1, x.object_index2, x.distance, x.time) + tuple(x.position_a)
                 + tuple(x.position_b) for x in ca.find(-1.0)]
        ca.close()
    with pytest.raises(G.GpopError):
        ca = ctx.closest_approach((2024, 1, 1, 0, 0, 0.0), 30.0, r, v, ids)
        try:
            ca.set_rows(10, 64)  # not on a tile boundary
        finally:
            ca.close()
    ctx.close()
    # the same tiles and the same trajectory: bit-identical per-pair results
    for key in got:
        assert np.array_equal(got[key], pairs[key].astype(np.float64)), key
    assert len(recs) == P
    assert np.array_equal(np.array(recs), full)


@pytest.mark.gpu
def test_sharded_job_one_rank_equals_fused():
    import sharded_screen_worker as W
    n, phases = 600, [100, 60]
    full, _, _, _, _ = _fused(n, 13, phases, -1.0)
    recs, sec = W.gpu_job(n, 13, phases, 48, -1.0)
    got = np.array([(a, b, d, t) + tuple(pa) + tuple(pb) for a, b, d, t, pa, pb in recs])
    assert len(full) > 0 and got.shape == full.shape
    assert np.array_equal(got[:, :2], full[:, :2])
    # the propagator's launches split at other steps; the arithmetic of every step is the same
    assert np.abs(got[:, 2:] - full[:, 2:]).max() <= 1e-9 * np.abs(full[:, 2:]).max()
    assert sec["propagation"] > 0 and sec["screen"] > 0


@pytest.mark.gpu
def test_sharded_job_two_ranks_on_one_gpu_equals_fused(tmp_path):
    import torch.multiprocessing as mp
    import sharded_screen_worker as W
    n, phases = 600, [100, 60]
    full, _, _, _, _ = _fused(n, 13, phases, -1.0)
    out = str(tmp_path / "gpu2.npy")
    mp.spawn(W.run_gpu, args=(2, _port(), out, n, 13, phases, 48, -1.0), nprocs=2, join=True)
    got = np.load(out)
    assert got.shape == full.shape
    assert np.array_equal(got[:, :2], full[:, :2])
    assert np.abs(got[:, 2:] - full[:, 2:]).max() <= 1e-9 * np.abs(full[:, 2:]).max()


@pytest.mark.gpu
def test_unreserved_appends_reproduce_the_fused_screen():
    # appends of uneven sizes with no reserve: the store grows by doubling, keeps every row, and
    # the running minima match one fused propagation over the same trajectory
    import torch
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    n, chunks = 300, [1, 2, 5, 3, 10, 16]
    r, v = orbits.leo(n, 17)
    ids = np.concatenate([np.arange(30), np.full(n - 30, 30)]).astype(np.uint32)
    ctx = G.Context(gravity_degree=20)
    ca = ctx.closest_approach((2024, 1, 1, 0, 0, 0.0), 30.0, r, v, ids)
    ca.propagate(sum(chunks))
    traj = ca.trajectory()
    want = ca.pairs()
    ca.close()
    ext = G.ClosestApproach(ctx, (2024, 1, 1, 0, 0, 0.0), 30.0, r, v, ids, kind="external")
    s = 0
    for k in chunks:
        rows = [torch.tensor(np.ascontiguousarray(t[s:s + k].transpose(0, 2, 1)), device="cuda")
                for t in traj]
        ext.append(k, *rows)
        s += k
    got = ext.pairs()
    got_traj = ext.trajectory()
    ext.close()
    ctx.close()
    for a, b in zip(got_traj, traj):
        assert np.array_equal(a, b)
    for key in want:
        assert np.array_equal(got[key], want[key]), key
