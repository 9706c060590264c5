"""Multi-GPU sharding of the propagation path: one process per GPU.

Propagation units are independent (objects of one request, whole requests of a batch, adjoint
units), so N GPUs each take a share and the results are concatenated; the only collectives are
the timing reduction (max over ranks) and, where a caller wants the results on one rank, a
gather at the end. The closest-approach screen has one real exchange: every rank propagates its
share of the objects, the ranks all-gather each window of trajectory steps, and each rank screens
and refines the pairs whose first object lies in its block of rows (closest_approach_sharded).
Works with any torch.distributed backend (NCCL on GPUs, gloo on CPUs).
"""
import heapq

import numpy as np


def object_shards(n, world):
    """Contiguous, balanced [start, end) ranges of n objects over `world` ranks."""
    base, extra = divmod(int(n), int(world))
    out, start = [], 0
    for r in range(world):
        end = start + base + (1 if r < extra else 0)
        out.append((start, end))
        start = end
    return out


def gravity_terms(L):
    return (L + 1) * (L + 2) // 2 - 3


def request_cost(n, steps, degree):
    """Cost model of a request: objects x steps x (7 W(L) + 500) flops, W(L) = 24 T(L) + 15 L + 60."""
    return float(n) * float(steps) * (7.0 * (24 * gravity_terms(degree) + 15 * degree + 60) + 500.0)


def lpt_partition(costs, world):
    """Longest-processing-time bin packing: request indices per rank, largest costs first onto the
    least-loaded rank. The makespan is at most 4/3 of the optimum (Graham's bound)."""
    order = sorted(range(len(costs)), key=lambda i: -costs[i])
    heap = [(0.0, r) for r in range(world)]
    bins = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        bins[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(b) for b in bins]


def max_over_ranks(value, device=None):
    """Maximum of a float over all ranks of the default process group (the job's time)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_rows(local, n_total, device=None):
    """Concatenates each rank's rows (its object_shards range, in rank order) on every rank."""
    import torch
    import torch.distributed as dist
    local = np.ascontiguousarray(local, dtype=np.float64)
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return local
    world = dist.get_world_size()
    shards = object_shards(n_total, world)
    width = int(np.prod(local.shape[1:])) if local.ndim > 1 else 1
    cap = max(e - s for s, e in shards)
    buf = torch.zeros((cap, width), dtype=torch.float64, device=device)
    buf[: local.shape[0]] = torch.from_numpy(local.reshape(local.shape[0], width)).to(buf.device)
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    rows = [p[: e - s].cpu().numpy() for p, (s, e) in zip(parts, shards)]
    return np.concatenate(rows).reshape((n_total,) + local.shape[1:])


SCREEN_TILE = 64  # rows of one screen tile: row blocks start on multiples of it


def _world():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(), dist.get_rank()
    return 1, 0


def pairs_per_row(set_ids):
    """Pairs (a, b) with b in a later set, per first object a (the PartitionParameters staircase,
    partition_parameters.cuh:94-135): n minus the first index of the next set, 0 in the last set."""
    ids = np.asarray(set_ids, dtype=np.int64)
    n = ids.shape[0]
    starts = np.searchsorted(ids, np.arange(int(ids[-1]) + 2), side="left")
    bound = starts[np.minimum(ids + 1, int(ids[-1]) + 1)]
    return (n - bound).astype(np.int64)


def screen_rows(set_ids, world, tile=SCREEN_TILE):
    """Row blocks [begin, end) per rank for the sharded screen: boundaries on multiples of the
    screen tile, each placed where the running pair count comes closest to an equal share."""
    per_row = pairs_per_row(set_ids)
    n = per_row.shape[0]
    cum = np.concatenate([[0], np.cumsum(per_row)])
    cands = np.unique(np.concatenate([np.arange(0, n, tile), [n]]))
    total = cum[-1]
    cuts = [0]
    for k in range(1, world):
        target = total * k / world
        c = cands[np.argmin(np.abs(cum[cands] - target))]
        cuts.append(int(max(c, cuts[-1])))
    cuts.append(n)
    return [(cuts[k], cuts[k + 1]) for k in range(world)]


def gather_window(buf, k, n_total, parts=3):
    """All-gathers one window of trajectory rows and returns them in the order of all objects.

    buf holds `parts` consecutive segments of k * 3 * m_max doubles (m_max: the largest object
    shard); in segment i the first k * 3 * m entries are this rank's [k][3][m] rows (SoA, as
    GpuPropagator::Step writes them). Returns `parts` contiguous [k][n_total][3] tensors (AoS,
    what ClosestApproach's append takes) on buf's device. NCCL gathers device memory in place;
    other backends gather through host memory."""
    import torch
    import torch.distributed as dist
    world, _ = _world()
    shards = object_shards(n_total, world)
    m_max = max(e - s for s, e in shards)
    seg = k * 3 * m_max
    local = buf[: parts * seg]
    if world == 1:
        full = local.unsqueeze(0)
    elif dist.get_backend() == "nccl":
        full = torch.empty((world, parts * seg), dtype=buf.dtype, device=buf.device)
        dist.all_gather_into_tensor(full, local)
    else:
        host = local.cpu()
        pieces = [torch.empty_like(host) for _ in range(world)]
        dist.all_gather(pieces, host)
        full = torch.stack(pieces).to(buf.device)
    outs = []
    for i in range(parts):
        aos = torch.empty((k, n_total, 3), dtype=buf.dtype, device=buf.device)
        for j, (s, e) in enumerate(shards):
            m = e - s
            if m:
                aos[:, s:e, :] = full[j, i * seg: i * seg + k * 3 * m].view(k, 3, m).permute(0, 2, 1)
        outs.append(aos)
    return outs


def _phase_start(start, h, steps_done, flags):
    # the reference's phases keep the first epoch; GPOP_FIX_PHASE_EPOCH advances it
    from opengpop_b200 import FIX_PHASE_EPOCH
    if not flags & FIX_PHASE_EPOCH:
        return start
    y, mo, d, hh, mi, sec = start
    return (y, mo, d, hh, mi, float(sec) + steps_done * float(h))


def closest_approach_sharded(ctx, start, h, r, v, set_ids, phases, threshold=-1.0, window=240,
                             make_propagator=None, make_ca=None):
    """ClosestApproach (closest_approach.cu:47-209) over the ranks of the default process group,
    one GPU each (no group: one rank).

    Every rank propagates its object_shards share for each phase (a fresh startup per phase, as
    ClosestApproach::Propagate does), all-gathers every `window` steps of positions, velocities
    and accelerations, and screens them for the pairs of its screen_rows block; after the last
    phase it refines those pairs and the records below `threshold` (all pairs if negative) are
    gathered on every rank, sorted by (object_index1, object_index2). Returns (records, seconds):
    records are tuples (i, j, distance, time, position_a, position_b); seconds holds this rank's
    device seconds of propagation, exchange, screen and refinement.
    make_propagator / make_ca replace the library's Propagator and ClosestApproach (tests)."""
    import torch
    import torch.distributed as dist
    import opengpop_b200 as G
    world, rank = _world()
    r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1, 3)
    v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1, 3)
    n = r.shape[0]
    phases = [int(p) for p in phases]
    if not phases or min(phases) <= 0:
        raise ValueError("every phase needs a positive number of steps")
    if v.shape[0] != n or len(set_ids) != n:
        raise ValueError("positions, velocities and set ids differ in length")
    shards = object_shards(n, world)
    o0, o1 = shards[rank]
    m, m_max = o1 - o0, max(e - s for s, e in shards)
    make_propagator = make_propagator or G.Propagator
    make_ca = make_ca or (lambda *a: G.ClosestApproach(*a, kind="external"))
    ca = make_ca(ctx, start, h, r, v, set_ids)
    try:
        ca.set_rows(*screen_rows(set_ids, world)[rank])
        ca.reserve(sum(phases))
        dev = torch.device("cuda", ctx.device) if torch.cuda.is_available() else torch.device("cpu")
        r_loc = torch.tensor(r[o0:o1], device=dev)
        v_loc = torch.tensor(v[o0:o1], device=dev)
        win = max(1, min(int(window), max(phases)))
        buf = torch.zeros(3 * win * 3 * m_max, dtype=torch.float64, device=dev)
        timed = dev.type == "cuda"
        t_prop = t_gather = 0.0
        done = 0
        for steps in phases:
            p = make_propagator(ctx, _phase_start(start, h, done, ctx.flags), h, steps, r_loc, v_loc) if m else None
            try:
                left = steps
                while left > 0:
                    k = min(win, left)
                    seg = k * 3 * m_max
                    if timed:
                        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
                        ev[0].record()
                    if p is not None:
                        p.step(k, buf[0: k * 3 * m], buf[seg: seg + k * 3 * m], buf[2 * seg: 2 * seg + k * 3 * m])
                    if timed:
                        ev[1].record()
                    rows = gather_window(buf, k, n)
                    if timed:
                        ev[2].record()
                        ev[2].synchronize()
                        t_prop += ev[0].elapsed_time(ev[1]) / 1e3
                        t_gather += ev[1].elapsed_time(ev[2]) / 1e3
                    ca.append(k, *rows)
                    left -= k
            finally:
                if p is not None:
                    p.close()
            done += steps
        recs = [(int(x.object_index1), int(x.object_index2), float(x.distance), float(x.time),
                 tuple(x.position_a), tuple(x.position_b)) for x in ca.find(threshold)]
        ds = ca.device_seconds()
    finally:
        ca.close()
    if world > 1:
        everyone = [None] * world
        dist.all_gather_object(everyone, recs)
        recs = [x for part in everyone for x in part]
    recs.sort(key=lambda x: (x[0], x[1]))
    return recs, {"propagation": t_prop, "exchange": t_gather, "screen": float(ds[1]),
                  "refinement": float(ds[2])}
