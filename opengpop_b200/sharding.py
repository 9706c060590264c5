"""Multi-GPU sharding of the propagation path: one process per GPU, no exchange on the data path.

Propagation units are independent (objects of one request, whole requests of a batch, adjoint
units), so N GPUs each take a share and the results are concatenated; the only collectives are
the timing reduction (max over ranks) and, where a caller wants the results on one rank, a
gather at the end. Works with any torch.distributed backend (NCCL on GPUs, gloo on CPUs).
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
