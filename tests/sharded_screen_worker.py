"""Rank bodies of the sharded closest-approach tests (sharding.closest_approach_sharded).

run_fake: gloo ranks on the CPU with a stand-in propagator and closest-approach object, which
check the window exchange, the phase loop and the record gather without a GPU.
run_gpu: gloo ranks that share one GPU, each with its own library context; the ranks' kernels
never wait on one another (the exchange is a host-side gloo all-gather)."""
import datetime
import os
import sys
from types import SimpleNamespace

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

H = 30.0


def traj_value(part, gstep, comp, obj):
    """Trajectory entry written by FakePropagator: part 0/1/2 = r/v/a, gstep counted from 1 over
    all phases, obj the global object index."""
    return np.sin(0.37 * obj + 0.11 * gstep + 1.3 * comp + 2.1 * part) * (1.0 + obj)


class FakePropagator:
    """Stand-in for Propagator: objects carry their global index in r[:, 0]; the global step of
    the phase's first step comes from the phase start (FIX_PHASE_EPOCH advances it by h a step)."""

    def __init__(self, ctx, start, h, max_steps, r, v):
        self.ids = r[:, 0].cpu().numpy().astype(np.int64)
        self.first = int(round(float(start[5]) / h))
        self.max_steps = max_steps
        self.done = 0
        ctx.log.append(("phase", self.first, max_steps, len(self.ids)))

    def step(self, k, tr, tv, ta):
        import torch
        assert self.done + k <= self.max_steps
        m = len(self.ids)
        for part, t in enumerate((tr, tv, ta)):
            out = np.empty((k, 3, m))
            for j in range(k):
                for c in range(3):
                    out[j, c] = traj_value(part, self.first + self.done + j + 1, c, self.ids)
            t.copy_(torch.from_numpy(out.reshape(-1)))
        self.done += k

    def close(self):
        pass


class FakeClosestApproach:
    """Stand-in for the external ClosestApproach: keeps the appended rows and, for each pair of
    its rows block, reports a checksum of both objects' r, v and a over every appended step."""

    def __init__(self, ctx, start, h, r, v, set_ids):
        self.ids = np.asarray(set_ids)
        self.n = len(self.ids)
        self.rows = (0, self.n)
        self.parts = [[], [], []]

    def set_rows(self, b, e):
        self.rows = (b, e)

    def reserve(self, total_steps):
        self.reserved = total_steps

    def append(self, k, R, V, A):
        for part, t in enumerate((R, V, A)):
            assert tuple(t.shape) == (k, self.n, 3) and t.is_contiguous()
            self.parts[part].append(t.cpu().numpy().copy())

    def find(self, threshold):
        traj = [np.concatenate(p) for p in self.parts]  # [steps][n][3]
        w = np.arange(1, traj[0].shape[0] + 1, dtype=np.float64)[:, None]
        recs = []
        for a in range(*self.rows):
            for b in range(a + 1, self.n):
                if self.ids[b] <= self.ids[a]:
                    continue
                d = sum(float(np.sum(w * (t[:, a] - t[:, b]) ** 2)) for t in traj)
                recs.append(SimpleNamespace(object_index1=a, object_index2=b, distance=d,
                                            time=float(traj[0].shape[0]),
                                            position_a=list(traj[0][-1, a]),
                                            position_b=list(traj[0][-1, b])))
        return recs

    def device_seconds(self):
        return np.zeros(3)

    def close(self):
        pass


def fake_job(n, set_ids, phases, window):
    from opengpop_b200 import FIX_PHASE_EPOCH, sharding
    ctx = SimpleNamespace(device=0, flags=FIX_PHASE_EPOCH, log=[])
    r = np.zeros((n, 3))
    r[:, 0] = np.arange(n)
    v = np.zeros((n, 3))
    recs, _ = sharding.closest_approach_sharded(
        ctx, (2024, 1, 1, 0, 0, 0.0), H, r, v, set_ids, phases, -1.0, window,
        make_propagator=FakePropagator, make_ca=FakeClosestApproach)
    return recs, ctx.log


def run_fake(rank, world, port, out_path, n, set_ids, phases, window):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        recs, log = fake_job(n, set_ids, phases, window)
        if rank == 0:
            np.save(out_path, np.array([(a, b, d, t) for a, b, d, t, _, _ in recs]))
        np.save(out_path.replace(".npy", "_log%d.npy" % rank), np.array(log, dtype=object),
                allow_pickle=True)
    finally:
        dist.destroy_process_group()


def gpu_job(n, seed, phases, window, threshold):
    import opengpop_b200 as G
    from opengpop_b200 import orbits, sharding
    r, v = orbits.leo(n, seed)
    set_ids = np.concatenate([np.arange(n // 10), np.full(n - n // 10, n // 10)]).astype(np.uint32)
    ctx = G.Context(gravity_degree=20)
    try:
        recs, sec = sharding.closest_approach_sharded(ctx, (2024, 1, 1, 0, 0, 0.0), H, r, v,
                                                      set_ids, phases, threshold, window)
    finally:
        ctx.close()
    return recs, sec


def run_gpu(rank, world, port, out_path, n, seed, phases, window, threshold):
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        recs, _ = gpu_job(n, seed, phases, window, threshold)
        if rank == 0:
            np.save(out_path, np.array([(a, b, d, t) + tuple(pa) + tuple(pb)
                                        for a, b, d, t, pa, pb in recs]))
    finally:
        dist.destroy_process_group()
