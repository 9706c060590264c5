#!/usr/bin/env python
"""Benchmark of the propagation hot path (object-steps/s at 70x70 gravity, mixed vs FP64).

Workload (the mixed-precision configuration): 65,536 seeded synthetic objects (70% LEO, 20% MEO,
10% GEO), 70x70 JGM3 gravity, 30 s GJ8 step with RK8 startup, epoch 2024-01-01T00:00:00 UTC.
A bench step propagates every object through --prop-steps GJ8 steps (default 64) of a continuing
propagation (startup runs in the warm-up). `value` is the mixed-precision throughput; the FP64
build is measured on the same workload and reported beside it. `e2e` times the public call a user
makes (gpop_propagate with pinned host buffers: upload, frame tables, startup, steps, download).

Multi-GPU (torchrun): every rank propagates its own 65,536 objects (weak scaling, no collective on
the data path); the time is the max over ranks.

--impl reference times the CPU FP64 restatement of the reference method (the oracle port; the
reference has no CPU implementation of this path) on the host cores, on a bounded sample.
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_OBJECTS = 65536
H = 30.0
DEGREE = 70
START = (2024, 1, 1, 0, 0, 0.0)
SEED = 20240101
# The headline metric; both arms (this build and --impl reference) print this same string, unit and
# direction so that the two lines can be divided.
METRIC = "object-steps/s @70x70: mixed vs FP64 at <=1 m/7 d err; conj pairs/s"
UNIT = "object-steps/s"

# Algorithmic work (FMA = 2 flops): gravity evaluation W(L) = 24 T(L) + 15 L + 60, T(L) the number
# of (n, m) terms with 2 <= n <= L; an object-step is 7 distinct evaluations plus ~500 flops of
# GJ8 predictor/corrector arithmetic.
def terms(L):
    return (L + 1) * (L + 2) // 2 - 3


def flops_per_object_step(L=DEGREE):
    return 7 * (24 * terms(L) + 15 * L + 60) + 500


def fp32_flops_per_object_step(L=DEGREE):
    # the mixed build runs the degree > 8 terms in FP32
    return 7 * 24 * (terms(L) - terms(8))


# DRAM bytes (read + write) of one mixed GJ8 launch over 65,536 objects (the split block), from an
# ncu capture (dram__bytes_read.sum 20.66 MB, dram__bytes_write.sum 0;
# profiles/gj8_kernels_65536obj_70x70.md).
MIXED_GJ8_DRAM_BYTES = 20.66e6


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for name, val in zip(names, p[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_baseline(seconds_target=15.0):
    """Oracle (CPU FP64 restatement of the reference method, OpenMP over objects) on a bounded
    sample of the same workload; returns object-steps/s and a description."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_api as O
    from opengpop_b200 import orbits
    data = O.Data(degree=DEGREE)
    cores = cpu_cores()
    n = max(32, 8 * cores)
    r0, v0 = orbits.mixed_population(N_OBJECTS, SEED)
    r0, v0 = r0[:n], v0[:n]
    # calibrate: two lengths, so the startup cost cancels out of the per-step rate
    t0 = time.perf_counter()
    O.propagate(data, "gravity", START, H, 8, r0, v0, threads=cores)
    t8 = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.propagate(data, "gravity", START, H, 40, r0, v0, threads=cores)
    t40 = time.perf_counter() - t0
    per_step = max((t40 - t8) / 32.0, 1e-6)
    steps = int(min(4000, max(40, seconds_target / per_step)))
    t0 = time.perf_counter()
    O.propagate(data, "gravity", START, H, steps, r0, v0, threads=cores)
    dt = time.perf_counter() - t0
    rate = n * steps / dt
    return rate, cores, ("%d of the %d objects x %d steps (30 s, 70x70, startup included), "
                         "%.1f s of CPU work" % (n, N_OBJECTS, steps, dt))


def run_reference(args):
    rank = env_int("RANK", 0)
    if rank != 0:
        return 0
    rates = []
    cores = cpu_cores()
    desc = ""
    for i in range(args.warmup + args.steps):
        rate, cores, desc = cpu_baseline(seconds_target=max(2.0, 30.0 / (args.steps + args.warmup)))
        if i >= args.warmup:
            rates.append(rate)
    value = float(np.mean(rates)) if rates else 0.0
    line = {
        "impl": "reference", "metric": METRIC, "value": value,
        "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "65,536 objects (70% LEO / 20% MEO / 10% GEO), 70x70, 30 s step",
                   "sample": desc},
        "cpu_baseline": {"value": value, "unit": "object-steps/s", "cores": cores, "kind": "port",
                         "sample": desc},
        "e2e": {"value": value, "unit": "object-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def probe_peak(torch, fp64, dev):
    """Measured FMA throughput (TFLOP/s) of this GPU: independent FMA chains on every SM."""
    lib = C.CDLL(os.path.join(ROOT, "opengpop_b200", "lib", "libgpop_probe.so"))
    lib.gpop_probe_fma.restype = C.c_int
    lib.gpop_probe_fma.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                   C.POINTER(C.c_double)]
    scratch = torch.zeros(16, dtype=torch.float64, device=dev)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    stream = torch.cuda.current_stream()
    flops = C.c_double()
    best = 0.0
    for it in range(4):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = lib.gpop_probe_fma(int(fp64), sms * 8, 2000, C.c_void_p(scratch.data_ptr()),
                                C.c_void_p(stream.cuda_stream), C.byref(flops))
        e1.record(stream)
        torch.cuda.synchronize()
        if rc != 0:
            return None
        if it:
            best = max(best, flops.value / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    return best


def probe_pipes(torch, dev):
    """Milliseconds of 6 packed FP32 FMA chains, 6 FP64 FMA chains, and both interleaved, per
    thread, one 256-thread block per SM (libgpop_probe.so): whether the FP64 pipe can work beside
    the FMA pipe (both interleaved taking the longer of the two times) or not (their sum)."""
    lib = C.CDLL(os.path.join(ROOT, "opengpop_b200", "lib", "libgpop_probe.so"))
    lib.gpop_probe_mix.restype = C.c_int
    lib.gpop_probe_mix.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    scratch = torch.zeros(16, dtype=torch.float32, device=dev)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    stream = torch.cuda.current_stream()
    out = {}
    for mode, name in ((0, "fp32x2_ms"), (1, "fp64_ms"), (2, "interleaved_ms")):
        best = None
        for it in range(4):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rc = lib.gpop_probe_mix(mode, sms, 4000, C.c_void_p(scratch.data_ptr()),
                                    C.c_void_p(stream.cuda_stream))
            e1.record(stream)
            torch.cuda.synchronize()
            if rc != 0:
                return None
            if it:
                ms = e0.elapsed_time(e1)
                best = ms if best is None else min(best, ms)
        out[name] = best
    return out


# ---- auxiliary workloads (one GPU; each prints its own JSON line) ----
def w_jac(L):
    """FP64 flops of one gravity evaluation with its 3x3 Jacobian at degree L: per (n, m) term
    the Q and dQ/deps recursions (7) and 18 sums (36) plus n Q (1); per column about 100."""
    return 44 * terms(L) + 100 * (L + 1) + 200


def _peaks(torch, dev, clocks):
    """FP64 and FP32 peaks (TFLOP/s) at the SM clock sampled during the timed region (the FMA
    probe's figures when no clock was sampled)."""
    p64, p32 = clock_peaks(clocks.get("sm_mhz"), dev)
    if p64:
        return p64, p32
    return probe_peak(torch, True, dev), probe_peak(torch, False, dev)


def _common(args, metric, value, unit, dtype, config, extra):
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": dtype, "data": "synthetic", "config": config}
    line.update(extra)
    print(json.dumps(line), flush=True)


def batch_cpu_baseline(reqs, seconds_target=12.0, max_object_steps=200000):
    """Oracle (CPU FP64 restatement, OpenMP over objects) on whole requests of the batch, in a
    seeded random order, until about seconds_target of CPU work; requests of more than
    max_object_steps object-steps are left out of the sample. Returns object-steps/s, cores and a
    description."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_api as O
    cores = cpu_cores()
    data = {}
    order = np.random.default_rng(SEED).permutation(len(reqs))
    done, osteps, t_all, used = 0, 0, 0.0, 0
    for i in order:
        q = reqs[i]
        n = q["r"].shape[0]
        if q["steps"] == 0 or n * q["steps"] > max_object_steps:
            continue
        L = q["degree"]
        if L not in data:
            data[L] = O.Data(degree=L)
        t0 = time.perf_counter()
        O.propagate(data[L], "gravity", q["start"], q["h"], q["steps"], q["r"], q["v"], threads=cores)
        t_all += time.perf_counter() - t0
        osteps += n * q["steps"]
        used += 1
        if t_all >= seconds_target:
            break
    return osteps / max(t_all, 1e-9), cores, ("%d of the %d requests (seeded random order; those of "
                                              "at most %d object-steps), %d object-steps, %.1f s of "
                                              "CPU work" % (used, len(reqs), max_object_steps, osteps,
                                                            t_all))


def adjoint_cpu_baseline(r, v, pairs, steps, seconds_target=12.0):
    """Miss-distance gradients on the CPU by central differences of the oracle (FP64, 25 runs of
    the pair per gradient, OpenMP over the runs): gradients per second on pairs taken in order
    until about seconds_target of CPU work."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_api as O
    data = O.Data()
    cores = cpu_cores()
    t_all, k = 0.0, 0
    while t_all < seconds_target and k < len(pairs):
        a, b = pairs[k]
        t0 = time.perf_counter()
        O.miss_fd_ld(data, START, H, steps, r[a], v[a], r[b], v[b], 1.0, 1e-3, threads=cores,
                     long=False)
        t_all += time.perf_counter() - t0
        k += 1
    return k / max(t_all, 1e-9), cores, ("%d pairs over %d steps, gradient by central differences "
                                         "(25 FP64 propagations of the pair each), %.1f s of CPU "
                                         "work" % (k, steps, t_all))


def run_batch(args, torch, G, dev):
    """Batched uneven requests: 4,096 requests in one persistent launch under a captured graph.
    Under torchrun the requests are split over the ranks by longest-processing-time bin packing of
    the cost model (no exchange while propagating); the time is the max over ranks."""
    import torch.distributed as dist
    from opengpop_b200 import orbits, sharding
    rank, world = env_int("RANK", 0), env_int("WORLD_SIZE", 1)
    all_reqs = orbits.batch_requests(args.batch_requests, SEED, max_days=args.batch_max_days)
    bins = sharding.lpt_partition([sharding.request_cost(q["r"].shape[0], q["steps"], q["degree"])
                                   for q in all_reqs], world)
    reqs = [all_reqs[i] for i in bins[rank]]
    osteps_all = sum(q["r"].shape[0] * q["steps"] for q in all_reqs)
    osteps = sum(q["r"].shape[0] * q["steps"] for q in reqs)
    f_total = sum(q["r"].shape[0] * q["steps"] * flops_per_object_step(q["degree"]) for q in reqs)
    f32 = sum(q["r"].shape[0] * q["steps"] * fp32_flops_per_object_step(q["degree"])
              for q in reqs if q["degree"] > 8)
    ctx = G.Context(device=dev.index, precision=G.MIXED)
    t0 = time.perf_counter()
    if not args.no_tune:
        ctx.tune()
    tune_s = time.perf_counter() - t0
    lpo, est = ctx.batch_plan(reqs)
    sampler = ClockSampler(torch.cuda.current_device())
    for _ in range(args.warmup):
        ctx.propagate_batch(reqs)
    sampler.start()
    dev_t, wall_t = [], []
    launches0 = ctx.kernel_launches
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ctx.propagate_batch(reqs)
        wall_t.append(time.perf_counter() - t0)
        dev_t.append(ctx.batch_device_seconds)
    clocks = sampler.stop()
    launches = ctx.kernel_launches - launches0
    warps = ctx.batch_warps_per_sm
    ctx.close()
    t = sharding.max_over_ranks(sum(dev_t) / len(dev_t), dev)
    t_wall = sharding.max_over_ranks(sum(wall_t) / len(wall_t), dev)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    peak64, peak32 = _peaks(torch, dev, clocks)
    cpu = None
    if not args.no_cpu_baseline:
        rate, cores, desc = batch_cpu_baseline(all_reqs)
        cpu = {"value": rate, "unit": "object-steps/s", "cores": cores, "kind": "port", "sample": desc}
    achieved = f_total / t / 1e12
    t_min = (f_total - f32) / (peak64 * 1e12) + f32 / (peak32 * 1e12) if peak64 and peak32 else None
    io = sum(q["r"].shape[0] for q in all_reqs) * 6 * 8
    args.gpus = world
    _common(args, "object-steps/s, batched uneven requests (mixed precision)", osteps_all / t,
            "object-steps/s", "f64+f32",
            {"workload": "%d requests (objects log-uniform 1-512, 1 h-7 d, h in {10,30,60,120} s, "
                         "degree in {8,20,36,70}, seed %d), one persistent launch per batch"
                         % (len(all_reqs), SEED),
             "object_steps_per_batch": osteps_all, "l2": "inputs (and state) larger than L2",
             "parallelism": "replicas" if world == 1 else "requests over %d ranks (LPT)" % world,
             "lanes_per_object_histogram": np.bincount(lpo, minlength=33)[[1, 2, 4, 8, 16, 32]].tolist(),
             "planner_estimate_s": est, "tune_s": tune_s},
            {"n_gpus": world, "scaling": "strong",
             "ms_per_step": 1e3 * t,
             "requests_per_s": len(all_reqs) / t,
             "e2e": {"value": osteps_all / t_wall, "unit": "object-steps/s",
                     "h2d_bytes_per_step": io, "d2h_bytes_per_step": io,
                     "call": "gpop_propagate_batch (host buffers, packing, copies)"},
             "roofline": {"bound": "fp64+fp32", "achieved": achieved,
                          "peak": f_total / t_min / 1e12 if t_min else None, "unit": "TFLOP/s",
                          "frac": achieved / (f_total / t_min / 1e12) if t_min else None,
                          "traffic": None},
             "warps_per_sm": warps,
             "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": launches})
    return 0


def run_screen(args, torch, G, dev):
    """Closest approach: 20,000 LEO objects, 2,000 seed-chosen objects against all (2,000
    singleton sets plus one set of 18,000: 37,999,000 pairs), 70x70, 30 s, 3 days, 5 km.
    Under torchrun each rank propagates its share of the objects, the ranks all-gather the
    trajectory in windows and each screens and refines its block of pair rows; every time is the
    max over ranks."""
    import torch.distributed as dist
    from opengpop_b200 import orbits, sharding
    rank, world = env_int("RANK", 0), env_int("WORLD_SIZE", 1)
    n, steps, thr = args.screen_objects, args.screen_steps, 5000.0
    n_sel = n // 10
    r, v = orbits.leo(n, SEED)
    sel = np.random.default_rng(SEED).choice(n, n_sel, replace=False)
    order = np.concatenate([sel, np.setdiff1d(np.arange(n), sel)])
    r, v = r[order], v[order]
    set_ids = np.concatenate([np.arange(n_sel), np.full(n - n_sel, n_sel)]).astype(np.uint32)
    ctx = G.Context(device=dev.index, precision=G.FP64)
    sampler = ClockSampler(torch.cuda.current_device())
    res = []
    launches0 = 0
    for i in range(args.warmup + args.steps):
        if i == args.warmup:
            sampler.start()
            launches0 = ctx.kernel_launches
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        if world == 1:
            ca = ctx.closest_approach(START, H, r, v, set_ids)
            ca.propagate(steps)
            recs = ca.find(thr)
            wall = time.perf_counter() - t0
            dt = list(ca.device_seconds())
            dt.insert(1, 0.0)
            pairs = ca.num_pairs
            ca.close()
        else:
            recs, sec = sharding.closest_approach_sharded(ctx, START, H, r, v, set_ids, [steps], thr)
            wall = time.perf_counter() - t0
            dt = [sec["propagation"], sec["exchange"], sec["screen"], sec["refinement"]]
            pairs = int(sharding.pairs_per_row(set_ids).sum())
        if i >= args.warmup:
            res.append((wall, dt))
    clocks = sampler.stop()
    launches = int(sharding.max_over_ranks(ctx.kernel_launches - launches0, dev))
    ctx.close()
    wall = sharding.max_over_ranks(float(np.mean([x[0] for x in res])), dev)
    t_prop, t_exch, t_screen, t_refine = (sharding.max_over_ranks(float(np.mean([x[1][k] for x in res])), dev)
                                          for k in range(4))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    args.gpus = world
    pair_steps = pairs * steps
    peak64 = _peaks(torch, dev, clocks)[0]
    cpu = None
    if not args.no_cpu_baseline:
        rate, cores, desc = screen_cpu_baseline(torch, G, r, v)
        cpu = {"value": rate, "unit": "pair-steps/s", "cores": cores, "kind": "port", "sample": desc}
    achieved = 9.0 * pair_steps / t_screen / 1e12
    _common(args, "conjunction pair-steps/s of the screen (FP64)", pair_steps / t_screen,
            "pair-steps/s", "f64",
            {"workload": "%d LEO objects (seed %d), %d vs all = %d pairs, 70x70, 30 s, "
                         "%d steps, threshold 5 km" % (n, SEED, n_sel, pairs, steps),
             "pairs": pairs, "steps": steps,
             "l2": "trajectory store %.1f GB" % (n * steps * 72 / 1e9),
             "parallelism": "one GPU" if world == 1 else
             "object shards x%d, trajectory all-gather per 240 steps, pair rows x%d" % (world, world)},
            {"n_gpus": world, "scaling": "strong", "ms_per_step": 1e3 * wall,
             "device_seconds": {"propagation": t_prop, "exchange": t_exch, "screen": t_screen,
                                "refinement": t_refine},
             "pairs_per_s_whole_job": pairs / wall,
             "found_below_threshold": len(recs),
             "e2e": {"value": pair_steps / wall, "unit": "pair-steps/s",
                     "h2d_bytes_per_step": n * 6 * 8 + n * 4, "d2h_bytes_per_step": len(recs) * 64,
                     "call": "gpop_ca_create + gpop_ca_propagate + gpop_ca_find" if world == 1 else
                     "sharding.closest_approach_sharded (gpop_propagator_step, NCCL all-gather, "
                     "gpop_ca_append, gpop_ca_find)"},
             "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                          "frac": achieved / peak64 if peak64 else None, "traffic": None,
                          "per_unit": "9 FP64 flops per pair-step"},
             "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": launches})
    return 0


def run_adjoint(args, torch, G, dev):
    """Differentiation: 10,000 pairs (24 h, 30 s, 70x70, FP64), adjoint gradient of each miss
    distance; and 8,192 state transition matrices by the forward variational equations."""
    from opengpop_b200 import orbits
    n_pairs, steps = args.adjoint_pairs, args.adjoint_steps
    r, v, pairs = orbits.conjunction_pairs(n_pairs, SEED)
    n_stm = min(args.stm_objects, r.shape[0])  # the STMs run on the pairs' first objects
    ctx = G.Context(precision=G.FP64)
    sampler = ClockSampler(torch.cuda.current_device())
    t_miss, t_stm = [], []
    launches0 = 0
    for i in range(args.warmup + args.steps):
        if i == args.warmup:
            sampler.start()
            launches0 = ctx.kernel_launches
        t0 = time.perf_counter()
        ctx.miss_gradient(START, H, steps, r, v, pairs)
        t1 = time.perf_counter()
        ctx.stm(START, H, steps, r[:n_stm], v[:n_stm])
        t2 = time.perf_counter()
        if i >= args.warmup:
            t_miss.append(t1 - t0)
            t_stm.append(t2 - t1)
    clocks = sampler.stop()
    launches = ctx.kernel_launches - launches0
    ctx.close()
    tm, ts = float(np.mean(t_miss)), float(np.mean(t_stm))
    # work of the miss-gradient call: forward propagation of 2 n_pairs objects, then per unit
    # (pair side) a recomputed forward pass (7 W + 500 per step), the reverse pass (one Jacobian
    # per step) and the tangent startup (145 Jacobian evaluations); of the STM: the primal step,
    # one Jacobian and six tangent steps per object-step
    W = 24 * terms(DEGREE) + 15 * DEGREE + 60
    units = 2 * n_pairs
    f_miss = units * steps * (2 * flops_per_object_step() + w_jac(DEGREE)) + units * 145 * w_jac(DEGREE)
    f_stm = n_stm * steps * (flops_per_object_step() + w_jac(DEGREE) + 6 * 500) + n_stm * 145 * w_jac(DEGREE)
    peak64 = _peaks(torch, dev, clocks)[0]
    cpu = None
    if not args.no_cpu_baseline:
        rate, cores, desc = adjoint_cpu_baseline(r, v, pairs, steps)
        cpu = {"value": rate, "unit": "pairs/s", "cores": cores, "kind": "port", "sample": desc}
    ach = f_miss / tm / 1e12
    _common(args, "miss-distance gradients/s (adjoint, FP64)", n_pairs / tm, "pairs/s", "f64",
            {"workload": "%d LEO pairs (seed %d), 70x70, 30 s, %d steps (24 h), checkpoint every 64 "
                         "steps; %d STMs over the same span" % (n_pairs, SEED, steps, n_stm)},
            {"ms_per_step": 1e3 * tm,
             "stm": {"value": n_stm * steps / ts, "unit": "object-steps/s (with 6x6 STM)",
                     "seconds": ts, "roofline_frac": (f_stm / ts / 1e12) / peak64 if peak64 else None},
             "e2e": {"value": n_pairs / tm, "unit": "pairs/s", "h2d_bytes_per_step": units * 48,
                     "d2h_bytes_per_step": n_pairs * 14 * 8, "call": "gpop_miss_gradient"},
             "roofline": {"bound": "fp64", "achieved": ach, "peak": peak64, "unit": "TFLOP/s",
                          "frac": ach / peak64 if peak64 else None, "traffic": None,
                          "per_unit": "per unit-step 2 (7 W + 500) + W_J, W(70) = %d, "
                                      "W_J(70) = %d flops" % (W, w_jac(DEGREE))},
             "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": launches})
    return 0


def accuracy_7d(G, n_sample):
    """Mixed vs FP64 position error after 7 days (20,160 steps) on n_sample objects spread over
    the population, propagated together (at the default, the whole population: the kernels and
    launch shapes of the headline)."""
    from opengpop_b200 import orbits
    r, v = orbits.mixed_population(N_OBJECTS, SEED)
    idx = np.linspace(0, N_OBJECTS - 1, n_sample).astype(int)
    out = {}
    for name, prec in (("fp64", G.FP64), ("mixed", G.MIXED)):
        c = G.Context(precision=prec)
        out[name] = c.propagate(START, H, 20160, r[idx], v[idx])
        c.close()
    err = np.linalg.norm(out["mixed"][0] - out["fp64"][0], axis=1)
    return {"objects": int(n_sample), "days": 7, "steps": 20160, "max_m": float(err.max()),
            "p99_m": float(np.percentile(err, 99)), "median_m": float(np.median(err)),
            "bound_m": 1.0}


def screen_problem(n=20000, seed=SEED):
    """The closest-approach configuration: n LEO objects, n/10 seed-chosen objects first as
    singleton sets, the rest one set (each chosen object against all others)."""
    from opengpop_b200 import orbits
    n_sel = n // 10
    r, v = orbits.leo(n, seed)
    sel = np.random.default_rng(seed).choice(n, n_sel, replace=False)
    order = np.concatenate([sel, np.setdiff1d(np.arange(n), sel)])
    set_ids = np.concatenate([np.arange(n_sel), np.full(n - n_sel, n_sel)]).astype(np.uint32)
    return r[order], v[order], set_ids


def screen_cpu_baseline(torch, G, r, v, rows=40, window=240, seconds_target=10.0):
    """Oracle screen (CPU FP64 restatement of UpdateClosestApproachKernel, OpenMP over pairs) on a
    row sample of the closest-approach configuration: `rows` set objects against all others over
    the first steps of the GPU trajectory. Returns pair-steps/s, cores and a description."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_api as O
    n = r.shape[0]
    ctx = G.Context(precision=G.FP64)
    rd = torch.tensor(r, dtype=torch.float64, device="cuda")
    vd = torch.tensor(v, dtype=torch.float64, device="cuda")
    prop = ctx.propagator(START, H, window, rd, vd)
    tr = torch.empty((window, 3, n), dtype=torch.float64, device="cuda")
    tv, ta = torch.empty_like(tr), torch.empty_like(tr)
    prop.step(window, tr, tv, ta)
    torch.cuda.synchronize()
    arrs = [np.ascontiguousarray(x.cpu().numpy().transpose(0, 2, 1)) for x in (tr, tv, ta)]
    prop.close()
    ctx.close()
    ids = np.concatenate([np.arange(rows), np.full(n - rows, rows)]).astype(np.uint32)
    part = O.partition(ids)
    P = int(part["num_pairs"])
    cores = cpu_cores()

    def run(steps):
        # `steps` screened steps: the window's steps, the window again (the state carries on) as
        # often as needed
        md = np.zeros(P)
        cs = np.zeros(P, np.uint32)
        nodes = np.zeros(P * 54)
        last = np.zeros(n * 9)
        st = O.OrCaState(md.ctypes.data, cs.ctypes.data, nodes.ctypes.data, last.ctypes.data)
        t0 = time.perf_counter()
        done = 0
        while done < steps:
            k = min(window, steps - done)
            O.lib().or_ca_screen(n, k, O.ptr(arrs[0]), O.ptr(arrs[1]), O.ptr(arrs[2]), O.ptr(ids),
                                 done, int(done == 0), C.byref(st), cores)
            done += k
        return time.perf_counter() - t0

    steps = 8
    for _ in range(4):  # the first runs are dominated by the state set-up: scale until the work dominates
        dt = run(steps)
        if dt >= 0.5 * seconds_target:
            break
        steps = int(steps * seconds_target / max(dt, 1e-3))
    return P * steps / dt, cores, ("%d set objects against the other %d objects (%d pairs) x %d "
                                   "steps (the first %d steps of the GPU trajectory, repeated), "
                                   "%.1f s of CPU work" % (rows, n - rows, P, steps, window, dt))


def screen_leg(torch, G, dev, steps, warmup=1, cpu=True):
    """One closest-approach job of the configuration (20,000 LEO objects, 2,000 against all,
    `steps` 30 s steps, 5 km) through the public calls: host buffers in, records out."""
    r, v, set_ids = screen_problem()
    n = r.shape[0]
    res = None
    ctx = G.Context(device=dev.index, precision=G.FP64)
    launches0 = 0
    for i in range(warmup + 1):
        if i == warmup:
            launches0 = ctx.kernel_launches
        t0 = time.perf_counter()
        ca = ctx.closest_approach(START, H, r, v, set_ids)
        ca.propagate(steps)
        recs = ca.find(5000.0)
        wall = time.perf_counter() - t0
        secs = ca.device_seconds()
        pairs = ca.num_pairs
        ca.close()
        res = (wall, secs, len(recs))
    launches = ctx.kernel_launches - launches0
    ctx.close()
    wall, secs, found = res
    pair_steps = pairs * steps
    out = {"value": pair_steps / secs[1], "unit": "pair-steps/s",
           "what": "screen kernel: pairs x steps / device time of the screen (CUDA events)",
           "workload": "%d LEO objects (seed %d), %d against all = %d pairs, 70x70, 30 s, %d steps, "
                       "threshold 5 km, FP64" % (n, SEED, n // 10, pairs, steps),
           "pairs_per_s_whole_job": pairs / wall, "job_seconds": wall,
           "device_seconds": {"propagation": float(secs[0]), "screen": float(secs[1]),
                              "refinement": float(secs[2])},
           "found_below_threshold": found, "gpu_launches": launches,
           "e2e": {"value": pair_steps / wall, "unit": "pair-steps/s",
                   "h2d_bytes_per_step": n * 6 * 8 + n * 4, "d2h_bytes_per_step": found * 64,
                   "call": "gpop_ca_create + gpop_ca_propagate + gpop_ca_find (host buffers)"}}
    if cpu:
        rate, cores, desc = screen_cpu_baseline(torch, G, r, v)
        out["cpu_baseline"] = {"value": rate, "unit": "pair-steps/s", "cores": cores, "kind": "port",
                               "sample": desc}
    return out


def reference_cuda_rate(n=16384, s1=8, s2=40):
    """The reference's own CUDA build (compiled from its sources into oracle/_ref/libref.so), timed
    on this GPU in child processes: object-steps/s of its step loop from two durations (startup
    cancels), FP64 at 70x70 on n objects of the mixed population. None when that build is absent."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import ref_build_runner as RB
    from opengpop_b200 import orbits
    if not RB.available():
        return None
    r0, v0 = orbits.mixed_population(n, SEED)
    RB.run("propagate", START, H, 2, r0[:256], v0[:256])  # loads its kernels
    t = [min(float(RB.run("propagate", START, H, s, r0, v0)["ms"]) * 1e-3 for _ in range(2))
         for s in (s1, s2)]
    rate = n * (s2 - s1) / max(t[1] - t[0], 1e-9)
    return {"value": rate, "unit": "object-steps/s", "kind": "reference CUDA build",
            "sample": "%d objects of the mixed population, 70x70, 30 s, FP64; step loop of %d and %d "
                      "steps (CUDA events), rate from the difference" % (n, s1, s2)}


def clock_peaks(sm_mhz, dev):
    """FP64 and FP32 FMA peaks (TFLOP/s) from the SM count and the SM clock sampled under load:
    64 FP64 and 128 FP32 FMAs per SM per cycle."""
    import torch
    if not sm_mhz:
        return None, None
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    return sms * 64 * 2 * sm_mhz * 1e6 / 1e12, sms * 128 * 2 * sm_mhz * 1e6 / 1e12


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 10; batch 2, screen and adjoint 1)")
    ap.add_argument("--warmup", type=int, default=None,
                    help="warm-up steps (default 3; batch, screen and adjoint 1)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--prop-steps", type=int, default=64, help="GJ8 steps per bench step")
    ap.add_argument("--objects", type=int, default=N_OBJECTS)
    ap.add_argument("--e2e-steps", type=int, default=960, help="GJ8 steps per e2e call")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="propagate",
                    choices=["propagate", "batch", "screen", "adjoint"],
                    help="propagate: the headline line; the others print their own line (1 GPU)")
    ap.add_argument("--batch-requests", type=int, default=4096)
    ap.add_argument("--batch-max-days", type=float, default=7.0)
    ap.add_argument("--no-tune", action="store_true", help="batch: plan with the untuned model")
    ap.add_argument("--screen-objects", type=int, default=20000)
    ap.add_argument("--screen-steps", type=int, default=8640)
    ap.add_argument("--adjoint-pairs", type=int, default=10000)
    ap.add_argument("--adjoint-steps", type=int, default=2880)
    ap.add_argument("--stm-objects", type=int, default=8192)
    ap.add_argument("--accuracy-objects", type=int, default=N_OBJECTS,
                    help="objects of the 7-day mixed-vs-FP64 error sample (0 = skip)")
    ap.add_argument("--no-screen", action="store_true",
                    help="headline: skip the closest-approach job (conj pairs/s)")
    ap.add_argument("--no-reference-cuda", action="store_true",
                    help="headline: skip timing the reference's own CUDA build")
    args = ap.parse_args()
    short = args.workload != "propagate"  # whole-job workloads of several seconds per step
    if args.steps is None:
        args.steps = {"batch": 2, "screen": 1, "adjoint": 1}.get(args.workload, 10)
    if args.warmup is None:
        args.warmup = 1 if short else 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload != "propagate":
        import torch
        import opengpop_b200 as G
        dev = torch.device("cuda", env_int("LOCAL_RANK", 0))
        torch.cuda.set_device(dev)
        if args.workload in ("batch", "screen"):
            if env_int("WORLD_SIZE", 1) > 1:
                import datetime
                import torch.distributed as dist
                dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
            return (run_batch if args.workload == "batch" else run_screen)(args, torch, G, dev)
        if env_int("RANK", 0) != 0:
            return 0
        return run_adjoint(args, torch, G, dev)

    import torch
    import torch.distributed as dist
    import opengpop_b200 as G
    from opengpop_b200 import orbits

    rank = env_int("RANK", 0)
    world = env_int("WORLD_SIZE", 1)
    local = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
    n = args.objects
    r0, v0 = orbits.mixed_population(n, SEED + rank)
    total_steps = (args.warmup + args.steps) * args.prop_steps + 1

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def run(precision):
        ctx = G.Context(device=local, precision=precision)
        r = torch.tensor(r0, dtype=torch.float64, device=dev)
        v = torch.tensor(v0, dtype=torch.float64, device=dev)
        prop = ctx.propagator(START, H, total_steps, r, v)
        stream = torch.cuda.current_stream()
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
        prop.step(1)  # startup (RK8 + 7 corrector passes) + step 1
        for _ in range(args.warmup):
            prop.step(args.prop_steps)
        torch.cuda.synchronize()
        barrier()
        launches0 = ctx.kernel_launches
        times = []
        for _ in range(args.steps):
            flush.fill_(1.0)  # L2 flush between timed steps (256 MB > 126 MB L2)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            prop.step(args.prop_steps)
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) * 1e-3)
        barrier()
        launches = ctx.kernel_launches - launches0
        rv = float(r.abs().sum().item())
        prop.close()
        ctx.close()
        return times, launches, rv

    sampler = ClockSampler(local)
    sampler.start()
    times_mixed, launches_mixed, chk_m = run(G.MIXED)
    times_fp64, launches_fp64, chk_d = run(G.FP64)
    clocks = sampler.stop()

    t_mixed = max_over_ranks(sum(times_mixed))
    t_fp64 = max_over_ranks(sum(times_fp64))
    osteps = n * args.prop_steps * args.steps
    value = world * osteps / t_mixed
    value_fp64 = world * osteps / t_fp64

    # ---- end to end through the public call (host pinned in/out) ----
    ctx = G.Context(device=local, precision=G.MIXED)
    rin = torch.tensor(r0, dtype=torch.float64).pin_memory()
    vin = torch.tensor(v0, dtype=torch.float64).pin_memory()
    rout = torch.empty_like(rin).pin_memory()
    vout = torch.empty_like(vin).pin_memory()
    rin_np, vin_np, rout_np, vout_np = (x.numpy() for x in (rin, vin, rout, vout))
    e2e_steps = args.e2e_steps
    ctx.propagate(START, H, e2e_steps, rin_np, vin_np)  # warm-up call
    barrier()
    e2e_calls = max(1, min(args.steps, 3))
    t0 = time.perf_counter()
    for _ in range(e2e_calls):
        lib = G.load_library()
        st = lib.gpop_propagate(ctx._h, C.byref(G.as_time(START)), H, e2e_steps, n,
                                rin_np.ctypes.data_as(C.c_void_p), vin_np.ctypes.data_as(C.c_void_p),
                                rout_np.ctypes.data_as(C.c_void_p),
                                vout_np.ctypes.data_as(C.c_void_p))
        ctx._check(st)
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    e2e_value = world * n * e2e_steps * e2e_calls / t_e2e
    ctx.close()

    # ---- roofline of the dominant kernel (the mixed GJ8 kernel) ----
    # denominators: the FMA rates per SM and cycle at the SM clock sampled during the timed runs
    # (the probe's live FMA-chain figures are reported beside them)
    probe64 = probe_peak(torch, True, dev)
    probe32 = probe_peak(torch, False, dev)
    pipes = probe_pipes(torch, dev)
    peak64, peak32 = clock_peaks(clocks.get("sm_mhz"), dev)
    if not peak64:
        peak64, peak32 = probe64, probe32
    launch_t = sum(times_mixed) / max(1, launches_mixed)
    steps_per_launch = args.prop_steps * args.steps / max(1, launches_mixed)
    f_total = flops_per_object_step() * n * steps_per_launch
    f32 = fp32_flops_per_object_step() * n * steps_per_launch
    f64 = f_total - f32
    achieved = f_total / launch_t / 1e12
    t_min = f64 / (peak64 * 1e12) + f32 / (peak32 * 1e12) if peak64 and peak32 else None
    eff_peak = f_total / t_min / 1e12 if t_min else None
    fp64_launch_t = sum(times_fp64) / max(1, launches_fp64)
    fp64_achieved = flops_per_object_step() * n * steps_per_launch / fp64_launch_t / 1e12

    accuracy = accuracy_7d(G, args.accuracy_objects) if args.accuracy_objects > 0 and rank == 0 else None
    # the metric's second half (conj pairs/s) and the reference's CUDA build: one GPU only
    screen = None
    if world == 1 and not args.no_screen:
        screen = screen_leg(torch, G, dev, args.screen_steps, cpu=not args.no_cpu_baseline)
        screen["roofline"] = {"bound": "fp64", "achieved": 9.0 * screen["value"] / 1e12,
                              "peak": peak64, "unit": "TFLOP/s",
                              "frac": 9.0 * screen["value"] / 1e12 / peak64 if peak64 else None,
                              "traffic": None, "per_unit": "9 FP64 flops per pair-step"}
    ref_cuda = None
    if world == 1 and not args.no_reference_cuda:
        try:
            ref_cuda = reference_cuda_rate()
        except Exception as e:  # the reference build exits on its own errors; report, do not fail
            ref_cuda = {"unavailable": str(e)[:200]}

    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline:
            rate, cores, desc = cpu_baseline()
            cpu = {"value": rate, "unit": "object-steps/s", "cores": cores, "kind": "port",
                   "sample": desc}
        line = {
            "metric": METRIC,
            "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_mixed / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
            "data": "synthetic",
            "config": {"workload": "65,536 objects (70%% LEO / 20%% MEO / 10%% GEO, seed %d), "
                                   "70x70 JGM3, 30 s GJ8 step, %d GJ8 steps per bench step"
                                   % (SEED, args.prop_steps),
                       "objects_per_gpu": n, "degree": DEGREE, "step_s": H,
                       "l2": "flushed (256 MB write) between timed steps",
                       "parallelism": "replicas" if world == 1 else "object shards x%d" % world},
            "fp64": {"value": value_fp64, "unit": "object-steps/s",
                     "ms_per_step": 1e3 * t_fp64 / args.steps,
                     "roofline": {"bound": "fp64", "achieved": fp64_achieved, "peak": peak64,
                                  "unit": "TFLOP/s",
                                  "frac": fp64_achieved / peak64 if peak64 else None,
                                  "frac_vs_probe": fp64_achieved / probe64 if probe64 else None}},
            "mixed_vs_fp64": value / value_fp64,
            "accuracy_7d": accuracy,
            "e2e": {"value": e2e_value, "unit": "object-steps/s",
                    "h2d_bytes_per_step": 2 * n * 3 * 8, "d2h_bytes_per_step": 2 * n * 3 * 8,
                    "call": "gpop_propagate, %d GJ8 steps per call incl. startup" % e2e_steps},
            "roofline": {"bound": "fp64+fp32", "achieved": achieved, "peak": eff_peak,
                         "unit": "TFLOP/s", "frac": achieved / eff_peak if eff_peak else None,
                         "traffic": MIXED_GJ8_DRAM_BYTES,
                         "traffic_note": "a stated constant, not measured in this run: dram "
                                         "read+write bytes of one launch of this kernel from an "
                                         "ncu capture (65,536 objects, 4-step launch; the state "
                                         "is read once per launch, later steps hit L2); "
                                         "algorithmic state bytes per launch %d" % (600 * n),
                         "peak_note": "not in MEASURED_PEAKS.json (HBM and bf16 only): SMs x "
                                      "(64 FP64 | 128 FP32 FMAs per cycle) x 2 x the median SM "
                                      "clock sampled during the timed runs",
                         "frac_vs_probe": (achieved / (f_total / (f64 / (probe64 * 1e12)
                                                                  + f32 / (probe32 * 1e12)) / 1e12)
                                           if probe64 and probe32 else None),
                         "peaks_measured": {"fp64_tflops": probe64, "fp32_tflops": probe32,
                                            "how": "live FMA-chain probe (libgpop_probe.so)"},
                         "peaks_clock": {"fp64_tflops": peak64, "fp32_tflops": peak32},
                         "fp64_beside_fp32_probe": pipes},
            "cpu_baseline": cpu,
            "screen": screen,
            "reference_cuda": ref_cuda,
            "clocks": clocks,
            "gpu_launches": launches_mixed,
            "checksum": [chk_m, chk_d],
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
