"""Parity with the reference's own CUDA build (oracle/_ref/libref.so, compiled from the reference
sources by oracle/ref/build.sh) on the same inputs, on the GPU. Skipped when that build is absent.
Each test prints the reference build's step-loop time next to this build's for the same case."""
import numpy as np
import pytest

import ref_build_runner as RB

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not RB.available(), reason="reference build not present")]

START = (2024, 1, 1, 0, 0, 0.0)


def test_propagation_matches_reference_build_1day():
    import time
    import torch
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    r0, v0 = orbits.mixed_population(64, seed=41)
    steps, h = 2880, 30.0  # 1 day
    ref = RB.run("propagate", START, h, steps, r0, v0)
    ctx = G.Context()
    r = torch.tensor(r0, dtype=torch.float64, device="cuda")
    v = torch.tensor(v0, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.propagate_device(START, h, steps, r, v)
    torch.cuda.synchronize()
    t_ours = time.perf_counter() - t0
    err = np.abs(r.cpu().numpy() - ref["r"]).max()
    verr = np.abs(v.cpu().numpy() - ref["v"]).max()
    print("\n64 objects x 1 day: |dr| max %.3e m, |dv| max %.3e m/s; reference step loop %.1f ms, "
          "this build %.1f ms (incl. startup)" % (err, verr, float(ref["ms"]), 1e3 * t_ours))
    assert err < 1e-2  # 1 cm
    assert verr < 1e-5


def test_propagation_matches_reference_build_20x20():
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    r0, v0 = orbits.leo(32, seed=42)
    steps, h = 1440, 60.0  # the 1,024-object configuration's 20x20 / 60 s / 24 h, on 32 objects
    ref = RB.run("propagate", START, h, steps, r0, v0, degree=20)
    ctx = G.Context(gravity_degree=20)
    r, v = ctx.propagate(START, h, steps, r0, v0)
    assert np.abs(r - ref["r"]).max() < 1e-2
    assert np.abs(v - ref["v"]).max() < 1e-5


def test_closest_approach_matches_reference_build():
    # One object against 31: all 31 pairs sit in one warp of the reference's screen kernel, so its
    # racy "last" arrays (device.cu:87-90) are read before they are overwritten and the
    # reference's own refinement is valid for every pair.
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    n = 32
    r0, v0 = orbits.leo(n, seed=43)
    r0[1:9] = r0[0] + np.array([[800.0 * k, -500.0, 250.0 + 30 * k] for k in range(1, 9)])
    v0[1:9] = v0[0] * (1.0 + 3e-6 * np.arange(1, 9))[:, None]
    sets = np.array([0] + [1] * (n - 1), np.uint32)
    steps, h = 240, 30.0
    ref = RB.run("ca", START, h, steps, r0, v0, set_ids=sets)
    ctx = G.Context()
    ca = ctx.closest_approach(START, h, r0, v0, sets)
    ca.propagate(steps)
    recs = ca.find()
    assert [(x.object_index1, x.object_index2) for x in recs] == list(zip(ref["obj1"], ref["obj2"]))
    d = np.array([x.distance for x in recs])
    t = np.array([x.time for x in recs])
    close = ref["distance"] < 20e3
    assert close.sum() >= 6
    # parity bar of the closest-approach path: TCA within 1 ms, miss distance within 1 m
    assert np.abs(t[close] - ref["time"][close]).max() < 1e-3
    assert np.abs(d[close] - ref["distance"][close]).max() < 1.0


def test_fp64_build_at_least_as_fast_as_reference_build():
    # the plain FP64 build against the reference's CUDA build on 16,384 objects of the mixed
    # population at 70x70; the step-loop rate comes from two durations (startup cancels)
    import time
    import torch
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    n, h, s1, s2 = 16384, 30.0, 8, 40
    r0, v0 = orbits.mixed_population(n, seed=42)
    # the first run of a fresh process loads (and may JIT) the reference's kernels inside its
    # timed loop, so a short run goes first and each duration is the shorter of two runs
    RB.run("propagate", START, h, 2, r0[:256], v0[:256])
    t_ref = [min(float(RB.run("propagate", START, h, s, r0, v0)["ms"]) * 1e-3 for _ in range(2))
             for s in (s1, s2)]
    assert t_ref[1] > t_ref[0], "reference build timings not ordered: %s" % t_ref
    ctx = G.Context(precision=G.FP64)
    t_ours = []
    for s in (s1, s2):
        r = torch.tensor(r0, dtype=torch.float64, device="cuda")
        v = torch.tensor(v0, dtype=torch.float64, device="cuda")
        ctx.propagate_device(START, h, 4, r.clone(), v.clone())  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.propagate_device(START, h, s, r, v)
        torch.cuda.synchronize()
        t_ours.append(time.perf_counter() - t0)
    ctx.close()
    rate_ref = n * (s2 - s1) / max(t_ref[1] - t_ref[0], 1e-9)
    rate_ours = n * (s2 - s1) / max(t_ours[1] - t_ours[0], 1e-9)
    print("\n%d objects, 70x70: reference CUDA build %.3e object-steps/s, this FP64 build %.3e "
          "(x%.1f)" % (n, rate_ref, rate_ours, rate_ours / rate_ref))
    assert rate_ours >= rate_ref
