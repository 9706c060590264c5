"""The GJ8 walks of the propagation kernels (one or two objects per thread; 4..32 lanes per object;
two lanes per pair of objects) give the same propagation to rounding, FP64 and mixed, and the
FP64 walks agree with the CPU oracle. The walk is forced per context with GPOP_WALK_MODE."""
import os

import numpy as np
import pytest

import oracle_api as O

pytestmark = pytest.mark.gpu

START = (2024, 1, 1, 0, 0, 0.0)


def _run(walk, precision, r, v, steps):
    import opengpop_b200 as G
    old = os.environ.get("GPOP_WALK_MODE")
    os.environ["GPOP_WALK_MODE"] = str(walk)
    try:
        c = G.Context(precision=precision)
    finally:
        if old is None:
            del os.environ["GPOP_WALK_MODE"]
        else:
            os.environ["GPOP_WALK_MODE"] = old
    try:
        return c.propagate(START, 30.0, steps, r, v)
    finally:
        c.close()


@pytest.mark.parametrize("n", [37, 3000, 20000])
@pytest.mark.parametrize("precision", [0, 1])
def test_walks_agree(n, precision):
    from opengpop_b200 import orbits
    r, v = orbits.mixed_population(n, seed=60 + n)
    steps = 40
    ref_r, ref_v = _run(2, precision, r, v, steps)  # two objects per thread
    for walk in (1, 3, 4):
        rr, vv = _run(walk, precision, r, v, steps)
        # summation order differs between walks: FP64 agrees to rounding; the mixed walks differ
        # by FP32 rounding of the degree > 8 sums
        tol_r, tol_v = (1e-6, 1e-9) if precision == 0 else (1e-3, 1e-6)
        assert np.abs(rr - ref_r).max() < tol_r, (walk, np.abs(rr - ref_r).max())
        assert np.abs(vv - ref_v).max() < tol_v


def test_lane_walks_match_oracle(oracle_data):
    from opengpop_b200 import orbits
    r, v = orbits.mixed_population(24, seed=71)
    steps = 30
    ro, vo = O.propagate(oracle_data, "gravity", START, 30.0, steps, r, v)
    for walk in (3, 4):
        rr, vv = _run(walk, 0, r, v, steps)
        assert np.abs(rr - ro).max() < 1e-6 and np.abs(vv - vo).max() < 1e-9


@pytest.mark.parametrize("n", [40000, 50000, 65536])
@pytest.mark.parametrize("precision", [0, 1])
def test_split_block_agrees_with_plain_block_and_oracle(n, precision, oracle_data):
    """Two objects per thread at 5 to 7 sets of 64 objects per SM run in the split block (owner
    warps carry the objects and walk the gravity columns m >= 4, the other warps walk columns
    0..3 of the owners' objects). The low and high column totals are formed apart and added, so
    the propagation matches the plain two-object block to rounding, not bit for bit; objects
    taken across the whole range (first and second slot of a thread, block ends, the last
    object) match the CPU oracle."""
    import torch
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    per_sm = -(-n // sms)
    assert G.split_block(n, sms) == (-(-per_sm // 64) if 4 < -(-per_sm // 64) < 8 else 0)
    r, v = orbits.mixed_population(n, seed=80 + n % 7)
    steps = 12
    ref_r, ref_v = _run(5, precision, r, v, steps)  # plain block
    rr, vv = _run(2, precision, r, v, steps)  # split block where the sizes call for it
    assert np.abs(rr - ref_r).max() < 1e-6, np.abs(rr - ref_r).max()
    assert np.abs(vv - ref_v).max() < 1e-9
    if precision == 0:
        gown = sms * 32 * max(G.split_block(n, sms), 1)
        pick = np.unique(np.clip(np.r_[0, 1, 31, 32, 223, 224, gown - 1, gown, gown + 1,
                                       n // 3, n // 2, n - 2, n - 1,
                                       np.linspace(0, n - 1, 24).astype(int)], 0, n - 1))
        ro, vo = O.propagate(oracle_data, "gravity", START, 30.0, steps, r[pick], v[pick])
        assert np.abs(rr[pick] - ro).max() < 1e-6, np.abs(rr[pick] - ro).max()
        assert np.abs(vv[pick] - vo).max() < 1e-9


@pytest.mark.parametrize("n,precision", [(4096, 0), (20000, 0), (9472, 1), (20000, 1)])
def test_lane_pair_walk(n, precision, oracle_data):
    """Lanes per group of two objects, the default walk in its bands: 20,000 FP64 objects run as
    18,944 in a wave of 8 warps per SM with four lanes per group and the other 1,056 in a second
    launch with more lanes. The propagation matches the one-object lane walk to rounding, and
    FP64 objects from both launches match the CPU oracle."""
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    assert G.walk_policy(n, 148, precision)[0] == 4
    r, v = orbits.mixed_population(n, seed=90 + n % 11)
    steps = 12
    ref_r, ref_v = _run(3, precision, r, v, steps)  # lanes per object
    rr, vv = _run(0, precision, r, v, steps)  # default: lanes per group of two objects
    tol_r, tol_v = (1e-6, 1e-9) if precision == 0 else (1e-3, 1e-6)
    assert np.abs(rr - ref_r).max() < tol_r, np.abs(rr - ref_r).max()
    assert np.abs(vv - ref_v).max() < tol_v
    if precision == 0:
        pick = np.unique(np.clip(np.r_[0, 1, 2, 3, n // 2, 18943, 18944, 18945, n - 2, n - 1,
                                       np.linspace(0, n - 1, 20).astype(int)], 0, n - 1))
        ro, vo = O.propagate(oracle_data, "gravity", START, 30.0, steps, r[pick], v[pick])
        assert np.abs(rr[pick] - ro).max() < 1e-6, np.abs(rr[pick] - ro).max()
        assert np.abs(vv[pick] - vo).max() < 1e-9


@pytest.mark.parametrize("precision", [0, 1])
def test_more_objects_than_one_wave(precision, oracle_data):
    """100,000 objects: one wave of 8 warps per SM at two objects per thread (75,776 objects on 148
    SMs), then the other 24,224 with the walk their own number takes (FP64: two lanes per object;
    mixed: two objects per thread). Matches the plain two-object block over all objects to
    rounding, and FP64 objects on both sides of the boundary match the CPU oracle."""
    import torch
    from opengpop_b200 import orbits
    n = 100000
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    r, v = orbits.mixed_population(n, seed=97)
    steps = 12
    ref_r, ref_v = _run(5, precision, r, v, steps)  # plain block over all objects
    rr, vv = _run(0, precision, r, v, steps)
    tol_r, tol_v = (1e-6, 1e-9) if precision == 0 else (1e-3, 1e-6)
    assert np.abs(rr - ref_r).max() < tol_r, np.abs(rr - ref_r).max()
    assert np.abs(vv - ref_v).max() < tol_v
    if precision == 0:
        wave = sms * 512
        pick = np.unique(np.clip(np.r_[0, 1, wave // 2, wave - 2, wave - 1, wave, wave + 1,
                                       n - 2, n - 1, np.linspace(0, n - 1, 16).astype(int)],
                                 0, n - 1))
        ro, vo = O.propagate(oracle_data, "gravity", START, 30.0, steps, r[pick], v[pick])
        assert np.abs(rr[pick] - ro).max() < 1e-6, np.abs(rr[pick] - ro).max()
        assert np.abs(vv[pick] - vo).max() < 1e-9


def test_split_block_trajectory():
    """The trajectory outputs of the split block (positions, velocities and accelerations of
    every step, [step][xyz][object]) match the plain two-object block's to rounding at 40,000
    objects (5 owner warps per SM)."""
    import torch
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    n, steps = 40000, 10
    r0, v0 = orbits.mixed_population(n, seed=41)
    out = {}
    for walk in (5, 2):
        os.environ["GPOP_WALK_MODE"] = str(walk)
        try:
            c = G.Context(precision=G.FP64)
        finally:
            del os.environ["GPOP_WALK_MODE"]
        r = torch.tensor(r0, dtype=torch.float64, device="cuda")
        v = torch.tensor(v0, dtype=torch.float64, device="cuda")
        tr, tv, ta = (torch.zeros(steps, 3, n, dtype=torch.float64, device="cuda") for _ in range(3))
        c.propagate_trajectory(START, 30.0, steps, r, v, tr, tv, ta)
        torch.cuda.synchronize()
        out[walk] = [t.cpu().numpy() for t in (tr, tv, ta)]
        c.close()
    for a, b, tol in zip(out[5], out[2], (1e-6, 1e-9, 1e-12)):
        assert np.isfinite(b).all() and np.abs(a - b).max() < tol, np.abs(a - b).max()


def test_trajectory_over_more_than_one_wave():
    """80,000 FP64 objects (one wave of 75,776 at two objects per thread, then 4,224 in lanes per
    group of two objects): every step's trajectory row matches the plain two-object block over all
    objects to rounding."""
    import torch
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    n, steps = 80000, 8
    r0, v0 = orbits.mixed_population(n, seed=43)
    out = {}
    for walk in (5, 0):
        os.environ["GPOP_WALK_MODE"] = str(walk)
        try:
            c = G.Context(precision=G.FP64)
        finally:
            del os.environ["GPOP_WALK_MODE"]
        r = torch.tensor(r0, dtype=torch.float64, device="cuda")
        v = torch.tensor(v0, dtype=torch.float64, device="cuda")
        tr = torch.zeros(steps, 3, n, dtype=torch.float64, device="cuda")
        c.propagate_trajectory(START, 30.0, steps, r, v, tr)
        torch.cuda.synchronize()
        out[walk] = tr.cpu().numpy()
        c.close()
    assert np.isfinite(out[0]).all() and np.abs(out[0] - out[5]).max() < 1e-6


def test_compensated_sums_at_split_sizes():
    """The compensated mixed walk has no split-block form: at 40,000 objects it runs the plain
    block and agrees with the default mixed walk (split block) within the FP32 rounding of the
    degree > 8 sums."""
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    r0, v0 = orbits.mixed_population(40000, seed=44)
    ref = G.Context(precision=G.MIXED)
    rr, vr = ref.propagate(START, 30.0, 12, r0, v0)
    ref.close()
    comp = G.Context(precision=G.MIXED, flags=G.MIXED_COMPENSATED)
    rc, vc = comp.propagate(START, 30.0, 12, r0, v0)
    comp.close()
    assert np.abs(rc - rr).max() < 1e-3 and np.abs(vc - vr).max() < 1e-6
