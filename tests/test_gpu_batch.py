"""GPU parity of the batched propagation (gpop_propagate_batch): many uneven requests in one
persistent launch must give each request the result of its own exec propagate call
(exec/runner.cu:11-70, one GpuPropagator per request in gpu_propagator.cu:121-136), i.e. of
gpop_propagate on a context of the request's degree, and of the CPU oracle."""
import os

import numpy as np
import pytest

import oracle_api as O

pytestmark = pytest.mark.gpu

START = (2024, 1, 1, 0, 0, 0.0)


@pytest.fixture(scope="module")
def contexts():
    import opengpop_b200 as G
    made = {}

    def get(degree, precision=G.FP64):
        key = (degree, precision)
        if key not in made:
            made[key] = G.Context(gravity_degree=degree, precision=precision)
        return made[key]
    yield get
    for c in made.values():
        c.close()


def _requests(spec, seed):
    from opengpop_b200 import orbits
    rng = np.random.default_rng(seed)
    out = []
    for i, (n, steps, h, degree) in enumerate(spec):
        r, v = orbits.mixed_population(n, seed=int(rng.integers(1 << 30)))
        start = START if i % 3 else (2024, 3, 5, 6, 30, 12.5)
        out.append(dict(start=start, h=h, steps=steps, degree=degree, r=r, v=v))
    return out


# (objects, steps, step size, degree): single objects, ragged groups, steps 0..4 (startup replay
# only), longer runs, four step sizes and three degrees.
SPEC = [(1, 40, 30.0, 70), (3, 0, 60.0, 20), (1, 1, 10.0, 8), (5, 2, 120.0, 70), (2, 3, 30.0, 36),
        (7, 4, 60.0, 20), (33, 5, 30.0, 70), (100, 24, 60.0, 8), (64, 12, 10.0, 36),
        (17, 60, 120.0, 20), (250, 9, 30.0, 70), (1, 7, 30.0, 20)]


def _compare(outs, reqs, ctx_of, rtol_r, rtol_v):
    for q, (ro, vo) in zip(reqs, outs):
        if q["steps"] == 0:
            assert np.array_equal(ro, q["r"]) and np.array_equal(vo, q["v"])
            continue
        ref_r, ref_v = ctx_of(q).propagate(q["start"], q["h"], q["steps"], q["r"], q["v"])
        dr = np.linalg.norm(ro - ref_r, axis=1).max()
        dv = np.linalg.norm(vo - ref_v, axis=1).max()
        assert dr <= rtol_r and dv <= rtol_v, (q["steps"], q["degree"], q["r"].shape[0], dr, dv)


def test_batch_matches_single_requests_fp64(contexts):
    import opengpop_b200 as G
    ctx = contexts(70)
    reqs = _requests(SPEC, 1)
    outs = ctx.propagate_batch(reqs)
    # the lane split reorders the gravity sums: agreement to rounding over <= 60 steps
    _compare(outs, reqs, lambda q: contexts(q["degree"]), 1e-6, 1e-9)
    assert ctx.kernel_launches > 0


def test_batch_matches_oracle(contexts, oracle_data):
    ctx = contexts(70)
    reqs = _requests([(9, 30, 30.0, 70), (1, 20, 60.0, 70)], 2)
    outs = ctx.propagate_batch(reqs)
    for q, (ro, vo) in zip(reqs, outs):
        rr, vv = O.propagate(oracle_data, "gravity", q["start"], q["h"], q["steps"], q["r"], q["v"])
        assert np.linalg.norm(ro - rr, axis=1).max() < 1e-6
        assert np.linalg.norm(vo - vv, axis=1).max() < 1e-9


def test_batch_mixed_precision(contexts):
    import opengpop_b200 as G
    ctx = contexts(70, G.MIXED)
    reqs = _requests(SPEC, 3)
    outs = ctx.propagate_batch(reqs)
    # against the FP64 single-request path: the mixed gravity error stays far below 1 mm here
    _compare(outs, reqs, lambda q: contexts(q["degree"]), 1e-3, 1e-6)


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_of_single_lane_items(contexts, precision):
    # enough objects that every request keeps one lane per object: the persistent kernel then
    # walks two gravity columns at a time on the lane-layout table (degree 8 in mixed mode takes
    # the one-column lane walk inside the same kernel)
    ctx = contexts(70, precision)
    # (more degree-70 items than warps, so none of them is longer than the mean warp load; the
    # degree-36 and degree-8 items are shorter still)
    reqs = _requests([(20000, 6, 30.0, 70), (20000, 6, 60.0, 70), (20000, 6, 10.0, 70),
                      (20000, 6, 120.0, 70), (8000, 4, 30.0, 36), (8000, 10, 60.0, 8)], 6)
    lpo, _ = ctx.batch_plan(reqs)
    assert all(int(p) == 1 for p in lpo), lpo
    outs = ctx.propagate_batch(reqs)
    tol = (1e-6, 1e-9) if precision == 0 else (1e-3, 1e-6)
    _compare(outs, reqs, lambda q: contexts(q["degree"]), *tol)


def test_batch_graph_replay_new_inputs(contexts):
    ctx = contexts(70)
    a = _requests(SPEC[:6], 4)
    b = _requests(SPEC[:6], 5)  # same shapes, other states: the cached graph is replayed
    outs_a = ctx.propagate_batch(a)
    outs_b = ctx.propagate_batch(b)
    _compare(outs_a, a, lambda q: contexts(q["degree"]), 1e-6, 1e-9)
    _compare(outs_b, b, lambda q: contexts(q["degree"]), 1e-6, 1e-9)
    outs_a2 = ctx.propagate_batch(a)
    for (r1, v1), (r2, v2) in zip(outs_a, outs_a2):
        assert np.array_equal(r1, r2) and np.array_equal(v1, v2)


def test_batch_plan_lanes(contexts):
    ctx = contexts(70)
    from opengpop_b200 import orbits
    r, v = orbits.leo(4096, seed=6)
    reqs = [dict(start=START, h=10.0, steps=20000, degree=70, r=r[:1], v=v[:1]),
            dict(start=START, h=60.0, steps=20, degree=8, r=r, v=v),
            dict(start=START, h=60.0, steps=20, degree=70, r=r[:3], v=v[:3])]
    lpo, est = ctx.batch_plan(reqs)
    assert lpo[0] == 32  # one object: the whole warp splits its columns
    assert lpo[1] == 1  # many objects, short run: one lane each
    assert lpo[2] == 8  # three objects fill 24 lanes
    assert est > 0


def test_batch_rejects_bad_requests(contexts):
    import opengpop_b200 as G
    ctx = contexts(70)
    good = _requests([(2, 5, 30.0, 70)], 7)[0]
    for bad in (dict(good, h=0.0), dict(good, steps=-1), dict(good, start=(2024, 13, 1, 0, 0, 0.0))):
        with pytest.raises(G.GpopError):
            ctx.propagate_batch([good, bad])


def test_tune_cache_roundtrip(contexts, tmp_path):
    import opengpop_b200 as G
    ctx = contexts(70, G.MIXED)
    path = str(tmp_path / "eta.txt")
    ctx.tune(path)
    lines = open(path).read().split("\n")
    rows = [l.split() for l in lines if l.strip()]
    assert len(rows) == 48  # (warps per SM 4 | 8) x degrees {8, 20, 36, 70} x lanes 1..32
    eta = {(int(W), int(L), int(P)): float(e) for _, W, L, P, e in rows}
    assert all(e > 0 for e in eta.values())
    for W in (4, 8):
        assert eta[(W, 8, 1)] > eta[(W, 70, 1)]  # lower degree, more object-steps per second
    ctx.tune(path)  # read back from the cache
    reqs = _requests(SPEC[:4], 8)
    _compare(ctx.propagate_batch(reqs), reqs, lambda q: contexts(q["degree"]), 1e-3, 1e-6)


def test_planner_block_shape(contexts):
    """The planner picks the persistent grid's block shape: a batch with fewer work items than
    schedulers runs four warps per SM (one item per scheduler), a batch that fills many waves
    eight; the results are those of single requests either way."""
    ctx = contexts(70)
    few = _requests([(20, 30, 30.0, 70), (40, 25, 60.0, 36), (9, 12, 30.0, 20)], 5)
    outs = ctx.propagate_batch(few)
    assert ctx.batch_warps_per_sm == 4
    _compare(outs, few, lambda q: contexts(q["degree"]), 1e-6, 1e-9)
    many = _requests([(512, 40, 30.0, 70)] * 120, 6)
    outs = ctx.propagate_batch(many)
    assert ctx.batch_warps_per_sm == 8
    _compare(outs[:3], many[:3], lambda q: contexts(q["degree"]), 1e-6, 1e-9)
