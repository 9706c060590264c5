"""Parity at the sizes and spans of the stated configurations, on the GPU.

- The 65,536-object mixed population over 7 days (30 s steps, 20,160 steps, 70x70), on 64 objects
  spread over LEO, MEO and GEO, against the FP64 CPU oracle: the FP64 build within 1 cm, the
  mixed-precision build (two-level and compensated FP32 sums) within 1 m; both propagated alone
  and inside the whole 65,536-object propagation.
- The 1,024-object configuration in full (20x20, 60 s, 24 h) against the oracle: within 1 cm.
- The closest-approach configuration (20,000 LEO objects, 2,000 seed-chosen objects against all,
  3 days, 5 km) screened by the CUDA path, against the oracle's screen of the very same GPU
  trajectory for a sample of 40 of the 2,000 set rows (every pair that involves one of them): the
  closest steps and the set of pairs below 5 km bit-exact, distance and time to rounding.
- The per-epoch ITRS->GCRS matrices against the reference's own CUDA build
  (TimePointParamsKernel and the DGEMM chain of ComputeITRStoGCRS, time_points.cu:26-71,146-201)
  on the 7-day epoch grid, the RK8 midpoints and the 1,024-object configuration's grid.
"""
import ctypes as C

import numpy as np
import pytest

import oracle_api as O
import ref_build_runner as RB

pytestmark = pytest.mark.gpu

START = (2024, 1, 1, 0, 0, 0.0)
SEED = 20240101


@pytest.fixture(scope="module")
def week():
    """64 objects of the mixed population and the oracle's FP64 state after 7 days."""
    from opengpop_b200 import orbits
    r, v = orbits.mixed_population(65536, SEED)
    idx = np.linspace(0, 65535, 64).astype(int)
    r0, v0 = r[idx], v[idx]
    ro, vo = O.propagate(O.Data(), "gravity", START, 30.0, 20160, r0, v0)
    return r0, v0, ro, vo


@pytest.mark.parametrize("precision,flags,bound_m", [(0, 0, 1e-2), (1, 0, 1.0), (1, 8, 1.0)],
                         ids=["fp64", "mixed", "mixed-compensated"])
def test_seven_days_against_oracle(week, precision, flags, bound_m):
    import opengpop_b200 as G
    r0, v0, ro, vo = week
    ctx = G.Context(precision=precision, flags=flags)
    r, v = ctx.propagate(START, 30.0, 20160, r0, v0)
    ctx.close()
    err = np.linalg.norm(r - ro, axis=1)
    verr = np.linalg.norm(v - vo, axis=1)
    print("\n7 days, %s: position error max %.3e m (object %d), median %.3e m; velocity error max "
          "%.3e m/s" % ({0: "FP64", 1: "mixed"}[precision] + (", compensated" if flags else ""),
                        err.max(), int(err.argmax()), np.median(err), verr.max()))
    assert err.max() <= bound_m


@pytest.mark.parametrize("precision,bound_m", [(0, 1e-2), (1, 1.0)], ids=["fp64", "mixed"])
def test_seven_days_all_objects_against_oracle(week, precision, bound_m):
    """The configuration itself: all 65,536 objects propagated together for 7 days (the split
    block: 7 owner warps per SM and one walking the low gravity columns), the same 64 objects
    against the oracle."""
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    r0, v0, ro, vo = week
    r, v = orbits.mixed_population(65536, SEED)
    idx = np.linspace(0, 65535, 64).astype(int)
    assert np.array_equal(r[idx], r0)
    assert G.split_block(65536) == 7
    ctx = G.Context(precision=precision)
    rr, vv = ctx.propagate(START, 30.0, 20160, r, v)
    ctx.close()
    err = np.linalg.norm(rr[idx] - ro, axis=1)
    print("\n7 days, all 65,536 objects, %s: position error max %.3e m (object %d), median %.3e m"
          % ({0: "FP64", 1: "mixed"}[precision], err.max(), int(idx[err.argmax()]), np.median(err)))
    assert np.isfinite(rr).all() and err.max() <= bound_m


def test_thousand_objects_20x20_one_day_against_oracle():
    """The 1,024-object configuration in full: 20x20, 60 s steps, 24 h (1,440 steps)."""
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    r0, v0 = orbits.leo(1024, SEED)
    ctx = G.Context(gravity_degree=20)
    r, v = ctx.propagate(START, 60.0, 1440, r0, v0)
    ctx.close()
    ro, vo = O.propagate(O.Data(degree=20), "gravity", START, 60.0, 1440, r0, v0)
    err = np.linalg.norm(r - ro, axis=1)
    print("\n1,024 objects, 20x20, 24 h: position error max %.3e m, velocity max %.3e m/s"
          % (err.max(), np.linalg.norm(v - vo, axis=1).max()))
    assert err.max() <= 1e-2


def _pair_of(p, idx):
    """(first, second) object of pair indices idx under partition p (the reference's map)."""
    A = np.searchsorted(p["map_offsets"][:p["num_sets"] - 1], idx, side="right") - 1
    rel = idx - p["map_offsets"][A].astype(np.int64)
    nh = p["num_higher"][A].astype(np.int64)
    return (rel // nh + p["set_offsets"][A]).astype(np.int64), \
        (rel % nh + p["set_offsets"][A + 1]).astype(np.int64)


def _index_of(p, a, b):
    """Pair index of (a, b), a < b in different sets, under partition p."""
    A = p["ids"][a].astype(np.int64)
    return (p["map_offsets"][A].astype(np.int64)
            + (a - p["set_offsets"][A].astype(np.int64)) * p["num_higher"][A].astype(np.int64)
            + (b - p["set_offsets"][A + 1].astype(np.int64)))


def test_closest_approach_configuration_row_sample():
    import torch
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    n, n_sel, steps, h, thr = 20000, 2000, 8640, 30.0, 5000.0
    r, v = orbits.leo(n, SEED)
    sel = np.random.default_rng(SEED).choice(n, n_sel, replace=False)
    order = np.concatenate([sel, np.setdiff1d(np.arange(n), sel)])
    r, v = r[order], v[order]
    set_ids = np.concatenate([np.arange(n_sel), np.full(n - n_sel, n_sel)]).astype(np.uint32)
    ctx = G.Context(precision=G.FP64)
    # the CUDA path: one closest-approach job over all 37,999,000 pairs
    ca = ctx.closest_approach(START, h, r, v, set_ids)
    ca.propagate(steps)
    g = ca.pairs()
    recs = ca.find(thr)
    ca.close()
    full = O.partition(set_ids)
    # 40 of the set rows; the oracle screens every pair with one of them, on the same trajectory
    rows = np.sort(np.random.default_rng(7).choice(n_sel, 40, replace=False))
    sub_order = np.concatenate([rows, np.setdiff1d(np.arange(n), rows)])
    sub_ids = np.concatenate([np.arange(40), np.full(n - 40, 40)]).astype(np.uint32)
    sub = O.partition(sub_ids)
    P = int(sub["num_pairs"])
    md = np.zeros(P)
    cs = np.zeros(P, np.uint32)
    nodes = np.zeros(P * 54)
    last = np.zeros(n * 9)
    st = O.OrCaState(md.ctypes.data, cs.ctypes.data, nodes.ctypes.data, last.ctypes.data)
    lib = O.lib()
    # the GPU trajectory, window by window (the same kernels and epochs as the job above)
    rd = torch.tensor(r, dtype=torch.float64, device="cuda")
    vd = torch.tensor(v, dtype=torch.float64, device="cuda")
    prop = ctx.propagator(START, h, steps, rd, vd)
    win = 240
    tr = torch.empty((win, 3, n), dtype=torch.float64, device="cuda")
    tv = torch.empty_like(tr)
    ta = torch.empty_like(tr)
    for w0 in range(0, steps, win):
        prop.step(win, tr, tv, ta)
        arrs = [np.ascontiguousarray(x.cpu().numpy().transpose(0, 2, 1)[:, sub_order, :])
                for x in (tr, tv, ta)]
        lib.or_ca_screen(n, win, O.ptr(arrs[0]), O.ptr(arrs[1]), O.ptr(arrs[2]),
                         O.ptr(sub["ids"]), w0, int(w0 == 0), C.byref(st), 0)
    prop.close()
    ctx.close()
    dist = np.zeros(P)
    tim = np.zeros(P)
    pa = np.zeros((P, 3))
    pb = np.zeros((P, 3))
    lib.or_ca_refine(n, O.ptr(sub["ids"]), h, steps, C.byref(st), O.ptr(dist), O.ptr(tim),
                     O.ptr(pa), O.ptr(pb), 0)
    # oracle pair k -> objects of the job -> the job's pair index
    ka, kb = _pair_of(sub, np.arange(P, dtype=np.int64))
    a, b = sub_order[ka], sub_order[kb]
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    gi = _index_of(full, lo, hi)
    assert np.array_equal(g["closest_step"][gi], cs)
    assert np.allclose(g["distance"][gi], dist, rtol=1e-9, atol=1e-6)
    assert np.allclose(g["time"][gi], tim, rtol=0, atol=1e-6)
    # the pairs below 5 km that involve a sampled row: the same set
    rowset = set(rows.tolist())
    got = sorted((x.object_index1, x.object_index2) for x in recs
                 if x.object_index1 in rowset or x.object_index2 in rowset)
    exp = sorted(zip(lo[dist < thr].tolist(), hi[dist < thr].tolist()))
    print("\n%d pairs of 40 rows over 8,640 steps: %d below 5 km (all rows: %d)"
          % (P, len(exp), len(recs)))
    assert got == exp


@pytest.mark.skipif(not RB.available(), reason="reference build not present")
@pytest.mark.parametrize("h,count,midpoints", [(30.0, 20165, False), (30.0, 80, True),
                                               (60.0, 1445, False), (60.0, 80, True)],
                         ids=["7d-30s", "rk8-30s", "1d-60s", "rk8-60s"])
def test_frame_matrices_against_reference_build(h, count, midpoints):
    import torch
    import opengpop_b200 as G
    ctx = G.Context()
    m = torch.zeros(count, 9, dtype=torch.float64, device="cuda")
    mjd = torch.zeros(count, dtype=torch.float64, device="cuda")
    ctx.frame_matrices(START, h, count, m, mjd, use_midpoints=midpoints, before_epoch=4)
    torch.cuda.synchronize()
    ctx.close()
    rm, rmjd = RB.frames(START, h, count, midpoints=midpoints, before=4)
    dm = np.abs(m.cpu().numpy() - rm).max()
    dmjd = np.abs(mjd.cpu().numpy() - rmjd).max()
    print("\n%d epochs (h %g s%s): matrix entries max |diff| %.3e, MJD max |diff| %.3e d"
          % (count, h, ", RK8 midpoints" if midpoints else "", dm, dmjd))
    assert dm <= 1e-12
    assert dmjd <= 2e-11  # a few units in the last place of an MJD near 60,310
