"""The seeded synthetic workloads behind every benchmark (opengpop_b200/orbits.py): deterministic
for a seed, element distributions as documented, and Keplerian states that round-trip through
the two-body invariants (energy gives the semi-major axis, the angular momentum the eccentricity)."""
import numpy as np

from opengpop_b200 import orbits


def _elements(r, v, gm=orbits.GM):
    rn = np.linalg.norm(r, axis=1)
    v2 = np.sum(v * v, axis=1)
    a = 1.0 / (2.0 / rn - v2 / gm)
    hvec = np.cross(r, v)
    evec = np.cross(v, hvec) / gm - r / rn[:, None]
    inc = np.degrees(np.arccos(hvec[:, 2] / np.linalg.norm(hvec, axis=1)))
    return a, np.linalg.norm(evec, axis=1), inc


def test_kepler_round_trip():
    g = np.random.default_rng(3)
    n = 200
    a = g.uniform(6.7e6, 4.3e7, n)
    e = g.uniform(0.0, 0.3, n)
    inc = np.radians(g.uniform(0.0, 180.0, n))
    r, v = orbits.kepler_to_cartesian(a, e, inc, *(np.radians(g.uniform(0, 360, n)) for _ in range(3)))
    a2, e2, inc2 = _elements(r, v)
    assert np.allclose(a2, a, rtol=1e-12)
    assert np.allclose(e2, e, atol=1e-12)
    assert np.allclose(inc2, np.degrees(inc), atol=1e-9)


def test_generators_are_seeded():
    for f in (lambda s: orbits.leo(50, s), lambda s: orbits.mixed_population(50, s)):
        r1, v1 = f(11)
        r2, v2 = f(11)
        r3, _ = f(12)
        assert np.array_equal(r1, r2) and np.array_equal(v1, v2)
        assert not np.array_equal(r1, r3)


def test_mixed_population_bands():
    n = 10000
    a, e, _ = _elements(*orbits.mixed_population(n, 5))
    a_km = a / 1e3
    n_leo, n_meo = int(round(0.7 * n)), int(round(0.2 * n))
    assert np.all((a_km[:n_leo] > 6700 - 1e-6) & (a_km[:n_leo] < 8000 + 1e-6)) and e[:n_leo].max() <= 0.02
    meo = slice(n_leo, n_leo + n_meo)
    assert np.all((a_km[meo] > 20000 - 1e-6) & (a_km[meo] < 27000 + 1e-6)) and e[meo].max() <= 0.05
    geo = slice(n_leo + n_meo, n)
    assert np.all(np.abs(a_km[geo] - 42164) <= 50 + 1e-6) and e[geo].max() <= 0.001


def test_leo_band():
    a, e, inc = _elements(*orbits.leo(5000, 9))
    assert np.all((a / 1e3 > 6700 - 1e-6) & (a / 1e3 < 7500 + 1e-6))
    assert e.max() <= 0.02 and inc.min() >= 0.0 and inc.max() <= 180.0


def test_batch_requests_distributions():
    reqs = orbits.batch_requests(1024, 20240101)
    n = np.array([q["r"].shape[0] for q in reqs])
    dur = np.array([q["steps"] * q["h"] for q in reqs])
    assert n.min() >= 1 and n.max() <= 512
    assert set(q["h"] for q in reqs) == {10.0, 30.0, 60.0, 120.0}
    assert set(q["degree"] for q in reqs) == {8, 20, 36, 70}
    # durations within [1 h, 7 d] up to the rounding of the step count
    assert dur.min() >= 3600.0 - 60.0 and dur.max() <= 7 * 86400.0 + 60.0
    # log-uniform object counts: about half the requests below sqrt(512) ~ 22.6
    assert 0.4 < np.mean(n < 22.6) < 0.6
    again = orbits.batch_requests(8, 20240101)
    assert all(np.array_equal(x["r"], y["r"]) and x["steps"] == y["steps"]
               for x, y in zip(again, reqs[:8]))


def test_conjunction_pairs_are_disjoint():
    r, v, pairs = orbits.conjunction_pairs(500, 4)
    assert r.shape == (1000, 3) and pairs.shape == (500, 2)
    assert np.array_equal(np.sort(pairs.ravel()), np.arange(1000))
