"""Seeded synthetic orbits: Keplerian elements drawn from a seed, converted to GCRS r, v in FP64.

These stand in for catalogue data (no dataset ships with the reference). GM and R are those of the
JGM3 gravity field the propagator uses.
"""
import numpy as np

GM = 0.3986004415e15
R_EARTH = 0.6378136300e7
EPOCH = (2024, 1, 1, 0, 0, 0.0)


def kepler_to_cartesian(a, e, inc, raan, argp, M, gm=GM):
    """Elements (arrays, radians, metres) -> r, v [n, 3] (m, m/s)."""
    a, e, inc, raan, argp, M = (np.asarray(x, np.float64) for x in (a, e, inc, raan, argp, M))
    E = M.copy()
    for _ in range(50):  # Newton on E - e sin E = M
        d = (E - e * np.sin(E) - M) / (1.0 - e * np.cos(E))
        E -= d
        if np.max(np.abs(d)) < 1e-15:
            break
    cE, sE = np.cos(E), np.sin(E)
    fac = np.sqrt(1.0 - e * e)
    x = a * (cE - e)
    y = a * fac * sE
    rn = a * (1.0 - e * cE)
    vs = np.sqrt(gm * a) / rn
    vx = -vs * sE
    vy = vs * fac * cE
    cO, sO = np.cos(raan), np.sin(raan)
    cw, sw = np.cos(argp), np.sin(argp)
    ci, si = np.cos(inc), np.sin(inc)
    # perifocal -> inertial: R3(-raan) R1(-inc) R3(-argp)
    p = np.stack([cO * cw - sO * sw * ci, sO * cw + cO * sw * ci, sw * si], -1)
    q = np.stack([-cO * sw - sO * cw * ci, -sO * sw + cO * cw * ci, cw * si], -1)
    r = x[:, None] * p + y[:, None] * q
    v = vx[:, None] * p + vy[:, None] * q
    return r, v


def leo(n, seed, a_km=(6700.0, 7500.0), e_max=0.02):
    """LEO population of the 1,024-object and closest-approach configurations."""
    g = np.random.default_rng(seed)
    a = g.uniform(a_km[0], a_km[1], n) * 1e3
    e = g.uniform(0.0, e_max, n)
    inc = np.radians(g.uniform(0.0, 180.0, n))
    raan, argp, M = (np.radians(g.uniform(0.0, 360.0, n)) for _ in range(3))
    return kepler_to_cartesian(a, e, inc, raan, argp, M)


def mixed_population(n, seed):
    """65,536-object population: 70% LEO (a 6,700-8,000 km, e <= 0.02), 20% MEO
    (a 20,000-27,000 km, e <= 0.05), 10% GEO (a 42,164 +- 50 km, e <= 0.001); angles uniform."""
    g = np.random.default_rng(seed)
    n_leo = int(round(0.7 * n))
    n_meo = int(round(0.2 * n))
    n_geo = n - n_leo - n_meo
    a = np.concatenate([g.uniform(6700, 8000, n_leo), g.uniform(20000, 27000, n_meo),
                        g.uniform(42164 - 50, 42164 + 50, n_geo)]) * 1e3
    e = np.concatenate([g.uniform(0, 0.02, n_leo), g.uniform(0, 0.05, n_meo),
                        g.uniform(0, 0.001, n_geo)])
    inc = np.radians(g.uniform(0.0, 180.0, n))
    raan, argp, M = (np.radians(g.uniform(0.0, 360.0, n)) for _ in range(3))
    return kepler_to_cartesian(a, e, inc, raan, argp, M)


def batch_requests(n_req, seed, start=EPOCH, max_days=7.0):
    """Uneven propagation requests of the batched configuration: object counts log-uniform in
    [1, 512], durations log-uniform in [1 h, 7 d], step sizes uniform in {10, 30, 60, 120} s, gravity
    degrees uniform in {8, 20, 36, 70}; states from the mixed population. Returns dicts with keys
    start, h, steps, degree, r, v (the argument of Context.propagate_batch). max_days < 7 scales
    the durations down (small cases for profiling)."""
    g = np.random.default_rng(seed)
    out = []
    scale = max_days / 7.0
    for _ in range(n_req):
        n = int(round(np.exp(g.uniform(0.0, np.log(512.0)))))
        dur = scale * float(np.exp(g.uniform(np.log(3600.0), np.log(7 * 86400.0))))
        h = float(g.choice([10.0, 30.0, 60.0, 120.0]))
        degree = int(g.choice([8, 20, 36, 70]))
        steps = max(1, int(round(dur / h)))
        r, v = mixed_population(n, int(g.integers(1 << 30)))
        out.append(dict(start=start, h=h, steps=steps, degree=degree, r=r, v=v))
    return out


def conjunction_pairs(n_pairs, seed):
    """The differentiation configuration's pairs: 2 n_pairs LEO objects (distribution of the
    1,024-object configuration) matched at random into disjoint pairs. Returns r, v, pairs [p, 2]."""
    r, v = leo(2 * n_pairs, seed)
    pairs = np.random.default_rng(seed + 1).permutation(2 * n_pairs).astype(np.int32).reshape(-1, 2)
    return r, v, pairs
