"""GPU parity of the force model: fused gravity kernel (FP64 and mixed), per-epoch frame kernel,
and a full propagation against the CPU oracle and the reference's golden vectors."""
import numpy as np
import pytest

import oracle_api as O
from test_oracle_golden import GRAV_EXP, GRAV_POS

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import opengpop_b200 as G
    c = G.Context()
    yield c
    c.close()


def _grav(ctx, r, frame=None, precision=0):
    from gpu_util import dev, host, zeros
    a = zeros(r.shape[0], 3)
    ctx.gravity(dev(r), a, None if frame is None else dev(frame), precision=precision)
    return host(a)


def test_gravity_golden_vectors(ctx):
    # fm_gravity_source_test.cu:79-180 at 1e-10 m/s^2 (identity frame, 70x70)
    a = _grav(ctx, GRAV_POS)
    assert np.abs(a - GRAV_EXP).max() <= 1e-10
    for i in range(10):
        assert np.abs(_grav(ctx, GRAV_POS[i:i + 1])[0] - GRAV_EXP[i]).max() <= 1e-10


def test_gravity_matches_oracle_random(ctx, oracle_data):
    from opengpop_b200 import orbits
    r, _ = orbits.mixed_population(4096, seed=11)
    m, _ = O.frame_matrices(oracle_data, (2024, 1, 1, 0, 0, 0.0), 30.0, 1, before=0)
    a = _grav(ctx, r, m[0])
    b = O.gravity(oracle_data, r, m[0])
    rel = np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)
    assert rel.max() < 1e-13


def test_gravity_mixed_precision_error(ctx, oracle_data):
    from opengpop_b200 import orbits
    r, _ = orbits.mixed_population(4096, seed=12)
    a = _grav(ctx, r, precision=1)
    b = O.gravity(oracle_data, r)
    err = np.linalg.norm(a - b, axis=1)
    # degree > 8 terms in FP32: absolute error far below the 1e-10 m/s^2 gravity tolerance
    assert err.max() < 1e-9, err.max()


def test_gravity_batch_invariance(ctx):
    # force_model_test.cu:38-88
    r = np.tile([-3884872.0, -5749111.0, 14723.0], (8, 1))
    a = _grav(ctx, r)
    assert np.all(a == a[0])


def test_frame_matrices_match_oracle(ctx, oracle_data):
    from gpu_util import host, zeros
    for start, h, cnt, mid in [((2024, 1, 1, 0, 0, 0.0), 30.0, 2000, False),
                               ((2015, 5, 4, 22, 22, 2.0), 60.0, 80, True),
                               ((2025, 10, 22, 11, 0, 0.0), 86400.0 * 50, 40, False)]:
        m = zeros(cnt, 9)
        mjd = zeros(cnt)
        ctx.frame_matrices(start, h, cnt, m, mjd, use_midpoints=mid, before_epoch=4)
        om, omjd = O.frame_matrices(oracle_data, start, h, cnt, midpoints=mid, before=4)
        assert np.abs(host(m) - om).max() < 1e-12
        assert np.abs(host(mjd) - omjd).max() == 0.0


def test_propagation_matches_oracle(ctx, oracle_data):
    from opengpop_b200 import orbits
    r0, v0 = orbits.leo(24, seed=5)
    start = (2024, 1, 1, 0, 0, 0.0)
    steps = 240  # 2 h at 30 s
    r, v = ctx.propagate(start, 30.0, steps, r0, v0)
    orr, ov = O.propagate(oracle_data, "gravity", start, 30.0, steps, r0, v0)
    assert np.abs(r - orr).max() < 1e-4  # m
    assert np.abs(v - ov).max() < 1e-7  # m/s


def test_propagation_trajectory_matches_oracle(ctx, oracle_data):
    from gpu_util import dev, host, zeros
    from opengpop_b200 import orbits
    r0, v0 = orbits.leo(16, seed=6)
    start = (2015, 5, 4, 22, 22, 2.0)
    steps = 30
    r, v = dev(r0), dev(v0)
    tr, tv, ta = zeros(steps, 3, 16), zeros(steps, 3, 16), zeros(steps, 3, 16)
    ctx.propagate_trajectory(start, 30.0, steps, r, v, tr, tv, ta)
    _, _, ors, ovs, oas = O.propagate(oracle_data, "gravity", start, 30.0, steps, r0, v0,
                                      per_step=True)
    tr, tv, ta = (host(x).transpose(0, 2, 1) for x in (tr, tv, ta))
    assert np.abs(tr - ors).max() < 1e-5
    assert np.abs(tv - ovs).max() < 1e-8
    assert np.abs(ta - oas).max() < 1e-11


def test_propagator_batch_invariance(ctx):
    # propagator_test.cu:38-83: 8 identical objects stay bitwise identical
    from gpu_util import dev, host, zeros
    r0 = np.tile([-3884872.0, -5749111.0, 14723.0], (8, 1))
    v0 = np.tile([-795.304, 573.772, 7518.179], (8, 1))
    r, v = dev(r0), dev(v0)
    tr = zeros(10, 3, 8)
    ctx.propagate_trajectory((2015, 5, 4, 22, 22, 2.0), 30.0, 10, r, v, tr)
    t = host(tr)
    assert np.all(t == t[:, :, :1])


def test_propagation_zero_steps_is_identity(ctx):
    from opengpop_b200 import orbits
    r0, v0 = orbits.leo(4, seed=1)
    r, v = ctx.propagate((2024, 1, 1, 0, 0, 0.0), 30.0, 0, r0, v0)
    assert np.all(r == r0) and np.all(v == v0)
