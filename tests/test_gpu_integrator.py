"""GPU parity of the integrator kernels with analytic forces: the reference's RK8, startup,
predictor, corrector and GJ8 known-answer tests, run through the CUDA kernels (libgpop.so) and
compared with the golden values and with the CPU oracle."""
import ctypes as C

import numpy as np
import pytest

import oracle_api as O

pytestmark = pytest.mark.gpu

POLY = {
    "zero": lambda t: 0.0,
    "poly7": lambda t: t ** 7 - t ** 3,
    "poly8": lambda t: t ** 8 - t ** 7 + 2 * t ** 6 - 5 * t ** 5 - 10 * t ** 4 + t ** 3 - t ** 2,
    "poly9": lambda t: (t ** 9 + t ** 8 - t ** 7 + 2 * t ** 6 - 5 * t ** 5 - 10 * t ** 4 + t ** 3
                        - t ** 2),
}


def ulps(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return np.abs(a - b) / np.spacing(np.maximum(np.abs(b), 1e-300))


@pytest.fixture(scope="module")
def ctx():
    import opengpop_b200 as G
    c = G.Context()
    yield c
    c.close()


def _startup(ctx, kind, h, ncorr, r0, v0):
    from gpu_util import dev, host, zeros
    out = [zeros(27) for _ in range(5)]
    ctx.startup(kind, None, h, ncorr, dev(r0), dev(v0), out)
    return [host(x).reshape(9, 3) for x in out]


@pytest.mark.parametrize("kind", ["zero", "poly7", "poly8"])
def test_rk8_exact(ctx, kind):
    # rk8_test.cu:197-250 through the CUDA RK8 (n_corrections = 0 returns the RK8 guess)
    r, *_ = _startup(ctx, kind, 1.0, 0, np.zeros(3), np.zeros(3))
    exp = np.array([[POLY[kind](i)] * 3 for i in range(-4, 5)])
    assert np.all((ulps(r, exp) <= 16) | (np.abs(r - exp) < 1e-15))


def test_rk8_degree9_not_exact(ctx):
    r, *_ = _startup(ctx, "poly9", 1.0, 0, np.zeros(3), np.zeros(3))
    exp = np.array([[POLY["poly9"](i)] * 3 for i in range(-4, 5)])
    assert np.abs(r - exp).max() > 1e-10


@pytest.mark.parametrize("kind,tol", [("zero", 0.0), ("poly7", 1e-10), ("poly8", 1e-13)])
def test_startup_exact(ctx, kind, tol):
    # startup_test.cu:111-144 (bound max(tol, 2 ulp): values reach 9e4)
    r, *_ = _startup(ctx, kind, 1.0, 5, np.zeros(3), np.zeros(3))
    exp = np.array([[POLY[kind](i)] * 3 for i in range(-4, 5)])
    assert np.all((np.abs(r - exp) <= tol) | (ulps(r, exp) <= 2))


def test_startup_matches_oracle_damped(ctx):
    # the full startup state (r, v, a, s, S) against the oracle at 1e-12 relative
    g = _startup(ctx, "damped", 0.1, 7, np.ones(3), np.zeros(3))
    L = O.lib()
    out = [np.zeros(27) for _ in range(5)]
    st = O.OrTime(2000, 1, 1, 0, 0, 0.0)
    L.or_startup(None, O.FORCE["damped"], C.byref(st), 0.1, 7, O.ptr(np.ones(3)),
                 O.ptr(np.zeros(3)), 0, *[O.ptr(x) for x in out])
    for a, b in zip(g, out):
        b = b.reshape(9, 3)
        assert np.allclose(a, b, rtol=1e-12, atol=1e-14)


def _corrector(ctx, kind, h, op, pm, vm):
    from gpu_util import dev, host, zeros
    t = [dev(pm), dev(vm), zeros(27), zeros(27), zeros(27)]
    ctx.corrector_unit(kind, h, op, *t)
    return [host(x).reshape(9, 3) for x in t]


def test_corrector_s0_hand_values(ctx):
    m = np.repeat(np.arange(9.0), 3)
    _, _, _, s, S = _corrector(ctx, "exp", 2.0, 1, m, m)
    assert np.all(ulps(s[4], 2.075075590567601) <= 4)
    assert np.all(np.abs(S[4] - 0.924524968616072) <= 1e-7 * 0.9245)


def test_corrector_s_hand_values(ctx):
    m = np.repeat(np.arange(9.0), 3)
    _, _, _, s, S = _corrector(ctx, "exp", 2.0, 2, m, m)
    es = [-1.954319917555107e3, -0.262126527287875e3, -0.033113055524935e3,
          -0.002119452458898e3, 0.002075075590568e3, 0.002642743232186e3, 0.002719568693249e3,
          0.002729965888781e3, 0.002731372996184e3]
    eS = [5.294164844621613e2, 0.655755604279188e2, 0.051634298864115e2, -0.006505506219515e2,
          0.009245249686161e2, 0.034996005591837e2, 0.062100114329879e2, 0.089387379456808e2,
          0.116699432105504e2]
    for i in range(9):
        assert np.all(np.abs(s[i] - es[i]) <= 1e-6 * abs(es[i]))
        assert np.all(np.abs(S[i] - eS[i]) <= 1e-6 * abs(eS[i]))


def test_corrector_acceleration_matrix(ctx):
    vm = np.repeat([8, 6, 4, 2, 0, -2, -4, -6, -8.0], 3)
    pm = np.repeat([-15, -8, -3, 0, 1, 0, 3, 8, 15.0], 3)
    _, _, a, _, _ = _corrector(ctx, "damped", 2.0, 0, pm, vm)
    assert np.all(a[:, 0] == [14, 4, -2, -4, -2, 4, 2, -4, -14])


def test_predictor_and_finalize_hand_values(ctx):
    from gpu_util import dev, host
    r, v = dev(np.zeros(3)), dev(np.zeros(3))
    a = dev(np.repeat(np.arange(1, 10, dtype=float), 3))
    s, S = dev(np.full(3, 2.0)), dev(np.ones(3))
    ctx.predict_unit("poly7", 0.1, 5, r, v, a, s, S)
    assert np.all(np.abs(host(r) - 0.083333333333333) <= 1e-7 * 0.0833)
    # the predictor sum cancels (sum |c_k a_k| / |sum c_k a_k| ~ 60): bound 1e-14 relative
    assert np.all(np.abs(host(v) - 1.141666666666669) <= 1e-14 * 1.1417)
    r, v = dev(np.ones(3)), dev(np.full(3, 2.0))
    a = dev(np.repeat(np.arange(1, 10, dtype=float), 3))
    ctx.finalize_correction_unit(0.1, r, v, a, dev(np.full(3, 4.0)), dev(np.full(3, 3.0)))
    assert np.all(np.abs(host(v) - 0.408277901785714) <= 1e-7 * 0.408)
    assert np.all(np.abs(host(r) - 0.045496538487554) <= 1e-7 * 0.0455)


def _prop(ctx, kind, h, steps, r0, v0, ncorr=7):
    from gpu_util import dev, host, zeros
    r0 = np.asarray(r0, float).reshape(-1, 3)
    n = r0.shape[0]
    r, v = dev(r0), dev(np.asarray(v0, float).reshape(-1, 3))
    tr, tv, ta = zeros(steps, 3, n), zeros(steps, 3, n), zeros(steps, 3, n)
    ctx.propagate_analytic(kind, h, steps, r, v, n_corrections=ncorr, traj_r=tr, traj_v=tv,
                           traj_a=ta)
    tr, tv, ta = (host(x).transpose(0, 2, 1) for x in (tr, tv, ta))
    return host(r), host(v), tr, tv, ta


def test_integrator_stationary_and_constant_speed(ctx):
    # integrator_test.cu:54-110
    r0 = np.array([[0, 0, 0], [1, 1, 1.0]])
    _, _, rs, vs, _ = _prop(ctx, "zero", 1.0, 10, r0, np.zeros((2, 3)))
    assert np.all(rs == r0[None]) and np.all(vs == 0.0)
    _, _, rs, vs, _ = _prop(ctx, "zero", 1.0, 10, r0, np.ones((2, 3)))
    for i in range(10):
        assert np.all(ulps(rs[i], r0 + i + 1) <= 4)
        assert np.all(vs[i] == 1.0)


@pytest.mark.parametrize("kind,bound", [("poly7", 1e-13), ("poly8", 2e-13)])
def test_integrator_polynomial_global_error(ctx, kind, bound):
    # integrator_test.cu:166-188
    _, _, rs, _, _ = _prop(ctx, kind, 0.1, 20, np.zeros(3), np.zeros(3), ncorr=1)
    err = max(np.linalg.norm(rs[i, 0] - POLY[kind]((i + 1) * 0.1)) for i in range(20))
    assert err <= bound


def test_integrator_convergence(ctx):
    # integrator_test.cu:190-205
    exact = lambda t: np.exp(-t) * (np.sin(t) + np.cos(t))
    prev = np.inf
    for nc in range(1, 6):
        _, _, rs, _, _ = _prop(ctx, "damped", 0.1, 40, np.ones(3), np.zeros(3), ncorr=nc)
        err = max(np.linalg.norm(rs[i, 0] - exact((i + 1) * 0.1)) for i in range(40))
        assert err < prev
        prev = err


def test_integrator_matches_oracle(ctx):
    # per-step states and exported accelerations against the oracle (damped oscillator)
    g = np.random.default_rng(3)
    r0 = g.normal(size=(33, 3))
    v0 = g.normal(size=(33, 3))
    _, _, rs, vs, as_ = _prop(ctx, "damped", 0.05, 60, r0, v0)
    _, _, ors, ovs, oas = O.propagate(None, "damped", None, 0.05, 60, r0, v0, per_step=True)
    for a, b in ((rs, ors), (vs, ovs), (as_, oas)):
        assert np.allclose(a, b, rtol=1e-11, atol=1e-13)
