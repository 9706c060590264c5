"""Pins the CPU oracle against the reference's own golden vectors and known-answer tests.

Every case below restates a test of the reference's unit_tests/ directory (file:line cited). Where
the reference compares with EXPECT_DOUBLE_EQ against values whose last bits depend on cuBLAS's
(unspecified) summation order, the bound here is a few units in the last place and says so.
"""
import ctypes as C

import numpy as np
import pytest

import oracle_api as O

# unit_tests/fm_gravity_source_test.cu:79-107
GRAV_POS = np.array([
    6.778136300000000e+06, 1.000000000000000e+03, 1.000000000000000e+03,
    0.000000000000000e+00, 6.878136300000000e+06, 5.000000000000000e+03,
    1.000000000000000e+03, 2.000000000000000e+03, -6.978136300000000e+06,
    5.217130210248624e+06, 5.217130210248623e+06, 1.000000000000000e+04,
    -7.000000000000000e+06, -5.000000000000000e+06, 3.000000000000000e+06,
    2.000000000000000e+07, 0.000000000000000e+00, 0.000000000000000e+00,
    0.000000000000000e+00, -2.500000000000000e+07, 1.000000000000000e+05,
    6.378136300000000e+06, 6.378136300000000e+06, 6.378136300000000e+06,
    -8.000000000000000e+06, 8.000000000000000e+06, -8.000000000000000e+06,
    -6.578136300000000e+06, 6.578136300000000e+06, -6.578136300000000e+06]).reshape(10, 3)
GRAV_EXP = np.array([
    -8.688512585751166e+00, -1.306014485437521e-03, -1.257696785446421e-03,
    -2.582667093861692e-04, -8.437050803978574e+00, -6.163521917854259e-03,
    -1.030412992305426e-03, -2.285861566359708e-03, 8.163505409516388e+00,
    -5.183755318186486e+00, -5.183875047834164e+00, -9.957411924758089e-03,
    3.691249064843031e+00, 2.636634693149141e+00, -1.584503282402068e+00,
    -9.966668939635662e-01, -2.945383387897605e-07, 1.037052511930428e-07,
    1.569778426358556e-07, 6.378123760414850e-01, -2.551886609172898e-03,
    -1.884989255869376e+00, -1.885012768325866e+00, -1.887034359138477e+00,
    1.198326115108038e+00, -1.198330866500345e+00, 1.199158569758444e+00,
    1.772149453385123e+00, -1.772160848876822e+00, 1.773973126474241e+00]).reshape(10, 3)

POLY = {
    "poly7": lambda t: t ** 7 - t ** 3,
    "poly8": lambda t: t ** 8 - t ** 7 + 2 * t ** 6 - 5 * t ** 5 - 10 * t ** 4 + t ** 3 - t ** 2,
    "poly9": lambda t: (t ** 9 + t ** 8 - t ** 7 + 2 * t ** 6 - 5 * t ** 5 - 10 * t ** 4 + t ** 3
                        - t ** 2),
    "zero": lambda t: 0.0,
}


def ulps(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return np.abs(a - b) / np.spacing(np.maximum(np.abs(b), 1e-300))


def test_data_sets(oracle_data):
    d = oracle_data
    assert d.degree == 70
    assert d.gm == 0.3986004415e15 and d.radius == 0.6378136300e7
    L = O.lib()
    # IERS tables: 1320 + 38 lon terms, 1037 + 19 obl terms
    assert [L.or_data_nut_count(d.h, i) for i in range(4)] == [1320, 38, 1037, 19]
    assert L.or_data_eop_count(d.h) == 19794
    assert L.or_data_leap_count(d.h) == 28


def test_gravity_golden_one_by_one(oracle_data):
    # fm_gravity_source_test.cu:109-138, tolerance 1e-10 m/s^2, identity frame
    for i in range(10):
        a = O.gravity(oracle_data, GRAV_POS[i:i + 1])
        assert np.all(np.abs(a[0] - GRAV_EXP[i]) <= 1e-10)


def test_gravity_golden_batched(oracle_data):
    # fm_gravity_source_test.cu:140-180
    a = O.gravity(oracle_data, GRAV_POS)
    assert np.abs(a - GRAV_EXP).max() <= 1e-10


def test_gravity_batch_invariance(oracle_data):
    # force_model_test.cu:38-88: identical objects give bitwise-identical accelerations
    r = np.tile([-3884872.0, -5749111.0, 14723.0], (8, 1))
    m, _ = O.frame_matrices(oracle_data, (2015, 5, 4, 22, 22, 2.0), 30.0, 1, before=0)
    a = O.gravity(oracle_data, r, m[0])
    assert np.all(a == a[0])


def test_refsys_rotations():
    # fm_ref_sys_trans_test.cu:49-88 build Rx/Ry/Rz(0.45); the column-major layout is the contract
    L = O.lib()
    c, s = np.cos(0.45), np.sin(0.45)
    exp = {0: [[1, 0, 0], [0, c, s], [0, -s, c]], 1: [[c, 0, -s], [0, 1, 0], [s, 0, c]],
           2: [[c, s, 0], [-s, c, 0], [0, 0, 1]]}
    for axis in range(3):
        out = np.zeros(9)
        L.or_rot(axis, 0.45, O.ptr(out))
        assert np.allclose(out.reshape(3, 3).T, exp[axis], atol=1e-15)


def test_calendar_and_ntp():
    L = O.lib()
    # 2000-01-01 12:00 = MJD 51544.5 ; fm_ref_sys_trans_test.cu:89-104 style check
    assert L.or_calendar_to_mjd(2000, 1, 1, 12, 0, 0.0) == 51544.5
    assert abs(L.or_calendar_to_mjd(2024, 1, 1, 0, 0, 0.0) - 60310.0) < 1e-12
    # fm_ref_sys_trans_test.cu:311-326: NTP epoch, one day, J2000 noon
    assert abs(L.or_ntp_to_mjd(0) - 15020.0) < 1e-10
    assert abs(L.or_ntp_to_mjd(86400) - 15021.0) < 1e-10
    assert abs(L.or_ntp_to_mjd(3155716800) - 51544.5) < 1e-10


def test_leap_and_eop(oracle_data):
    L = O.lib()
    d = oracle_data
    assert L.or_data_leap_seconds(d.h, 41317.0) == 10.0
    assert L.or_data_leap_seconds(d.h, 60000.0) == 37.0
    assert L.or_data_leap_seconds(d.h, 30000.0) == 10.0  # before the table: first entry
    out = np.zeros(4)
    L.or_data_eop_record(d.h, 41684.0, O.ptr(out))  # first record, clamped
    assert out[0] == 41684.0 and abs(out[3] - 0.8084178) < 1e-15
    L.or_data_eop_record(d.h, 41684.5, O.ptr(out))  # halfway: linear interpolation
    assert abs(out[3] - 0.5 * (0.8084178 + 0.8056163)) < 1e-15
    L.or_data_eop_record(d.h, 1e6, O.ptr(out))  # beyond the table: clamped to the last (Q8)
    assert out[0] == 61477.0


def test_frame_matrix_is_rotation(oracle_data):
    m, mjd = O.frame_matrices(oracle_data, (2024, 1, 1, 0, 0, 0.0), 30.0, 9, before=4)
    for k in range(9):
        M = m[k].reshape(3, 3).T
        assert np.abs(M @ M.T - np.eye(3)).max() < 1e-14
        assert abs(np.linalg.det(M) - 1.0) < 1e-14
    assert abs(mjd[4] - 60310.0) < 1e-12
    assert abs((mjd[5] - mjd[4]) * 86400.0 - 30.0) < 1e-6


def _rk8(kind, h=1.0):
    L = O.lib()
    r27 = np.zeros(27)
    v27 = np.zeros(27)
    st = O.OrTime(2000, 1, 1, 0, 0, 0.0)
    L.or_rk8(None, O.FORCE[kind], C.byref(st), h, O.ptr(np.zeros(3)), O.ptr(np.zeros(3)), 0,
             O.ptr(r27), O.ptr(v27))
    return r27.reshape(9, 3), v27.reshape(9, 3)


def test_rk8_stationary():
    # rk8_test.cu:34-155
    L = O.lib()
    r27 = np.zeros(27)
    v27 = np.zeros(27)
    st = O.OrTime(2000, 1, 1, 0, 0, 0.0)
    L.or_rk8(None, O.FORCE["zero"], C.byref(st), 1.0, O.ptr(np.ones(3)), O.ptr(np.zeros(3)), 0,
             O.ptr(r27), O.ptr(v27))
    assert np.all(r27 == 1.0) and np.all(v27 == 0.0)


@pytest.mark.parametrize("kind", ["zero", "poly7", "poly8"])
def test_rk8_exact_to_degree8(kind):
    # rk8_test.cu:197-250 (EXPECT_DOUBLE_EQ; here: within 16 ulp, cuBLAS order differs)
    r, _ = _rk8(kind)
    exp = np.array([[POLY[kind](i)] * 3 for i in range(-4, 5)])
    assert np.all((ulps(r, exp) <= 16) | (np.abs(r - exp) < 1e-15))


def test_rk8_degree9_not_exact():
    # rk8_test.cu:252-261
    r, _ = _rk8("poly9")
    exp = np.array([[POLY["poly9"](i)] * 3 for i in range(-4, 5)])
    assert np.abs(r - exp).max() > 1e-10


def _startup(kind, h, ncorr, r0, v0):
    L = O.lib()
    out = [np.zeros(27) for _ in range(5)]
    st = O.OrTime(2000, 1, 1, 0, 0, 0.0)
    L.or_startup(None, O.FORCE[kind], C.byref(st), h, ncorr, O.ptr(O.f64(r0)), O.ptr(O.f64(v0)),
                 0, *[O.ptr(x) for x in out])
    return [x.reshape(9, 3) for x in out]


@pytest.mark.parametrize("kind,tol", [("zero", 0.0), ("poly7", 1e-10), ("poly8", 1e-13)])
def test_startup_exact(kind, tol):
    # startup_test.cu:111-144 (EXPECT_NEAR with 0 / 1e-10 / 1e-13; values up to 9e4, so the
    # bound here is max(tol, 2 ulp))
    r, *_ = _startup(kind, 1.0, 5, np.zeros(3), np.zeros(3))
    exp = np.array([[POLY[kind](i)] * 3 for i in range(-4, 5)])
    err = np.abs(r - exp)
    assert np.all((err <= tol) | (ulps(r, exp) <= 2))


def _corrector(kind, h, op, pm, vm):
    L = O.lib()
    pm = O.f64(pm).copy()
    vm = O.f64(vm).copy()
    a = np.zeros(27)
    s = np.zeros(27)
    S = np.zeros(27)
    L.or_corrector_unit(O.FORCE[kind], h, op, O.ptr(pm), O.ptr(vm), O.ptr(a), O.ptr(s), O.ptr(S))
    return pm.reshape(9, 3), vm.reshape(9, 3), a.reshape(9, 3), s.reshape(9, 3), S.reshape(9, 3)


def test_startup_s0_hand_values():
    # startup_test.cu:146-200: s0 = 2.075075590567601, S0 = 0.924524968616072
    m = np.repeat(np.arange(9.0), 3)
    _, _, _, s, S = _corrector("exp", 2.0, 1, m, m)
    assert np.all(ulps(s[4], 2.075075590567601) <= 4)
    assert np.all(np.abs(S[4] - 0.924524968616072) <= 1e-7 * 0.924524968616072)


def test_startup_corrector_s_hand_values():
    # startup_test.cu:202-262 (EXPECT_FLOAT_EQ)
    m = np.repeat(np.arange(9.0), 3)
    _, _, _, s, S = _corrector("exp", 2.0, 2, m, m)
    es = [-1.954319917555107e3, -0.262126527287875e3, -0.033113055524935e3,
          -0.002119452458898e3, 0.002075075590568e3, 0.002642743232186e3, 0.002719568693249e3,
          0.002729965888781e3, 0.002731372996184e3]
    eS = [5.294164844621613e2, 0.655755604279188e2, 0.051634298864115e2, -0.006505506219515e2,
          0.009245249686161e2, 0.034996005591837e2, 0.062100114329879e2, 0.089387379456808e2,
          0.116699432105504e2]
    for i in range(9):
        assert np.all(np.abs(s[i] - es[i]) <= 1e-6 * abs(es[i]))
        assert np.all(np.abs(S[i] - eS[i]) <= 1e-6 * abs(eS[i]))


def test_startup_corrector_acceleration_matrix():
    # startup_test.cu:278-341 (damped oscillator, EXPECT_DOUBLE_EQ)
    vm = np.repeat([8, 6, 4, 2, 0, -2, -4, -6, -8.0], 3)
    pm = np.repeat([-15, -8, -3, 0, 1, 0, 3, 8, 15.0], 3)
    _, _, a, _, _ = _corrector("damped", 2.0, 0, pm, vm)
    assert np.all(a[:, 0] == [14, 4, -2, -4, -2, 4, 2, -4, -14])


def test_startup_oscillator_convergence():
    # startup_test.cu:264-276: error falls with every extra correction (1..4)
    exact = lambda t: np.exp(-t) * (np.sin(t) + np.cos(t))
    exp = np.array([[exact(i * 0.1)] * 3 for i in range(-4, 5)])
    prev = np.inf
    for nc in range(1, 5):
        r, *_ = _startup("damped", 0.1, nc, np.ones(3), np.zeros(3))
        err = np.linalg.norm(r - exp)
        assert err < prev
        prev = err


def test_predictor_hand_values():
    # integrator_prediction_test.cu:26-101
    L = O.lib()
    r = np.zeros(3)
    v = np.zeros(3)
    a = np.repeat(np.arange(1, 10, dtype=float), 3)
    s = np.full(3, 2.0)
    S = np.ones(3)
    L.or_predict_unit(O.FORCE["poly7"], 0.1, 5, O.ptr(r), O.ptr(v), O.ptr(a), O.ptr(s), O.ptr(S))
    assert np.all(np.abs(r - 0.083333333333333) <= 1e-7 * 0.0833)
    # the predictor sum cancels (sum |c_k a_k| / |sum c_k a_k| ~ 60): bound 1e-14 relative
    assert np.all(np.abs(v - 1.141666666666669) <= 1e-14 * 1.1417)


def test_finalize_correction_hand_values():
    # integrator_test.cu:207-261
    L = O.lib()
    r = np.ones(3)
    v = np.full(3, 2.0)
    a = np.repeat(np.arange(1, 10, dtype=float), 3)
    L.or_finalize_correction_unit(0.1, O.ptr(r), O.ptr(v), O.ptr(a), O.ptr(np.full(3, 4.0)),
                                  O.ptr(np.full(3, 3.0)))
    assert np.all(np.abs(v - 0.408277901785714) <= 1e-7 * 0.408)
    assert np.all(np.abs(r - 0.045496538487554) <= 1e-7 * 0.0455)


def test_integrator_stationary_and_constant_speed():
    # integrator_test.cu:54-110
    r0 = np.array([[0, 0, 0], [1, 1, 1.0]])
    _, _, rs, vs, _ = O.propagate(None, "zero", None, 1.0, 10, r0, np.zeros((2, 3)),
                                  per_step=True)
    assert np.all(rs == r0[None]) and np.all(vs == 0.0)
    _, _, rs, vs, _ = O.propagate(None, "zero", None, 1.0, 10, r0, np.ones((2, 3)), per_step=True)
    for i in range(10):
        assert np.all(ulps(rs[i], r0 + i + 1) <= 4)
        assert np.all(vs[i] == 1.0)


@pytest.mark.parametrize("kind,bound", [("poly7", 1e-13), ("poly8", 2e-13)])
def test_integrator_polynomial_global_error(kind, bound):
    # integrator_test.cu:166-188 (20 steps of 0.1, one correction)
    _, _, rs, _, _ = O.propagate(None, kind, None, 0.1, 20, np.zeros(3), np.zeros(3), ncorr=1,
                                 per_step=True)
    err = max(np.linalg.norm(rs[i, 0] - POLY[kind]((i + 1) * 0.1)) for i in range(20))
    assert err <= bound


def test_integrator_convergence():
    # integrator_test.cu:190-205
    exact = lambda t: np.exp(-t) * (np.sin(t) + np.cos(t))
    prev = np.inf
    for nc in range(1, 6):
        _, _, rs, _, _ = O.propagate(None, "damped", None, 0.1, 40, np.ones(3), np.zeros(3),
                                     ncorr=nc, per_step=True)
        err = max(np.linalg.norm(rs[i, 0] - exact((i + 1) * 0.1)) for i in range(40))
        assert err < prev
        prev = err


def test_propagator_batch_invariance(oracle_data):
    # propagator_test.cu:38-83 (8 identical objects, 10 steps, real force model)
    r0 = np.tile([-3884872.0, -5749111.0, 14723.0], (8, 1))
    v0 = np.tile([-795.304, 573.772, 7518.179], (8, 1))
    _, _, rs, vs, _ = O.propagate(oracle_data, "gravity", (2015, 5, 4, 22, 22, 2.0), 30.0, 10, r0,
                                  v0, per_step=True)
    assert np.all(rs == rs[:, :1]) and np.all(vs == vs[:, :1])


# ---------------- closest approach (closest_approach_utils_test.cu, closest_approach_test.cu) ----

def test_partition_parameters():
    # closest_approach_utils_test.cu:29-47
    p = O.partition([0, 0, 0, 1, 1, 2, 2, 2, 3, 3])
    assert p["num_sets"] == 4
    assert list(p["set_offsets"]) == [0, 3, 5, 8]
    assert list(p["num_higher"]) == [7, 5, 2, 0]
    assert list(p["map_offsets"]) == [0, 21, 31, 37]


def test_partition_invalid():
    # closest_approach_utils_test.cu:49-60
    assert O.partition([0, 0, 0, 1, 1, 2, 2, 2, 3, 0]) is None
    assert O.partition([0, 0, 0, 1, 1, 2, 2, 2, 3, 5]) is None
    assert O.partition([0, 0, 0, 1, 1, 3, 2, 2, 3, 3]) is None


def _map_idx(p, a, b):
    L = O.lib()
    return L.or_partition_map_idx(O.ptr(p["ids"]), p["num_sets"], O.ptr(p["set_offsets"]),
                                  O.ptr(p["num_higher"]), O.ptr(p["map_offsets"]), a, b)


def _map_pair(p, idx):
    L = O.lib()
    a = C.c_uint32()
    b = C.c_uint32()
    ok = L.or_partition_map_pair(p["num_sets"], O.ptr(p["set_offsets"]), O.ptr(p["num_higher"]),
                                 O.ptr(p["map_offsets"]), idx, C.byref(a), C.byref(b))
    return (a.value, b.value) if ok else None


def test_partition_valid_pairs():
    # closest_approach_utils_test.cu:62-94
    p = O.partition([0, 0, 0, 1, 1, 1, 2])
    assert _map_idx(p, 0, 3) == 0 and _map_idx(p, 1, 6) == 7 and _map_idx(p, 1, 3) == 4
    assert _map_idx(p, 3, 6) == 12 and _map_idx(p, 6, 5) == 14
    assert _map_pair(p, 0) == (0, 3) and _map_pair(p, 7) == (1, 6) and _map_pair(p, 4) == (1, 3)
    assert _map_pair(p, 12) == (3, 6) and _map_pair(p, 14) == (5, 6)


def test_partition_one_set_and_invalid_pairs():
    # closest_approach_utils_test.cu:96-129
    p = O.partition([0, 0, 0, 0])
    assert p["num_sets"] == 1 and p["num_pairs"] == 0
    p = O.partition([0, 0, 0, 1, 1, 2, 2, 2, 3, 3])
    assert _map_idx(p, 0, 1) == -1 and _map_idx(p, 8, 9) == -1
    assert _map_pair(p, 37) is None


def _herm(q, dt):
    c = np.zeros(9)
    O.lib().or_hermite_coeffs(O.ptr(O.f64(q)), dt, O.ptr(c))
    return c


def test_hermite_cases():
    L = O.lib()
    # constant (closest_approach_utils_test.cu:131-154)
    c = _herm([5, 0, 0, 5, 0, 0, 5, 0, 0], 1.0)
    assert c[0] == 5 and np.all(c[1:] == 0)
    # linear 2t+1 (:156-180)
    c = _herm([1, 2, 0, 3, 2, 0, 5, 2, 0], 1.0)
    assert c[0] == 1 and c[1] == 2 and np.all(c[2:] == 0)
    for t, val in [(0.5, 2.0), (1.5, 4.0), (2.0, 5.0)]:
        assert L.or_hermite_eval(O.ptr(c), 1.0, t) == val
        assert L.or_hermite_deriv(O.ptr(c), 1.0, t) == 2.0
    # quadratic t^2 with dt=2 (:182-204)
    c = _herm([0, 0, 2, 4, 4, 2, 16, 8, 2], 2.0)
    assert list(c[:3]) == [0, 0, 1] and np.all(c[3:] == 0)
    assert L.or_hermite_eval(O.ptr(c), 2.0, 3.0) == 9.0
    assert L.or_hermite_deriv(O.ptr(c), 2.0, 3.0) == 6.0
    # t^3 - t (:206-234)
    c = _herm([0, -1, 0, 0, 2, 6, 6, 11, 12], 1.0)
    assert list(c[:4]) == [0, -1, 0, 1] and np.all(c[4:] == 0)
    assert L.or_hermite_eval(O.ptr(c), 1.0, 0.5) == -0.375
    assert L.or_hermite_deriv(O.ptr(c), 1.0, 0.5) == -0.25
    # extrapolation t^2 (:236-253)
    c = _herm([0, 0, 2, 1, 2, 2, 4, 4, 2], 1.0)
    assert L.or_hermite_eval(O.ptr(c), 1.0, -1.0) == 1.0
    assert L.or_hermite_deriv(O.ptr(c), 1.0, 3.0) == 6.0


def test_find_root_cases():
    # closest_approach_utils_test.cu:267-296
    L = O.lib()
    assert abs(L.or_find_root_test(0, 0.0, 1.0, 1e-7, 100) - 2.0) < 1e-7
    assert abs(L.or_find_root_test(1, 1.0, 5.0, 1e-7, 100) - 3.0) < 1e-7
    assert abs(L.or_find_root_test(1, -1.0, -5.0, 1e-7, 100) + 3.0) < 1e-7
    assert L.or_find_root_test(2, -2.0, 2.0, 1e-7, 100) == 2.0


def _approach_objects():
    ax = [0, 1, 0, 1, 1, 0, 2, 1, 0]
    ay = [2, 0, 0, 2, 0, 0, 2, 0, 0]
    az = [0] * 9
    by = [0, -3, 1, -2.5, -2, 1, -4, -1, 1]
    return O.f64(ax + ay + az), O.f64(ax + by + az)


def test_approach_func_and_root():
    # closest_approach_utils_test.cu:298-346
    L = O.lib()
    A, B = _approach_objects()
    for t, val in [(0.0, 6.0), (1.0, 9.0), (2.0, 6.0), (3.0, 0.0), (4.0, -6.0)]:
        assert L.or_approach_func(O.ptr(A), O.ptr(B), 1.0, t) == val
    root = L.or_find_root_approach(O.ptr(A), O.ptr(B), 1.0, 2.0, 10.0, 1e-12, 100)
    assert abs(root - 3.0) < 1e-12


def _ca(pos, vel, sets, h, phases):
    total = sum(phases)
    rs_all, vs_all, as_all = [], [], []
    r = np.array(pos, float)
    v = np.array(vel, float)
    for n in phases:  # each Propagate() call runs its own startup from the current state
        rf, vf, rs, vs, as_ = O.propagate(None, "zero", None, h, n, r, v, per_step=True)
        rs_all.append(rs)
        vs_all.append(vs)
        as_all.append(as_)
        r, v = rf, vf
    res = O.closest_approach(np.concatenate(rs_all), np.concatenate(vs_all),
                             np.concatenate(as_all), sets, h, phases=phases)
    assert total == sum(phases)
    return res


def test_ca_head_on():
    # closest_approach_test.cu:60-88
    res = _ca([[0, 0, 0], [10, 0, 0]], [[1, 0, 0], [-1, 0, 0]], [0, 1], 0.5, [10])
    assert abs(res["distance"][0]) < 1e-14 and abs(res["time"][0] - 5.0) < 1e-14


def test_ca_parallel():
    # closest_approach_test.cu:90-117
    res = _ca([[0, 0, 0], [5, 0, 0]], [[0, 2, 0], [0, 2, 0]], [0, 1], 0.5, [20])
    assert res["distance"][0] == 5.0 and res["time"][0] >= 0.0


def test_ca_multi_phase_global_minimum():
    # closest_approach_test.cu:119-157
    pos = [[0, 0, 0], [10, 0, 0]]
    vel = [[0, 0, 0], [-1, 0, 0]]
    res = _ca(pos, vel, [0, 1], 0.1, [40])
    assert abs(res["distance"][0] - 6.0) < 1e-14
    res = _ca(pos, vel, [0, 1], 0.1, [40, 60])
    assert abs(res["distance"][0]) < 1e-14 and abs(res["time"][0] - 10.0) < 1e-14
    res = _ca(pos, vel, [0, 1], 0.1, [40, 60, 50])
    assert abs(res["distance"][0]) < 1e-14 and abs(res["time"][0] - 10.0) < 1e-14


def test_ca_between_steps():
    # closest_approach_test.cu:159-186
    res = _ca([[0, 0, 0], [0.5, 3, 0]], [[0, 0, 0], [-2, 0, 0]], [0, 1], 0.1, [5])
    assert abs(res["distance"][0] - 3.0) < 1e-14 and abs(res["time"][0] - 0.25) < 1e-14


def test_ca_multi_object_sets():
    # closest_approach_test.cu:188-229
    pos = [[0, 0, 0], [10, 5, 0], [3, 0, 8]]
    vel = [[0, 0, 0], [-1, 0, 0], [0, 0, -2]]
    res = _ca(pos, vel, [0, 1, 1], 0.1, [120])
    p = res["partition"]
    i01 = _map_idx(p, 0, 1)
    i02 = _map_idx(p, 0, 2)
    assert abs(res["distance"][i01] - 5.0) < 1e-14 and abs(res["time"][i01] - 10.0) < 1e-14
    assert abs(res["distance"][i02] - 3.0) < 1e-14 and abs(res["time"][i02] - 4.0) < 1e-14


def test_long_double_miss_matches_double_oracle(oracle_data):
    # the extended-precision copy of the oracle's propagation, screen and refinement (used only for
    # finite differences) agrees with the double oracle on the miss distance and TCA of a pair
    from opengpop_b200 import orbits
    r, v, pairs = orbits.conjunction_pairs(2, 20240101)
    a, b = pairs[0]
    start, h, steps = (2024, 1, 1, 0, 0, 0.0), 30.0, 60
    m_ld, t_ld, grad = O.miss_fd_ld(oracle_data, start, h, steps, r[a], v[a], r[b], v[b], 1.0, 1e-3)
    _, _, rs, vs, as_ = O.propagate(oracle_data, "gravity", start, h, steps, r[[a, b]], v[[a, b]],
                                    per_step=True)
    o = O.closest_approach(rs, vs, as_, np.array([0, 1], np.uint32), h)
    assert abs(m_ld[0] - o["distance"][0]) <= 1e-9 * o["distance"][0]
    assert abs(t_ld[0] - o["time"][0]) <= 1e-6
    # d miss / d r0_A along the line of sight is close to the unit vector early on: bounded, finite
    assert np.all(np.isfinite(grad)) and np.linalg.norm(grad[0, :3]) < 10.0
