"""Argument checks of the force-free integrator pieces (gpop_rk8_stage ... gpop_gj8_coefficients),
the C ABI behind the per-evaluation path of the C++ mirror. They are rejected on the host before
any CUDA call, with a NULL context, so these run without a GPU."""
import ctypes as C

import pytest

INVALID = 1
OK = 0


@pytest.fixture(scope="module")
def lib():
    import opengpop_b200 as G
    return C.CDLL(G.LIB_PATH)


def _p(x=1):
    # a non-NULL pointer that is never dereferenced (every call below fails or returns first)
    return C.c_void_p(x * 4096)


def test_rk8_stage_checks(lib):
    f = lib.gpop_rk8_stage
    f.restype = C.c_int32
    f.argtypes = [C.c_void_p, C.c_int64, C.c_double, C.c_int32, C.c_int32] + [C.c_void_p] * 7
    args = [_p()] * 6 + [None]
    assert f(None, -1, 30.0, 1, 0, *args) == INVALID  # negative n
    assert f(None, 4, 0.0, 1, 0, *args) == INVALID  # step size
    assert f(None, 4, 30.0, 0, 0, *args) == INVALID  # startup step 0
    assert f(None, 4, 30.0, 5, 0, *args) == INVALID  # beyond +-4
    assert f(None, 4, 30.0, -1, 10, *args) == INVALID  # stage 10
    assert f(None, 0, 30.0, 1, 3, *args) == OK  # nothing to do
    assert f(None, 4, 30.0, 1, 3, None, None, None, None, None, None, None) == INVALID  # buffers


def test_startup_and_gj8_checks(lib):
    fin = lib.gpop_rk8_finish
    fin.restype = C.c_int32
    fin.argtypes = [C.c_void_p, C.c_int64, C.c_double, C.c_int32] + [C.c_void_p] * 5
    assert fin(None, 4, 30.0, -5, _p(), _p(), _p(), _p(), None) == INVALID
    assert fin(None, 4, 30.0, 2, None, _p(), _p(), _p(), None) == INVALID
    init = lib.gpop_startup_init
    init.restype = C.c_int32
    init.argtypes = [C.c_void_p, C.c_int64] + [C.c_void_p] * 8
    assert init(None, 4, None, _p(), _p(), _p(), None, None, None, None) == INVALID
    assert init(None, -2, _p(), _p(), _p(), _p(), None, None, None, None) == INVALID
    cor = lib.gpop_startup_correct
    cor.restype = C.c_int32
    cor.argtypes = [C.c_void_p, C.c_int64, C.c_double] + [C.c_void_p] * 6
    assert cor(None, 4, -30.0, _p(), _p(), _p(), _p(), _p(), None) == INVALID
    assert cor(None, 4, 30.0, _p(), _p(), None, _p(), _p(), None) == INVALID
    for name in ("gpop_gj8_predict", "gpop_gj8_correct"):
        g = getattr(lib, name)
        g.restype = C.c_int32
        g.argtypes = [C.c_void_p, C.c_int64, C.c_double] + [C.c_void_p] * 9
        bufs = [_p()] * 8
        assert g(None, 4, float("nan"), *bufs, None) == INVALID
        assert g(None, 4, 30.0, *(bufs[:-1] + [None]), None) == INVALID
        assert g(None, 0, 30.0, *bufs, None) == OK


def test_matrix_column_checks(lib):
    f = lib.gpop_matrix_column
    f.restype = C.c_int32
    f.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_int32,
                  C.c_void_p]
    assert f(None, 4, _p(), 9, 9, _p(), 0, None) == INVALID  # column outside [0, 9)
    assert f(None, 4, _p(), 0, 0, _p(), 0, None) == INVALID  # no columns
    assert f(None, 4, _p(), 10, -1, _p(), 1, None) == INVALID
    assert f(None, 4, None, 9, 8, _p(), 0, None) == INVALID
    assert f(None, 0, None, 9, 8, None, 0, None) == OK


def test_coefficients_without_buffers(lib):
    f = lib.gpop_gj8_coefficients
    f.restype = C.c_int32
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    assert f(None, None, None, None) == OK


def test_closest_approach_row_calls_without_object(lib):
    # the sharded screen's entry points reject a missing object before any CUDA call
    rows = lib.gpop_ca_set_rows
    rows.restype = C.c_int32
    rows.argtypes = [C.c_void_p, C.c_int64, C.c_int64]
    assert rows(None, 0, 64) == INVALID
    rng = lib.gpop_ca_pair_range
    rng.restype = C.c_int32
    rng.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lo, hi = C.c_int64(), C.c_int64()
    assert rng(None, C.byref(lo), C.byref(hi)) == INVALID
    res = lib.gpop_ca_reserve
    res.restype = C.c_int32
    res.argtypes = [C.c_void_p, C.c_int32]
    assert res(None, 100) == INVALID
