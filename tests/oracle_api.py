"""ctypes binding of the CPU oracle (oracle/liboracle.so).

Test infrastructure only: the oracle is the checker for the CUDA product and is never imported by
the product package.
"""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
DATA_DIR = os.path.join(ROOT, "opengpop_b200", "data")

FORCE = {"gravity": 0, "zero": 1, "const": 2, "poly7": 3, "poly8": 4, "poly9": 5, "exp": 6,
         "damped": 7}
FLAG_FIX_Q1 = 1
FLAG_FIX_Q3 = 2


class OrTime(C.Structure):
    _fields_ = [("year", C.c_int32), ("month", C.c_int32), ("day", C.c_int32),
                ("hour", C.c_int32), ("min", C.c_int32), ("sec", C.c_double)]


class OrCaState(C.Structure):
    _fields_ = [("min_dist", C.c_void_p), ("closest_step", C.c_void_p), ("nodes", C.c_void_p),
                ("last", C.c_void_p)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(ORACLE_DIR, "liboracle.so")
        if not os.path.exists(path):
            subprocess.check_call(["make", "-s", "-C", ORACLE_DIR])
        _lib = C.CDLL(path)
        _lib.or_data_load.restype = C.c_void_p
        _lib.or_data_load.argtypes = [C.c_char_p, C.c_int32]
        for fn in ("or_data_gm", "or_data_radius", "or_calendar_to_mjd", "or_gast",
                   "or_ntp_to_mjd", "or_data_leap_seconds", "or_hermite_eval", "or_hermite_deriv",
                   "or_approach_func", "or_find_root_approach", "or_find_root_test"):
            getattr(_lib, fn).restype = C.c_double
        _lib.or_data_degree.restype = C.c_int32
        for fn in ("or_data_eop_count", "or_data_leap_count", "or_data_nut_count",
                   "or_partition_map_idx"):
            getattr(_lib, fn).restype = C.c_int64
        _lib.or_calendar_to_mjd.argtypes = [C.c_int32] * 5 + [C.c_double]
        _lib.or_gast.argtypes = [C.c_double] * 4 + [C.c_void_p]
        _lib.or_ntp_to_mjd.argtypes = [C.c_int64]
        _lib.or_data_leap_seconds.argtypes = [C.c_void_p, C.c_double]
        _lib.or_hermite_eval.argtypes = [C.c_void_p, C.c_double, C.c_double]
        _lib.or_hermite_deriv.argtypes = [C.c_void_p, C.c_double, C.c_double]
        _lib.or_hermite_coeffs.argtypes = [C.c_void_p, C.c_double, C.c_void_p]
        _lib.or_approach_func.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_double]
        _lib.or_find_root_approach.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_double,
                                               C.c_double, C.c_double, C.c_int32]
        _lib.or_find_root_test.argtypes = [C.c_int32, C.c_double, C.c_double, C.c_double,
                                           C.c_int32]
        _lib.or_ftable.argtypes = [C.c_double, C.c_void_p]
        _lib.or_precession.argtypes = [C.c_double, C.c_void_p]
        _lib.or_nutation.argtypes = [C.c_void_p, C.c_double, C.c_void_p]
        _lib.or_rot.argtypes = [C.c_int32, C.c_double, C.c_void_p]
        _lib.or_data_eop_record.argtypes = [C.c_void_p, C.c_double, C.c_void_p]
        _lib.or_data_coef.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]
        for fn in ("or_data_gm", "or_data_radius", "or_data_degree", "or_data_eop_count",
                   "or_data_leap_count", "or_data_free"):
            getattr(_lib, fn).argtypes = [C.c_void_p]
        _lib.or_data_nut_count.argtypes = [C.c_void_p, C.c_int32]
        _lib.or_frame_matrices.argtypes = [C.c_void_p, C.POINTER(OrTime), C.c_double, C.c_int32,
                                           C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]
        _lib.or_gravity.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.or_rk8.argtypes = [C.c_void_p, C.c_int32, C.POINTER(OrTime), C.c_double, C.c_void_p,
                                C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
        _lib.or_startup.argtypes = [C.c_void_p, C.c_int32, C.POINTER(OrTime), C.c_double,
                                    C.c_int32, C.c_void_p, C.c_void_p, C.c_uint32] + [C.c_void_p] * 5
        _lib.or_corrector_unit.argtypes = [C.c_int32, C.c_double, C.c_int32] + [C.c_void_p] * 5
        _lib.or_predict_unit.argtypes = [C.c_int32, C.c_double, C.c_int32] + [C.c_void_p] * 5
        _lib.or_finalize_correction_unit.argtypes = [C.c_double] + [C.c_void_p] * 5
        _lib.or_propagate.restype = C.c_int32
        _lib.or_propagate.argtypes = [C.c_void_p, C.c_int32, C.POINTER(OrTime), C.c_double,
                                      C.c_int32, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p,
                                      C.c_uint32] + [C.c_void_p] * 5 + [C.c_int32]
        _lib.or_partition.restype = C.c_int32
        _lib.or_partition.argtypes = [C.c_void_p, C.c_int64] + [C.c_void_p] * 5
        _lib.or_partition_map_idx.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                              C.c_void_p, C.c_uint32, C.c_uint32]
        _lib.or_partition_map_pair.restype = C.c_int32
        _lib.or_partition_map_pair.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                               C.c_uint64, C.c_void_p, C.c_void_p]
        _lib.or_ca_screen.argtypes = [C.c_int64, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_uint32, C.c_int32, C.POINTER(OrCaState),
                                      C.c_int32]
        _lib.or_ca_refine.argtypes = [C.c_int64, C.c_void_p, C.c_double, C.c_uint32,
                                      C.POINTER(OrCaState)] + [C.c_void_p] * 4 + [C.c_int32]
        for fn in ("or_miss_fd_ld", "or_miss_fd"):
            getattr(_lib, fn).restype = C.c_int32
            getattr(_lib, fn).argtypes = [C.c_void_p, C.POINTER(OrTime), C.c_double, C.c_int32,
                                          C.c_int32, C.c_int64] + [C.c_void_p] * 4 + [
                C.c_double, C.c_double] + [C.c_void_p] * 3 + [C.c_int32]
    return _lib


def ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Data:
    """Loaded model data sets (gravity field, nutation, EOP, leap seconds)."""

    def __init__(self, degree=0, data_dir=DATA_DIR):
        self.h = lib().or_data_load(data_dir.encode(), degree)
        if not self.h:
            raise RuntimeError("oracle could not load data from %s" % data_dir)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.or_data_free(self.h)
            self.h = None

    @property
    def degree(self):
        return lib().or_data_degree(self.h)

    @property
    def gm(self):
        return lib().or_data_gm(self.h)

    @property
    def radius(self):
        return lib().or_data_radius(self.h)


def tstruct(t):
    return OrTime(*t) if not isinstance(t, OrTime) else t


def gravity(data, r, m9=None):
    r = f64(r).reshape(-1, 3)
    a = np.zeros_like(r)
    lib().or_gravity(data.h, r.shape[0], ptr(r), None if m9 is None else ptr(f64(m9)), ptr(a))
    return a


def frame_matrices(data, start, h, count, midpoints=False, before=4):
    m = np.zeros((count, 9))
    mjd = np.zeros(count)
    lib().or_frame_matrices(data.h, C.byref(tstruct(start)), h, count, int(midpoints), before,
                            ptr(m), ptr(mjd))
    return m, mjd


def propagate(data, kind, start, h, steps, r0, v0, ncorr=7, flags=0, per_step=False, threads=0):
    r0 = f64(r0).reshape(-1, 3)
    v0 = f64(v0).reshape(-1, 3)
    n = r0.shape[0]
    rf = np.zeros_like(r0)
    vf = np.zeros_like(v0)
    rs = vs = as_ = None
    if per_step:
        rs = np.zeros((steps, n, 3))
        vs = np.zeros((steps, n, 3))
        as_ = np.zeros((steps, n, 3))
    k = FORCE[kind] if isinstance(kind, str) else kind
    st = tstruct(start if start is not None else (2000, 1, 1, 0, 0, 0.0))
    rc = lib().or_propagate(data.h if data is not None else None, k, C.byref(st), h, steps, ncorr,
                            n, ptr(r0), ptr(v0), flags, ptr(rs), ptr(vs), ptr(as_), ptr(rf),
                            ptr(vf), threads)
    if rc != 0:
        raise RuntimeError("oracle propagate failed")
    return (rf, vf, rs, vs, as_) if per_step else (rf, vf)


def partition(set_ids):
    ids = np.ascontiguousarray(set_ids, dtype=np.uint32)
    n = ids.shape[0]
    so = np.zeros(n, np.uint32)
    nh = np.zeros(n, np.uint32)
    mo = np.zeros(n, np.uint64)
    ns = C.c_uint32()
    npairs = C.c_uint64()
    ok = lib().or_partition(ptr(ids), n, C.byref(ns), C.byref(npairs), ptr(so), ptr(nh), ptr(mo))
    if not ok:
        return None
    k = ns.value
    return dict(ids=ids, num_sets=k, num_pairs=npairs.value, set_offsets=so[:k].copy(),
                num_higher=nh[:k].copy(), map_offsets=mo[:k].copy())


def closest_approach(r_steps, v_steps, a_steps, set_ids, h, phases=None, threads=0):
    """Reference semantics over a trajectory (steps x n x 3 arrays). Returns per-pair arrays
    (distance, time, posA, posB, closest_step) in the reference's pair order."""
    r_steps, v_steps, a_steps = f64(r_steps), f64(v_steps), f64(a_steps)
    steps, n, _ = r_steps.shape
    p = partition(set_ids)
    P = p["num_pairs"]
    md = np.zeros(P)
    cs = np.zeros(P, np.uint32)
    nodes = np.zeros(P * 54)
    last = np.zeros(n * 9)
    st = OrCaState(md.ctypes.data, cs.ctypes.data, nodes.ctypes.data, last.ctypes.data)
    ids = p["ids"]
    bounds = phases if phases is not None else [steps]
    off = 0
    for i, cnt in enumerate(bounds):
        lib().or_ca_screen(n, cnt, ptr(r_steps[off:off + cnt]), ptr(v_steps[off:off + cnt]),
                           ptr(a_steps[off:off + cnt]), ptr(ids), off, int(i == 0), C.byref(st),
                           threads)
        off += cnt
    dist = np.zeros(P)
    tim = np.zeros(P)
    pa = np.zeros((P, 3))
    pb = np.zeros((P, 3))
    lib().or_ca_refine(n, ptr(ids), h, off, C.byref(st), ptr(dist), ptr(tim), ptr(pa), ptr(pb),
                       threads)
    return dict(distance=dist, time=tim, posA=pa, posB=pb, closest_step=cs, min_sampled=md,
                partition=p)


def miss_fd_ld(data, start, h, steps, rA, vA, rB, vB, dr, dv, ncorr=7, threads=0, long=True):
    """Miss distance, TCA and the central-difference gradient of the miss distance (steps dr in
    m, dv in m/s) per pair, computed in long double (or_miss_fd_ld; double with long=False).
    Returns (miss, tca, grad [n, 12] ordered r0_A, v0_A, r0_B, v0_B)."""
    rA, vA, rB, vB = (f64(x).reshape(-1, 3) for x in (rA, vA, rB, vB))
    n = rA.shape[0]
    miss = np.zeros(n)
    tca = np.zeros(n)
    grad = np.zeros((n, 12))
    fn = lib().or_miss_fd_ld if long else lib().or_miss_fd
    rc = fn(data.h, C.byref(tstruct(start)), h, steps, ncorr, n, ptr(rA), ptr(vA), ptr(rB), ptr(vB),
            dr, dv, ptr(miss), ptr(tca), ptr(grad), threads)
    if rc != 0:
        raise RuntimeError("oracle or_miss_fd_ld failed")
    return miss, tca, grad
