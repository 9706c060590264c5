"""opengpop_b200 -- B200 (sm_100a) propagation and closest-approach library.

Python binding of the C ABI in include/gpop.h (libgpop.so, built in-tree into
opengpop_b200/lib/). Device memory for the *_device calls comes from torch tensors (plumbing only);
every computation runs in the library's own CUDA kernels. Importing works without a GPU; creating a
Context needs the built library and a CUDA device, and fails loudly otherwise.
"""
import ctypes as C
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libgpop.so")
DATA_DIR = os.path.join(PKG_DIR, "data")

OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "model data error",
          4: "out of memory", 5: "device wait timed out", 6: "unsupported", 7: "call out of order"}
FP64, MIXED = 0, 1
FIX_BACKWARD_RK8_EPOCH = 1
FIX_STARTUP_EXPORT_ACC = 2
FIX_PHASE_EPOCH = 4
MIXED_COMPENSATED = 8
FORCE = {"gravity": 0, "zero": 1, "const": 2, "poly7": 3, "poly8": 4, "poly9": 5, "exp": 6,
         "damped": 7}

# Every symbol include/gpop.h declares (checked by the test suite against the built library).
EXPORTS = (
    "gpop_config_default", "gpop_create", "gpop_destroy", "gpop_last_error", "gpop_status_string",
    "gpop_gravity_degree", "gpop_kernel_launches", "gpop_propagate", "gpop_propagate_device",
    "gpop_propagate_device_noalloc", "gpop_propagate_trajectory", "gpop_propagator_create", "gpop_propagator_step",
    "gpop_propagator_steps_done", "gpop_propagator_destroy", "gpop_propagate_analytic",
    "gpop_propagate_batch", "gpop_propagate_batch_status", "gpop_batch_plan", "gpop_batch_warps_per_sm", "gpop_tune", "gpop_batch_device_seconds", "gpop_gravity_jacobian", "gpop_stm", "gpop_propagate_vjp",
    "gpop_miss_gradient", "gpop_sample_states", "gpop_startup", "gpop_corrector_unit",
    "gpop_predict_unit", "gpop_finalize_correction_unit", "gpop_rk8_stage", "gpop_rk8_finish",
    "gpop_startup_init", "gpop_startup_correct", "gpop_gj8_predict", "gpop_gj8_correct",
    "gpop_matrix_column", "gpop_gj8_coefficients", "gpop_gravity", "gpop_frame_matrices",
    "gpop_ca_create", "gpop_ca_create_analytic", "gpop_ca_create_external", "gpop_ca_append", "gpop_ca_propagate", "gpop_ca_find", "gpop_ca_pairs", "gpop_ca_num_pairs",
    "gpop_ca_set_rows", "gpop_ca_pair_range", "gpop_ca_reserve", "gpop_walk_policy", "gpop_split_block", "gpop_ca_trajectory", "gpop_ca_device_seconds", "gpop_ca_destroy",
)


class GpopError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s (%d): %s" % (STATUS.get(status, "?"), status, message))
        self.status = status


class Time(C.Structure):
    """TimeData of the reference (lib/common/types/types/Parameters.hpp:19-22)."""
    _fields_ = [("year", C.c_int32), ("month", C.c_int32), ("day", C.c_int32),
                ("hour", C.c_int32), ("min", C.c_int32), ("sec", C.c_double)]


class Config(C.Structure):
    _fields_ = [("data_dir", C.c_char_p), ("device", C.c_int32), ("gravity_degree", C.c_int32),
                ("n_corrections", C.c_int32), ("precision", C.c_int32), ("flags", C.c_uint32)]


class Request(C.Structure):
    _fields_ = [("start", Time), ("h", C.c_double), ("steps", C.c_int32), ("degree", C.c_int32),
                ("n", C.c_int64), ("r_in", C.c_void_p), ("v_in", C.c_void_p),
                ("r_out", C.c_void_p), ("v_out", C.c_void_p)]


class CaRecord(C.Structure):
    _fields_ = [("object_index1", C.c_uint32), ("object_index2", C.c_uint32),
                ("distance", C.c_double), ("time", C.c_double),
                ("position_a", C.c_double * 3), ("position_b", C.c_double * 3)]


_lib = None
_VP = C.c_void_p


def load_library(path=LIB_PATH):
    """Loads libgpop.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError("libgpop.so not built (%s): run __graft_entry__.build() or make -C "
                      "opengpop_b200/csrc" % path)
    lib = C.CDLL(path)
    i32, i64, f64 = C.c_int32, C.c_int64, C.c_double
    sig = {
        "gpop_config_default": (None, [C.POINTER(Config)]),
        "gpop_create": (i32, [C.POINTER(Config), C.POINTER(_VP)]),
        "gpop_destroy": (None, [_VP]),
        "gpop_last_error": (C.c_char_p, [_VP]),
        "gpop_status_string": (C.c_char_p, [i32]),
        "gpop_gravity_degree": (i32, [_VP]),
        "gpop_kernel_launches": (i64, [_VP]),
        "gpop_propagate": (i32, [_VP, C.POINTER(Time), f64, i32, i64, _VP, _VP, _VP, _VP]),
        "gpop_propagate_device": (i32, [_VP, C.POINTER(Time), f64, i32, i64, _VP, _VP, _VP]),
        "gpop_propagate_device_noalloc": (i32, [_VP, C.POINTER(Time), f64, i32, i64, _VP, _VP,
                                                _VP]),
        "gpop_propagate_trajectory": (i32, [_VP, C.POINTER(Time), f64, i32, i64] + [_VP] * 6),
        "gpop_propagator_create": (i32, [_VP, C.POINTER(Time), f64, i32, i64, _VP, _VP,
                                         C.POINTER(_VP)]),
        "gpop_propagator_step": (i32, [_VP, i32, _VP, _VP, _VP, _VP]),
        "gpop_propagator_steps_done": (i32, [_VP]),
        "gpop_propagator_destroy": (None, [_VP]),
        "gpop_propagate_analytic": (i32, [_VP, i32, f64, i32, i32, i64] + [_VP] * 6),
        "gpop_propagate_batch": (i32, [_VP, _VP, i32]),
        "gpop_propagate_batch_status": (i32, [_VP, _VP, i32, _VP]),
        "gpop_batch_plan": (i32, [_VP, _VP, i32, _VP, C.POINTER(f64)]),
        "gpop_tune": (i32, [_VP, C.c_char_p]),
        "gpop_batch_warps_per_sm": (i32, [_VP]),
        "gpop_batch_device_seconds": (f64, [_VP]),
        "gpop_gravity_jacobian": (i32, [_VP, i64, _VP, _VP, _VP, _VP, _VP]),
        "gpop_sample_states": (i32, [_VP, _VP, _VP, f64, f64, C.c_uint64, i64, _VP, _VP, _VP]),
        "gpop_stm": (i32, [_VP, C.POINTER(Time), f64, i32, i64] + [_VP] * 5),
        "gpop_propagate_vjp": (i32, [_VP, C.POINTER(Time), f64, i32, i64] + [_VP] * 6),
        "gpop_miss_gradient": (i32, [_VP, C.POINTER(Time), f64, i32, i64, _VP, _VP, i64]
                               + [_VP] * 4),
        "gpop_startup": (i32, [_VP, i32, C.POINTER(Time), f64, i32] + [_VP] * 8),
        "gpop_corrector_unit": (i32, [_VP, i32, f64, i32] + [_VP] * 6),
        "gpop_predict_unit": (i32, [_VP, i32, f64, i32] + [_VP] * 6),
        "gpop_finalize_correction_unit": (i32, [_VP, f64] + [_VP] * 6),
        "gpop_gravity": (i32, [_VP, i64, _VP, _VP, _VP, i32, _VP]),
        "gpop_frame_matrices": (i32, [_VP, C.POINTER(Time), f64, i32, i32, i32, _VP, _VP, _VP]),
        "gpop_ca_create": (i32, [_VP, C.POINTER(Time), f64, i64, _VP, _VP, _VP, C.POINTER(_VP)]),
        "gpop_ca_create_analytic": (i32, [_VP, i32, f64, i64, _VP, _VP, _VP, C.POINTER(_VP)]),
        "gpop_ca_create_external": (i32, [_VP, f64, i64, _VP, _VP, _VP, C.POINTER(_VP)]),
        "gpop_ca_append": (i32, [_VP, i32, _VP, _VP, _VP]),
        "gpop_ca_propagate": (i32, [_VP, i32]),
        "gpop_ca_find": (i32, [_VP, f64, _VP, i64, C.POINTER(i64)]),
        "gpop_ca_pairs": (i32, [_VP] * 6),
        "gpop_ca_num_pairs": (i64, [_VP]),
        "gpop_ca_set_rows": (i32, [_VP, i64, i64]),
        "gpop_ca_reserve": (i32, [_VP, i32]),
        "gpop_walk_policy": (i32, [i64, i32, i32, C.POINTER(i32)]),
        "gpop_split_block": (i32, [i64, i32, i32]),
        "gpop_ca_pair_range": (i32, [_VP, C.POINTER(i64), C.POINTER(i64)]),
        "gpop_ca_trajectory": (i32, [_VP] * 4 + [C.POINTER(i32)]),
        "gpop_ca_device_seconds": (i32, [_VP, _VP]),
        "gpop_ca_destroy": (None, [_VP]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


WALKS = {1: "one object per thread", 2: "two objects per thread", 3: "lanes",
         4: "lanes per group of two objects"}


def walk_policy(n, num_sms=148, precision=FP64):
    """(walk, lanes per object) the propagation takes for n objects (gpop_walk_policy)."""
    lanes = C.c_int32()
    w = load_library().gpop_walk_policy(int(n), int(num_sms), int(precision), C.byref(lanes))
    if w < 0:
        raise GpopError(1, "invalid arguments to gpop_walk_policy")
    return w, lanes.value


def split_block(n, num_sms=148, degree=70):
    """Owner warps of the split block two objects per thread take for n objects (0: a plain
    block; gpop_split_block)."""
    s = load_library().gpop_split_block(int(n), int(num_sms), int(degree))
    if s < 0:
        raise GpopError(1, "invalid arguments to gpop_split_block")
    return s


def as_time(t):
    if isinstance(t, Time):
        return t
    y, mo, d, hh, mi, s = t
    return Time(int(y), int(mo), int(d), int(hh), int(mi), float(s))


def _host(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a.reshape(shape) if shape is not None else a


def _dptr(t):
    """Device pointer of a CUDA torch tensor (or None)."""
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("expected a contiguous CUDA tensor")
    return C.c_void_p(t.data_ptr())


def _stream_ptr(stream):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream) if hasattr(stream, "cuda_stream") else C.c_void_p(stream)


class Context:
    """A loaded force model and device tables (replaces ForceModel + PreInitialize)."""

    def __init__(self, data_dir=DATA_DIR, device=0, gravity_degree=0, n_corrections=7,
                 precision=FP64, flags=0):
        lib = load_library()
        cfg = Config()
        lib.gpop_config_default(C.byref(cfg))
        self._dir = data_dir.encode()
        cfg.data_dir = self._dir
        cfg.device = device
        cfg.gravity_degree = gravity_degree
        cfg.n_corrections = n_corrections
        cfg.precision = precision
        cfg.flags = flags
        h = _VP()
        st = lib.gpop_create(C.byref(cfg), C.byref(h))
        self._h = h.value
        if st != OK:
            msg = lib.gpop_last_error(self._h).decode() if self._h else ""
            if self._h:
                lib.gpop_destroy(self._h)
                self._h = None
            raise GpopError(st, msg)
        self.device = device
        self.precision = precision
        self.flags = flags

    def close(self):
        if getattr(self, "_h", None):
            load_library().gpop_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != OK:
            raise GpopError(st, load_library().gpop_last_error(self._h).decode())

    @property
    def degree(self):
        return load_library().gpop_gravity_degree(self._h)

    @property
    def kernel_launches(self):
        return load_library().gpop_kernel_launches(self._h)

    # ---- propagation ----
    def propagate(self, start, h, steps, r, v):
        """Host in, host out (exec propagate): returns (r_end, v_end) as [n, 3] arrays."""
        r = _host(r).reshape(-1, 3)
        v = _host(v).reshape(-1, 3)
        ro = np.empty_like(r)
        vo = np.empty_like(v)
        self._check(load_library().gpop_propagate(
            self._h, C.byref(as_time(start)), float(h), int(steps), r.shape[0],
            r.ctypes.data_as(_VP), v.ctypes.data_as(_VP), ro.ctypes.data_as(_VP),
            vo.ctypes.data_as(_VP)))
        return ro, vo

    def propagate_device(self, start, h, steps, r, v, stream=None):
        """In place on CUDA tensors r, v of shape [n, 3] (float64)."""
        self._check(load_library().gpop_propagate_device(
            self._h, C.byref(as_time(start)), float(h), int(steps), r.shape[0], _dptr(r), _dptr(v),
            _stream_ptr(stream)))

    def propagate_trajectory(self, start, h, steps, r, v, traj_r=None, traj_v=None, traj_a=None,
                             stream=None):
        self._check(load_library().gpop_propagate_trajectory(
            self._h, C.byref(as_time(start)), float(h), int(steps), r.shape[0], _dptr(r), _dptr(v),
            _dptr(traj_r), _dptr(traj_v), _dptr(traj_a), _stream_ptr(stream)))

    def propagator(self, start, h, max_steps, r, v):
        """GpuPropagator over CUDA tensors r, v [n, 3] (updated in place by step())."""
        return Propagator(self, start, h, max_steps, r, v)

    def propagate_analytic(self, kind, h, steps, r, v, n_corrections=7, traj_r=None,
                           traj_v=None, traj_a=None, stream=None):
        k = FORCE[kind] if isinstance(kind, str) else kind
        self._check(load_library().gpop_propagate_analytic(
            self._h, k, float(h), int(steps), int(n_corrections), r.shape[0], _dptr(r), _dptr(v),
            _dptr(traj_r), _dptr(traj_v), _dptr(traj_a), _stream_ptr(stream)))

    def startup(self, kind, start, h, n_corrections, r0, v0, out):
        """out: five CUDA tensors [27] (r, v, a, s, S)."""
        k = FORCE[kind] if isinstance(kind, str) else kind
        t = as_time(start if start is not None else (2000, 1, 1, 0, 0, 0.0))
        self._check(load_library().gpop_startup(
            self._h, k, C.byref(t), float(h), int(n_corrections), _dptr(r0), _dptr(v0),
            *[_dptr(x) for x in out], _stream_ptr(None)))

    def corrector_unit(self, kind, h, op, r27, v27, a27, s27, S27):
        k = FORCE[kind] if isinstance(kind, str) else kind
        self._check(load_library().gpop_corrector_unit(
            self._h, k, float(h), int(op), _dptr(r27), _dptr(v27), _dptr(a27), _dptr(s27),
            _dptr(S27), _stream_ptr(None)))

    def predict_unit(self, kind, h, step, r3, v3, a27, s3, S3):
        k = FORCE[kind] if isinstance(kind, str) else kind
        self._check(load_library().gpop_predict_unit(
            self._h, k, float(h), int(step), _dptr(r3), _dptr(v3), _dptr(a27), _dptr(s3),
            _dptr(S3), _stream_ptr(None)))

    def finalize_correction_unit(self, h, r3, v3, a27, s3, S3):
        self._check(load_library().gpop_finalize_correction_unit(
            self._h, float(h), _dptr(r3), _dptr(v3), _dptr(a27), _dptr(s3), _dptr(S3),
            _stream_ptr(None)))

    # ---- batched propagation ----
    def _requests(self, reqs):
        """reqs: list of dicts (start, h, steps, degree, r, v); returns the ctypes array and the
        output arrays (kept alive with the inputs)."""
        arr = (Request * len(reqs))()
        keep = []
        for i, q in enumerate(reqs):
            r = _host(q["r"]).reshape(-1, 3)
            v = _host(q["v"]).reshape(-1, 3)
            ro = np.empty_like(r)
            vo = np.empty_like(v)
            keep.append((r, v, ro, vo))
            arr[i].start = as_time(q["start"])
            arr[i].h = float(q["h"])
            arr[i].steps = int(q["steps"])
            arr[i].degree = int(q.get("degree", 0))
            arr[i].n = r.shape[0]
            arr[i].r_in = r.ctypes.data
            arr[i].v_in = v.ctypes.data
            arr[i].r_out = ro.ctypes.data
            arr[i].v_out = vo.ctypes.data
        return arr, keep

    def propagate_batch(self, reqs):
        """Returns [(r_end, v_end)] per request."""
        arr, keep = self._requests(reqs)
        self._check(load_library().gpop_propagate_batch(self._h, arr, len(reqs)))
        return [(k[2], k[3]) for k in keep]

    def propagate_batch_status(self, reqs):
        """Requests that cannot run are refused alone. Returns ([(r_end, v_end) or None per
        request], per-request status array, the call's status, its error message or None)."""
        arr, keep = self._requests(reqs)
        status = np.zeros(len(reqs), np.int32)
        st = load_library().gpop_propagate_batch_status(self._h, arr, len(reqs),
                                                        status.ctypes.data_as(_VP))
        msg = None if st == OK else load_library().gpop_last_error(self._h).decode()
        out = [(k[2], k[3]) if status[i] == OK else None for i, k in enumerate(keep)]
        return out, status, st, msg

    @property
    def batch_warps_per_sm(self):
        """Block shape (warps per SM) the planner chose for the last batch."""
        return load_library().gpop_batch_warps_per_sm(self._h)

    def batch_plan(self, reqs):
        arr, keep = self._requests(reqs)
        lpo = np.zeros(len(reqs), np.int32)
        est = C.c_double()
        self._check(load_library().gpop_batch_plan(self._h, arr, len(reqs),
                                                   lpo.ctypes.data_as(_VP), C.byref(est)))
        return lpo, est.value

    @property
    def batch_device_seconds(self):
        """Device time of the last propagate_batch launch (without host copies)."""
        return load_library().gpop_batch_device_seconds(self._h)

    def tune(self, cache_path=None):
        self._check(load_library().gpop_tune(
            self._h, None if cache_path is None else cache_path.encode()))

    # ---- variational equations and adjoint (FP64) ----
    def sample_states(self, r_nominal, v_nominal, sigma_r, sigma_v, seed, r_out, v_out, stream=None):
        """Monte Carlo ensemble on the device: r_out, v_out [n, 3] CUDA tensors."""
        rn = np.ascontiguousarray(r_nominal, dtype=np.float64).reshape(3)
        vn = np.ascontiguousarray(v_nominal, dtype=np.float64).reshape(3)
        self._check(load_library().gpop_sample_states(
            self._h, rn.ctypes.data, vn.ctypes.data, float(sigma_r), float(sigma_v), int(seed),
            int(r_out.shape[0]), _dptr(r_out), _dptr(v_out), _stream_ptr(stream)))

    def gravity_jacobian(self, r, jac, frame9=None, acc=None, stream=None):
        """FP64 acceleration Jacobian [n, 3, 3] (device tensors) at GCRS positions r [n, 3]."""
        self._check(load_library().gpop_gravity_jacobian(
            self._h, int(r.shape[0]), _dptr(r), None if frame9 is None else _dptr(frame9),
            None if acc is None else _dptr(acc), _dptr(jac), _stream_ptr(stream)))

    def stm(self, start, h, steps, r, v):
        """Returns (r_end, v_end, stm [n, 6, 6]) with stm[i, j] = d x_N,i / d x0_j, x = (r, v)."""
        r = _host(r).reshape(-1, 3)
        v = _host(v).reshape(-1, 3)
        ro, vo = np.empty_like(r), np.empty_like(v)
        phi = np.empty((r.shape[0], 6, 6))
        self._check(load_library().gpop_stm(
            self._h, C.byref(as_time(start)), float(h), int(steps), r.shape[0], r.ctypes.data,
            v.ctypes.data, ro.ctypes.data, vo.ctypes.data, phi.ctypes.data))
        return ro, vo, phi

    def propagate_vjp(self, start, h, steps, r, v, r_bar=None, v_bar=None):
        """Adjoint: d(sum r_bar . r_N + v_bar . v_N) / d(r0, v0) as two [n, 3] arrays."""
        r = _host(r).reshape(-1, 3)
        v = _host(v).reshape(-1, 3)
        rb = None if r_bar is None else _host(r_bar).reshape(-1, 3)
        vb = None if v_bar is None else _host(v_bar).reshape(-1, 3)
        gr, gv = np.empty_like(r), np.empty_like(v)
        self._check(load_library().gpop_propagate_vjp(
            self._h, C.byref(as_time(start)), float(h), int(steps), r.shape[0], r.ctypes.data,
            v.ctypes.data, None if rb is None else rb.ctypes.data,
            None if vb is None else vb.ctypes.data, gr.ctypes.data, gv.ctypes.data))
        return gr, gv

    def miss_gradient(self, start, h, steps, r, v, pairs):
        """Closest approach of listed pairs and the adjoint gradient of each miss distance:
        returns (tca [p], miss [p], grad [p, 12] = d miss / d(r0_a, v0_a, r0_b, v0_b))."""
        r = _host(r).reshape(-1, 3)
        v = _host(v).reshape(-1, 3)
        pr = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
        tca = np.empty(pr.shape[0])
        miss = np.empty(pr.shape[0])
        grad = np.empty((pr.shape[0], 12))
        self._check(load_library().gpop_miss_gradient(
            self._h, C.byref(as_time(start)), float(h), int(steps), r.shape[0], r.ctypes.data,
            v.ctypes.data, pr.shape[0], pr.ctypes.data, tca.ctypes.data, miss.ctypes.data,
            grad.ctypes.data))
        return tca, miss, grad

    # ---- force model ----
    def gravity(self, r, a, frame9=None, precision=None, stream=None):
        p = self.precision if precision is None else precision
        self._check(load_library().gpop_gravity(
            self._h, r.shape[0], _dptr(r), _dptr(frame9), _dptr(a), int(p), _stream_ptr(stream)))

    def frame_matrices(self, start, h, count, m_out, mjd_out=None, use_midpoints=False,
                       before_epoch=4, stream=None):
        self._check(load_library().gpop_frame_matrices(
            self._h, C.byref(as_time(start)), float(h), int(count), int(use_midpoints),
            int(before_epoch), _dptr(m_out), _dptr(mjd_out), _stream_ptr(stream)))

    # ---- closest approach ----
    def closest_approach(self, start, h, r, v, set_ids, kind="gravity"):
        return ClosestApproach(self, start, h, r, v, set_ids, kind)


class Propagator:
    """GpuPropagator of the reference (gpu_propagator.cuh:26-59): step(k) = Step() k times."""

    def __init__(self, ctx, start, h, max_steps, r, v):
        lib = load_library()
        self.ctx = ctx
        self._keep = (r, v)
        out = _VP()
        ctx._check(lib.gpop_propagator_create(ctx._h, C.byref(as_time(start)), float(h),
                                              int(max_steps), r.shape[0], _dptr(r), _dptr(v),
                                              C.byref(out)))
        self._h = out.value

    def step(self, steps=1, traj_r=None, traj_v=None, traj_a=None, stream=None):
        self.ctx._check(load_library().gpop_propagator_step(
            self._h, int(steps), _dptr(traj_r), _dptr(traj_v), _dptr(traj_a),
            _stream_ptr(stream)))

    @property
    def steps_done(self):
        return load_library().gpop_propagator_steps_done(self._h)

    def close(self):
        if getattr(self, "_h", None):
            load_library().gpop_propagator_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ClosestApproach:
    """ClosestApproach of the reference (lib/closest_approach/closest_approach.cuh:36-88)."""

    def __init__(self, ctx, start, h, r, v, set_ids, kind="gravity"):
        lib = load_library()
        self.ctx = ctx
        r = _host(r).reshape(-1, 3)
        v = _host(v).reshape(-1, 3)
        ids = np.ascontiguousarray(set_ids, dtype=np.uint32)
        if ids.shape[0] != r.shape[0]:
            raise GpopError(1, "set_ids size mismatch")
        out = _VP()
        k = -1 if kind == "external" else FORCE[kind] if isinstance(kind, str) else kind
        if k == -1:
            # trajectory supplied by append() (per-evaluation path, sharded screen)
            ctx._check(lib.gpop_ca_create_external(ctx._h, float(h), r.shape[0],
                                                   r.ctypes.data_as(_VP), v.ctypes.data_as(_VP),
                                                   ids.ctypes.data_as(_VP), C.byref(out)))
        elif k == 0:
            ctx._check(lib.gpop_ca_create(ctx._h, C.byref(as_time(start)), float(h), r.shape[0],
                                          r.ctypes.data_as(_VP), v.ctypes.data_as(_VP),
                                          ids.ctypes.data_as(_VP), C.byref(out)))
        else:
            ctx._check(lib.gpop_ca_create_analytic(ctx._h, k, float(h), r.shape[0],
                                                   r.ctypes.data_as(_VP), v.ctypes.data_as(_VP),
                                                   ids.ctypes.data_as(_VP), C.byref(out)))
        self._h = out.value
        self.n = r.shape[0]

    def close(self):
        if getattr(self, "_h", None):
            load_library().gpop_ca_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def num_pairs(self):
        return load_library().gpop_ca_num_pairs(self._h)

    def propagate(self, steps):
        self.ctx._check(load_library().gpop_ca_propagate(self._h, int(steps)))

    def append(self, steps, r, v, a):
        """Screens `steps` more steps of an external object: device tensors [steps][n][3]."""
        for t in (r, v, a):
            if tuple(t.shape) != (int(steps), self.n, 3) or not t.is_contiguous():
                raise GpopError(1, "append wants contiguous [steps][n][3] device arrays")
        self.ctx._check(load_library().gpop_ca_append(self._h, int(steps), _dptr(r), _dptr(v),
                                                      _dptr(a)))

    def reserve(self, total_steps):
        """Sizes the trajectory store for total_steps steps in all (no regrowth up to there)."""
        self.ctx._check(load_library().gpop_ca_reserve(self._h, int(total_steps)))

    def set_rows(self, begin, end):
        """Screen and refine only the pairs whose first object is in rows [begin, end)."""
        self.ctx._check(load_library().gpop_ca_set_rows(self._h, int(begin), int(end)))

    @property
    def pair_range(self):
        lo, hi = C.c_int64(), C.c_int64()
        self.ctx._check(load_library().gpop_ca_pair_range(self._h, C.byref(lo), C.byref(hi)))
        return lo.value, hi.value

    def find(self, threshold=-1.0):
        lib = load_library()
        cnt = C.c_int64()
        self.ctx._check(lib.gpop_ca_find(self._h, float(threshold), None, 0, C.byref(cnt)))
        recs = (CaRecord * max(cnt.value, 1))()
        self.ctx._check(lib.gpop_ca_find(self._h, float(threshold), recs, cnt.value, C.byref(cnt)))
        return [recs[i] for i in range(cnt.value)]

    def pairs(self):
        """Per-pair results in the reference's pair order (num_pairs entries); after set_rows only
        the entries of pair_range are filled, the others stay zero."""
        P = self.num_pairs
        d = np.zeros(P)
        t = np.zeros(P)
        pa = np.zeros((P, 3))
        pb = np.zeros((P, 3))
        cs = np.zeros(P, np.uint32)
        self.ctx._check(load_library().gpop_ca_pairs(
            self._h, d.ctypes.data_as(_VP), t.ctypes.data_as(_VP), pa.ctypes.data_as(_VP),
            pb.ctypes.data_as(_VP), cs.ctypes.data_as(_VP)))
        return dict(distance=d, time=t, posA=pa, posB=pb, closest_step=cs)

    def device_seconds(self):
        """Cumulative device seconds (propagation, screen, refinement)."""
        out = np.zeros(3)
        self.ctx._check(load_library().gpop_ca_device_seconds(self._h, out.ctypes.data_as(_VP)))
        return out

    def trajectory(self):
        lib = load_library()
        steps = C.c_int32()
        self.ctx._check(lib.gpop_ca_trajectory(self._h, None, None, None, C.byref(steps)))
        k = steps.value
        r = np.zeros((k, 3, self.n))
        v = np.zeros((k, 3, self.n))
        a = np.zeros((k, 3, self.n))
        self.ctx._check(lib.gpop_ca_trajectory(self._h, r.ctypes.data_as(_VP),
                                               v.ctypes.data_as(_VP), a.ctypes.data_as(_VP),
                                               C.byref(steps)))
        return r, v, a
