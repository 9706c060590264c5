"""Runs the reference's own CUDA build (oracle/_ref/libref.so) in a child process.

TEST INFRASTRUCTURE ONLY. The reference reads its data files at ../../data/ relative to the working
directory and calls exit() on errors, so each run happens in a fresh process, in a scratch
directory two levels below a data/ directory that holds the same model files as
opengpop_b200/data (with the gfc header's max_degree rewritten for a lower degree).

    python ref_build_runner.py in.npz out.npz
"""
import ctypes as C
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libref.so")
DATA = os.path.join(ROOT, "opengpop_b200", "data")


def available():
    return os.path.exists(LIB)


def frames(start, h, count, midpoints=False, before=4):
    """The reference's own per-epoch ITRS->GCRS matrices [count, 9] (column-major) and UTC MJDs."""
    out = run("frames", start, h, 0, np.zeros((1, 3)), np.zeros((1, 3)), count=count,
              midpoints=int(midpoints), before=before)
    return out["m"], out["mjd"]


def _stage_data(tmp, degree):
    d = os.path.join(tmp, "data")
    os.makedirs(d)
    for f in os.listdir(DATA):
        if f.endswith(".md"):
            continue
        if f == "JGM3.gfc" and degree and degree < 70:
            with open(os.path.join(DATA, f)) as src, open(os.path.join(d, f), "w") as dst:
                for line in src:
                    if line.split()[:1] == ["max_degree"]:
                        line = "max_degree %d\n" % degree
                    dst.write(line)
        else:
            os.symlink(os.path.join(DATA, f), os.path.join(d, f))
    run = os.path.join(tmp, "run", "here")
    os.makedirs(run)
    return run


def child(inp, outp):
    z = dict(np.load(inp, allow_pickle=False))
    tmp = tempfile.mkdtemp(prefix="gpop_ref_")
    try:
        os.chdir(_stage_data(tmp, int(z["degree"])))
        lib = C.CDLL(LIB)
        st = [int(x) for x in z["start"][:5]] + [float(z["start"][5])]
        r = np.ascontiguousarray(z["r"], np.float64)
        v = np.ascontiguousarray(z["v"], np.float64)
        n = r.shape[0]
        ms = C.c_double()
        vp = C.c_void_p
        if str(z["mode"]) == "frames":
            cnt = int(z["count"])
            m = np.zeros((cnt, 9))
            mjd = np.zeros(cnt)
            lib.ref_frame_matrices.argtypes = [C.c_int] * 5 + [C.c_double, C.c_double] + [C.c_int] * 3 + [vp, vp]
            rc = lib.ref_frame_matrices(*st, float(z["h"]), cnt, int(z["midpoints"]),
                                        int(z["before"]), m.ctypes.data_as(vp), mjd.ctypes.data_as(vp))
            np.savez(outp, rc=rc, m=m, mjd=mjd, ms=0.0)
        elif str(z["mode"]) == "propagate":
            ro = np.zeros_like(r)
            vo = np.zeros_like(v)
            lib.ref_propagate.argtypes = [C.c_int] * 5 + [C.c_double, C.c_double, C.c_int, C.c_int,
                                                          vp, vp, vp, vp, C.POINTER(C.c_double)]
            rc = lib.ref_propagate(*st, float(z["h"]), int(z["steps"]), n, r.ctypes.data_as(vp),
                                   v.ctypes.data_as(vp), ro.ctypes.data_as(vp),
                                   vo.ctypes.data_as(vp),
                                   C.byref(ms))
            np.savez(outp, rc=rc, r=ro, v=vo, ms=ms.value)
        else:
            ids = np.ascontiguousarray(z["set_ids"], np.uint32)
            P = int(sum(1 for i in range(n) for j in range(i + 1, n) if ids[i] != ids[j]))
            o1 = np.zeros(P, np.int32)
            o2 = np.zeros(P, np.int32)
            dist = np.zeros(P)
            tim = np.zeros(P)
            pa = np.zeros((P, 3))
            pb = np.zeros((P, 3))
            cnt = C.c_longlong()
            lib.ref_closest_approach.argtypes = [C.c_int] * 5 + [C.c_double, C.c_double, C.c_int,
                                                                 C.c_int] + [vp] * 9 + [
                C.POINTER(C.c_longlong), C.POINTER(C.c_double)]
            rc = lib.ref_closest_approach(*st, float(z["h"]), int(z["steps"]), n,
                                          r.ctypes.data_as(vp), v.ctypes.data_as(vp),
                                          ids.ctypes.data_as(vp), o1.ctypes.data_as(vp),
                                          o2.ctypes.data_as(vp), dist.ctypes.data_as(vp),
                                          tim.ctypes.data_as(vp), pa.ctypes.data_as(vp),
                                          pb.ctypes.data_as(vp), C.byref(cnt), C.byref(ms))
            np.savez(outp, rc=rc, obj1=o1, obj2=o2, distance=dist, time=tim, posA=pa, posB=pb,
                     ms=ms.value)
    finally:
        os.chdir("/")
        shutil.rmtree(tmp, ignore_errors=True)


def run(mode, start, h, steps, r, v, set_ids=None, degree=70, timeout=1800, **extra):
    """Runs the reference build in a child process; returns the result arrays."""
    tmp = tempfile.mkdtemp(prefix="gpop_refio_")
    try:
        inp = os.path.join(tmp, "in.npz")
        outp = os.path.join(tmp, "out.npz")
        kw = dict(mode=mode, start=np.array(start, float), h=h, steps=steps,
                  r=np.asarray(r, float), v=np.asarray(v, float), degree=degree)
        if set_ids is not None:
            kw["set_ids"] = np.asarray(set_ids, np.uint32)
        kw.update(extra)
        np.savez(inp, **kw)
        p = subprocess.run([sys.executable, os.path.abspath(__file__), inp, outp],
                           capture_output=True, text=True, timeout=timeout)
        if p.returncode != 0 or not os.path.exists(outp):
            raise RuntimeError("reference build failed (rc=%d): %s" % (p.returncode,
                                                                        p.stderr[-2000:]))
        out = dict(np.load(outp))
        if int(out["rc"]) != 0:
            raise RuntimeError("reference build returned %d" % int(out["rc"]))
        return out
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    child(sys.argv[1], sys.argv[2])
