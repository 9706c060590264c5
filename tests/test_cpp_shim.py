"""The C++ mirror classes of include/gpop.hpp (ForceModel, GpuPropagator, ClosestApproach,
ClosestApproachData with the reference's signatures): they compile and link against libgpop.so
(CPU), and on the GPU give exactly what the C ABI gives for the same calls."""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = "/usr/local/cuda"


def _build(tmp_path):
    exe = str(tmp_path / "shim_check")
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I", CUDA + "/include",
           os.path.join(ROOT, "tests", "cpp", "shim_check.cpp"), "-o", exe,
           "-L", os.path.join(ROOT, "opengpop_b200", "lib"), "-lgpop", "-L", CUDA + "/lib64", "-lcudart",
           "-Wl,-rpath," + os.path.join(ROOT, "opengpop_b200", "lib") + ":" + CUDA + "/lib64"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_shim_compiles_and_links(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_shim_matches_c_abi(tmp_path):
    import opengpop_b200 as G
    exe = _build(tmp_path)
    out = subprocess.run([exe, G.DATA_DIR], check=True, capture_output=True, text=True).stdout
    res = {}
    for line in out.splitlines():
        res.update(json.loads(line))
    n, h, steps = 8, 30.0, 100
    r = np.zeros((n, 3))
    v = np.zeros((n, 3))
    for i in range(n):
        a, ph, inc = 7.0e6 + 1.0e4 * i, 0.3 * i, 0.2 + 0.1 * i
        sp = np.sqrt(3.986004415e14 / a)
        r[i] = [a * np.cos(ph), a * np.sin(ph) * np.cos(inc), a * np.sin(ph) * np.sin(inc)]
        v[i] = [-sp * np.sin(ph), sp * np.cos(ph) * np.cos(inc), sp * np.cos(ph) * np.sin(inc)]
    start = (2024, 1, 1, 0, 0, 0.0)
    ctx = G.Context(precision=G.FP64)
    # GpuPropagator: 100 Step() calls == one propagate call of 100 steps (same kernels)
    r_end, v_end = ctx.propagate(start, h, steps, r, v)
    assert np.array_equal(np.array(res["r_end"]).reshape(n, 3), r_end)
    assert np.array_equal(np.array(res["v_end"]).reshape(n, 3), v_end)
    # ForceModel hook: column 2 of the [N][27] matrix = gravity at propagation epoch 5
    from gpu_util import dev, host, zeros
    m = zeros(15 * 9)
    ctx.frame_matrices(start, h, 15, m, before_epoch=4)
    acc = zeros(n, 3)
    ctx.gravity(dev(r), acc, m[5 * 9:6 * 9].contiguous(), precision=G.FP64)
    mat = np.array(res["acc_matrix"]).reshape(n, 9, 3)
    assert np.array_equal(mat[:, 2, :], host(acc)) and not mat[:, [0, 1, 3], :].any()
    # ClosestApproach: Get(a, b) for every pair of objects vs the C ABI's records
    ca = ctx.closest_approach(start, h, r, v, np.array([0, 0, 0, 1, 1, 2, 2, 2], np.uint32))
    ca.propagate(60)
    ca.propagate(40)
    recs = {(x.object_index1, x.object_index2): x for x in ca.find()}
    ca.close()
    sets = [0, 0, 0, 1, 1, 2, 2, 2]
    for a, b, d, t, pa0, pb2 in np.array(res["approaches"]).reshape(-1, 6):
        a, b = int(a), int(b)
        if a == b:
            assert d == 0.0 and t == 0.0
        elif sets[a] == sets[b]:
            assert d == -1.0 and t == -1.0
        else:
            x = recs[(min(a, b), max(a, b))]
            assert (d, t, pa0, pb2) == (x.distance, x.time, x.position_a[0], x.position_b[2])
    ctx.close()
