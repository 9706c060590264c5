"""The per-evaluation path of the C++ mirror (include/gpop.hpp): GpuPropagator, GpuStartup and
Predictor with an IForceModel that is not the library's ForceModel, as the reference runs them with
its mock force models (gpu_startup.cu, prediction.cu, gpu_propagator.cu). The program compiles and
links on the CPU; on the GPU the path gives the fused path's result when the library's gravity sits
behind the hooks, integrates a harmonic oscillator to its closed form, and calls the hooks in the
reference's numbers; ClosestApproach over such a model screens and refines as the fused path does."""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = "/usr/local/cuda"


def _build(tmp_path):
    exe = str(tmp_path / "generic_check")
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I", CUDA + "/include",
           os.path.join(ROOT, "tests", "cpp", "generic_check.cpp"), "-o", exe,
           "-L", os.path.join(ROOT, "opengpop_b200", "lib"), "-lgpop", "-L", CUDA + "/lib64", "-lcudart",
           "-Wl,-rpath," + os.path.join(ROOT, "opengpop_b200", "lib") + ":" + CUDA + "/lib64"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_generic_path_compiles_and_links(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_generic_path(tmp_path):
    import opengpop_b200 as G
    exe = _build(tmp_path)
    out = subprocess.run([exe, G.DATA_DIR], check=True, capture_output=True, text=True).stdout
    res = {}
    for line in out.splitlines():
        res.update(json.loads(line))
    # the library's gravity behind the hooks: the fused path's state and last acceleration
    for key in ("r", "v", "a"):
        fused = np.array(res["fused_" + key])
        generic = np.array(res["generic_" + key])
        assert np.abs(generic - fused).max() <= 1e-9 * np.abs(fused).max(), key
    # harmonic oscillator a = -r (w = 1) over t = 10: r = r0 cos t + v0 sin t
    t = res["osc_t"]
    r0, v0 = np.array(res["osc_r0"]), np.array(res["osc_v0"])
    assert np.abs(np.array(res["osc_r"]) - (r0 * np.cos(t) + v0 * np.sin(t))).max() < 1e-9
    assert np.abs(np.array(res["osc_v"]) - (-r0 * np.sin(t) + v0 * np.cos(t))).max() < 1e-9
    # hook calls: PreInitialize and InitializeGeneration/-Propagation once, 8 x 10 RK8 stages,
    # 9 + 7 x 8 startup-corrector evaluations, then 1 + 7 per step from step 5 (200 steps)
    pre, init_gen, gen, init_prop, prop = res["osc_calls"]
    assert (pre, init_gen, init_prop) == (1, 1, 1)
    assert gen == 80
    assert prop == 9 + 7 * 8 + (200 - 4) * 8
    # the reference mock's polynomial force, from rest: r = -t^3 + t^7, v = -3 t^2 + 7 t^6 at t = 6
    t = res["poly_t"]
    r_ex, v_ex = -t ** 3 + t ** 7, -3 * t ** 2 + 7 * t ** 6
    assert np.abs(np.array(res["poly_r"]) - r_ex).max() <= 1e-9 * r_ex
    assert np.abs(np.array(res["poly_v"]) - v_ex).max() <= 1e-9 * v_ex
    # ClosestApproach: the per-evaluation phases screen and refine as the fused ones do
    fused = np.array(res["ca_fused"]).reshape(-1, 4)
    generic = np.array(res["ca_generic"]).reshape(-1, 4)
    assert np.array_equal(fused[:, :2], generic[:, :2])
    screened = fused[:, 2] > 0
    assert screened.sum() == 42  # cross-set pairs of sets of 3, 2 and 3 objects, both orders
    assert np.array_equal(fused[~screened, 2:], generic[~screened, 2:])  # -1 or 0 entries
    assert np.abs(generic[screened, 2] - fused[screened, 2]).max() <= 1e-6 * fused[screened, 2].max()
    assert np.abs(generic[screened, 3] - fused[screened, 3]).max() < 1e-3
