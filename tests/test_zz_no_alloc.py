"""The no-alloc propagation entry point (gpop_propagate_device_noalloc), through the C ABI.

It serves callers that may not allocate device memory while running: services that reserve their
whole device-memory budget at start-up, and hosts whose device memory another allocator's pool
already holds, where a cudaMalloc in mid-run would fail. Its scratch is a fixed array inside the
library instead of on-demand cudaMalloc. It runs the same walk, tables and kernels as
gpop_propagate_device, so its results must equal that entry point's bit for bit, call after call
(the shared array keeps the previous call's contents, which must not leak into the next result).
This file is collected last so that a run that stops at the first failure has run every other test
first; it also passes on its own.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = "/usr/local/cuda"
START = (2024, 1, 1, 0, 0, 0.0)


def _call(lib, ctx, start, h, steps, r, v, stream):
    import opengpop_b200 as G
    return lib.gpop_propagate_device_noalloc(ctx._h, C.byref(G.as_time(start)), h, steps,
                                             r.shape[0], C.c_void_p(r.data_ptr()),
                                             C.c_void_p(v.data_ptr()), stream)


def _both(lib, ctx, stream, h, steps, r0, v0):
    """(allocating result, no-alloc result) on device copies of the same inputs."""
    import torch
    ra = torch.tensor(r0, dtype=torch.float64, device="cuda")
    va = torch.tensor(v0, dtype=torch.float64, device="cuda")
    ctx.propagate_device(START, h, steps, ra, va)
    rb = torch.tensor(r0, dtype=torch.float64, device="cuda")
    vb = torch.tensor(v0, dtype=torch.float64, device="cuda")
    st = _call(lib, ctx, START, h, steps, rb, vb, stream)
    assert st == 0, lib.gpop_last_error(ctx._h)
    torch.cuda.synchronize()
    return (ra, va), (rb, vb)


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_noalloc_equals_allocating_entry_point_twice(precision):
    """Two calls in a row, of different sizes and step signs: bit-identical to
    gpop_propagate_device (same walk, tables and kernels)."""
    import torch
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    lib = G.load_library()
    ctx = G.Context(precision=precision)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call, (n, h, steps, seed) in enumerate([(300, 30.0, 150, 1), (97, -60.0, 40, 2)]):
        r0, v0 = orbits.mixed_population(n, seed)
        (ra, va), (rb, vb) = _both(lib, ctx, stream, h, steps, r0, v0)
        assert torch.equal(ra, rb) and torch.equal(va, vb), (call, (ra - rb).abs().max().item())
    ctx.close()


def test_noalloc_fixed_backward_epoch_flag():
    """The device-side epoch arithmetic also follows the fixed backward RK8 epochs."""
    import torch
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    lib = G.load_library()
    ctx = G.Context(flags=G.FIX_BACKWARD_RK8_EPOCH)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    r0, v0 = orbits.leo(40, 5)
    (ra, va), (rb, vb) = _both(lib, ctx, stream, 30.0, 25, r0, v0)
    assert torch.equal(ra, rb) and torch.equal(va, vb)
    ctx.close()


def test_noalloc_against_oracle():
    """FP64 no-alloc result against the CPU FP64 oracle: 24 objects, 2 h."""
    import torch
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    import oracle_api as O
    lib = G.load_library()
    ctx = G.Context()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    r0, v0 = orbits.mixed_population(24, 11)
    r = torch.tensor(r0, dtype=torch.float64, device="cuda")
    v = torch.tensor(v0, dtype=torch.float64, device="cuda")
    st = _call(lib, ctx, START, 30.0, 240, r, v, stream)
    assert st == 0, lib.gpop_last_error(ctx._h)
    ro, vo = O.propagate(O.Data(), "gravity", START, 30.0, 240, r0, v0)
    assert np.abs(r.cpu().numpy() - ro).max() <= 1e-4
    assert np.abs(v.cpu().numpy() - vo).max() <= 1e-7
    ctx.close()


def test_noalloc_rejects_sizes_beyond_its_limit():
    import torch
    import opengpop_b200 as G
    lib = G.load_library()
    ctx = G.Context()
    r = torch.zeros(4097, 3, dtype=torch.float64, device="cuda")
    v = torch.zeros(4097, 3, dtype=torch.float64, device="cuda")
    st = _call(lib, ctx, START, 30.0, 10, r, v, None)
    assert st == 1
    assert b"4096 objects" in lib.gpop_last_error(ctx._h)
    r = torch.zeros(8, 3, dtype=torch.float64, device="cuda")
    v = torch.zeros(8, 3, dtype=torch.float64, device="cuda")
    st = _call(lib, ctx, START, 30.0, 20161, r, v, None)
    assert st == 1
    ctx.close()


def test_noalloc_after_device_reset(tmp_path):
    """A context made after cudaDeviceReset finds the new CUDA context's scratch array and gives
    the bits it gave before the reset. Runs as a child process that does not use torch, so the
    reset invalidates no memory another allocator still holds."""
    import opengpop_b200 as G
    exe = str(tmp_path / "noalloc_reset_check")
    lib_dir = os.path.join(ROOT, "opengpop_b200", "lib")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I",
                    CUDA + "/include", os.path.join(ROOT, "tests", "cpp", "noalloc_reset_check.cpp"),
                    "-o", exe, "-L", lib_dir, "-lgpop", "-L", CUDA + "/lib64", "-lcudart",
                    "-Wl,-rpath," + lib_dir + ":" + CUDA + "/lib64"],
                   check=True, capture_output=True, text=True)
    out = subprocess.run([exe, G.DATA_DIR], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.strip().endswith("ok"), out.stdout + out.stderr
