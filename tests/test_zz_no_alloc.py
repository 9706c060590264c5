"""The no-alloc propagation entry point (gpop_propagate_device_noalloc), through the C ABI.

It serves callers that may not allocate device memory while running: its scratch is a fixed array
inside the library instead of on-demand cudaMalloc. Its results must equal those of
gpop_propagate_device on the same inputs, call after call (the shared array keeps the previous
call's contents, which must not leak into the next result). This file is collected last so that a
run that stops at the first failure has run every other test first; it also passes on its own.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call(lib, ctx, start, h, steps, r, v, stream):
    import opengpop_b200 as G
    return lib.gpop_propagate_device_noalloc(ctx._h, C.byref(G.as_time(start)), h, steps,
                                             r.shape[0], C.c_void_p(r.data_ptr()),
                                             C.c_void_p(v.data_ptr()), stream)


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    import opengpop_b200 as G
    from opengpop_b200 import orbits
    lib = G.load_library()
    ctx = G.Context()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    start = (2024, 1, 1, 0, 0, 0.0)
    for call, (n, steps, seed) in enumerate([(300, 150, 1), (97, 40, 2)]):
        r0, v0 = orbits.mixed_population(n, seed)
        # reference result from the allocating entry point
        ra = torch.tensor(r0, dtype=torch.float64, device="cuda")
        va = torch.tensor(v0, dtype=torch.float64, device="cuda")
        ctx.propagate_device(start, 30.0, steps, ra, va)
        # the no-alloc entry point on fresh copies of the same inputs
        rb = torch.tensor(r0, dtype=torch.float64, device="cuda")
        vb = torch.tensor(v0, dtype=torch.float64, device="cuda")
        st = _call(lib, ctx, start, 30.0, steps, rb, vb, stream)
        assert st == 0, lib.gpop_last_error(ctx._h)
        torch.cuda.synchronize()
        dr = (ra - rb).abs().max().item()
        dv = (va - vb).abs().max().item()
        # same kernels and epoch tables: agreement to well below the 1e-4 m parity bound
        assert dr <= 1e-6 and dv <= 1e-9, (call, dr, dv)
    ctx.close()


def test_noalloc_rejects_sizes_beyond_its_limit():
    import torch
    import opengpop_b200 as G
    lib = G.load_library()
    ctx = G.Context()
    r = torch.zeros(4097, 3, dtype=torch.float64, device="cuda")
    v = torch.zeros(4097, 3, dtype=torch.float64, device="cuda")
    st = _call(lib, ctx, (2024, 1, 1, 0, 0, 0.0), 30.0, 10, r, v, None)
    assert st == 1
    assert b"4096 objects" in lib.gpop_last_error(ctx._h)
    r = torch.zeros(8, 3, dtype=torch.float64, device="cuda")
    v = torch.zeros(8, 3, dtype=torch.float64, device="cuda")
    st = _call(lib, ctx, (2024, 1, 1, 0, 0, 0.0), 30.0, 20161, r, v, None)
    assert st == 1
    ctx.close()
