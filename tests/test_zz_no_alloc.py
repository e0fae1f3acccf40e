"""qmt_grid_total_noalloc: the grid total for callers that must not allocate device memory.

Some callers cannot let a library call cudaMalloc: a framework that owns all device memory
through its own pool, or a serving loop that cannot accept the device-wide synchronisation that
cudaMalloc and cudaFree can cause.  This entry point keeps its partial sums in a fixed array
compiled into the library (limit 33,554,432 points) and must agree with qmt_grid_total.

The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from qmtools import _native as N

MAX_POINTS = 4096 * 8192


def _total(lib, name, x, n):
    out = C.c_double()
    st = getattr(lib, name)(C.c_void_p(x.data_ptr()), n, C.byref(out), None)
    assert st == N.OK, lib.qmt_last_error().decode()
    return out.value


@pytest.mark.gpu
def test_noalloc_total_matches_grid_total_on_two_calls():
    import torch
    N.ensure_device(None)
    lib = N.load()
    g = torch.Generator(device="cuda").manual_seed(17)
    x = torch.rand(5_000_003, generator=g, device="cuda", dtype=torch.float32) * 2.0 - 0.5
    # a large call, then a smaller one that reads fewer slots than the first one wrote
    for n in (5_000_003, 70_001):
        ref = _total(lib, "qmt_grid_total", x, n)
        got = _total(lib, "qmt_grid_total_noalloc", x, n)
        assert abs(got - ref) <= 1e-9 * abs(ref)
        exact = float(x[:n].double().sum().item())
        assert abs(got - exact) <= 1e-9 * abs(exact)


def test_noalloc_total_rejects_sizes_beyond_its_scratch():
    lib = N.load()
    out = C.c_double()
    # rejected before any device work, so no buffer of that size is needed
    st = lib.qmt_grid_total_noalloc(C.c_void_p(256), MAX_POINTS + 1, C.byref(out), None)
    assert st == N.BAD_ARG
    assert b"fixed scratch limit" in lib.qmt_last_error()
