"""The allocation-free CFL step, checked against the regular entry point.

gcs_local_timestep_noalloc serves callers that cannot call cudaMalloc when
they need a time step (device arrays owned by another allocator, or a
driver that forbids device allocation after start-up): they pass their own
device arrays in the reference layout and the reduction keeps its scratch
in a fixed static device array.  This file is collected last so that a run
stopping at the first failure has already run every other test; it also
passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from gamera_cube_b200 import abi
from oracle import oracle_cases

pytestmark = pytest.mark.gpu

RTOL = 1e-12


@pytest.fixture(scope="module")
def lib():
    import gamera_cube_b200
    lib = gamera_cube_b200.lib
    P = C.POINTER
    fn = lib.gcs_local_timestep_noalloc
    fn.restype = C.c_int
    fn.argtypes = [P(C.c_size_t), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                   P(C.c_size_t), P(C.c_size_t), P(abi.TimestepOptions),
                   P(C.c_double)]
    lib.gcs_noalloc_last_error.restype = C.c_char_p
    lib.gcs_noalloc_scratch_bytes.restype = C.c_size_t
    return lib


def _device_bytes(ptr, nbytes):
    """Copy host memory into a caller-owned device buffer (the test plays
    the caller that owns its device arrays)."""
    import torch
    host = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_uint8)), shape=(nbytes,))
    return torch.from_numpy(host.copy()).to("cuda")


def _face_inputs(case, f):
    g = case.grid[f]
    ext = tuple(g.cell_extent)
    ncell = ext[0] * ext[1] * ext[2]
    s = case.storage[f]
    bg = case.background[f]
    return {
        "extent": (C.c_size_t * 3)(*ext),
        "cells": _device_bytes(g.cell, ncell * C.sizeof(abi.CellGeometry)),
        "u": _device_bytes(s.conserved, ncell * 5 * 8),
        "b": _device_bytes(s.cell_magnetic, ncell * 24),
        "b0": _device_bytes(bg.cell_magnetic, ncell * 24),
    }


def _noalloc_min(lib, case, inputs):
    g, act = case.ghost, case.active
    lower = (C.c_size_t * 3)(g, g, g)
    upper = (C.c_size_t * 3)(g + act[0], g + act[1], g + act[2])
    best = float("inf")
    for f in range(6):
        x = inputs[f]
        dt = C.c_double()
        rc = lib.gcs_local_timestep_noalloc(
            x["extent"], x["cells"].data_ptr(), x["u"].data_ptr(),
            x["b"].data_ptr(), x["b0"].data_ptr(), lower, upper,
            case.timestep_options, C.byref(dt))
        assert rc == 0, lib.gcs_noalloc_last_error()
        best = min(best, dt.value)
    return best


def test_noalloc_timestep_matches_context_entry_point(lib):
    import torch
    torch.cuda.init()
    case = oracle_cases.Case("wind", 12, 10, 7)
    ctx = lib.gcs_context_create(case.grid, case.active, case.ghost)
    assert ctx, lib.gcs_last_error()
    try:
        assert lib.gcs_context_upload_background(ctx, case.background) == 0
        assert lib.gcs_context_upload_state(ctx, case.storage) == 0
        inputs = [_face_inputs(case, f) for f in range(6)]
        torch.cuda.synchronize()
        free = []
        for call in range(2):       # two calls in a row share the scratch
            want = C.c_double()
            assert lib.gcs_context_timestep(ctx, case.timestep_options,
                                            C.byref(want)) == 0
            got = _noalloc_min(lib, case, inputs)
            free.append(torch.cuda.mem_get_info()[0])
            assert abs(got - want.value) <= RTOL * want.value, (call, got,
                                                               want.value)
            assert abs(got - case.local_timestep()) <= RTOL * got
        # once the library is loaded, a call changes the device footprint
        # by nothing
        got = _noalloc_min(lib, case, inputs)
        assert torch.cuda.mem_get_info()[0] == free[-1], (free, got)
        assert 0 < lib.gcs_noalloc_scratch_bytes() < 1 << 20
    finally:
        lib.gcs_context_destroy(ctx)


def test_noalloc_rejects_oversized_box(lib):
    """Boxes above the stated maximum are refused before any device work."""
    ext = (C.c_size_t * 3)(300, 300, 300)
    lower = (C.c_size_t * 3)(0, 0, 0)
    upper = (C.c_size_t * 3)(300, 300, 300)
    opts = abi.TimestepOptions(5.0 / 3.0, 1e-6, 1e-8, 0.3, 10.0, True, True,
                               False)
    dt = C.c_double(-1.0)
    dummy = C.c_void_p(16)
    rc = lib.gcs_local_timestep_noalloc(ext, dummy, dummy, dummy, None, lower,
                                        upper, C.byref(opts), C.byref(dt))
    assert rc == -1 and dt.value == -1.0
    assert b"exceed the maximum" in lib.gcs_noalloc_last_error()
