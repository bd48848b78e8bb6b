"""GPU parity of the six-face step against the unmodified reference.

Each case is built twice through the reference setup API; one copy is
advanced by the reference CPU step (oracle/_ref), the other by this
library's drop-in entry point gamera_cs_advance_six_with_background_planned
through the C-ABI.  Tolerance: 1e-12 normwise relative per step in FP64
(the plain-path target), div B at round-off.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import refbind
from tests.parity_util import STATE_ARRAYS, compare_state, divergence

pytestmark = pytest.mark.gpu

RTOL_STEP = 1e-12


@pytest.fixture(scope="module")
def lib():
    import gamera_cube_b200
    return gamera_cube_b200.lib


def _gpu_plan(lib, case):
    plan = C.c_void_p()
    assert lib.gamera_cs_halo_plan_create(case.grid, case.active, case.ghost,
                                          C.byref(plan)) == 0, \
        lib.gcs_last_error()
    return plan


def _gpu_step(lib, case, plan, ratio, dt):
    return lib.gamera_cs_advance_six_with_background_planned(
        case.grid, case.storage, case.active, case.ghost, ratio, dt,
        case.options, case.background, plan, None, 0.0, 0.0, None)


def _pair(kind, nr=0, n=0, seed=7):
    a = refbind.Case(kind, nr, n, seed)
    b = refbind.Case(kind, nr, n, seed)
    return a, b


def _assert_close(res, rtol, what):
    bad = {k: v for k, v in res.items() if not v[0] <= rtol}
    assert not bad, "%s: arrays beyond rtol %g: %s" % (what, rtol, bad)


@pytest.mark.parametrize("kind,nr,n,steps,rtol", [
    (refbind.FX_UNIFORM, 0, 0, 1, RTOL_STEP),
    (refbind.FX_SHOCK, 0, 0, 1, RTOL_STEP),
    (refbind.FX_SHOCK, 0, 0, 10, 1e-10),
])
def test_fixed_dt_cases(lib, kind, nr, n, steps, rtol):
    ref, gpu = _pair(kind, nr, n)
    plan = _gpu_plan(lib, gpu)
    try:
        for s in range(steps):
            assert ref.step(ref.ratio, ref.dt) == 0
            assert _gpu_step(lib, gpu, plan, gpu.ratio, gpu.dt) == 0
        res = compare_state(gpu, ref)
        _assert_close(res, rtol, "kind %d after %d steps" % (kind, steps))
        for f in range(6):
            assert divergence(gpu, f) <= 1e-9
    finally:
        lib.gamera_cs_halo_plan_destroy(plan)


def test_wind_driver_steps(lib):
    """Solar wind + dipole background + Boris + HOGS, driver dt sequence."""
    ref, gpu = _pair(refbind.FX_WIND, 12, 10)
    plan = _gpu_plan(lib, gpu)
    try:
        dt_prev = 0.0
        for s in range(3):
            local = ref.local_timestep()
            dt = 0.5 * local if dt_prev == 0.0 else min(0.5 * local,
                                                        1.25 * dt_prev)
            ratio = 0.0 if dt_prev == 0.0 else 0.5 * dt / dt_prev
            assert ref.step(ratio, dt) == 0
            assert _gpu_step(lib, gpu, plan, ratio, dt) == 0
            res = compare_state(gpu, ref)
            _assert_close(res, RTOL_STEP * 10 ** s, "wind step %d" % s)
            dt_prev = dt
    finally:
        lib.gamera_cs_halo_plan_destroy(plan)


def test_step_uniform_preserved(lib):
    """Known answer of test_cubedsphere_six_mhd.c:63-96 on the GPU path:
    a uniform state stays uniform (|dU| <= 5e-6) with div B <= 1e-10."""
    _, gpu = _pair(refbind.FX_UNIFORM)
    plan = _gpu_plan(lib, gpu)
    try:
        expected = gpu.arrays(0)["conserved"][6, 6, 6].copy()
        for _ in range(3):
            assert _gpu_step(lib, gpu, plan, 0.5, 0.01) == 0
        g, act = gpu.ghost, gpu.active
        for f in range(6):
            u = gpu.arrays(f)["conserved"][g:g + act[0], g:g + act[1],
                                           g:g + act[2]]
            assert np.max(np.abs(u - expected)) <= 5e-6
            assert divergence(gpu, f) <= 1e-10
    finally:
        lib.gamera_cs_halo_plan_destroy(plan)
