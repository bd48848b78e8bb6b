"""GPU parity of the six-face step (plain FP64 path).

Each case is built twice with identical inputs; one copy is advanced by the
oracle on the CPU, the other by this library's drop-in entry point
gamera_cs_advance_six_with_background_planned through the C-ABI.  The oracle
is the CPU restatement (bit-exact with the reference, tests/test_oracle.py)
and, where it was built, the compiled reference itself.  The golden test
compares the device result with values recorded from the reference.

Tolerance: 1e-12 normwise relative per step in FP64 (the plain-path
target); div B at round-off.
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import oracle_cases, refbind
from tests.parity_util import compare_state, divergence

pytestmark = pytest.mark.gpu

RTOL_STEP = 1e-12
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_steps.npz")


@pytest.fixture(scope="module")
def lib():
    import gamera_cube_b200
    return gamera_cube_b200.lib


def _oracle_pair(backend, kind, nr=0, n=0, seed=7):
    if backend == "reference":
        if not refbind.ref_available():
            pytest.skip("reference library not built")
        k = oracle_cases.KINDS[kind]
        return refbind.Case(k, nr, n, seed), refbind.Case(k, nr, n, seed)
    return oracle_cases.pair(kind, nr, n, seed)


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


def _assert_close(res, rtol, what):
    bad = {k: v for k, v in res.items() if not v[0] <= rtol}
    assert not bad, "%s: arrays beyond rtol %g: %s" % (what, rtol, bad)


def _driver_dt(oracle, dt_prev):
    local = oracle.local_timestep()
    dt = 0.5 * local if dt_prev == 0.0 else min(0.5 * local, 1.25 * dt_prev)
    ratio = 0.0 if dt_prev == 0.0 else 0.5 * dt / dt_prev
    return ratio, dt


@pytest.mark.parametrize("backend", ["restatement", "reference"])
@pytest.mark.parametrize("kind,steps,rtol", [
    ("uniform", 1, RTOL_STEP),
    ("shock", 1, RTOL_STEP),
    ("shock", 10, 1e-10),
])
def test_fixed_dt_cases(lib, backend, kind, steps, rtol):
    ref, gpu = _oracle_pair(backend, kind)
    plan = _gpu_plan(lib, gpu)
    try:
        for _ in range(steps):
            assert ref.step(ref.ratio, ref.dt) == 0
            assert _gpu_step(lib, gpu, plan, gpu.ratio, gpu.dt) == 0
        _assert_close(compare_state(gpu, ref), rtol,
                      "%s after %d steps" % (kind, steps))
        for f in range(6):
            assert divergence(gpu, f) <= 1e-9
    finally:
        lib.gamera_cs_halo_plan_destroy(plan)


@pytest.mark.parametrize("backend", ["restatement", "reference"])
def test_wind_driver_steps(lib, backend):
    """Solar wind + dipole background + Boris + HOGS, driver dt sequence:
    each step compared after identical inputs (1e-12), three steps chained."""
    ref, gpu = _oracle_pair(backend, "wind", 12, 10)
    plan = _gpu_plan(lib, gpu)
    try:
        dt_prev = 0.0
        for s in range(3):
            ratio, dt = _driver_dt(ref, dt_prev)
            assert ref.step(ratio, dt) == 0
            assert _gpu_step(lib, gpu, plan, ratio, dt) == 0
            _assert_close(compare_state(gpu, ref), RTOL_STEP * 10 ** s,
                          "wind step %d" % s)
            dt_prev = dt
    finally:
        lib.gamera_cs_halo_plan_destroy(plan)


@pytest.mark.parametrize("name,kind,nr,n,steps", [
    ("uniform", "uniform", 0, 0, 2),
    ("shock", "shock", 0, 0, 3),
    ("wind", "wind", 12, 10, 2),
])
def test_against_reference_golden(lib, name, kind, nr, n, steps):
    """Device steps against the sampled values recorded from the reference
    (tests/golden/make_golden.py), same per-step time steps."""
    from tests.golden.make_golden import ARRAYS, sample_indices
    golden = np.load(GOLDEN)
    _, gpu = oracle_cases.pair(kind, nr, n, 7)
    plan = _gpu_plan(lib, gpu)
    try:
        for s, (ratio, dt) in enumerate(golden["%s/dts" % name][:steps]):
            assert _gpu_step(lib, gpu, plan, ratio, dt) == 0
            prefix = "%s/step%d" % (name, s + 1)
            for name_a in ARRAYS:
                scale = max(float(np.max(np.abs(
                    golden["%s/f%d/%s/sample" % (prefix, f, name_a)])))
                    for f in range(6)) or 1.0
                for f in range(6):
                    flat = np.ascontiguousarray(
                        gpu.arrays(f)[name_a]).reshape(-1)
                    got = flat[sample_indices(flat.size)]
                    want = golden["%s/f%d/%s/sample" % (prefix, f, name_a)]
                    err = np.max(np.abs(got - want)) / scale
                    assert err <= RTOL_STEP * 10 ** s, (prefix, f, name_a, err)
    finally:
        lib.gamera_cs_halo_plan_destroy(plan)


def test_step_uniform_preserved(lib):
    """Known answer of test_cubedsphere_six_mhd.c:63-96 on the GPU path:
    a uniform state stays uniform (|dU| <= 5e-6) with div B <= 1e-10."""
    _, gpu = oracle_cases.pair("uniform")
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


def test_shock_thirty_steps_known_answer(lib):
    """Known answer of test_cubedsphere_mhd_shock.c:171-219 on the GPU path."""
    _, gpu = oracle_cases.pair("shock")
    plan = _gpu_plan(lib, gpu)
    try:
        for _ in range(30):
            assert _gpu_step(lib, gpu, plan, 0.5, 0.001) == 0
        g, act = gpu.ghost, gpu.active
        rho_max = 0.0
        for f in range(6):
            u = gpu.arrays(f)["conserved"][g:g + act[0], g:g + act[1],
                                           g:g + act[2]]
            rho = u[..., 0]
            p = (2.0 / 3.0) * (u[..., 4] - 0.5 * np.sum(u[..., 1:4] ** 2, -1) / rho)
            assert rho.min() > 0 and p.min() > 0
            rho_max = max(rho_max, rho.max())
            assert divergence(gpu, f) <= 1e-9
        assert rho_max >= 0.9
    finally:
        lib.gamera_cs_halo_plan_destroy(plan)
