"""GPU checks of the post-step pressure control (nonorthogonal_step.c:74-171).

Chain of parity: the device call on an uploaded state equals the oracle
(whole conserved arrays bit for bit, counts and maxima exactly, a failing
cell included; the oracle is pinned to the reference by
tests/test_pressure_host.py); in the device driver loop, one step with the
control equals one step followed by the direct call, the next step size is
the CFL step of the controlled state, and the CUDA-graph loop equals the
launch-by-launch loop."""
import ctypes as C

import numpy as np
import pytest

from gamera_cube_b200 import abi
from gamera_cube_b200.host import HostStorage
from oracle import oracle_cases
from tests import pressure_util as pu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import gamera_cube_b200
    return gamera_cube_b200.lib


def download(lib, ctx):
    act = (C.c_size_t * 3)()
    g = C.c_size_t()
    assert lib.gcs_context_dims(ctx, act, C.byref(g)) == 0
    hs = HostStorage(list(act), g.value)
    assert lib.gcs_context_download_state(ctx, hs.storage, 0) == 0
    return hs


def config(light, thr, low_sound):
    return abi.PressureControl(pu.GAMMA, pu.RHO_FLOOR, pu.P_FLOOR, light, thr, low_sound)


def device_call(lib, ctx, grid, dt, cfg):
    nl, nh = C.c_size_t(), C.c_size_t()
    s, p = C.c_double(), C.c_double()
    rc = lib.gcs_context_pressure_control(ctx, grid, dt, C.byref(cfg), C.byref(nl),
                                          C.byref(nh), C.byref(s), C.byref(p))
    return rc, nl.value, nh.value, s.value, p.value


@pytest.mark.parametrize("poison", [False, True])
def test_device_call_matches_oracle(lib, poison):
    case = oracle_cases.Case("wind", 12, 10, 7)
    assert case.step(0.0, 0.5 * case.local_timestep()) == 0
    act, g = list(case.active), case.ghost
    light, thr, low_sound = pu.parameters([case.arrays(f) for f in range(6)], g, act)
    if poison:
        case.arrays(2)["conserved"][g + 3, g + 4, g + 5, 0] = -1.0
    ctx = lib.gcs_context_create(case.grid, case.active, case.ghost)
    assert ctx, lib.gcs_last_error()
    try:
        assert lib.gcs_context_upload_background(ctx, case.background) == 0
        assert lib.gcs_context_upload_state(ctx, case.storage) == 0
        got = device_call(lib, ctx, case.grid, pu.DT, config(light, thr, low_sound))
        want = pu.apply_faces(case.lib.gcso_apply_pressure_control, case.storage, case.grid,
                              g, act, pu.DT, light, thr, low_sound)
        assert got == want
        assert want[0] == (-1 if poison else 0) and want[1] > 0 and want[2] > 0
        hs = download(lib, ctx)
        for f in range(6):
            np.testing.assert_array_equal(hs.arrays(f)["conserved"],
                                          case.arrays(f)["conserved"], err_msg="face %d" % f)
        # invalid arguments change nothing
        bad = config(light, thr, low_sound)
        bad.light_speed = 0.0
        assert device_call(lib, ctx, case.grid, pu.DT, bad)[0] == -1
        assert device_call(lib, ctx, case.grid, 0.0, config(light, thr, low_sound))[0] == -1
        hs2 = download(lib, ctx)
        for f in range(6):
            np.testing.assert_array_equal(hs2.arrays(f)["conserved"], hs.arrays(f)["conserved"])
    finally:
        lib.gcs_context_destroy(ctx)


def test_device_built_case_needs_no_grid(lib):
    ctx = lib.gcs_context_create_case(2, 12, 10, 7)
    assert ctx, lib.gcs_last_error()
    try:
        hs = download(lib, ctx)
        light, thr, low_sound = pu.parameters([hs.arrays(f) for f in range(6)], 4, [12, 10, 10])
        rc, low, hot, ms, mp = device_call(lib, ctx, None, pu.DT, config(light, thr, low_sound))
        assert rc == 0 and low > 0 and hot > 0 and ms > 1.5 * light and mp > 0.0
        for f in range(6):
            assert np.isfinite(download(lib, ctx).arrays(f)["conserved"]).all()
    finally:
        lib.gcs_context_destroy(ctx)


def params(lib, ctx):
    dt, ratio, cfl = C.c_double(), C.c_double(), C.c_double()
    steps = C.c_int()
    assert lib.gcs_context_params(ctx, C.byref(dt), C.byref(ratio), C.byref(cfl),
                                  C.byref(steps)) == 0
    return dt.value, ratio.value, steps.value


def test_driver_loop_control(lib):
    o, t = abi.AdvanceOptions(), abi.TimestepOptions()
    assert lib.gcs_case_options(2, C.byref(o), C.byref(t)) == 0
    ctxs = [lib.gcs_context_create_case(2, 20, 10, 5) for _ in range(4)]
    assert all(ctxs), lib.gcs_last_error()
    a, b, c, d = ctxs
    try:
        hs = download(lib, a)
        cfg = config(*pu.parameters([hs.arrays(f) for f in range(6)], 4, [20, 10, 10]))
        local0 = C.c_double()
        assert lib.gcs_context_timestep(c, C.byref(t), C.byref(local0)) == 0
        dt0 = 0.5 * local0.value
        # one step with the control == one step, then the direct call
        assert lib.gcs_context_set_pressure_control(d, None, C.byref(cfg)) == 0
        assert lib.gcs_context_run(d, C.byref(o), C.byref(t), 0.5, 1, 1) == 0
        assert lib.gcs_context_sync(d) == 0
        assert lib.gcs_context_run(c, C.byref(o), C.byref(t), 0.5, 1, 1) == 0
        assert lib.gcs_context_sync(c) == 0
        rc, low, hot, _, _ = device_call(lib, c, None, dt0, cfg)
        assert rc == 0 and low > 0 and hot > 0
        hc, hd = download(lib, c), download(lib, d)
        for f in range(6):
            np.testing.assert_array_equal(hd.arrays(f)["conserved"], hc.arrays(f)["conserved"])
        nl, nh = C.c_size_t(), C.c_size_t()
        assert lib.gcs_context_pressure_control_stats(d, C.byref(nl), C.byref(nh), None,
                                                      None, 1) == 0
        assert (nl.value, nh.value) == (low, hot)
        # the next step size is the CFL step of the controlled state
        local1 = C.c_double()
        assert lib.gcs_context_timestep(c, C.byref(t), C.byref(local1)) == 0
        assert params(lib, d)[0] == min(0.5 * local1.value, 1.25 * dt0)
        # the graph loop equals the launch-by-launch loop
        for ctx, graph in ((a, 1), (b, 0)):
            assert lib.gcs_context_set_pressure_control(ctx, None, C.byref(cfg)) == 0
            assert lib.gcs_context_run(ctx, C.byref(o), C.byref(t), 0.5, 3, graph) == 0
            assert lib.gcs_context_sync(ctx) == 0
        ha, hb = download(lib, a), download(lib, b)
        for f in range(6):
            for name in ("conserved", "cell_magnetic", "face_flux0"):
                np.testing.assert_array_equal(ha.arrays(f)[name], hb.arrays(f)[name])
        assert params(lib, a) == params(lib, b) and params(lib, a)[2] == 3
        sa = [C.c_size_t(), C.c_size_t(), C.c_double(), C.c_double()]
        sb = [C.c_size_t(), C.c_size_t(), C.c_double(), C.c_double()]
        assert lib.gcs_context_pressure_control_stats(a, *[C.byref(x) for x in sa], 0) == 0
        assert lib.gcs_context_pressure_control_stats(b, *[C.byref(x) for x in sb], 0) == 0
        assert [x.value for x in sa] == [x.value for x in sb] and sa[0].value > 0
        # turning it off
        assert lib.gcs_context_set_pressure_control(a, None, None) == 0
        assert lib.gcs_context_run(a, C.byref(o), C.byref(t), 0.5, 1, 1) == 0
        assert lib.gcs_context_sync(a) == 0
    finally:
        for ctx in ctxs:
            lib.gcs_context_destroy(ctx)
