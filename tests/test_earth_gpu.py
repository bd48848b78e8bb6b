"""GPU parity of the device Earth radial boundary (no-MI wall).

The same reference-built wind case (grid, state, dipole background) is
advanced twice from identical inputs:
  * by the compiled reference's own step with its own callbacks
    gamera_cs_earth_fill_radial_ghosts / gamera_cs_earth_inner_fluid_flux /
    gamera_cs_earth_no_mi_emf (oracle/_ref), on the CPU;
  * by gcs_context_step_earth, the step with those callbacks as kernels.
The monitor series has three samples with linear interpolation, a tilted
planar front (By/Bz coefficients) and a time offset, so the ballistic
mapping, interpolation and upstream-to-tail weights all enter.  Tolerance:
1e-12 normwise per array per step (device libm may differ from the host's
in the last bit of sqrt/acos/exp), growing by 10x per chained step as the
plain step parity test allows.
"""
import ctypes as C

import numpy as np
import pytest

from gamera_cube_b200 import abi
from oracle import refbind
from tests.parity_util import compare_state

pytestmark = pytest.mark.gpu

NAMES = ["conserved", "old_conserved", "cell_magnetic", "old_cell_magnetic"] + \
        ["face_flux%d" % d for d in range(3)] + ["old_face_flux%d" % d for d in range(3)]


@pytest.fixture(scope="module")
def lib():
    import gamera_cube_b200
    return gamera_cube_b200.lib


def wind_series(keep):
    times = np.array([0.0, 0.004, 0.012])
    states = (abi.SolarWindState * 3)()
    for q, (rho, vx, by, bz) in enumerate([(5.0, -4.0, 0.05, -0.08),
                                           (7.5, -4.6, -0.02, 0.10),
                                           (4.0, -3.5, 0.03, -0.12)]):
        states[q].density = rho
        states[q].pressure = 0.6 * rho / 5.0
        states[q].velocity[:] = [vx, 0.2, -0.1]
        states[q].magnetic[:] = [0.02, by, bz]
    t = (C.c_double * 3)(*times)
    keep += [t, states]
    w = abi.SolarWindSeries()
    w.count = 3
    w.time = t
    w.state = states
    w.reference[:] = [28.0, 0.0, 0.0]
    w.time_offset = 0.001
    w.by_coefficient = 0.2
    w.bz_coefficient = -0.1
    w.linear_interpolation = 1
    return w


def boundary(startup, wind, background, strict):
    b = abi.EarthBoundary()
    b.startup = C.pointer(startup)
    b.wind = C.pointer(wind)
    b.background = background
    b.mi = None
    b.density_floor = 1e-6
    b.pressure_floor = 1e-8
    b.cfl = 0.3
    b.strict_inner_gas_wall = strict
    return b


@pytest.mark.parametrize("strict", [0, 1])
def test_earth_boundary_matches_reference(lib, strict):
    if not refbind.ref_available():
        pytest.skip("reference library not built")
    R = refbind.ref()
    ref = refbind.Case(refbind.FX_WIND, 12, 10, 7)
    gpu = refbind.Case(refbind.FX_WIND, 12, 10, 7)
    keep = []
    startup = abi.EarthStartup()
    startup.gamma = 5.0 / 3.0
    wind = wind_series(keep)
    b_ref = boundary(startup, wind, ref.background, strict)
    b_gpu = boundary(startup, wind, gpu.background, strict)

    ropts = abi.AdvanceOptions.from_buffer_copy(ref.options.contents)
    ropts.fluid_flux_sync = C.cast(R.gamera_cs_earth_inner_fluid_flux, C.c_void_p).value
    ropts.edge_emf_sync = C.cast(R.gamera_cs_earth_no_mi_emf, C.c_void_p).value
    ropts.edge_emf_context = C.cast(C.pointer(b_ref), C.c_void_p).value
    radial = C.cast(R.gamera_cs_earth_fill_radial_ghosts, C.c_void_p).value
    gopts = abi.AdvanceOptions.from_buffer_copy(gpu.options.contents)

    ctx = lib.gcs_context_create(gpu.grid, gpu.active, gpu.ghost)
    assert ctx, lib.gcs_last_error()
    earth = C.c_void_p()
    try:
        assert lib.gcs_context_upload_background(ctx, gpu.background) == 0
        assert lib.gcs_context_upload_state(ctx, gpu.storage) == 0
        assert lib.gcs_earth_create(ctx, gpu.grid, C.byref(b_gpu), C.byref(earth)) == 0, \
            lib.gcs_last_error()
        assert lib.gcs_earth_device_bytes(earth) > 0
        time, dt_prev = 0.0, 0.0
        for s in range(3):
            local = ref.local_timestep()
            dt = 0.5 * local if dt_prev == 0.0 else min(0.5 * local, 1.25 * dt_prev)
            ratio = 0.0 if dt_prev == 0.0 else 0.5 * dt / dt_prev
            prev = time if s == 0 else time - dt_prev
            b_ref.step_time, b_ref.step_dt = time, dt
            assert R.gamera_cs_advance_six_with_background_planned(
                ref.grid, ref.storage, ref.active, ref.ghost, ratio, dt, C.byref(ropts),
                ref.background, R.fx_plan(ref.handle), radial, time, prev,
                C.cast(C.pointer(b_ref), C.c_void_p)) == 0
            assert lib.gcs_context_step_earth(ctx, earth, C.byref(gopts), ratio, dt, time,
                                              prev) == 0, lib.gcs_context_error(ctx)
            assert lib.gcs_context_download_state(ctx, gpu.storage, 0) == 0
            res = compare_state(gpu, ref, NAMES)
            bad = {k: v for k, v in res.items() if not v[0] <= 1e-12 * 10 ** s}
            assert not bad, "step %d: %s" % (s, bad)
            time += dt
            dt_prev = dt
        # the boundary acted: inner ghosts mirror, outer ghosts follow the wind
        u = ref.arrays(0)["conserved"]
        assert not np.allclose(u[0], u[4]) or not np.allclose(u[-1], u[-5])
    finally:
        if earth:
            lib.gcs_earth_destroy(earth)
        lib.gcs_context_destroy(ctx)
        ref.close()
        gpu.close()


def test_earth_boundary_rejects_bad_input(lib):
    if not refbind.ref_available():
        pytest.skip("reference library not built")
    case = refbind.Case(refbind.FX_WIND, 12, 10, 7)
    ctx = lib.gcs_context_create(case.grid, case.active, case.ghost)
    assert ctx
    try:
        keep = []
        startup = abi.EarthStartup()
        startup.gamma = 5.0 / 3.0
        wind = wind_series(keep)
        b = boundary(startup, wind, case.background, 0)
        b.density_floor = 0.0
        earth = C.c_void_p()
        assert lib.gcs_earth_create(ctx, case.grid, C.byref(b), C.byref(earth)) == -1
        b.density_floor = 1e-6
        wind.count = 0
        assert lib.gcs_earth_create(ctx, case.grid, C.byref(b), C.byref(earth)) == -1
        assert not earth
    finally:
        lib.gcs_context_destroy(ctx)
        case.close()


def earth_options(cbs, case, b):
    o = abi.AdvanceOptions.from_buffer_copy(case.options.contents)
    o.fluid_flux_sync = C.cast(cbs.gamera_cs_earth_inner_fluid_flux, C.c_void_p).value
    o.edge_emf_sync = C.cast(cbs.gamera_cs_earth_no_mi_emf, C.c_void_p).value
    o.edge_emf_context = C.cast(C.pointer(b), C.c_void_p).value
    return o


@pytest.mark.parametrize("strict", [0, 1])
def test_drop_in_step_with_earth_callbacks(lib, strict):
    """A reference caller's unchanged Earth-driver step (the reference's
    callback symbols, resolved in this library) against the reference."""
    if not refbind.ref_available():
        pytest.skip("reference library not built")
    R = refbind.ref()
    abi.bind(R, abi.earth_callback_signatures())
    ref = refbind.Case(refbind.FX_WIND, 12, 10, 7)
    gpu = refbind.Case(refbind.FX_WIND, 12, 10, 7)
    keep = []
    startup = abi.EarthStartup()
    startup.gamma = 5.0 / 3.0
    wind = wind_series(keep)
    b_ref = boundary(startup, wind, ref.background, strict)
    b_gpu = boundary(startup, wind, gpu.background, strict)
    ropts, gopts = earth_options(R, ref, b_ref), earth_options(lib, gpu, b_gpu)
    plan = C.c_void_p()
    assert lib.gamera_cs_halo_plan_create(gpu.grid, gpu.active, gpu.ghost, C.byref(plan)) == 0
    try:
        time, dt_prev = 0.0, 0.0
        for s in range(3):
            local = ref.local_timestep()
            dt = 0.5 * local if dt_prev == 0.0 else min(0.5 * local, 1.25 * dt_prev)
            ratio = 0.0 if dt_prev == 0.0 else 0.5 * dt / dt_prev
            prev = time if s == 0 else time - dt_prev
            for bd in (b_ref, b_gpu):
                bd.step_time, bd.step_dt = time, dt
            assert R.gamera_cs_advance_six_with_background_planned(
                ref.grid, ref.storage, ref.active, ref.ghost, ratio, dt, C.byref(ropts),
                ref.background, R.fx_plan(ref.handle),
                C.cast(R.gamera_cs_earth_fill_radial_ghosts, C.c_void_p),
                time, prev, C.cast(C.pointer(b_ref), C.c_void_p)) == 0
            assert lib.gamera_cs_advance_six_with_background_planned(
                gpu.grid, gpu.storage, gpu.active, gpu.ghost, ratio, dt, C.byref(gopts),
                gpu.background, plan, C.cast(lib.gamera_cs_earth_fill_radial_ghosts,
                                             C.c_void_p),
                time, prev, C.cast(C.pointer(b_gpu), C.c_void_p)) == 0
            res = compare_state(gpu, ref, NAMES)
            bad = {k: v for k, v in res.items() if not v[0] <= 1e-12 * 10 ** s}
            assert not bad, "step %d: %s" % (s, bad)
            time += dt
            dt_prev = dt
    finally:
        lib.gamera_cs_halo_plan_destroy(plan)
        ref.close()
        gpu.close()


def test_direct_radial_fill_matches_reference(lib):
    """gamera_cs_earth_fill_radial_ghosts called on host storage (all faces,
    then one receiver face) against the reference's."""
    if not refbind.ref_available():
        pytest.skip("reference library not built")
    R = refbind.ref()
    abi.bind(R, abi.earth_callback_signatures())
    ref = refbind.Case(refbind.FX_WIND, 12, 10, 7)
    gpu = refbind.Case(refbind.FX_WIND, 12, 10, 7)
    one = refbind.Case(refbind.FX_WIND, 12, 10, 7)
    keep = []
    startup = abi.EarthStartup()
    startup.gamma = 5.0 / 3.0
    wind = wind_series(keep)
    try:
        for case, fn in ((ref, R), (gpu, lib)):
            bd = boundary(startup, wind, case.background, 0)
            keep.append(bd)
            assert fn.gamera_cs_earth_fill_radial_ghosts(case.grid, case.storage, case.active,
                                                         case.ghost, 0.006, 0.002,
                                                         C.byref(bd)) == 0
        res = compare_state(gpu, ref, NAMES)
        bad = {k: v for k, v in res.items() if not v[0] <= 1e-12}
        assert not bad, bad
        bd = boundary(startup, wind, one.background, 0)
        before = [one.arrays(f)["conserved"].copy() for f in range(6)]
        assert lib.gamera_cs_earth_fill_radial_ghosts_face(one.grid, one.storage, one.active,
                                                           one.ghost, 0.006, 0.002,
                                                           C.byref(bd), 2) == 0
        for f in range(6):
            now = one.arrays(f)["conserved"]
            if f == 2:
                np.testing.assert_allclose(now, ref.arrays(2)["conserved"], rtol=0,
                                           atol=1e-12 * np.max(np.abs(now)))
            else:
                np.testing.assert_array_equal(now, before[f])
    finally:
        ref.close()
        gpu.close()
        one.close()


def test_device_built_case_boundary_matches_host_grid(lib):
    """gcs_earth_create_case (boundary layers rebuilt on the device) against
    gcs_earth_create on the oracle's host grid of the same case: one Earth
    step agrees to the builders' level (1e-11).  As in the builder test,
    conserved ghost values are compared on active cells: the cube-corner
    diagonal ghosts take their donor by a projection tie that last-bit
    differences of the device-built centroids flip, and later steps carry
    that difference inward, in the plain step as well."""
    from oracle import oracle_cases
    host = oracle_cases.Case("wind", 12, 10, 7)
    keep = []
    startup = abi.EarthStartup()
    startup.gamma = 5.0 / 3.0
    wind = wind_series(keep)
    b_host = boundary(startup, wind, host.background, 0)
    b_dev = boundary(startup, wind, None, 0)
    opts = abi.AdvanceOptions.from_buffer_copy(host.options.contents)
    a = lib.gcs_context_create(host.grid, host.active, host.ghost)
    d = lib.gcs_context_create_case(2, 12, 10, 7)
    ea, ed = C.c_void_p(), C.c_void_p()
    try:
        assert a and d
        assert lib.gcs_context_upload_background(a, host.background) == 0
        assert lib.gcs_context_upload_state(a, host.storage) == 0
        assert lib.gcs_earth_create(a, host.grid, C.byref(b_host), C.byref(ea)) == 0
        assert lib.gcs_earth_create_case(d, C.byref(b_dev), C.byref(ed)) == 0, \
            lib.gcs_last_error()
        time, dt_prev = 0.0, 0.0
        for s in range(1):
            dt = 0.5 * host.local_timestep() if s == 0 else dt_prev
            ratio = 0.0 if s == 0 else 0.5
            prev = time if s == 0 else time - dt_prev
            for ctx, e in ((a, ea), (d, ed)):
                assert lib.gcs_context_step_earth(ctx, e, C.byref(opts), ratio, dt, time,
                                                  prev) == 0
            time += dt
            dt_prev = dt
        from tests.test_ensemble_gpu import download
        ha, hd = download(lib, a), download(lib, d)
        for name in ("conserved", "cell_magnetic", "face_flux0", "face_flux1", "face_flux2"):
            worst = scale = 0.0
            for f in range(6):
                x, y = ha.arrays(f)[name], hd.arrays(f)[name]
                g = host.ghost
                if name == "conserved":   # corner-diagonal ghosts: donor ties
                    x = x[g:-g, g:-g, g:-g]
                    y = y[g:-g, g:-g, g:-g]
                worst = max(worst, float(np.max(np.abs(x - y))))
                scale = max(scale, float(np.max(np.abs(x))))
            assert worst <= 1e-11 * scale, (name, worst / scale)
    finally:
        for e in (ea, ed):
            if e:
                lib.gcs_earth_destroy(e)
        for ctx in (a, d):
            if ctx:
                lib.gcs_context_destroy(ctx)


@pytest.mark.parametrize("strict", [0, 1])
def test_drop_in_step_with_mi_coupled_wall(lib, strict):
    """The Earth step with a ready MI coupling (potential views of both
    libraries holding the reference's solved potential of the coupling
    test): E x B drift ghost velocities and the inner-shell EMF from the
    potential, on the device, against the reference's host callbacks.
    Tolerance 1e-10: the drift is a central difference of the mapped
    potential over 1e-4 R_E, which turns the last-bit differences of the
    device's acos/asin/atan2 in the lookup into ~1e-12 relative in E."""
    if not refbind.ref_available():
        pytest.skip("reference library not built")
    import mi_util
    R = refbind.ref()
    abi.bind(R, abi.earth_callback_signatures())
    abi.bind(R, {"gamera_cs_mi_dipole_create_potential_view":
                 (C.c_int, [C.POINTER(abi.EarthStartup), C.POINTER(abi.MiDipoleConfig),
                            C.POINTER(C.c_void_p)])})
    cfg, startup = mi_util.coupling_config(), mi_util.coupling_startup()
    pot = np.ascontiguousarray(mi_util.golden()["coupling/potential"])
    P = C.POINTER(C.c_double)
    views = []
    for L in (R, lib):
        mi = C.c_void_p()
        assert L.gamera_cs_mi_dipole_create_potential_view(C.byref(startup), C.byref(cfg),
                                                           C.byref(mi)) == 0
        assert L.gamera_cs_mi_dipole_import_potential(mi, pot.ctypes.data_as(P), pot.size,
                                                      0.0, 10.0) == 0
        views.append(mi)
    ref = refbind.Case(refbind.FX_WIND, 12, 10, 7)
    gpu = refbind.Case(refbind.FX_WIND, 12, 10, 7)
    keep = []
    wind = wind_series(keep)
    b_ref = boundary(startup, wind, ref.background, strict)
    b_gpu = boundary(startup, wind, gpu.background, strict)
    b_ref.mi, b_gpu.mi = views[0].value, views[1].value
    ropts, gopts = earth_options(R, ref, b_ref), earth_options(lib, gpu, b_gpu)
    plan = C.c_void_p()
    assert lib.gamera_cs_halo_plan_create(gpu.grid, gpu.active, gpu.ghost, C.byref(plan)) == 0
    try:
        time, dt_prev = 0.0, 0.0
        for s in range(3):
            local = ref.local_timestep()
            dt = 0.5 * local if dt_prev == 0.0 else min(0.5 * local, 1.25 * dt_prev)
            ratio = 0.0 if dt_prev == 0.0 else 0.5 * dt / dt_prev
            prev = time if s == 0 else time - dt_prev
            for bd in (b_ref, b_gpu):
                bd.step_time, bd.step_dt = time, dt
            assert R.gamera_cs_advance_six_with_background_planned(
                ref.grid, ref.storage, ref.active, ref.ghost, ratio, dt, C.byref(ropts),
                ref.background, R.fx_plan(ref.handle),
                C.cast(R.gamera_cs_earth_fill_radial_ghosts, C.c_void_p),
                time, prev, C.cast(C.pointer(b_ref), C.c_void_p)) == 0
            assert lib.gamera_cs_advance_six_with_background_planned(
                gpu.grid, gpu.storage, gpu.active, gpu.ghost, ratio, dt, C.byref(gopts),
                gpu.background, plan, C.cast(lib.gamera_cs_earth_fill_radial_ghosts,
                                             C.c_void_p),
                time, prev, C.cast(C.pointer(b_gpu), C.c_void_p)) == 0
            res = compare_state(gpu, ref, NAMES)
            bad = {k: v for k, v in res.items() if not v[0] <= 1e-10 * 10 ** s}
            assert not bad, "step %d: %s" % (s, bad)
            time += dt
            dt_prev = dt
        # the MI wall acted: one reference step without the coupling differs
        plain = refbind.Case(refbind.FX_WIND, 12, 10, 7)
        b_plain = boundary(startup, wind, plain.background, strict)
        po = earth_options(R, plain, b_plain)
        once = refbind.Case(refbind.FX_WIND, 12, 10, 7)
        b_once = boundary(startup, wind, once.background, strict)
        b_once.mi = views[0].value
        oo = earth_options(R, once, b_once)
        dt = 0.5 * plain.local_timestep()
        for case, bd, o in ((plain, b_plain, po), (once, b_once, oo)):
            bd.step_time, bd.step_dt = 0.0, dt
            assert R.gamera_cs_advance_six_with_background_planned(
                case.grid, case.storage, case.active, case.ghost, 0.0, dt, C.byref(o),
                case.background, R.fx_plan(case.handle),
                C.cast(R.gamera_cs_earth_fill_radial_ghosts, C.c_void_p), 0.0, 0.0,
                C.cast(C.pointer(bd), C.c_void_p)) == 0
        assert any(not np.array_equal(plain.arrays(f)["edge_emf1"], once.arrays(f)["edge_emf1"])
                   for f in range(6))
        plain.close()
        once.close()
    finally:
        lib.gamera_cs_halo_plan_destroy(plan)
        R.gamera_cs_mi_dipole_destroy(views[0])
        lib.gamera_cs_mi_dipole_destroy(views[1])
        ref.close()
        gpu.close()


def test_earth_driver_loop_matches_stepwise(lib):
    """gcs_context_run_earth (device times, one CUDA graph per step) equals
    the same steps driven from the host with the reference driver's dt rule
    and times, bit for bit."""
    keep = []
    startup = abi.EarthStartup()
    startup.gamma = 5.0 / 3.0
    wind = wind_series(keep)
    o, t = abi.AdvanceOptions(), abi.TimestepOptions()
    assert lib.gcs_case_options(2, C.byref(o), C.byref(t)) == 0
    a = lib.gcs_context_create_case(2, 20, 10, 5)
    b = lib.gcs_context_create_case(2, 20, 10, 5)
    ea, eb = C.c_void_p(), C.c_void_p()
    try:
        for ctx, e in ((a, ea), (b, eb)):
            bd = boundary(startup, wind, None, 0)
            keep.append(bd)
            assert lib.gcs_earth_create_case(ctx, C.byref(bd), C.byref(e)) == 0
        assert lib.gcs_context_run_earth(a, ea, C.byref(o), C.byref(t), 0.5, 2, 1) == 0
        assert lib.gcs_context_run_earth(a, ea, C.byref(o), C.byref(t), 0.5, 2, 1) == 0
        assert lib.gcs_context_sync(a) == 0
        time, dt_prev = 0.0, 0.0
        for s in range(4):
            local = C.c_double()
            assert lib.gcs_context_timestep(b, C.byref(t), C.byref(local)) == 0
            dt = 0.5 * local.value if s == 0 else min(0.5 * local.value, 1.25 * dt_prev)
            ratio = 0.0 if s == 0 else 0.5 * dt / dt_prev
            prev = time if s == 0 else time - dt_prev
            assert lib.gcs_context_step_earth(b, eb, C.byref(o), ratio, dt, time, prev) == 0
            time += dt
            dt_prev = dt
        from tests.test_ensemble_gpu import download, assert_same_state
        ha, hb = download(lib, a), download(lib, b)
        assert_same_state(ha, hb)
    finally:
        for e in (ea, eb):
            if e:
                lib.gcs_earth_destroy(e)
        lib.gcs_context_destroy(a)
        lib.gcs_context_destroy(b)
