"""The ionosphere coupling updated inside the device driver loop's step
graph against the same coupling driven from the host.

Host-driven: before every step the host calls gamera_cs_mi_dipole_maybe_update
with the simulation time of the state (the reference Earth driver's loop,
test_cubedsphere_dipole_background.c:631), then runs one graph step.
In-graph: gcs_context_set_mi_coupling attaches the coupling and one
gcs_context_run call advances all the steps; the cadence
(cubedsphere_mi_dipole.c:372-378, 430-435), the FAC kernels and the two
solves run inside each step's graph with no host round trip.

The two must agree bit for bit: the state, the potentials, the FAC
statistics and the cadence (epoch, next update).  Cases: the reference's
time rule and an every-n-steps cadence on a plain wind run, and the Earth
boundary with the coupling as its MI wall (the potential feeds back into
the state).
"""
import ctypes as C

import numpy as np
import pytest

from gamera_cube_b200 import abi, cases

pytestmark = pytest.mark.gpu

STEPS = 12


@pytest.fixture(scope="module")
def lib():
    import gamera_cube_b200
    return gamera_cube_b200.lib


def _config():
    cfg = cases.mi_dipole_config(azimuth=64, colatitude=12, shell=1)
    # an update every three or four steps at this case's time step
    cfg.coupling_interval_s = 0.2
    return cfg


def _coupling(lib, ctx, startup, cfg):
    mi = C.c_void_p()
    assert lib.gcs_context_mi_dipole_create(ctx, C.byref(startup), C.byref(cfg),
                                            C.byref(mi)) == 0, lib.gcs_last_error()
    return mi


def _potential(lib, mi, cfg):
    n = 2 * cfg.azimuth_points * cfg.colatitude_points
    pot = np.zeros(n)
    epoch, nxt = C.c_double(), C.c_double()
    assert lib.gamera_cs_mi_dipole_export_potential(
        mi, pot.ctypes.data_as(C.POINTER(C.c_double)), n, C.byref(epoch),
        C.byref(nxt)) == 0
    fmin, fmax, pmin, pmax = (C.c_double() for _ in range(4))
    st = (abi.MiSolverStats * 2)()
    assert lib.gamera_cs_mi_dipole_stats(mi, C.byref(fmin), C.byref(fmax), C.byref(pmin),
                                         C.byref(pmax), st) == 0
    return pot, epoch.value, nxt.value, (fmin.value, fmax.value, st[0].iterations,
                                         st[1].iterations)


def _time(lib, ctx):
    t = C.c_double()
    assert lib.gcs_context_time(ctx, C.byref(t)) == 0
    return t.value


@pytest.mark.parametrize("every", [0, 3])
def test_in_graph_cadence_matches_host_driven(lib, every):
    from tests.test_ensemble_gpu import download, assert_same_state
    startup, cfg = cases.earth_startup(), _config()
    o, t = abi.AdvanceOptions(), abi.TimestepOptions()
    assert lib.gcs_case_options(2, C.byref(o), C.byref(t)) == 0
    a = lib.gcs_context_create_case(2, 20, 16, 5)
    b = lib.gcs_context_create_case(2, 20, 16, 5)
    ma, mb = _coupling(lib, a, startup, cfg), _coupling(lib, b, startup, cfg)
    try:
        updates = 0
        for s in range(STEPS):
            if every == 0:
                rc = lib.gamera_cs_mi_dipole_maybe_update(ma, _time(lib, a))
            elif s % every == 0:
                # the host-driven form of an every-n-steps cadence: the k-th
                # update at the time of the k-th coupling interval, where the
                # reference's rule makes it due
                rc = lib.gamera_cs_mi_dipole_maybe_update(
                    ma, updates * cfg.coupling_interval_s * cfg.speed_norm_m_s /
                    cfg.length_norm_m)
            else:
                rc = 0
            assert rc in (0, 1), lib.gcs_last_error()
            updates += rc
            assert lib.gcs_context_run(a, C.byref(o), C.byref(t), 0.5, 1, 1) == 0
        assert lib.gcs_context_sync(a) == 0
        assert updates >= 3
        assert lib.gcs_context_set_mi_coupling(b, mb, every) == 0
        assert lib.gcs_context_run(b, C.byref(o), C.byref(t), 0.5, STEPS, 1) == 0
        assert lib.gcs_context_sync(b) == 0, lib.gcs_context_error(b)
        assert_same_state(download(lib, a), download(lib, b))
        pa, ea, na, sa = _potential(lib, ma, cfg)
        pb, eb, nb, sb = _potential(lib, mb, cfg)
        assert np.array_equal(pa, pb)
        assert sa == sb
        if every == 0:
            assert (ea, na) == (eb, nb)
        assert lib.gcs_context_set_mi_coupling(b, None, 0) == 0
    finally:
        lib.gamera_cs_mi_dipole_destroy(ma)
        lib.gamera_cs_mi_dipole_destroy(mb)
        lib.gcs_context_destroy(a)
        lib.gcs_context_destroy(b)


def test_in_graph_coupling_feeds_the_earth_wall(lib):
    """Earth boundary with the coupling as its MI wall: the in-graph updates
    feed the wall's EMF and ghost drift exactly as host-driven ones do."""
    from tests.test_earth_gpu import boundary, wind_series
    from tests.test_ensemble_gpu import download, assert_same_state
    keep = []
    startup, cfg = cases.earth_startup(), _config()
    wind = wind_series(keep)
    o, t = abi.AdvanceOptions(), abi.TimestepOptions()
    assert lib.gcs_case_options(2, C.byref(o), C.byref(t)) == 0
    a = lib.gcs_context_create_case(2, 20, 16, 5)
    b = lib.gcs_context_create_case(2, 20, 16, 5)
    ma, mb = _coupling(lib, a, startup, cfg), _coupling(lib, b, startup, cfg)
    ea, eb = C.c_void_p(), C.c_void_p()
    try:
        for ctx, e, mi in ((a, ea, ma), (b, eb, mb)):
            bd = boundary(startup, wind, None, 0)
            bd.mi = mi
            keep.append(bd)
            assert lib.gcs_earth_create_case(ctx, C.byref(bd), C.byref(e)) == 0, \
                lib.gcs_last_error()
        for s in range(STEPS):
            assert lib.gamera_cs_mi_dipole_maybe_update(ma, _time(lib, a)) in (0, 1)
            assert lib.gcs_context_run_earth(a, ea, C.byref(o), C.byref(t), 0.5, 1, 1) == 0
        assert lib.gcs_context_sync(a) == 0
        assert lib.gcs_context_set_mi_coupling(b, mb, 0) == 0
        assert lib.gcs_context_run_earth(b, eb, C.byref(o), C.byref(t), 0.5, STEPS, 1) == 0
        assert lib.gcs_context_sync(b) == 0, lib.gcs_context_error(b)
        assert_same_state(download(lib, a), download(lib, b))
        pa, ea_, na, sa = _potential(lib, ma, cfg)
        pb, eb_, nb, sb = _potential(lib, mb, cfg)
        assert np.array_equal(pa, pb) and (ea_, na) == (eb_, nb) and sa == sb
    finally:
        for e in (ea, eb):
            if e:
                lib.gcs_earth_destroy(e)
        lib.gamera_cs_mi_dipole_destroy(ma)
        lib.gamera_cs_mi_dipole_destroy(mb)
        lib.gcs_context_destroy(a)
        lib.gcs_context_destroy(b)
