"""The library's host forms of the reference's per-face Earth callbacks
(gamera_cs_earth_inner_fluid_flux, gamera_cs_earth_no_mi_emf) against the
compiled reference's own, on copies of one stepped reference case: bit for
bit (both are host code with the same operation order).  No GPU needed."""
import ctypes as C

import numpy as np
import pytest

import gamera_cube_b200
from gamera_cube_b200 import abi
from oracle import refbind
from tests.test_earth_gpu import boundary, wind_series

pytestmark = pytest.mark.skipif(not refbind.ref_available(),
                                reason="reference library not built")


def stepped_pair():
    a = refbind.Case(refbind.FX_WIND, 12, 10, 7)
    assert a.step(0.0, 0.5 * a.local_timestep()) == 0
    b = refbind.Case(refbind.FX_WIND, 12, 10, 7)
    b.copy_from(a)
    return a, b


def bounds(case):
    g = case.ghost
    lower = (C.c_size_t * 3)(g, g, g)
    upper = (C.c_size_t * 3)(*[g + case.active[q] for q in range(3)])
    return lower, upper


@pytest.mark.parametrize("strict", [0, 1])
def test_host_emf_callback_matches_reference(strict):
    R = refbind.ref()
    abi.bind(R, abi.earth_callback_signatures())
    ours = gamera_cube_b200.lib
    a, b = stepped_pair()
    keep = []
    startup = abi.EarthStartup()
    startup.gamma = 5.0 / 3.0
    wind = wind_series(keep)
    ba = boundary(startup, wind, a.background, strict)
    bb = boundary(startup, wind, b.background, strict)
    for bd in (ba, bb):
        bd.step_time, bd.step_dt = 0.003, 0.0035
    lower, upper = bounds(a)
    before = [b.arrays(f)["edge_emf1"].copy() for f in range(6)]
    try:
        for f in range(6):
            assert R.gamera_cs_earth_no_mi_emf(C.byref(a.storage[f]), C.byref(a.grid[f]),
                                               lower, upper, C.byref(ba)) == 0
            assert ours.gamera_cs_earth_no_mi_emf(C.byref(b.storage[f]), C.byref(b.grid[f]),
                                                  lower, upper, C.byref(bb)) == 0
            assert R.gamera_cs_earth_inner_fluid_flux(C.byref(a.storage[f]),
                                                      C.byref(a.grid[f]), lower, upper,
                                                      None) == 0
            assert ours.gamera_cs_earth_inner_fluid_flux(C.byref(b.storage[f]),
                                                         C.byref(b.grid[f]), lower, upper,
                                                         None) == 0
        for f in range(6):
            A, B = a.arrays(f), b.arrays(f)
            for d in range(3):
                np.testing.assert_array_equal(A["edge_emf%d" % d], B["edge_emf%d" % d])
                np.testing.assert_array_equal(A["fluid_face_flux%d" % d],
                                              B["fluid_face_flux%d" % d])
        # the callbacks acted on the stepped state
        assert any(not np.array_equal(before[f], b.arrays(f)["edge_emf1"]) for f in range(6))
    finally:
        a.close()
        b.close()


def test_host_callbacks_reject_bad_input():
    ours = gamera_cube_b200.lib
    a = refbind.Case(refbind.FX_WIND, 12, 10, 7)
    try:
        lower, upper = bounds(a)
        keep = []
        startup = abi.EarthStartup()
        startup.gamma = 5.0 / 3.0
        bd = boundary(startup, wind_series(keep), a.background, 0)
        bd.step_time, bd.step_dt = 0.0, 0.0   # the EMF needs a positive step
        assert ours.gamera_cs_earth_no_mi_emf(C.byref(a.storage[0]), C.byref(a.grid[0]),
                                              lower, upper, C.byref(bd)) == -1
        bad_upper = (C.c_size_t * 3)(upper[0], 10 ** 6, upper[2])
        assert ours.gamera_cs_earth_inner_fluid_flux(C.byref(a.storage[0]),
                                                     C.byref(a.grid[0]), lower, bad_upper,
                                                     None) == -1
    finally:
        a.close()
