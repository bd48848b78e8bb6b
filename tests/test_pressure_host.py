"""CPU checks of the oracle's post-step pressure control
(nonorthogonal_step.c:74-171): against the golden vectors recorded from the
unmodified reference (tests/golden/reference_pressure.npz, made by
tests/golden/make_pressure_golden.py), against the reference library itself
when it is built here (whole arrays, a failing cell included), and the
reference's argument checks."""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import oracle_cases, refbind
from tests import pressure_util as pu
from tests.golden.make_golden import sample_indices

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_pressure.npz")


def stepped_wind():
    case = oracle_cases.Case("wind", 12, 10, 7)
    assert case.step(0.0, 0.5 * case.local_timestep()) == 0
    return case


def test_oracle_matches_golden():
    g = np.load(GOLDEN)
    case = stepped_wind()
    light, thr, low_sound, dt = g["params"]
    rc, low, hot, ms, mp = pu.apply_faces(case.lib.gcso_apply_pressure_control, case.storage,
                                          case.grid, case.ghost, list(case.active), dt,
                                          light, thr, low_sound)
    assert rc == 0
    assert [low, hot] == list(g["counts"])
    assert [ms, mp] == list(g["maxima"])
    for f in range(6):
        flat = np.ascontiguousarray(case.arrays(f)["conserved"]).reshape(-1)
        np.testing.assert_array_equal(flat[sample_indices(flat.size)], g["f%d/sample" % f])
        np.testing.assert_allclose([flat.sum(), np.abs(flat).sum()], g["f%d/sum" % f],
                                   rtol=1e-14, atol=0)


@pytest.mark.skipif(not refbind.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("poison", [False, True])
def test_oracle_matches_reference_bitwise(poison):
    ref = refbind.Case(refbind.FX_WIND, 12, 10, 7)
    orc = oracle_cases.Case("wind", 12, 10, 7)
    dt = 0.5 * ref.local_timestep()
    assert ref.step(0.0, dt) == 0 and orc.step(0.0, dt) == 0
    act, g = list(ref.active), ref.ghost
    light, thr, low_sound = pu.parameters([ref.arrays(f) for f in range(6)], g, act)
    if poison:   # one active cell the primitive conversion rejects
        for c in (ref, orc):
            c.arrays(2)["conserved"][g + 3, g + 4, g + 5, 0] = -1.0
    a = pu.apply_faces(ref.lib.gamera_no_apply_pressure_control, ref.storage, ref.grid, g,
                       act, pu.DT, light, thr, low_sound)
    b = pu.apply_faces(orc.lib.gcso_apply_pressure_control, orc.storage, orc.grid, g, act,
                       pu.DT, light, thr, low_sound)
    assert a == b
    assert a[0] == (-1 if poison else 0) and a[1] > 0 and a[2] > 0
    for f in range(6):
        np.testing.assert_array_equal(orc.arrays(f)["conserved"], ref.arrays(f)["conserved"])


def test_oracle_rejects_invalid_arguments():
    case = oracle_cases.Case("wind", 12, 10, 7)
    fn = case.lib.gcso_apply_pressure_control
    before = case.arrays(0)["conserved"].copy()
    for dt, gamma, c, thr, cs in [(0.0, pu.GAMMA, 1.0, 1.0, 0.0), (0.1, 1.0, 1.0, 1.0, 0.0),
                                  (0.1, pu.GAMMA, 0.0, 1.0, 0.0),
                                  (0.1, pu.GAMMA, 1.0, 0.0, 0.0),
                                  (0.1, pu.GAMMA, 1.0, 1.0, -1.0)]:
        lo = (C.c_size_t * 3)(4, 4, 4)
        hi = (C.c_size_t * 3)(16, 14, 14)
        assert fn(C.byref(case.storage[0]), C.byref(case.grid[0]), lo, hi, dt, gamma,
                  pu.RHO_FLOOR, pu.P_FLOOR, c, thr, cs, None, None, None, None) == -1
    np.testing.assert_array_equal(case.arrays(0)["conserved"], before)


def test_c_abi_rejects_missing_handles():
    """Host-side argument checks of the device entry points (no CUDA call is
    reached): a missing context, configuration or plan is -1."""
    import gamera_cube_b200
    from gamera_cube_b200 import abi
    lib = gamera_cube_b200.lib
    cfg = abi.PressureControl(pu.GAMMA, pu.RHO_FLOOR, pu.P_FLOOR, 10.0, 1e-3, 1e-7)
    assert lib.gcs_context_pressure_control(None, None, 0.1, C.byref(cfg), None, None,
                                            None, None) == -1
    assert lib.gcs_context_set_pressure_control(None, None, C.byref(cfg)) == -1
    assert lib.gcs_context_pressure_control_stats(None, None, None, None, None, 0) == -1
    assert lib.gcs_mi_tensor_plan_set_ordering(None, 1) == -1
    assert lib.gcs_mi_tensor_plan_set_schedule(None, 1) == -1
    assert lib.gcs_mi_tensor_plan_schedule(None, None, None) == -1
