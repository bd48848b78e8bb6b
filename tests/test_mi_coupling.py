"""Magnetosphere-ionosphere coupling (cubedsphere_mi_dipole.c) against the
reference.

Inputs: the wind fixture case (12 x 10 x 10 per face) with the analytic
residual field of the reference MI shell test on its active cells, the
reference Earth driver's MI configuration (192 x 22 per hemisphere, shell 1,
5 S) and one update at t = 0.  The golden outputs come from the reference
build (tests/golden/make_golden_mi.py).

Tolerances of the GPU comparison:
* FAC on the polar grids, shell J_parallel: 1e-11 of their maximum (the
  same formulas; the calibrated recovery and the sums run in a different
  order on the device);
* potential, lookups, wall EMF, ghost velocities: 5e-8 of their maximum
  (the potential solves agree to the solver tolerance, see test_mi_gpu.py);
* solver iterations within 3 %.
"""
import ctypes as C

import numpy as np
import pytest

import mi_util
from mi_util import POTENTIAL_RTOL, golden
from oracle import oracle_cases, refbind


def close(a, b, rtol):
    scale = float(np.max(np.abs(b)))
    return float(np.max(np.abs(a - b))) <= rtol * max(scale, 1e-300)


def input_case():
    kind, nr, n, seed = mi_util.COUPLING_CASE
    case = oracle_cases.Case(kind, nr, n, seed)
    mi_util.set_mi_field(case)
    return case


@pytest.mark.skipif(not refbind.ref_available(), reason="reference library not built")
def test_reference_reproduces_golden_and_inputs_match():
    """Pins the golden coupling outputs to the reference build, and the
    numpy-evaluated analytic field of the inputs to the fixture's C one."""
    R = refbind.ref()
    kind, nr, n, seed = mi_util.COUPLING_CASE
    ref_case = refbind.Case(refbind.FX_WIND, nr, n, seed)
    assert R.fx_set_mi_field(ref_case.handle) == 0
    ours = input_case()
    for f in range(6):
        a, b = ours.arrays(f), ref_case.arrays(f)
        for name in ("cell_magnetic", "old_cell_magnetic"):
            assert np.array_equal(a[name].view(np.uint64), b[name].view(np.uint64))
    cfg, startup = mi_util.coupling_config(), mi_util.coupling_startup()
    mi = R.fx_mi_create(ref_case.handle, C.byref(startup), C.byref(cfg))
    assert mi
    try:
        assert R.gamera_cs_mi_dipole_maybe_update(mi, 0.0) == 1
        out = mi_util.coupling_outputs(R, mi, ref_case, cfg)
    finally:
        R.gamera_cs_mi_dipole_destroy(mi)
    g = golden()
    for k, v in out.items():
        assert np.array_equal(np.asarray(v), g["coupling/" + k]), k


def test_potential_view_and_import_export_on_host():
    """The potential view needs no GPU work: import, export, lookups and
    the cadence rule (cubedsphere_mi_dipole.c:54-158, :372-378)."""
    import gamera_cube_b200
    L = gamera_cube_b200.lib
    cfg, startup = mi_util.coupling_config(), mi_util.coupling_startup()
    mi = C.c_void_p()
    assert L.gamera_cs_mi_dipole_create_potential_view(C.byref(startup), C.byref(cfg),
                                                       C.byref(mi)) == 0
    try:
        assert L.gamera_cs_mi_dipole_ready(mi) == 0
        assert L.gamera_cs_mi_dipole_update_due(mi, 0.0) == 1
        assert L.gamera_cs_mi_dipole_update_due(mi, -1.0) == -1
        g = golden()
        pot = np.ascontiguousarray(g["coupling/potential"])
        P = C.POINTER(C.c_double)
        assert L.gamera_cs_mi_dipole_import_potential(mi, pot.ctypes.data_as(P),
                                                      pot.size, 0.0, 10.0) == 0
        assert L.gamera_cs_mi_dipole_ready(mi) == 1
        # 10 s cadence: one code time is length/speed = 63.71 s
        assert L.gamera_cs_mi_dipole_update_due(mi, 9.0 / 63.71) == 0
        assert L.gamera_cs_mi_dipole_update_due(mi, 10.0 / 63.71) == 1
        back = np.zeros_like(pot)
        ep, nx = C.c_double(), C.c_double()
        assert L.gamera_cs_mi_dipole_export_potential(mi, back.ctypes.data_as(P), back.size,
                                                      C.byref(ep), C.byref(nx)) == 0
        assert np.array_equal(back, pot) and (ep.value, nx.value) == (0.0, 10.0)
        bad = pot.copy()
        bad[5] = np.nan
        assert L.gamera_cs_mi_dipole_import_potential(mi, bad.ctypes.data_as(P),
                                                      bad.size, 0.0, 10.0) == -1
        # lookups from the imported reference potential are the reference's
        look = np.zeros(len(mi_util.probe_points()))
        for q, p in enumerate(mi_util.probe_points()):
            v = mi_util.abi.Vec3()
            for a in range(3):
                v.value[a] = p[a]
            val = C.c_double()
            assert L.gamera_cs_mi_dipole_potential(mi, v, C.byref(val)) == 0
            look[q] = val.value
        assert np.array_equal(look, g["coupling/lookup"])
    finally:
        L.gamera_cs_mi_dipole_destroy(mi)


@pytest.mark.gpu
def test_update_against_reference():
    import gamera_cube_b200
    L = gamera_cube_b200.lib
    case = input_case()
    cfg, startup = mi_util.coupling_config(), mi_util.coupling_startup()
    mi = C.c_void_p()
    assert L.gamera_cs_mi_dipole_create(case.grid, case.storage, case.background,
                                        C.byref(startup), case.active, case.ghost,
                                        C.byref(cfg), C.byref(mi)) == 0, \
        L.gcs_last_error().decode()
    try:
        assert L.gamera_cs_mi_dipole_update_due(mi, 0.0) == 1
        assert L.gamera_cs_mi_dipole_maybe_update(mi, 0.0) == 1, \
            L.gcs_last_error().decode()
        assert L.gamera_cs_mi_dipole_maybe_update(mi, 0.0) == 0
        out = mi_util.coupling_outputs(L, mi, case, cfg)
    finally:
        L.gamera_cs_mi_dipole_destroy(mi)
    g = golden()

    def ref(k):
        return g["coupling/" + k]

    assert np.array_equal(out["times"], ref("times"))
    assert np.allclose(out["view"], ref("view"), rtol=1e-14, atol=0.0)
    assert close(out["fac"], ref("fac"), 1e-11)
    assert close(out["shell_j"], ref("shell_j"), 1e-11)
    assert np.array_equal(out["shell_mlat"], ref("shell_mlat"))
    assert np.array_equal(out["shell_phi"], ref("shell_phi"))
    assert close(out["potential"], ref("potential"), POTENTIAL_RTOL)
    assert close(out["lookup"], ref("lookup"), POTENTIAL_RTOL)
    assert close(out["wall_emf"], ref("wall_emf"), POTENTIAL_RTOL)
    assert close(out["ghost_velocity"], ref("ghost_velocity"), 1e-6)
    for h in range(2):
        assert abs(out["stats"][h] - ref("stats")[h]) <= max(3, 0.03 * ref("stats")[h])
    # FAC extremes: within the FAC tolerance of the reference's
    assert close(out["stats"][4:6], ref("stats")[4:6], 1e-11)


@pytest.mark.gpu
def test_device_built_case_coupling():
    """The coupling on a device-built case (no host grid) matches the one
    on the host grid of the same case."""
    import gamera_cube_b200
    from gamera_cube_b200 import abi
    L = gamera_cube_b200.lib
    kind, nr, n, seed = mi_util.COUPLING_CASE
    ctx = L.gcs_context_create_case(oracle_cases.KINDS[kind], nr, n, seed)
    assert ctx, L.gcs_last_error().decode()
    cfg, startup = mi_util.coupling_config(), mi_util.coupling_startup()
    mi = C.c_void_p()
    try:
        assert L.gcs_context_mi_dipole_create(ctx, C.byref(startup), C.byref(cfg),
                                              C.byref(mi)) == 0, \
            L.gcs_last_error().decode()
        assert L.gamera_cs_mi_dipole_maybe_update(mi, 0.0) == 1, \
            L.gcs_last_error().decode()
        view = abi.MiAnalysisView()
        assert L.gamera_cs_mi_dipole_analysis_view(mi, C.byref(view)) == 0
        per = cfg.azimuth_points * cfg.colatitude_points
        fac = np.concatenate([np.ctypeslib.as_array(view.fac_parallel_a_m2[h],
                                                    shape=(per,)).copy() for h in range(2)])
        st = (abi.MiSolverStats * 2)()
        mm = [C.c_double() for _ in range(4)]
        assert L.gamera_cs_mi_dipole_stats(mi, *[C.byref(v) for v in mm], st) == 0
        assert st[0].converged == 1 and st[1].converged == 1
        # uniform wind + IMF: the residual field is curl-free up to
        # round-off, so the coupling current is at round-off level
        assert np.isfinite(fac).all()
        assert float(np.max(np.abs(fac))) < 1e-14
        assert abs(view.sample_radius_re - golden()["coupling/view"][1]) < 1e-12
    finally:
        if mi:
            L.gamera_cs_mi_dipole_destroy(mi)
        L.gcs_context_destroy(ctx)
