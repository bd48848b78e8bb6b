"""Stand-alone halo fills and seam syncs (cubedsphere_halo.h,
cubedsphere_interface.h) on the GPU against the restatement oracle, bit for
bit, on a wind case whose state arrays carry seeded +-1 % perturbations so
every seam, halo and edge group is non-trivial."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle_cases

pytestmark = pytest.mark.gpu

ARRAYS = ["conserved", "old_conserved", "cell_magnetic", "old_cell_magnetic",
          "face_flux0", "face_flux1", "face_flux2", "old_face_flux0",
          "old_face_flux1", "old_face_flux2", "fluid_face_flux0", "fluid_face_flux1",
          "fluid_face_flux2", "maxwell_face_flux0", "maxwell_face_flux1",
          "maxwell_face_flux2", "edge_emf0", "edge_emf1", "edge_emf2"]


def glib():
    import gamera_cube_b200
    return gamera_cube_b200.lib


def perturbed_case():
    case = oracle_cases.Case("wind", 12, 10, 5)
    rng = np.random.default_rng(17)
    for f in range(6):
        arr = case.arrays(f)
        for name in ARRAYS:
            a = arr[name]
            a[...] = a * (1.0 + 0.01 * rng.uniform(-1.0, 1.0, size=a.shape)) + \
                (0.0 if name.endswith("conserved") else 1e-3 * rng.uniform(-1, 1, a.shape))
    return case


def same(a, b, faces=range(6)):
    for f in faces:
        for name in ARRAYS:
            x, y = a.arrays(f)[name], b.arrays(f)[name]
            if not np.array_equal(x.view(np.uint64), y.view(np.uint64)):
                return "face %d %s" % (f, name)
    return None


def test_cell_and_face_halos():
    O, L = oracle_cases.lib(), glib()
    ref, ours = perturbed_case(), perturbed_case()
    assert same(ref, ours) is None
    plan = C.c_void_p()
    assert O.gcso_halo_plan_create(ref.grid, ref.active, ref.ghost, C.byref(plan)) == 0
    try:
        assert O.gcso_fill_cell_halos(plan, ref.storage) == 0
        assert L.gamera_cs_fill_tangential_cell_halos(ours.grid, ours.storage, ours.active,
                                                      ours.ghost) == 0
        assert same(ref, ours) is None
        assert O.gcso_fill_face_halos(plan, ref.grid, ref.storage) == 0
        assert L.gamera_cs_fill_magnetic_face_halos(ours.grid, ours.storage, ours.active,
                                                    ours.ghost) == 0
        assert same(ref, ours) is None
    finally:
        O.gcso_halo_plan_destroy(plan)


def test_planned_face_variants_write_only_the_receiver():
    O, L = oracle_cases.lib(), glib()
    ref, ours, orig = perturbed_case(), perturbed_case(), perturbed_case()
    plan, gplan = C.c_void_p(), C.c_void_p()
    assert O.gcso_halo_plan_create(ref.grid, ref.active, ref.ghost, C.byref(plan)) == 0
    assert L.gamera_cs_halo_plan_create(ours.grid, ours.active, ours.ghost,
                                        C.byref(gplan)) == 0
    try:
        assert O.gcso_fill_cell_halos(plan, ref.storage) == 0
        assert O.gcso_fill_face_halos(plan, ref.grid, ref.storage) == 0
        assert L.gamera_cs_fill_tangential_cell_halos_planned_face(
            gplan, ours.grid, ours.storage, 2) == 0
        assert L.gamera_cs_fill_magnetic_face_halos_planned_face(
            gplan, ours.grid, ours.storage, 2) == 0
        assert same(ref, ours, faces=[2]) is None
        assert same(orig, ours, faces=[0, 1, 3, 4, 5]) is None
        assert L.gamera_cs_fill_magnetic_face_halos_planned_face(
            gplan, ours.grid, ours.storage, 6) == -1
    finally:
        O.gcso_halo_plan_destroy(plan)
        L.gamera_cs_halo_plan_destroy(gplan)


def test_radial_outflow():
    O, L = oracle_cases.lib(), glib()
    ref, ours, orig = perturbed_case(), perturbed_case(), perturbed_case()
    assert O.gcso_fill_radial_outflow(ref.storage, ref.active, ref.ghost) == 0
    assert L.gamera_cs_fill_radial_outflow_cells_face(ours.storage, ours.active,
                                                      ours.ghost, 4) == 0
    assert same(ref, ours, faces=[4]) is None
    assert same(orig, ours, faces=[0, 1, 2, 3, 5]) is None
    assert L.gamera_cs_fill_radial_outflow_cells(ours.storage, ours.active,
                                                 ours.ghost) == 0
    assert same(ref, ours) is None


def test_seam_syncs():
    O, L = oracle_cases.lib(), glib()
    ref, ours = perturbed_case(), perturbed_case()
    assert O.gcso_sync_faces(ref.storage, ref.active, ref.ghost, 1) == 0
    assert L.gamera_cs_sync_magnetic_face_flux(ours.storage, ours.active, ours.ghost) == 0
    assert same(ref, ours) is None
    assert O.gcso_sync_faces(ref.storage, ref.active, ref.ghost, 0) == 0
    assert L.gamera_cs_sync_mhd_face_fluxes(ours.storage, ours.active, ours.ghost) == 0
    assert same(ref, ours) is None


def test_edge_emf_syncs():
    O, L = oracle_cases.lib(), glib()
    ref, ours = perturbed_case(), perturbed_case()
    plan, gplan = C.c_void_p(), C.c_void_p()
    assert O.gcso_edge_plan_create(ref.active, ref.ghost, C.byref(plan)) == 0
    assert L.gamera_cs_edge_sync_plan_create(ours.grid, ours.active, ours.ghost,
                                             C.byref(gplan)) == 0
    try:
        assert O.gcso_sync_edges(plan, ref.storage) == 0
        assert L.gamera_cs_sync_edge_emf_planned(gplan, ours.storage) == 0
        assert same(ref, ours) is None
        assert O.gcso_sync_edges(plan, ref.storage) == 0
        assert L.gamera_cs_sync_edge_emf(ours.grid, ours.storage, ours.active,
                                         ours.ghost) == 0
        assert same(ref, ours) is None
    finally:
        O.gcso_edge_plan_destroy(plan)
        L.gamera_cs_edge_sync_plan_destroy(gplan)
