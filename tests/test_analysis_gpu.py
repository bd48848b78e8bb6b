"""GPU checks of the analysis output (cubedsphere_analysis_hdf5.c): the
device frame against the CPU restatement (oracle/analysis_oracle.py) bit for
bit, and the writer's file set (raw datasets + JSON metadata)."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from gamera_cube_b200 import abi
from oracle import analysis_oracle, oracle_cases

pytestmark = pytest.mark.gpu
GAMMA = 5.0 / 3.0


@pytest.fixture(scope="module")
def lib():
    import gamera_cube_b200
    return gamera_cube_b200.lib


def host_context(lib, case):
    ctx = lib.gcs_context_create(case.grid, case.active, case.ghost)
    assert ctx, lib.gcs_last_error()
    assert lib.gcs_context_upload_background(ctx, case.background) == 0
    assert lib.gcs_context_upload_state(ctx, case.storage) == 0
    return ctx


def expected(case):
    out = []
    for f in range(6):
        a = case.arrays(f)
        bg = case.background[f]
        n = int(np.prod(a["cell_magnetic"].shape[:3]))
        b0 = np.ctypeslib.as_array(C.cast(bg.cell_magnetic, C.POINTER(C.c_double)),
                                   shape=(3 * n,)).reshape(a["cell_magnetic"].shape)
        out.append(analysis_oracle.frame(a["conserved"], a["cell_magnetic"], b0, case.ghost,
                                         GAMMA))
    return np.stack(out)


def test_frame_matches_restatement(lib):
    case = oracle_cases.Case("wind", 12, 10, 7)
    assert case.step(0.0, 0.5 * case.local_timestep()) == 0
    ctx = host_context(lib, case)
    try:
        n = lib.gcs_analysis_frame_floats(ctx)
        assert n == 6 * 8 * 12 * 10 * 10
        host = np.zeros(n, np.float32)
        assert lib.gcs_context_analysis_frame(ctx, GAMMA, None, host.ctypes.data) == 0
        want = expected(case)
        np.testing.assert_array_equal(host.reshape(want.shape), want)
        # and the frames recorded through the reference's own conversion
        # (tests/golden/make_analysis_golden.py, same case and step)
        golden = np.load(os.path.join(os.path.dirname(__file__), "golden",
                                      "reference_analysis.npz"))["frames"]
        np.testing.assert_array_equal(host.reshape(golden.shape), golden)
        # an invalid state fails as the reference writer does
        case.arrays(3)["conserved"][6, 7, 8, 0] = -1.0
        assert lib.gcs_context_upload_state(ctx, case.storage) == 0
        assert lib.gcs_context_analysis_frame(ctx, GAMMA, None, host.ctypes.data) == -1
    finally:
        lib.gcs_context_destroy(ctx)


def test_writer_file_set(lib, tmp_path):
    case = oracle_cases.Case("wind", 12, 10, 7)
    ctx = host_context(lib, case)
    dev = lib.gcs_context_create_case(2, 12, 10, 7)
    try:
        d = str(tmp_path / "host")
        os.makedirs(d)
        assert lib.gcs_context_write_analysis(ctx, d.encode(), 3, 40, 0.25, 15.93, GAMMA,
                                              case.grid) == 0
        want = expected(case)
        for f in range(6):
            meta = json.load(open(os.path.join(d, "analysis_p%d_000003.json" % f)))
            assert meta["patch_id"] == f and meta["sequence"] == 3 and meta["step"] == 40
            assert meta["global_cells"] == [12, 10, 10]
            assert meta["field_names"] == ["rho", "p", "vx", "vy", "vz", "Bx", "By", "Bz"]
            assert meta["time_seconds"] == 15.93 and len(meta["normalization"]) == 10
            st = np.fromfile(os.path.join(d, meta["state"]["file"]), "<f4")
            np.testing.assert_array_equal(st.reshape(meta["state"]["shape"]), want[f])
            gm = json.load(open(os.path.join(d, "analysis_grid_p%d.json" % f)))
            xyz = np.fromfile(os.path.join(d, gm["coordinates"]["file"]), "<f8")
            xyz = xyz.reshape(gm["coordinates"]["shape"])
            cen = np.ctypeslib.as_array(case.grid[f].cell, shape=(20 * 18 * 18,))
            cen = np.asarray(cen["centroid"]["value"]).reshape(20, 18, 18, 3)[4:-4, 4:-4, 4:-4]
            np.testing.assert_array_equal(xyz, np.moveaxis(cen, -1, 0))
            vtx = np.fromfile(os.path.join(d, gm["vertices"]["file"]), "<f8")
            assert vtx.size == 3 * 13 * 11 * 11
        # a device-built case rebuilds its grid on the device
        d2 = str(tmp_path / "device")
        os.makedirs(d2)
        assert lib.gcs_context_write_analysis(dev, d2.encode(), 0, 0, 0.0, 0.0, GAMMA,
                                              None) == 0, lib.gcs_last_error()
        for f in range(6):
            a = np.fromfile(os.path.join(d, "analysis_grid_p%d.coordinates.f64" % f), "<f8")
            b = np.fromfile(os.path.join(d2, "analysis_grid_p%d.coordinates.f64" % f), "<f8")
            np.testing.assert_allclose(b, a, rtol=0, atol=1e-12 * np.abs(a).max())
            a = np.fromfile(os.path.join(d, "analysis_grid_p%d.vertices.f64" % f), "<f8")
            b = np.fromfile(os.path.join(d2, "analysis_grid_p%d.vertices.f64" % f), "<f8")
            np.testing.assert_allclose(b, a, rtol=0, atol=1e-12 * np.abs(a).max())
            s1 = np.fromfile(os.path.join(d, "analysis_p%d_000003.state.f32" % f), "<f4")
            s2 = np.fromfile(os.path.join(d2, "analysis_p%d_000000.state.f32" % f), "<f4")
            np.testing.assert_allclose(s2, s1, rtol=1e-6, atol=1e-6 * np.abs(s1).max())
    finally:
        lib.gcs_context_destroy(ctx)
        lib.gcs_context_destroy(dev)
