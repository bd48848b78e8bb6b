"""FP32-bulk precision variant against the plain FP64 path on the device.

Both copies of a device-built case advance through the same time levels
(gamera_cube_b200.precision.compare_bulk replays the FP64 run's adaptive
dt).  Bars: every state variable within 1e-5 of its maximum magnitude
(max over active cells), div B of the bulk copy at FP64 round-off
(<= 1e-13 of the largest face flux), and switching the precision back
leaves the plain path bit-identical.
"""
import ctypes as C

import numpy as np
import pytest

from gamera_cube_b200 import precision

pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.fixture(scope="module")
def lib():
    import gamera_cube_b200
    return gamera_cube_b200.lib


@pytest.mark.parametrize("kind,nr,n,steps", [(1, 12, 9, 50), (2, 12, 10, 300)])
def test_bulk_tracks_fp64(lib, kind, nr, n, steps):
    r = precision.compare_bulk(lib, kind, nr, n, steps)
    for name in precision.VARIABLES:
        assert r[name]["linf"] <= TOL, (name, r[name])
    assert r["div_b_bulk"] <= 1e-13
    assert r["div_b_fp64"] <= 1e-13


def test_bulk_split_layers(lib):
    """Wind + dipole case: the strong-dipole inner layers stay FP64, the
    threshold moves the split, and a case without background runs FP32
    everywhere."""
    ctx = lib.gcs_context_create_case(2, 48, 32, 7)
    try:
        assert lib.gcs_context_set_precision(ctx, 1) == 0
        split8 = lib.gcs_context_bulk_split(ctx)
        assert lib.gcs_context_set_bulk_threshold(ctx, 64.0) == 0
        split64 = lib.gcs_context_bulk_split(ctx)
        assert 4 < split64 < split8 < 4 + 48
        assert lib.gcs_context_set_bulk_threshold(ctx, -1.0) == -1
    finally:
        lib.gcs_context_destroy(ctx)
    ctx = lib.gcs_context_create_case(1, 12, 9, 7)
    try:
        assert lib.gcs_context_set_precision(ctx, 1) == 0
        assert lib.gcs_context_bulk_split(ctx) == 0
    finally:
        lib.gcs_context_destroy(ctx)


def test_switching_back_restores_fp64(lib):
    """Enabling the FP32-bulk path (allocating and converting its arrays)
    and switching it off again leaves the plain FP64 path bit-identical."""
    from gamera_cube_b200 import abi
    from gamera_cube_b200.host import HostStorage

    def run(toggle):
        ctx = lib.gcs_context_create_case(2, 12, 10, 7)
        o, ts = abi.AdvanceOptions(), abi.TimestepOptions()
        lib.gcs_case_options(2, C.byref(o), C.byref(ts))
        try:
            if toggle:
                assert lib.gcs_context_set_precision(ctx, 1) == 0
                assert lib.gcs_context_precision(ctx) == 1
                assert lib.gcs_context_set_precision(ctx, 0) == 0
                assert lib.gcs_context_precision(ctx) == 0
            assert lib.gcs_context_run(ctx, C.byref(o), C.byref(ts), 0.5, 3, 1) == 0
            assert lib.gcs_context_sync(ctx) == 0
            act = (C.c_size_t * 3)()
            g = C.c_size_t()
            lib.gcs_context_dims(ctx, act, C.byref(g))
            hs = HostStorage(list(act), g.value)
            assert lib.gcs_context_download_state(ctx, hs.storage, 0) == 0
            return hs
        finally:
            lib.gcs_context_destroy(ctx)

    a, b = run(False), run(True)
    for f in range(6):
        for name in ("conserved", "cell_magnetic", "face_flux0", "face_flux1",
                     "face_flux2"):
            x, y = a.arrays(f)[name], b.arrays(f)[name]
            assert np.array_equal(x.view(np.uint64), y.view(np.uint64)), name
