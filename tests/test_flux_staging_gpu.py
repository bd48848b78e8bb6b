"""The TMA-staged flux sweep against the per-face flux sweep it replaces.

Both read the same predictor outputs and run the same arithmetic per face;
only where the eight-cell Up7 stencil comes from differs (shared memory
filled by tiled bulk tensor copies, or per-face loads from global memory).
Cases built on the device are stepped with each sweep (plain FP64 and
FP32-bulk, the step graph with device dt) and must agree bit for bit: the
state after the steps and the fluid and Maxwell face fluxes of the last
step.  The sizes cover partial tiles along every axis (9, 10 and 32
angular cells per face; 12 and 48 radial) and the extra last face along
the sweep axis.
"""
import ctypes as C

import numpy as np
import pytest

from gamera_cube_b200 import abi
from gamera_cube_b200.host import HostStorage

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import gamera_cube_b200
    return gamera_cube_b200.lib


def _run(lib, kind, nr, n, steps, staged, bulk):
    ctx = lib.gcs_context_create_case(kind, nr, n, 7)
    assert ctx, lib.gcs_last_error()
    try:
        assert lib.gcs_context_set_flux_staging(ctx, staged) == 0
        if bulk:
            assert lib.gcs_context_set_precision(ctx, 1) == 0
        opts, ts = abi.AdvanceOptions(), abi.TimestepOptions()
        lib.gcs_case_options(kind, C.byref(opts), C.byref(ts))
        assert lib.gcs_context_run(ctx, C.byref(opts), C.byref(ts), 0.5, steps, 1) == 0
        assert lib.gcs_context_sync(ctx) == 0, lib.gcs_context_error(ctx)
        act = (C.c_size_t * 3)()
        g = C.c_size_t()
        lib.gcs_context_dims(ctx, act, C.byref(g))
        hs = HostStorage(list(act), g.value, scratch=True)
        assert lib.gcs_context_download_state(ctx, hs.storage, 1) == 0
        return hs
    finally:
        lib.gcs_context_destroy(ctx)


NAMES = ["conserved", "old_conserved", "cell_magnetic", "old_cell_magnetic"] + \
    ["face_flux%d" % d for d in range(3)] + \
    ["fluid_face_flux%d" % d for d in range(3)] + \
    ["maxwell_face_flux%d" % d for d in range(3)]


@pytest.mark.parametrize("bulk", [0, 1])
@pytest.mark.parametrize("kind,nr,n,steps", [
    (1, 12, 9, 3),      # radial shock, no background
    (2, 12, 10, 3),     # wind + dipole, Boris, HOGS, emergency diffusion
    (2, 48, 32, 2),     # configuration C1
])
def test_staged_flux_is_bitwise(lib, kind, nr, n, steps, bulk):
    a = _run(lib, kind, nr, n, steps, 0, bulk)
    b = _run(lib, kind, nr, n, steps, 1, bulk)
    for f in range(6):
        for name in NAMES:
            x, y = a.arrays(f)[name], b.arrays(f)[name]
            assert np.array_equal(x, y, equal_nan=True), (f, name,
                                                          float(np.nanmax(np.abs(x - y))))
