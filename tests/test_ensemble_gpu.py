"""GPU checks of the driven wind builder, the launch tiles, the autotuner and
ensembles.

Chain of parity: the driven device builder matches the oracle's driven case
(set-up and one step, to device-libm rounding, as the plain builder does);
tiles change no result bit; every run of an ensemble (runs sharing a grid,
one CUDA graph per ensemble step, FP64 or FP32-bulk) is bit-identical to the
same run stepped alone through gcs_context_run."""
import ctypes as C

import numpy as np
import pytest

from gamera_cube_b200 import abi
from gamera_cube_b200.host import HostStorage
from oracle import oracle_cases

pytestmark = pytest.mark.gpu

STATE = ["conserved", "old_conserved", "cell_magnetic", "old_cell_magnetic"] + \
        ["face_flux%d" % d for d in range(3)] + ["old_face_flux%d" % d for d in range(3)]

DRIVERS = [(12.0, -650.0, 1.5e5, 3.0), (2.0, -350.0, 6.0e4, -9.0),
           (18.0, -780.0, 1.9e5, -1.0), (5.0, -400.0, 1.0e5, -5.0)]


@pytest.fixture(scope="module")
def lib():
    import gamera_cube_b200
    return gamera_cube_b200.lib


def options(lib):
    o, t = abi.AdvanceOptions(), abi.TimestepOptions()
    assert lib.gcs_case_options(2, C.byref(o), C.byref(t)) == 0
    return o, t


def download(lib, ctx):
    act = (C.c_size_t * 3)()
    g = C.c_size_t()
    assert lib.gcs_context_dims(ctx, act, C.byref(g)) == 0
    hs = HostStorage(list(act), g.value)
    assert lib.gcs_context_download_state(ctx, hs.storage, 0) == 0
    return hs


def wind(lib, nr, n, seed, drv):
    ctx = lib.gcs_context_create_wind(nr, n, seed, C.byref(abi.WindDriver(*drv)))
    assert ctx, lib.gcs_last_error()
    return ctx


def assert_same_state(a, b):
    for f in range(6):
        A, B = a.arrays(f), b.arrays(f)
        for name in STATE:
            np.testing.assert_array_equal(A[name], B[name], err_msg="%s face %d" % (name, f))


def params(lib, ctx):
    dt, ratio, cfl = C.c_double(), C.c_double(), C.c_double()
    steps = C.c_int()
    assert lib.gcs_context_params(ctx, C.byref(dt), C.byref(ratio), C.byref(cfl),
                                  C.byref(steps)) == 0
    return dt.value, ratio.value, steps.value


@pytest.mark.parametrize("drv", DRIVERS[:2])
def test_driven_builder_matches_oracle(lib, drv):
    ctx = wind(lib, 12, 10, 7, drv)
    try:
        oracle = oracle_cases.Case("wind", 12, 10, 7, driver=drv)
        g, act = oracle.ghost, oracle.active
        active = (slice(g, g + act[0]), slice(g, g + act[1]), slice(g, g + act[2]))

        def worst(hs):
            out = 0.0
            for name in ("conserved", "cell_magnetic", "face_flux0", "face_flux1",
                         "face_flux2"):
                d = s = 0.0
                for f in range(6):
                    a, b = hs.arrays(f)[name], oracle.arrays(f)[name]
                    if name == "conserved":
                        a, b = a[active], b[active]
                    d = max(d, float(np.max(np.abs(a - b))))
                    s = max(s, float(np.max(np.abs(b))))
                out = max(out, d / s)
            return out

        assert worst(download(lib, ctx)) <= 1e-12
        dt = 0.5 * oracle.local_timestep()
        assert oracle.step(0.0, dt) == 0
        assert lib.gcs_context_step(ctx, oracle.options, 0.0, dt) == 0
        assert worst(download(lib, ctx)) <= 1e-11
    finally:
        lib.gcs_context_destroy(ctx)


def test_default_driver_is_the_wind_case(lib):
    a = lib.gcs_context_create_case(2, 12, 10, 7)
    b = wind(lib, 12, 10, 7, DRIVERS[3])
    try:
        assert_same_state(download(lib, a), download(lib, b))
    finally:
        lib.gcs_context_destroy(a)
        lib.gcs_context_destroy(b)


def test_tiles_change_no_result(lib):
    o, t = options(lib)
    a = wind(lib, 20, 10, 3, DRIVERS[0])
    b = wind(lib, 20, 10, 3, DRIVERS[0])
    try:
        for f, (bx, by) in enumerate([(64, 4), (32, 4), (32, 8), (64, 2), (64, 4),
                                      (32, 4), (128, 2)]):
            assert lib.gcs_context_set_tile(b, f, bx, by) == 0
            x, y = C.c_int(), C.c_int()
            assert lib.gcs_context_tile(b, f, C.byref(x), C.byref(y)) == 0
            assert (x.value, y.value) == (bx, by)
        assert lib.gcs_context_set_tile(b, 1, 256, 1) == -1   # above the flux limit
        assert lib.gcs_context_set_tile(b, 0, 48, 1) == -1    # not whole warps
        for ctx in (a, b):
            assert lib.gcs_context_run(ctx, C.byref(o), C.byref(t), 0.5, 3, 1) == 0
            assert lib.gcs_context_sync(ctx) == 0
        assert_same_state(download(lib, a), download(lib, b))
        assert params(lib, a) == params(lib, b)
    finally:
        lib.gcs_context_destroy(a)
        lib.gcs_context_destroy(b)


def test_autotune_keeps_state_and_picks_a_valid_tile(lib):
    o, t = options(lib)
    a = wind(lib, 24, 12, 5, DRIVERS[1])
    b = wind(lib, 24, 12, 5, DRIVERS[1])
    try:
        before = download(lib, a)
        best = (C.c_double * 7)()
        default = (C.c_double * 7)()
        assert lib.gcs_context_autotune(a, C.byref(o), C.byref(t), 3, best, default) == 0
        assert_same_state(before, download(lib, a))
        for f in range(7):
            bx, by = C.c_int(), C.c_int()
            assert lib.gcs_context_tile(a, f, C.byref(bx), C.byref(by)) == 0
            assert (bx.value * by.value) % 32 == 0
            assert bx.value * by.value <= lib.gcs_tile_limit(f)
            if f in (4, 5):
                assert best[f] == 0.0 and (bx.value, by.value) == (128, 1)
            else:
                assert 0.0 < best[f] <= default[f]
        # the tuned run steps exactly as the untuned one
        for ctx in (a, b):
            assert lib.gcs_context_run(ctx, C.byref(o), C.byref(t), 0.5, 3, 1) == 0
            assert lib.gcs_context_sync(ctx) == 0
        assert_same_state(download(lib, a), download(lib, b))
    finally:
        lib.gcs_context_destroy(a)
        lib.gcs_context_destroy(b)


def make_ensemble(lib, sizes, drivers, seed, bulk, tune):
    k = len(sizes)
    nr = (C.c_size_t * k)(*[s[0] for s in sizes])
    n = (C.c_size_t * k)(*[s[1] for s in sizes])
    drv = (abi.WindDriver * k)(*[abi.WindDriver(*d) for d in drivers])
    cfg = abi.EnsembleConfig(k, nr, n, drv, seed, bulk, tune, 0.5)
    e = lib.gcs_ensemble_create(C.byref(cfg))
    assert e, lib.gcs_last_error()
    return e, (nr, n, drv)


@pytest.mark.parametrize("bulk", [0, 1])
def test_ensemble_runs_equal_standalone_runs(lib, bulk):
    o, t = options(lib)
    sizes = [(20, 10), (24, 12), (20, 10), (20, 10), (24, 12)]
    drivers = [DRIVERS[0], DRIVERS[1], DRIVERS[2], DRIVERS[3], DRIVERS[2]]
    seed, steps = 11, 4
    e, keep = make_ensemble(lib, sizes, drivers, seed, bulk, 2 if bulk else 0)
    try:
        assert lib.gcs_ensemble_count(e) == 5
        assert [lib.gcs_ensemble_grid_owner(e, i) for i in range(5)] == [0, 1, 0, 0, 1]
        assert lib.gcs_ensemble_advance(e, steps - 1) == 0
        assert lib.gcs_ensemble_advance(e, 1) == 0
        failed = C.c_int()
        assert lib.gcs_ensemble_sync(e, C.byref(failed)) == 0, failed.value
        nodes, grids = C.c_int(), C.c_int()
        assert lib.gcs_ensemble_graph_info(e, C.byref(nodes), C.byref(grids)) == 0
        assert grids.value == 2 and nodes.value > 5 * 20
        for i, ((nr, n), drv) in enumerate(zip(sizes, drivers)):
            run = lib.gcs_ensemble_run_context(e, i)
            alone = wind(lib, nr, n, seed + i, drv)
            try:
                if bulk:
                    assert lib.gcs_context_set_precision(alone, 1) == 0
                assert lib.gcs_context_run(alone, C.byref(o), C.byref(t), 0.5, steps, 1) == 0
                assert lib.gcs_context_sync(alone) == 0
                assert params(lib, run) == params(lib, alone)
                assert params(lib, run)[2] == steps
                assert_same_state(download(lib, run), download(lib, alone))
            finally:
                lib.gcs_context_destroy(alone)
        # runs with different drivers differ
        h0 = download(lib, lib.gcs_ensemble_run_context(e, 0))
        h2 = download(lib, lib.gcs_ensemble_run_context(e, 2))
        assert not np.array_equal(h0.arrays(0)["conserved"], h2.arrays(0)["conserved"])
    finally:
        lib.gcs_ensemble_destroy(e)


def test_ensemble_rejects_what_does_not_fit(lib):
    k = 400
    nr = (C.c_size_t * k)(*([256, 200] * (k // 2)))
    n = (C.c_size_t * k)(*([128, 100] * (k // 2)))
    drv = (abi.WindDriver * k)(*[abi.WindDriver(*DRIVERS[0])] * k)
    # 400 runs on two 128- and 100-cell grids need far more than 180 GB
    cfg = abi.EnsembleConfig(k, nr, n, drv, 1, 1, 0, 0.5)
    assert not lib.gcs_ensemble_create(C.byref(cfg))
    assert b"device memory" in lib.gcs_last_error()
    bad = (abi.WindDriver * 1)(abi.WindDriver(-1.0, -400.0, 1e5, -5.0))
    one = (C.c_size_t * 1)(20)
    ten = (C.c_size_t * 1)(10)
    cfg = abi.EnsembleConfig(1, one, ten, bad, 1, 0, 0, 0.5)
    assert not lib.gcs_ensemble_create(C.byref(cfg))
    assert b"driver" in lib.gcs_last_error()
