"""Host-side checks of the ensemble support (no device calls): the seeded
draw of sizes and drivers, the device-memory estimate, tile limits, and the
oracle's driven wind case (the checker of the device builder's drivers)."""
import ctypes as C

import numpy as np
import pytest

import gamera_cube_b200
from gamera_cube_b200 import abi
from oracle import oracle_cases

lib = gamera_cube_b200.lib


def draw(seed, count):
    n = (C.c_size_t * count)()
    drv = (abi.WindDriver * count)()
    assert lib.gcs_ensemble_draw(seed, count, n, drv) == 0
    return list(n), [(d.density_cm3, d.velocity_x_kms, d.temperature_k, d.bz_nt) for d in drv]


def test_draw_is_seeded_and_in_range():
    n1, d1 = draw(2024, 64)
    n2, d2 = draw(2024, 64)
    n3, d3 = draw(2025, 64)
    assert n1 == n2 and d1 == d2
    assert d1 != d3
    assert set(n1) <= {48, 64, 96, 128} and len(set(n1)) == 4
    d = np.array(d1)
    assert np.all((d[:, 0] >= 1) & (d[:, 0] < 20))
    assert np.all((d[:, 1] >= -800) & (d[:, 1] < -300))
    assert np.all((d[:, 2] >= 5e4) & (d[:, 2] < 2e5))
    assert np.all((d[:, 3] >= -10) & (d[:, 3] < 5))
    # a prefix of a longer draw is the shorter draw
    n4, d4 = draw(2024, 16)
    assert n4 == n1[:16] and d4 == d1[:16]


def test_draw_rejects_bad_arguments():
    assert lib.gcs_ensemble_draw(1, 0, None, None) == -1
    assert lib.gcs_ensemble_draw(1, 4, None, None) == -1


def estimate(nr, n, bulk=1):
    k = len(n)
    a = (C.c_size_t * k)(*nr)
    b = (C.c_size_t * k)(*n)
    return lib.gcs_ensemble_estimate_bytes(k, a, b, bulk)


def test_memory_estimate_shares_grids():
    one = estimate([256], [128])
    two = estimate([256, 256], [128, 128])
    member = two - one
    # a run on a shared grid holds 22 doubles per node
    assert member == pytest.approx(6 * 265 * 137 * 137 * 22 * 8)
    assert member < 0.15 * one
    # sixteen runs of the largest size fit in one B200's HBM (180 GB)
    assert estimate([256] * 16, [128] * 16) < 170e9
    assert estimate([256, 128], [128, 64]) > one


@pytest.mark.parametrize("seed", [1, 2, 3, 2024])
def test_seeded_sixteen_run_ensembles_fit(seed):
    n, _ = draw(seed, 16)
    assert estimate([2 * x for x in n], n) < 170e9


def test_tile_limits():
    limits = [lib.gcs_tile_limit(f) for f in range(7)]
    assert limits == [256, 128, 256, 128, 256, 128, 256]
    assert lib.gcs_tile_limit(7) == -1
    assert lib.gcs_context_set_tile(None, 0, 128, 1) == -1


def test_oracle_driven_case_matches_default_wind():
    """The driven oracle case with the reference driver's values is the
    plain wind case bit for bit; other drivers set n and V as asked."""
    a = oracle_cases.Case("wind", 12, 10, 7)
    b = oracle_cases.Case("wind", 12, 10, 7, driver=(5.0, -400.0, 1.0e5, -5.0))
    for f in range(6):
        A, B = a.arrays(f), b.arrays(f)
        for name in ("conserved", "cell_magnetic", "face_flux0", "face_flux1",
                     "face_flux2"):
            np.testing.assert_array_equal(A[name], B[name])
    c = oracle_cases.Case("wind", 12, 10, 7, driver=(12.0, -650.0, 1.5e5, 3.0))
    u = c.arrays(0)["conserved"]
    assert abs(u[..., 0].mean() / 12.0 - 1.0) < 1e-3
    np.testing.assert_allclose(u[..., 1] / u[..., 0], -6.5, rtol=1e-14)
    # the northward IMF changes the face flux
    assert not np.array_equal(c.arrays(0)["face_flux0"], a.arrays(0)["face_flux0"])
