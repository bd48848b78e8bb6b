"""CPU checks of the restatement oracle (no GPU).

* Against the golden vectors recorded from the unmodified reference
  (tests/golden/reference_steps.npz, made by tests/golden/make_golden.py):
  every sampled value bit-exact.
* Against the reference library itself when it is built here: whole arrays
  bit-exact.
* The reference test suite's own known answers, applied to the oracle:
  uniform-state preservation (test_cubedsphere_six_mhd.c:63-96), radial
  shock positivity/div B (test_cubedsphere_mhd_shock.c:178-219) and halo
  weight bounds (test_cubedsphere_halo_bounded.c:1-33).
"""
import os

import numpy as np
import pytest

from oracle import oracle_cases, refbind
from tests.parity_util import STATE_ARRAYS, divergence

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_steps.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def _check_golden(case, golden, prefix):
    from tests.golden.make_golden import ARRAYS, sample_indices
    for f in range(6):
        arr = case.arrays(f)
        for name in ARRAYS:
            flat = np.ascontiguousarray(arr[name]).reshape(-1)
            key = "%s/f%d/%s" % (prefix, f, name)
            np.testing.assert_array_equal(flat[sample_indices(flat.size)],
                                          golden[key + "/sample"], err_msg=key)
            sums = np.array([flat.sum(), np.abs(flat).sum()])
            np.testing.assert_allclose(sums, golden[key + "/sum"], rtol=1e-14,
                                       atol=0, err_msg=key)


@pytest.mark.parametrize("name,kind,nr,n,steps", [
    ("uniform", "uniform", 0, 0, 2),
    ("shock", "shock", 0, 0, 3),
    ("wind", "wind", 12, 10, 2),
])
def test_restatement_matches_golden(golden, name, kind, nr, n, steps):
    case = oracle_cases.Case(kind, nr, n, 7)
    _check_golden(case, golden, "%s/step0" % name)
    dts = golden["%s/dts" % name]
    for s in range(steps):
        ratio, dt = dts[s]
        if kind == "wind":
            # the driver time step must also reproduce the reference's
            local = case.local_timestep()
            prev = dts[s - 1][1] if s else 0.0
            mine = 0.5 * local if s == 0 else min(0.5 * local, 1.25 * prev)
            assert mine == dt
        assert case.step(ratio, dt) == 0
        _check_golden(case, golden, "%s/step%d" % (name, s + 1))


@pytest.mark.skipif(not refbind.ref_available(),
                    reason="reference library not built here")
@pytest.mark.parametrize("kind", ["uniform", "shock"])
def test_restatement_matches_reference_bitwise(kind):
    ref = refbind.Case(oracle_cases.KINDS[kind], 0, 0, 3)
    orc = oracle_cases.Case(kind, 0, 0, 3)
    for _ in range(2):
        assert ref.step(ref.ratio, ref.dt) == 0
        assert orc.step(orc.ratio, orc.dt) == 0
    for f in range(6):
        a, b = orc.arrays(f), ref.arrays(f)
        for name in STATE_ARRAYS + ["predicted_conserved",
                                    "predicted_cell_magnetic"]:
            np.testing.assert_array_equal(a[name], b[name], err_msg=name)


def test_uniform_state_preserved():
    case = oracle_cases.Case("uniform")
    expected = case.arrays(0)["conserved"][6, 6, 6].copy()
    for _ in range(3):
        assert case.step(0.5, 0.01) == 0
    g, act = case.ghost, case.active
    for f in range(6):
        u = case.arrays(f)["conserved"][g:g + act[0], g:g + act[1], g:g + act[2]]
        assert np.max(np.abs(u - expected)) <= 5e-6
        assert divergence(case, f) <= 1e-10


def test_shock_positive_and_divergence_free():
    case = oracle_cases.Case("shock")
    for _ in range(30):
        assert case.step(0.5, 0.001) == 0
    g, act = case.ghost, case.active
    rho_max = 0.0
    for f in range(6):
        u = case.arrays(f)["conserved"][g:g + act[0], g:g + act[1], g:g + act[2]]
        rho = u[..., 0]
        kin = 0.5 * np.sum(u[..., 1:4] ** 2, axis=-1) / rho
        p = (5.0 / 3.0 - 1.0) * (u[..., 4] - kin)
        assert rho.min() > 0 and p.min() > 0
        rho_max = max(rho_max, rho.max())
        assert divergence(case, f) <= 1e-9
    assert rho_max >= 0.9


FRAME = [[[1, 0, 0], [0, 1, 0], [0, 0, 1]], [[-1, 0, 0], [0, -1, 0], [0, 0, 1]],
         [[0, 1, 0], [-1, 0, 0], [0, 0, 1]], [[0, -1, 0], [1, 0, 0], [0, 0, 1]],
         [[0, 0, 1], [1, 0, 0], [0, 1, 0]], [[0, 0, -1], [1, 0, 0], [0, -1, 0]]]


def _donor_weights(x, n):
    """Stencil start and 8 weights of cubedsphere_halo.c:25-57."""
    import math
    start = min(max(math.floor(x) - 3, 0), n - 8)
    logical = x - start
    if logical < 0:
        base, frac = 0, logical
    elif logical >= 7:
        base, frac = 6, logical - 6
    else:
        base = math.floor(logical)
        frac = logical - base
    w = [0.0] * 8
    w[base] = 1.0 - frac
    w[base + 1] = frac
    return w


def test_halo_weights_bounded():
    """Known answer of test_cubedsphere_halo_bounded.c:9-33: for ghost points
    up to half a cell past the cube corners the tensor-product donor weights
    sum to one within 1e-14 and their absolute sum stays <= 4."""
    import math
    qp = 0.25 * math.acos(-1.0)
    points = [(1, 1, 1), (1, -1, 1), (-1, 1, 1), (-1, -1, -1),
              (1, 1.01, 0.99), (1, 0.3, -1.02), (0.1, 1, 0.2)]
    for n in (16, 24, 32, 64, 256):
        for pt in points:
            # gamera_cs_inverse (cubedsphere_mesh.c:77-103)
            sel, dom = -1, 0.0
            for f in range(6):
                p = sum(pt[d] * FRAME[f][0][d] for d in range(3))
                if p > dom:
                    sel, dom = f, p
            a = math.atan2(sum(pt[d] * FRAME[sel][1][d] for d in range(3)), dom)
            b = math.atan2(sum(pt[d] * FRAME[sel][2][d] for d in range(3)), dom)
            for magnetic in (0, 1):
                if magnetic:
                    x = (a + qp) * n / (2.0 * qp) - 0.5
                    y = (b + qp) * n / (2.0 * qp) - 0.5
                else:
                    x = (a + qp) / (2.0 * qp / n) - 0.5
                    y = (b + qp) / (2.0 * qp / n) - 0.5
                wx, wy = _donor_weights(x, n), _donor_weights(y, n)
                s = sum(p * q for p in wx for q in wy)
                norm = sum(abs(p * q) for p in wx for q in wy)
                assert abs(s - 1.0) <= 1e-14 and norm <= 4.0 + 1e-12
