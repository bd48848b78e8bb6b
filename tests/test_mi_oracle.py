"""The CPU restatement of the ionosphere solvers against the reference.

The restatement (oracle/gcs_oracle_mi.inc) must reproduce the reference
solvers and operators (nonorthogonal_mi.c) bit for bit: golden vectors
recorded from the reference (tests/golden/make_golden_mi.py), and, where the
reference library is built here, direct comparisons on the 181 x 361
production polar grid.
"""
import ctypes as C

import numpy as np
import pytest

from mi_util import CASE_NAMES, golden, golden_case, ptr, stats_tuple, true_residual
from oracle import oracle_cases, refbind
from gamera_cube_b200 import abi, cases


def bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


def olib():
    return oracle_cases.lib()


def oracle_apply(cfg, p):
    out = np.zeros_like(p)
    assert olib().gcso_mi_apply_constant_pedersen(C.byref(cfg), ptr(p), ptr(out)) == 0
    return out


@pytest.mark.parametrize("name", CASE_NAMES)
def test_constant_pedersen_matches_golden(name):
    g = golden()
    cfg, d = golden_case(g, name)
    pot = d["guess"].copy()
    st = abi.MiSolverStats()
    rc = olib().gcso_mi_solve_constant_pedersen(C.byref(cfg), ptr(d["fac"]), ptr(pot),
                                                C.byref(st))
    assert rc == int(g[name + "/constant/rc"][0])
    assert np.array_equal(bits(pot), bits(g[name + "/constant/potential"]))
    assert np.array_equal(np.array(stats_tuple(st), dtype=np.float64),
                          g[name + "/constant/stats"])
    res = np.zeros_like(d["probe"])
    olib().gcso_mi_apply_constant_pedersen(C.byref(cfg), ptr(d["probe"]), ptr(res))
    assert np.array_equal(bits(res), bits(g[name + "/constant/apply"]))
    # the reference's own convergence claim holds for its potential
    norm, target = true_residual(oracle_apply, cfg, d["fac"], pot)
    assert norm <= target * (1 + 1e-9)


@pytest.mark.parametrize("name", [n for n in CASE_NAMES if n != "small_south_low"])
def test_conductance_tensor_matches_golden(name):
    g = golden()
    cfg, d = golden_case(g, name, tensor=True)
    pot = d["guess"].copy()
    st = abi.MiSolverStats()
    rc = olib().gcso_mi_solve_conductance_tensor(
        C.byref(cfg), ptr(d["fac"]), ptr(d["pedersen"]), ptr(d["hall"]), ptr(pot),
        C.byref(st))
    assert rc == int(g[name + "/tensor/rc"][0])
    assert np.array_equal(bits(pot), bits(g[name + "/tensor/potential"]))
    assert np.array_equal(np.array(stats_tuple(st), dtype=np.float64),
                          g[name + "/tensor/stats"])
    res = np.zeros_like(d["probe"])
    olib().gcso_mi_apply_conductance_tensor(C.byref(cfg), ptr(d["pedersen"]),
                                            ptr(d["hall"]), ptr(d["probe"]), ptr(res))
    assert np.array_equal(bits(res), bits(g[name + "/tensor/apply"]))


def test_invalid_arguments_rejected():
    L = olib()
    case = cases.mi_case(16, 9, seed=2)
    pot = case.potential.copy()
    st = abi.MiSolverStats()
    bad = cases.mi_config(16, 9, hall_siemens=1.0)
    assert L.gcso_mi_solve_constant_pedersen(C.byref(bad), ptr(case.fac), ptr(pot),
                                             C.byref(st)) == -1
    fac = case.fac.copy()
    fac[3, 5] = np.nan
    before = pot.copy()
    assert L.gcso_mi_solve_constant_pedersen(C.byref(case.config), ptr(fac), ptr(pot),
                                             C.byref(st)) == -1
    assert np.array_equal(pot, before)
    tcfg = cases.mi_config(16, 9, low_latitude_potential_v=10.0)
    assert L.gcso_mi_solve_conductance_tensor(
        C.byref(tcfg), ptr(case.fac), ptr(case.pedersen), ptr(case.hall), ptr(pot),
        C.byref(st)) == -1
    ped = case.pedersen.copy()
    ped[0, 0] = 0.0
    tcfg = cases.mi_config(16, 9)
    assert L.gcso_mi_solve_conductance_tensor(
        C.byref(tcfg), ptr(case.fac), ptr(ped), ptr(case.hall), ptr(pot),
        C.byref(st)) == -1


@pytest.mark.skipif(not refbind.ref_available(), reason="reference library not built")
def test_production_grid_bitwise_against_reference():
    R, L = refbind.ref(), olib()
    case = cases.mi_case(361, 181, seed=5, hemisphere=cases.SOUTH)
    out = []
    for lib, pre in ((R, "gamera_mi_"), (L, "gcso_mi_")):
        pot = case.potential.copy()
        st = abi.MiSolverStats()
        rc = getattr(lib, pre + "solve_constant_pedersen")(
            C.byref(case.config), ptr(case.fac), ptr(pot), C.byref(st))
        out.append((rc, pot, stats_tuple(st)))
    assert out[0][0] == out[1][0] == 0
    assert out[0][2] == out[1][2]
    assert np.array_equal(bits(out[0][1]), bits(out[1][1]))
