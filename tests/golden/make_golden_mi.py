"""Generate tests/golden/reference_mi.npz from the unmodified reference.

Run in a container that has the reference sources:

    make -C oracle ref && python tests/golden/make_golden_mi.py

Each case stores its inputs (field-aligned current, Pedersen and Hall
conductance, an initial potential) and the outputs of the reference's
ionosphere solvers and operators (nonorthogonal_mi.c): the
constant-Pedersen solve with its stats, the conductance-tensor solve with
its stats, and both operators applied to a fixed seeded potential.  The
inputs come from gamera_cube_b200.cases (seeded Region-1/2 currents over an
auroral-oval conductance); every output comes from the reference library
through its public API.  The grids are the polar grid of the reference's own
MI test (192 x 22, cubedsphere/tests/test_cubedsphere_mi_shell.c:82-87) and
two small ones.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import refbind  # noqa: E402
from gamera_cube_b200 import abi, cases  # noqa: E402

# (name, longitudes, colatitudes, max colatitude deg, hemisphere, low-latitude V)
CASES = [("small_north", 16, 9, 45.0, 1, 0.0),
         ("small_south_low", 24, 12, 40.0, -1, 1500.0),
         ("shell_192x22", 192, 22, 45.0, 1, 0.0)]
SEED = 11

P = C.POINTER(C.c_double)


def ptr(a):
    return a.ctypes.data_as(P)


def stats_array(st):
    return np.array([st.iterations, st.initial_residual, st.final_residual,
                     st.converged], dtype=np.float64)


def main():
    lib = refbind.ref()
    out = {}
    for name, npl, nt, deg, hemi, low in CASES:
        case = cases.mi_case(npl, nt, seed=SEED, hemisphere=hemi,
                             max_colatitude_deg=deg, low_latitude_potential_v=low,
                             max_iterations=4000)
        rng = np.random.default_rng(SEED + npl)
        guess = rng.uniform(-100.0, 100.0, size=(nt, npl))
        probe = rng.standard_normal((nt, npl)) * 1e3
        key = name + "/"
        out[key + "fac"] = case.fac
        out[key + "pedersen"] = case.pedersen
        out[key + "hall"] = case.hall
        out[key + "guess"] = guess
        out[key + "probe"] = probe
        out[key + "config"] = np.array([npl, nt, deg, hemi, low], dtype=np.float64)
        pot = guess.copy()
        st = abi.MiSolverStats()
        rc = lib.gamera_mi_solve_constant_pedersen(C.byref(case.config), ptr(case.fac),
                                                   ptr(pot), C.byref(st))
        out[key + "constant/rc"] = np.array([rc])
        out[key + "constant/potential"] = pot
        out[key + "constant/stats"] = stats_array(st)
        res = np.zeros_like(probe)
        lib.gamera_mi_apply_constant_pedersen(C.byref(case.config), ptr(probe), ptr(res))
        out[key + "constant/apply"] = res
        if low == 0.0:
            tcfg = cases.mi_config(npl, nt, deg, hemi, max_iterations=4000)
            pot = guess.copy()
            st = abi.MiSolverStats()
            rc = lib.gamera_mi_solve_conductance_tensor(
                C.byref(tcfg), ptr(case.fac), ptr(case.pedersen), ptr(case.hall),
                ptr(pot), C.byref(st))
            out[key + "tensor/rc"] = np.array([rc])
            out[key + "tensor/potential"] = pot
            out[key + "tensor/stats"] = stats_array(st)
            res = np.zeros_like(probe)
            lib.gamera_mi_apply_conductance_tensor(C.byref(tcfg), ptr(case.pedersen),
                                                   ptr(case.hall), ptr(probe), ptr(res))
            out[key + "tensor/apply"] = res
        print(name, "constant it", int(out[key + "constant/stats"][0]))
    coupling(lib, out)
    np.savez_compressed(os.path.join(HERE, "reference_mi.npz"), **out)


def coupling(lib, out):
    """The reference coupling (cubedsphere_mi_dipole.c) on the wind fixture
    case with the analytic residual field of the reference MI shell test:
    one update at t = 0 and every output the coupling tests compare."""
    sys.path.insert(0, os.path.dirname(HERE))
    import mi_util
    kind, nr, n, seed = mi_util.COUPLING_CASE
    case = refbind.Case(refbind.FX_WIND, nr, n, seed)
    assert lib.fx_set_mi_field(case.handle) == 0
    cfg = mi_util.coupling_config()
    startup = mi_util.coupling_startup()
    mi = lib.fx_mi_create(case.handle, C.byref(startup), C.byref(cfg))
    assert mi
    assert lib.gamera_cs_mi_dipole_update_due(mi, 0.0) == 1
    assert lib.gamera_cs_mi_dipole_maybe_update(mi, 0.0) == 1
    assert lib.gamera_cs_mi_dipole_update_due(mi, 0.0) == 0
    res = mi_util.coupling_outputs(lib, mi, case, cfg)
    for k, v in res.items():
        out["coupling/" + k] = v
    print("coupling iterations", res["stats"][:2], "fac range", res["stats"][4:6])
    lib.gamera_cs_mi_dipole_destroy(mi)


if __name__ == "__main__":
    main()
