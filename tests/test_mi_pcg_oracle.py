"""The restated Jacobi-PCG of the variable-Pedersen, Hall-free operator
(oracle gcso_mi_solve_pedersen_pcg, the CPU form of the device solve
gcs_mi_solve_pedersen_pcg) against the reference's own solver for that
operator: gamera_mi_solve_conductance_tensor with Hall = 0
(SSOR-BiCGStab, nonorthogonal_mi.c:966-1151) from the compiled reference.
Different methods, one operator and one residual rule: both converge to
relative residual 1e-8 and their potentials agree to the solves' accuracy."""
import ctypes as C

import numpy as np
import pytest

from gamera_cube_b200 import abi, cases
from oracle import oracle_cases, refbind

P = C.POINTER(C.c_double)


def pedersen_case(npl, nt, seed, hemisphere=cases.NORTH):
    c = cases.mi_case(npl, nt, seed=seed, hemisphere=hemisphere)
    ped = c.pedersen.copy()
    ped[0, :] = ped[0, :].mean()      # one conductance at the pole point
    return c, ped


@pytest.mark.parametrize("npl,nt,hemisphere", [(24, 12, cases.NORTH),
                                                (64, 33, cases.SOUTH)])
def test_restated_pcg_matches_reference_tensor_solve(npl, nt, hemisphere):
    if not refbind.ref_available():
        pytest.skip("reference library not built")
    c, ped = pedersen_case(npl, nt, 3, hemisphere)
    hall = np.zeros_like(ped)
    pcg, st = c.potential.copy(), abi.MiSolverStats()
    assert oracle_cases.lib().gcso_mi_solve_pedersen_pcg(
        C.byref(c.config), c.fac.ctypes.data_as(P), ped.ctypes.data_as(P),
        pcg.ctypes.data_as(P), C.byref(st)) == 0
    ref, st2 = c.potential.copy(), abi.MiSolverStats()
    assert refbind.ref().gamera_mi_solve_conductance_tensor(
        C.byref(c.config), c.fac.ctypes.data_as(P), ped.ctypes.data_as(P),
        hall.ctypes.data_as(P), ref.ctypes.data_as(P), C.byref(st2)) == 0
    assert st.converged and st2.converged
    assert st.final_residual <= st.initial_residual * 1e-6
    assert np.abs(pcg - ref).max() <= 1e-7 * np.abs(ref).max()
