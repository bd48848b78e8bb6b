"""The device Jacobi-PCG of the variable-Pedersen, Hall-free operator
(gcs_mi_solve_pedersen_pcg, gcs_mi_plan_create_pedersen) against its CPU
restatement (oracle gcso_mi_solve_pedersen_pcg: same algorithm, sequential
sums) and against the reference's own solver for that operator
(gamera_mi_solve_conductance_tensor with Hall = 0).  The device sums dot
products in a fixed parallel order, so its iterates differ from the
restatement's at rounding level: iterations within 3 %, potentials within
5e-8 of their maximum; against the reference (another method) within the
solves' accuracy, 1e-7."""
import ctypes as C

import numpy as np
import pytest

from gamera_cube_b200 import abi, cases
from oracle import oracle_cases, refbind
from tests.test_mi_pcg_oracle import pedersen_case

pytestmark = pytest.mark.gpu
P = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def lib():
    import gamera_cube_b200
    return gamera_cube_b200.lib


@pytest.mark.parametrize("npl,nt,hemisphere", [(24, 12, cases.NORTH),
                                                (64, 33, cases.SOUTH),
                                                (361, 181, cases.NORTH)])
def test_device_pcg_matches_restatement(lib, npl, nt, hemisphere):
    c, ped = pedersen_case(npl, nt, 3, hemisphere)
    dev, sd = c.potential.copy(), abi.MiSolverStats()
    assert lib.gcs_mi_solve_pedersen_pcg(C.byref(c.config), c.fac.ctypes.data_as(P),
                                         ped.ctypes.data_as(P), dev.ctypes.data_as(P),
                                         C.byref(sd)) == 0, lib.gcs_last_error()
    cpu, sc = c.potential.copy(), abi.MiSolverStats()
    assert oracle_cases.lib().gcso_mi_solve_pedersen_pcg(
        C.byref(c.config), c.fac.ctypes.data_as(P), ped.ctypes.data_as(P),
        cpu.ctypes.data_as(P), C.byref(sc)) == 0
    assert sd.converged and sc.converged
    assert abs(sd.iterations - sc.iterations) <= max(2, 0.03 * sc.iterations), \
        (sd.iterations, sc.iterations)
    assert np.abs(dev - cpu).max() <= 5e-8 * np.abs(cpu).max()
    if npl == 361 and refbind.ref_available():
        ref, st = c.potential.copy(), abi.MiSolverStats()
        hall = np.zeros_like(ped)
        assert refbind.ref().gamera_mi_solve_conductance_tensor(
            C.byref(c.config), c.fac.ctypes.data_as(P), ped.ctypes.data_as(P),
            hall.ctypes.data_as(P), ref.ctypes.data_as(P), C.byref(st)) == 0
        assert np.abs(dev - ref).max() <= 1e-7 * np.abs(ref).max()


def test_plan_solves_both_hemispheres(lib):
    """A two-system plan solves both hemispheres in one launch, each as the
    one-system call does."""
    import torch
    cs = [pedersen_case(361, 181, 5, h) for h in (cases.NORTH, cases.SOUTH)]
    cfgs = (abi.MiSolverConfig * 2)(*[c.config for c, _ in cs])
    ped = np.ascontiguousarray(np.concatenate([p.ravel() for _, p in cs]))
    plan = C.c_void_p()
    assert lib.gcs_mi_plan_create_pedersen(cfgs, ped.ctypes.data_as(P), 2,
                                           C.byref(plan)) == 0, lib.gcs_last_error()
    try:
        fac = torch.from_numpy(np.concatenate([c.fac.ravel() for c, _ in cs])).cuda()
        pot = torch.zeros_like(fac)
        assert lib.gcs_mi_solve_constant_pedersen_async(
            plan, C.c_void_p(fac.data_ptr()), C.c_void_p(pot.data_ptr()), None) == 0
        stats, status = (abi.MiSolverStats * 2)(), (C.c_int * 2)()
        assert lib.gcs_mi_plan_results(plan, stats, status) == 0
        assert status[0] == 0 and status[1] == 0
        got = pot.cpu().numpy().reshape(2, 181, 361)
        for h, (c, p) in enumerate(cs):
            one, st = np.zeros((181, 361)), abi.MiSolverStats()
            assert lib.gcs_mi_solve_pedersen_pcg(C.byref(c.config), c.fac.ctypes.data_as(P),
                                                 p.ctypes.data_as(P), one.ctypes.data_as(P),
                                                 C.byref(st)) == 0
            assert st.iterations == stats[h].iterations
            np.testing.assert_array_equal(got[h], one)
    finally:
        lib.gcs_mi_plan_destroy(plan)


@pytest.mark.parametrize("iterations", [1, 5, 20])
def test_first_iterations_follow_the_restatement(lib, iterations):
    """The variable-coefficient recurrence stopped after a few iterations
    equals the restatement's iterate to 1e-11 of its maximum."""
    c, ped = pedersen_case(361, 181, 3, cases.NORTH)
    cfg = abi.MiSolverConfig.from_buffer_copy(c.config)
    cfg.maximum_iterations = iterations
    dev, sd = c.potential.copy(), abi.MiSolverStats()
    lib.gcs_mi_solve_pedersen_pcg(C.byref(cfg), c.fac.ctypes.data_as(P),
                                  ped.ctypes.data_as(P), dev.ctypes.data_as(P), C.byref(sd))
    cpu, sc = c.potential.copy(), abi.MiSolverStats()
    oracle_cases.lib().gcso_mi_solve_pedersen_pcg(
        C.byref(cfg), c.fac.ctypes.data_as(P), ped.ctypes.data_as(P),
        cpu.ctypes.data_as(P), C.byref(sc))
    assert sd.iterations == sc.iterations == iterations
    assert np.abs(dev - cpu).max() <= 1e-11 * np.abs(cpu).max()
