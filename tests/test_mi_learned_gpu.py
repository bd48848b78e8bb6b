"""The flexible-GMRES conductance-tensor solves of gcs_learn.cu against the
oracle: the two-level preconditioned solve (ring-mean coarse correction and
damped Jacobi, left), and the solve with the learned network as the flexible
right preconditioner, briefly trained on the GPU.  Both must reach the
reference's residual target (or, for the learned one, fall back to the
reference algorithm) with the reference's accuracy: distance to the oracle's
1e-12 solve at most twice the oracle's own 1e-8 solve's, plus 5e-8 of max.
The learned test records the iteration counts with and without the network
(it asserts no gain: on these grids the trained network does not reduce the
iteration count of the two-level method)."""
import ctypes as C

import numpy as np
import pytest

from mi_util import POTENTIAL_RTOL, ptr
from oracle import oracle_cases

pytestmark = pytest.mark.gpu


def glib():
    import gamera_cube_b200
    return gamera_cube_b200.lib


def oracle(case, rel_tol):
    from gamera_cube_b200 import abi, cases
    c = cases.mi_case(case.config.longitude_count, case.config.colatitude_count,
                      seed=CASE_SEED, max_iterations=200000, rel_tol=rel_tol)
    pot = case.potential.copy()
    st = abi.MiSolverStats()
    rc = oracle_cases.lib().gcso_mi_solve_conductance_tensor(
        C.byref(c.config), ptr(case.fac), ptr(case.pedersen), ptr(case.hall), ptr(pot),
        C.byref(st))
    assert rc == 0
    return pot, st


CASE_SEED = 31


def check_accuracy(case, pot):
    truth, _ = oracle(case, 1e-12)
    ref, _ = oracle(case, 1e-8)
    scale = np.abs(truth).max()
    assert np.abs(pot - truth).max() <= 2.0 * np.abs(ref - truth).max() + POTENTIAL_RTOL * scale
    assert np.all(pot[0] == pot[0, 0]) and np.all(pot[-1] == 0.0)


@pytest.mark.parametrize("npl,nt", [(24, 12), (64, 40), (361, 181)])
def test_two_level_solve(npl, nt):
    from gamera_cube_b200 import cases, learn
    case = cases.mi_case(npl, nt, seed=CASE_SEED, max_iterations=5000)
    rc, pot, st, fb, _ = learn.solve(glib(), None, case, method=2)
    assert rc == 0, glib().gcs_last_error().decode()
    assert fb == 0 and st.converged == 1
    check_accuracy(case, pot)


def test_pieces_against_restatement():
    """The device's scaled operator and two-level step equal the numpy ones."""
    import scipy.sparse.linalg as spl
    from gamera_cube_b200 import cases, learn
    case = cases.mi_case(40, 22, seed=CASE_SEED)
    A, E = learn.scaled_operator(case.config, case.pedersen, case.hall)
    T = spl.splu((E.T @ A @ E).tocsc())
    v = np.random.default_rng(4).normal(size=A.shape[0])
    for what, method, ref in [(1, 1, A @ v), (0, 1, v / A.diagonal()),
                              (0, 2, learn.two_level(A, E, T, v))]:
        y = np.zeros_like(v)
        assert glib().gcs_mi_learned_apply(None, method, what, C.byref(case.config),
                                           ptr(case.pedersen), ptr(case.hall), ptr(v),
                                           ptr(y)) == 0
        assert np.abs(y - ref).max() <= 1e-12 * np.abs(ref).max()


def test_learned_solve_and_gain(record_property):
    from gamera_cube_b200 import cases, learn
    L = glib()
    case = cases.mi_case(64, 40, seed=CASE_SEED, max_iterations=3000)
    net = learn.create_net(L, case.config, batch=8, seed=3)
    try:
        pool = learn.Pool(L, npl=64, nt=40, random_fields=64, solved=4, conductances=4)
        losses = learn.train(L, net, pool, steps=300, batch=8, lr=1e-3)
        assert np.isfinite(losses).all() and np.mean(losses[-20:]) < np.mean(losses[:20])
        rc, pot, st, fb, sec = learn.solve(L, net, case, method=0)
        assert rc == 0, L.gcs_last_error().decode()
        check_accuracy(case, pot)
        rc2, _, st2, fb2, sec2 = learn.solve(L, None, case, method=2)
        assert rc2 == 0 and fb2 == 0
        record_property("iterations_with_network", st.iterations)
        record_property("iterations_without_network", st2.iterations)
        record_property("fallback_with_network", fb)
    finally:
        L.gcs_mi_net_destroy(net)
