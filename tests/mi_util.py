"""Shared helpers of the ionosphere-solve tests."""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
if REPO not in sys.path:
    sys.path.insert(0, REPO)

from gamera_cube_b200 import abi, cases  # noqa: E402

GOLDEN = os.path.join(HERE, "golden", "reference_mi.npz")
CASE_NAMES = ["small_north", "small_south_low", "shell_192x22"]

# Two solves that each reach relative residual 1e-8 differ by about 1.2e-9
# of max|potential| on these grids (measured against 1e-13 solves); the
# potential comparisons allow 5e-8.
POTENTIAL_RTOL = 5e-8

P = C.POINTER(C.c_double)


def ptr(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(P)


def golden():
    return np.load(GOLDEN)


def golden_case(g, name, tensor=False):
    npl, nt, deg, hemi, low = g[name + "/config"]
    npl, nt, hemi = int(npl), int(nt), int(hemi)
    if tensor:
        cfg = cases.mi_config(npl, nt, deg, hemi, max_iterations=4000)
    else:
        cfg = cases.mi_config(npl, nt, deg, hemi, low_latitude_potential_v=low,
                              max_iterations=4000)
    return cfg, {k: np.ascontiguousarray(g[name + "/" + k])
                 for k in ("fac", "pedersen", "hall", "guess", "probe")}


def stats_tuple(st):
    return (st.iterations, st.initial_residual, st.final_residual, st.converged)


def true_residual(apply_fn, cfg, fac, pot):
    """Residual norm and target of nonorthogonal_mi.c:415-431 and :506-509,
    evaluated with a full-layout operator apply_fn(cfg, p) -> A p."""
    npl, nt = cfg.longitude_count, cfg.colatitude_count
    ap = apply_fn(cfg, pot)
    dth = cfg.maximum_colatitude / (nt - 1)
    theta = dth * np.arange(1, nt - 1)
    c = np.cos(theta)
    inc = cfg.hemisphere * 2.0 * c / np.sqrt(1.0 + 3.0 * c * c)
    u = -(cfg.ionosphere_radius_m ** 2) * fac[1:nt - 1] * inc[:, None]
    res = u - ap[1:nt - 1]
    norm2 = npl * ap[0, 0] ** 2 + np.sum(res * res)
    rhs2 = npl * cfg.low_latitude_potential_v ** 2 + np.sum(u * u)
    target = max(cfg.absolute_tolerance,
                 cfg.relative_tolerance * max(np.sqrt(rhs2), 1.0))
    return float(np.sqrt(norm2)), float(target)
