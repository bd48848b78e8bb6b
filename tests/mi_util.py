"""Shared helpers of the ionosphere-solve and coupling tests."""
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


# ------------------------------------------------------------- coupling
COUPLING_CASE = ("wind", 12, 10, 7)     # kind, radial, angular, seed


def coupling_config(np_=192, nt=22, shell=1, max_iterations=4000):
    return cases.mi_dipole_config(np_, nt, shell, max_iterations)


def coupling_startup():
    return cases.earth_startup()


def cell_centroids(grid_face):
    n = 1
    for a in range(3):
        n *= grid_face.cell_extent[a]
    cells = np.ctypeslib.as_array(grid_face.cell, shape=(n,))
    return np.ascontiguousarray(cells["centroid"]["value"], dtype=np.float64)


def set_mi_field(case):
    """Analytic residual B of the reference MI shell test
    (cubedsphere/tests/test_cubedsphere_mi_shell.c:54-66) on every active
    cell of both time levels, evaluated in the same operation order."""
    g = case.ghost
    act = [case.active[a] for a in range(3)]
    for f in range(6):
        e = [case.grid[f].cell_extent[a] for a in range(3)]
        cen = cell_centroids(case.grid[f]).reshape(e[0], e[1], e[2], 3)
        arr = case.arrays(f)
        sl = (slice(g, g + act[0]), slice(g, g + act[1]), slice(g, g + act[2]))
        p = cen[sl]
        x, y, z = p[..., 0], p[..., 1], p[..., 2]
        r2 = x * x + y * y + z * z
        b = np.stack([0.03 * y / r2, -0.02 * x / r2, 0.01 * x * z / r2], axis=-1)
        for name in ("cell_magnetic", "old_cell_magnetic"):
            arr[name].reshape(e[0], e[1], e[2], 3)[sl] = b


def probe_points(seed=3, count=40):
    rng = np.random.default_rng(seed)
    d = rng.standard_normal((count, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    return d * rng.uniform(1.2, 3.0, size=(count, 1))


def coupling_outputs(lib, mi, case, cfg):
    """Everything the coupling tests compare, from library `lib` (this
    library or the reference build) after an update of coupling `mi` on
    `case`: polar FAC and potential, shell J_parallel, solver stats,
    potential lookups and ghost velocities at seeded probe points, and the
    wall EMF that apply_inner_emf writes on face 0."""
    P = C.POINTER(C.c_double)
    out = {}
    per = cfg.azimuth_points * cfg.colatitude_points
    pot = np.zeros(2 * per)
    ep, nx = C.c_double(), C.c_double()
    assert lib.gamera_cs_mi_dipole_export_potential(mi, pot.ctypes.data_as(P), 2 * per,
                                                    C.byref(ep), C.byref(nx)) == 0
    out["potential"] = pot
    out["times"] = np.array([ep.value, nx.value])
    view = abi.MiAnalysisView()
    assert lib.gamera_cs_mi_dipole_analysis_view(mi, C.byref(view)) == 0
    out["fac"] = np.concatenate([np.ctypeslib.as_array(view.fac_parallel_a_m2[h],
                                                       shape=(per,)).copy()
                                 for h in range(2)])
    out["view"] = np.array([view.maximum_colatitude_rad, view.sample_radius_re])
    nsh = 6 * case.active[1] * case.active[2]
    j, la, ph = np.zeros(nsh), np.zeros(nsh), np.zeros(nsh)
    assert lib.gamera_cs_mi_dipole_export_shell_current(
        mi, j.ctypes.data_as(P), la.ctypes.data_as(P), ph.ctypes.data_as(P), nsh) == 0
    out["shell_j"], out["shell_mlat"], out["shell_phi"] = j, la, ph
    st = (abi.MiSolverStats * 2)()
    mm = [C.c_double() for _ in range(4)]
    assert lib.gamera_cs_mi_dipole_stats(mi, *[C.byref(v) for v in mm], st) == 0
    out["stats"] = np.array([st[0].iterations, st[1].iterations, st[0].final_residual,
                             st[1].final_residual] + [v.value for v in mm])
    pts = probe_points()
    look = np.zeros(len(pts))
    ghost = np.zeros((len(pts), 3))
    for q, p in enumerate(pts):
        v = abi.Vec3()
        for a in range(3):
            v.value[a] = p[a]
        val = C.c_double()
        assert lib.gamera_cs_mi_dipole_potential(mi, v, C.byref(val)) == 0
        look[q] = val.value
        src = abi.Vec3()
        src.value[0], src.value[1], src.value[2] = 0.3, -0.2, 0.1
        gv = abi.Vec3()
        assert lib.gamera_cs_mi_dipole_ghost_velocity(mi, v, src, C.byref(gv)) == 0
        ghost[q] = [gv.value[a] for a in range(3)]
    out["lookup"], out["ghost_velocity"] = look, ghost
    arr = case.arrays(0)
    for d in (1, 2):
        arr["edge_emf%d" % d][...] = 0.0
    assert lib.gamera_cs_mi_dipole_apply_inner_emf(mi, C.byref(case.storage[0]),
                                                   C.byref(case.grid[0]),
                                                   case.ghost) == 0
    out["wall_emf"] = np.concatenate([arr["edge_emf%d" % d].ravel().copy()
                                      for d in (1, 2)])
    return out
