"""Shared pieces of the pressure-control parity checks: parameters that make
both branches of gamera_no_apply_pressure_control (nonorthogonal_step.c:74-171)
fire on a part of a case's cells, and a per-face driver of a CPU
implementation (the reference's or the oracle's) that sums the counts and
takes the maxima over the faces, as the device call does."""
import ctypes as C

import numpy as np

GAMMA = 5.0 / 3.0
RHO_FLOOR, P_FLOOR = 1e-6, 1e-8
DT = 0.05


def parameters(arrays, ghost, active):
    """(light speed, low-density threshold, low-density sound speed): the
    threshold at the 30th percentile of the active densities, 1.5 c at the
    60th percentile of the sound speeds."""
    g = ghost
    rho, cs = [], []
    for a in arrays:
        u = a["conserved"][g:g + active[0], g:g + active[1], g:g + active[2]]
        r = u[..., 0]
        v2 = sum((u[..., 1 + d] / r) ** 2 for d in range(3))
        p = np.maximum((GAMMA - 1.0) * (u[..., 4] - 0.5 * r * v2), P_FLOOR)
        rho.append(r.ravel())
        cs.append(np.sqrt(GAMMA * p / np.maximum(r, RHO_FLOOR)).ravel())
    rho, cs = np.concatenate(rho), np.concatenate(cs)
    return (float(np.quantile(cs, 0.6)) / 1.5, float(np.quantile(rho, 0.3)),
            0.5 * float(np.quantile(cs, 0.1)))


def apply_faces(fn, storage, grid, ghost, active, dt, light, threshold, low_sound):
    """Call fn (the reference's signature) on each face; (status, low, hot,
    max sound, max pressure) with status -1 when any face failed."""
    lo = (C.c_size_t * 3)(ghost, ghost, ghost)
    hi = (C.c_size_t * 3)(*[ghost + a for a in active])
    status, low, hot, ms, mp = 0, 0, 0, 0.0, 0.0
    for f in range(6):
        nl, nh = C.c_size_t(), C.c_size_t()
        s, p = C.c_double(), C.c_double()
        rc = fn(C.byref(storage[f]), C.byref(grid[f]), lo, hi, dt, GAMMA, RHO_FLOOR, P_FLOOR,
                light, threshold, low_sound, C.byref(nl), C.byref(nh), C.byref(s),
                C.byref(p))
        if rc != 0:
            status = -1
        low += nl.value
        hot += nh.value
        ms, mp = max(ms, s.value), max(mp, p.value)
    return status, low, hot, ms, mp
