"""CPU restatement of the reference's analysis frame
(cubedsphere/cubedsphere_analysis_hdf5.c:316-331 with
nonorthogonal_state.c:60-93): per face float32 [8][NI][NJ][NK] of rho, p,
vx, vy, vz from the conserved state (floors 1e-12) and the total B
(residual + cell B0) over the active cells.  Test infrastructure only.
Pinned bit for bit to frames recorded through the reference library's own
gamera_no_conserved_to_primitive (tests/golden/make_analysis_golden.py,
tests/test_analysis_oracle.py)."""
import numpy as np


def primitives(u, gamma, rho_floor=1e-12, p_floor=1e-12):
    """nonorthogonal_state.c:60-93 on an array [..., 5], same operation order."""
    raw = u[..., 0]
    vx = u[..., 1] / raw
    vy = u[..., 2] / raw
    vz = u[..., 3] / raw
    v2 = vx * vx
    v2 = v2 + vy * vy
    v2 = v2 + vz * vz
    kinetic = 0.5 * raw * v2
    rho = np.maximum(raw, rho_floor)
    p = np.maximum((gamma - 1.0) * (u[..., 4] - kinetic), p_floor)
    return rho, p, vx, vy, vz


def frame(conserved, cell_b, b0, ghost, gamma):
    """One face's frame from its reference-layout arrays ([E0,E1,E2,5],
    [E0,E1,E2,3], B0 [E0,E1,E2,3] or None)."""
    g = ghost
    act = (slice(g, -g), slice(g, -g), slice(g, -g))
    u = conserved[act]
    rho, p, vx, vy, vz = primitives(u, gamma)
    b = cell_b[act] + (b0[act] if b0 is not None else 0.0)
    fields = [rho, p, vx, vy, vz, b[..., 0], b[..., 1], b[..., 2]]
    return np.stack([f.astype(np.float32) for f in fields])
