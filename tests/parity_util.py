"""Helpers shared by the parity tests: array comparison over the regions the
reference step defines."""
import numpy as np

from gamera_cube_b200 import abi

STATE_ARRAYS = ["conserved", "old_conserved", "cell_magnetic",
                "old_cell_magnetic"] + \
    ["face_flux%d" % d for d in range(3)] + \
    ["old_face_flux%d" % d for d in range(3)]


def compare_state(case_a, case_b, names=STATE_ARRAYS, region=None):
    """Normwise relative difference per array: max|a-b| / max|b| over the
    six faces.  Returns {name: (rel, max_abs)}."""
    out = {}
    for name in names:
        worst_abs, scale = 0.0, 0.0
        for f in range(abi.FACE_COUNT):
            a = case_a.arrays(f)[name]
            b = case_b.arrays(f)[name]
            if region is not None:
                a = a[region(name)]
                b = b[region(name)]
            worst_abs = max(worst_abs, float(np.max(np.abs(a - b))))
            scale = max(scale, float(np.max(np.abs(b))))
        out[name] = (worst_abs / scale if scale > 0 else worst_abs, worst_abs)
    return out


def divergence(case, face):
    """Max |net face flux| / volume over active cells (the div B check of
    test_cubedsphere_six_mhd.c:81-83)."""
    g = case.ghost
    act = case.active
    arr = case.arrays(face)
    f0, f1, f2 = arr["face_flux0"], arr["face_flux1"], arr["face_flux2"]
    s = (slice(g, g + act[0]), slice(g, g + act[1]), slice(g, g + act[2]))
    net = (f0[g + 1:g + act[0] + 1, s[1], s[2]] - f0[s]
           + f1[s[0], g + 1:g + act[1] + 1, s[2]] - f1[s]
           + f2[s[0], s[1], g + 1:g + act[2] + 1] - f2[s])
    grid = case.grid[face]
    ext = tuple(grid.cell_extent)
    vol = np.array([grid.cell[n].volume for n in range(ext[0] * ext[1] * ext[2])]
                   ).reshape(ext)[s]
    return float(np.max(np.abs(net) / vol))
