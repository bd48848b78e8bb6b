"""Golden analysis frames from the unmodified reference.

The analysis frame of cubedsphere/cubedsphere_analysis_hdf5.c:314-331 is,
per active cell, the reference's gamera_no_conserved_to_primitive
(nonorthogonal_state.c:60-93, floors 1e-12) followed by the total field
B + B0 and a cast of the eight values to float32.  The HDF5 writer itself
needs MPI and HDF5, which are absent here, so this script calls the
reference library's gamera_no_conserved_to_primitive (built by
`make -C oracle ref`) cell by cell on a case built and stepped by the
reference (the 12 x 10 x 10 wind case, seed 7, one driver step) and records
the float32 frames of the six faces:

    make -C oracle ref && python tests/golden/make_analysis_golden.py
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from gamera_cube_b200 import abi  # noqa: E402
from oracle import refbind  # noqa: E402

GAMMA = 5.0 / 3.0
NR, N, SEED = 12, 10, 7


class Primitive(C.Structure):
    """nonorthogonal_flux.h:21-25"""
    _fields_ = [("density", C.c_double), ("velocity", abi.Vec3),
                ("pressure", C.c_double)]


def main():
    lib = refbind.ref()
    fn = lib.gamera_no_conserved_to_primitive
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(C.c_double), C.c_double, C.c_double, C.c_double,
                   C.POINTER(Primitive)]
    case = refbind.Case(refbind.FX_WIND, NR, N, SEED)
    assert case.step(0.0, 0.5 * case.local_timestep()) == 0
    g = case.ghost
    frames = []
    for f in range(6):
        a = case.arrays(f)
        ext = a["conserved"].shape[:3]
        ncell = ext[0] * ext[1] * ext[2]
        b0 = np.ctypeslib.as_array(
            C.cast(case.background[f].cell_magnetic, C.POINTER(C.c_double)),
            shape=(3 * ncell,)).reshape(ext + (3,))
        u = np.ascontiguousarray(a["conserved"])
        out = np.zeros((8, NR, N, N), np.float32)
        p = Primitive()
        for i in range(NR):
            for j in range(N):
                for k in range(N):
                    cell = u[i + g, j + g, k + g]
                    assert fn(cell.ctypes.data_as(C.POINTER(C.c_double)), GAMMA, 1e-12,
                              1e-12, C.byref(p)) == 0
                    b = a["cell_magnetic"][i + g, j + g, k + g]
                    bb = b0[i + g, j + g, k + g]
                    vals = [p.density, p.pressure, p.velocity.value[0],
                            p.velocity.value[1], p.velocity.value[2],
                            b[0] + bb[0], b[1] + bb[1], b[2] + bb[2]]
                    out[:, i, j, k] = np.array(vals, np.float64).astype(np.float32)
        frames.append(out)
    path = os.path.join(HERE, "reference_analysis.npz")
    np.savez_compressed(path, frames=np.stack(frames))
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
