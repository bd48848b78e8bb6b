"""The C-ABI library loads and exports every function its headers declare
(no device calls: runs without a GPU)."""
import ctypes as C
import os
import re

import gamera_cube_b200
from gamera_cube_b200 import abi

INCLUDE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                       "include")


def declared_functions():
    names = set()
    for fname in os.listdir(INCLUDE):
        if not fname.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, fname)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b([a-z_][a-z0-9_]*)\s*\(", text):
            name = m.group(1)
            if name.startswith(("gamera_cs_", "gamera_mi_", "gcs_")):
                names.add(name)
    return names


def test_library_exports_every_declared_function():
    lib = C.CDLL(gamera_cube_b200.LIBRARY_PATH)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layouts_match_reference_abi():
    # sizes of the reference structs on x86-64 (LP64)
    assert C.sizeof(abi.Vec3) == 24
    assert C.sizeof(abi.FaceGeometry) == 128
    assert C.sizeof(abi.CellGeometry) == 8 + 24 + 6 * 128 + 24
    assert C.sizeof(abi.EdgeGeometry) == 80
    assert C.sizeof(abi.SweepOptions) == 7 * 8 + 8
    assert C.sizeof(abi.EmfOptions) == 6 * 8 + 8
    assert C.sizeof(abi.MiSolverConfig) == 2 * 8 + 5 * 8 + 2 * 4 + 2 * 8


def test_halo_valid_state_predicate():
    lib = gamera_cube_b200.lib
    good = (C.c_double * 5)(1.0, 0.1, 0.2, 0.3, 1.0)
    bad_energy = (C.c_double * 5)(1.0, 1.0, 1.0, 1.0, 0.5)
    bad_rho = (C.c_double * 5)(0.0, 0.0, 0.0, 0.0, 1.0)
    nan = (C.c_double * 5)(float("nan"), 0.0, 0.0, 0.0, 1.0)
    assert lib.gamera_cs_halo_valid_state(good) == 1
    assert lib.gamera_cs_halo_valid_state(bad_energy) == 0
    assert lib.gamera_cs_halo_valid_state(bad_rho) == 0
    assert lib.gamera_cs_halo_valid_state(nan) == 0
