"""ctypes binding of the CPU restatement oracle (oracle/libgcs_oracle.so).

Test infrastructure: builds cases with the restatement's own set-up code and
advances them with its restated step.  The class mirrors refbind.Case so a
test can use either the restatement or the compiled reference as the oracle.
"""
import ctypes as C
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
if REPO not in sys.path:
    sys.path.insert(0, REPO)

from gamera_cube_b200 import abi  # noqa: E402
from oracle.refbind import RESTATEMENT_PATH  # noqa: E402

KINDS = {"uniform": 0, "shock": 1, "wind": 2, "pulse": 3}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(RESTATEMENT_PATH):
            subprocess.run(["make", "-C", HERE, "restatement"], check=True)
        L = C.CDLL(RESTATEMENT_PATH, mode=os.RTLD_LOCAL)
        P = C.POINTER
        for name, res, args in [
                ("gcso_case_create", C.c_void_p, [C.c_int, C.c_size_t, C.c_size_t,
                                                  C.c_ulonglong]),
                ("gcso_case_create_driven", C.c_void_p,
                 [C.c_size_t, C.c_size_t, C.c_ulonglong, C.c_double, C.c_double,
                  C.c_double, C.c_double]),
                ("gcso_case_destroy", None, [C.c_void_p]),
                ("gcso_case_grid", P(abi.Grid), [C.c_void_p]),
                ("gcso_case_storage", P(abi.Storage), [C.c_void_p]),
                ("gcso_case_background", P(abi.BackgroundField), [C.c_void_p]),
                ("gcso_case_options", P(abi.AdvanceOptions), [C.c_void_p]),
                ("gcso_case_timestep_options", P(abi.TimestepOptions),
                 [C.c_void_p]),
                ("gcso_case_active", P(C.c_size_t), [C.c_void_p]),
                ("gcso_case_ghost", C.c_size_t, [C.c_void_p]),
                ("gcso_case_default_dt", C.c_double, [C.c_void_p]),
                ("gcso_case_default_ratio", C.c_double, [C.c_void_p]),
                ("gcso_case_local_timestep", C.c_int, [C.c_void_p, P(C.c_double)]),
                ("gcso_case_step", C.c_int, [C.c_void_p, C.c_double, C.c_double]),
                ("gcso_case_copy_storage", C.c_int, [C.c_void_p, C.c_void_p]),
                ("gcso_halo_plan_create", C.c_int, [P(abi.Grid), P(C.c_size_t),
                                                    C.c_size_t, P(C.c_void_p)]),
                ("gcso_halo_plan_destroy", None, [C.c_void_p]),
                ("gcso_edge_plan_create", C.c_int, [P(C.c_size_t), C.c_size_t,
                                                    P(C.c_void_p)]),
                ("gcso_edge_plan_destroy", None, [C.c_void_p]),
                ("gcso_fill_cell_halos", C.c_int, [C.c_void_p, P(abi.Storage)]),
                ("gcso_fill_face_halos", C.c_int, [C.c_void_p, P(abi.Grid),
                                                   P(abi.Storage)]),
                ("gcso_fill_radial_outflow", C.c_int, [P(abi.Storage), P(C.c_size_t),
                                                       C.c_size_t]),
                ("gcso_sync_faces", C.c_int, [P(abi.Storage), P(C.c_size_t),
                                              C.c_size_t, C.c_int]),
                ("gcso_sync_edges", C.c_int, [C.c_void_p, P(abi.Storage)]),
                ("gcso_apply_pressure_control", C.c_int,
                 [P(abi.Storage), P(abi.Grid), P(C.c_size_t), P(C.c_size_t), C.c_double,
                  C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                  C.c_double, P(C.c_size_t), P(C.c_size_t), P(C.c_double),
                  P(C.c_double)]),
                ("gcso_mi_apply_constant_pedersen", C.c_int,
                 [P(abi.MiSolverConfig), P(C.c_double), P(C.c_double)]),
                ("gcso_mi_solve_constant_pedersen", C.c_int,
                 [P(abi.MiSolverConfig), P(C.c_double), P(C.c_double),
                  P(abi.MiSolverStats)]),
                ("gcso_mi_apply_conductance_tensor", C.c_int,
                 [P(abi.MiSolverConfig), P(C.c_double), P(C.c_double),
                  P(C.c_double), P(C.c_double)]),
                ("gcso_mi_solve_pedersen_pcg", C.c_int,
                 [P(abi.MiSolverConfig), P(C.c_double), P(C.c_double), P(C.c_double),
                  P(abi.MiSolverStats)]),
                ("gcso_mi_solve_conductance_tensor", C.c_int,
                 [P(abi.MiSolverConfig), P(C.c_double), P(C.c_double),
                  P(C.c_double), P(C.c_double), P(abi.MiSolverStats)])]:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class Case:
    """A six-face case built and advanced by the restatement oracle."""

    def __init__(self, kind, nr=0, n=0, seed=1, driver=None):
        """driver: (density cm^-3, Vx km/s, T K, Bz nT) of a wind case."""
        if isinstance(kind, str):
            kind = KINDS[kind]
        self.lib = lib()
        if driver is not None:
            if kind != KINDS["wind"]:
                raise ValueError("a driver needs the wind case")
            self.handle = self.lib.gcso_case_create_driven(nr, n, seed, *map(float, driver))
        else:
            self.handle = self.lib.gcso_case_create(kind, nr, n, seed)
        if not self.handle:
            raise RuntimeError("oracle case construction failed")
        self.kind = kind
        self.grid = self.lib.gcso_case_grid(self.handle)
        self.storage = self.lib.gcso_case_storage(self.handle)
        bg = self.lib.gcso_case_background(self.handle)
        self.background = bg if bg else None
        self.options = self.lib.gcso_case_options(self.handle)
        self.timestep_options = self.lib.gcso_case_timestep_options(self.handle)
        act = self.lib.gcso_case_active(self.handle)
        self.active = (C.c_size_t * 3)(act[0], act[1], act[2])
        self.ghost = self.lib.gcso_case_ghost(self.handle)
        self.dt = self.lib.gcso_case_default_dt(self.handle)
        self.ratio = self.lib.gcso_case_default_ratio(self.handle)

    def local_timestep(self):
        v = C.c_double()
        if self.lib.gcso_case_local_timestep(self.handle, C.byref(v)) != 0:
            raise RuntimeError("oracle timestep failed")
        return v.value

    def step(self, ratio, dt):
        return self.lib.gcso_case_step(self.handle, ratio, dt)

    def copy_from(self, other):
        if self.lib.gcso_case_copy_storage(self.handle, other.handle) != 0:
            raise RuntimeError("copy failed")

    def arrays(self, face):
        return abi.storage_arrays(self.storage[face])

    def close(self):
        if self.handle:
            self.lib.gcso_case_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pair(kind, nr=0, n=0, seed=7):
    """Two identical cases: one for the oracle, one to hand to the library."""
    return Case(kind, nr, n, seed), Case(kind, nr, n, seed)
