"""ctypes binding of the oracle libraries (test infrastructure only).

* oracle/_ref/libgamera_ref.so: the unmodified reference C library built by
  oracle/Makefile from the reference sources, plus ref_fixture.c (case
  construction through the reference's public setup API).
* oracle/libgcs_oracle.so: this repository's CPU restatement of the hot path
  (gcs_oracle.c), pinned against the reference.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module; the product library never does.
"""
import ctypes as C
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_PATH = os.path.join(HERE, "_ref", "libgamera_ref.so")
RESTATEMENT_PATH = os.path.join(HERE, "libgcs_oracle.so")
REPO = os.path.dirname(HERE)
if REPO not in sys.path:
    sys.path.insert(0, REPO)

from gamera_cube_b200 import abi  # noqa: E402  (ctypes struct mirrors only)

FX_UNIFORM, FX_SHOCK, FX_WIND, FX_PULSE = 0, 1, 2, 3


def ref_available():
    return os.path.exists(REF_PATH)


def _bind_common(lib):
    P = C.POINTER
    c_sz3 = C.c_size_t * 3
    sigs = {
        "gamera_cs_advance_six_with_background_planned": (
            C.c_int, [P(abi.Grid), P(abi.Storage), c_sz3, C.c_size_t, C.c_double,
                      C.c_double, P(abi.AdvanceOptions), P(abi.BackgroundField),
                      C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_void_p]),
        "gamera_cs_halo_plan_create": (C.c_int, [P(abi.Grid), c_sz3, C.c_size_t,
                                                 P(C.c_void_p)]),
        "gamera_cs_halo_plan_destroy": (None, [C.c_void_p]),
        "gamera_cs_fill_tangential_cell_halos_planned": (
            C.c_int, [C.c_void_p, P(abi.Grid), P(abi.Storage)]),
        "gamera_cs_fill_magnetic_face_halos_planned": (
            C.c_int, [C.c_void_p, P(abi.Grid), P(abi.Storage)]),
        "gamera_no_apply_pressure_control": (
            C.c_int, [P(abi.Storage), P(abi.Grid), P(C.c_size_t), P(C.c_size_t),
                      C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                      C.c_double, C.c_double, P(C.c_size_t), P(C.c_size_t),
                      P(C.c_double), P(C.c_double)]),
        "gamera_mi_solve_constant_pedersen": (
            C.c_int, [P(abi.MiSolverConfig), P(C.c_double), P(C.c_double),
                      P(abi.MiSolverStats)]),
        "gamera_mi_apply_constant_pedersen": (
            C.c_int, [P(abi.MiSolverConfig), P(C.c_double), P(C.c_double)]),
        "gamera_mi_solve_conductance_tensor": (
            C.c_int, [P(abi.MiSolverConfig), P(C.c_double), P(C.c_double),
                      P(C.c_double), P(C.c_double), P(abi.MiSolverStats)]),
        "gamera_mi_apply_conductance_tensor": (
            C.c_int, [P(abi.MiSolverConfig), P(C.c_double), P(C.c_double),
                      P(C.c_double), P(C.c_double)]),
    }
    for name, (res, args) in sigs.items():
        if hasattr(lib, name):
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
    return lib


_ref = None


def ref():
    """The reference library with the fixture harness."""
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(REF_PATH + " (build with make -C oracle ref)")
        lib = C.CDLL(REF_PATH, mode=os.RTLD_LOCAL)
        P = C.POINTER
        for name, res, args in [
                ("fx_create", C.c_void_p, [C.c_int, C.c_size_t, C.c_size_t,
                                           C.c_ulonglong]),
                ("fx_destroy", None, [C.c_void_p]),
                ("fx_grid", P(abi.Grid), [C.c_void_p]),
                ("fx_storage", P(abi.Storage), [C.c_void_p]),
                ("fx_background", P(abi.BackgroundField), [C.c_void_p]),
                ("fx_options", P(abi.AdvanceOptions), [C.c_void_p]),
                ("fx_timestep_options", P(abi.TimestepOptions), [C.c_void_p]),
                ("fx_plan", C.c_void_p, [C.c_void_p]),
                ("fx_active", P(C.c_size_t), [C.c_void_p]),
                ("fx_ghost", C.c_size_t, [C.c_void_p]),
                ("fx_default_dt", C.c_double, [C.c_void_p]),
                ("fx_default_ratio", C.c_double, [C.c_void_p]),
                ("fx_local_timestep", C.c_int, [C.c_void_p, P(C.c_double)]),
                ("fx_step", C.c_int, [C.c_void_p, C.c_double, C.c_double]),
                ("fx_copy_storage", C.c_int, [C.c_void_p, C.c_void_p]),
                ("fx_noise", C.c_double, [C.c_ulonglong, C.c_int, C.c_size_t]),
                ("fx_magnetic_norm_tesla", C.c_double, [])]:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        abi.bind(lib, abi.mi_dipole_signatures())
        P = C.POINTER
        abi.bind(lib, {"fx_set_mi_field": (C.c_int, [C.c_void_p]),
                       "fx_mi_create": (C.c_void_p, [C.c_void_p, P(abi.EarthStartup),
                                                     P(abi.MiDipoleConfig)])})
        _ref = _bind_common(lib)
    return _ref


class Case:
    """A six-face case built by the reference setup API (see ref_fixture.c)."""

    def __init__(self, kind, nr=0, n=0, seed=1):
        self.lib = ref()
        self.handle = self.lib.fx_create(kind, nr, n, seed)
        if not self.handle:
            raise RuntimeError("reference case construction failed")
        self.kind = kind
        self.grid = self.lib.fx_grid(self.handle)
        self.storage = self.lib.fx_storage(self.handle)
        bg = self.lib.fx_background(self.handle)
        self.background = bg if bg else None
        self.options = self.lib.fx_options(self.handle)
        self.timestep_options = self.lib.fx_timestep_options(self.handle)
        act = self.lib.fx_active(self.handle)
        self.active = (C.c_size_t * 3)(act[0], act[1], act[2])
        self.ghost = self.lib.fx_ghost(self.handle)
        self.dt = self.lib.fx_default_dt(self.handle)
        self.ratio = self.lib.fx_default_ratio(self.handle)

    def local_timestep(self):
        v = C.c_double()
        if self.lib.fx_local_timestep(self.handle, C.byref(v)) != 0:
            raise RuntimeError("reference timestep failed")
        return v.value

    def step(self, ratio, dt):
        return self.lib.fx_step(self.handle, ratio, dt)

    def copy_from(self, other):
        if self.lib.fx_copy_storage(self.handle, other.handle) != 0:
            raise RuntimeError("copy failed")

    def arrays(self, face):
        return abi.storage_arrays(self.storage[face])

    def close(self):
        if self.handle:
            self.lib.fx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
