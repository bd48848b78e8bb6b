"""Python host interface of libgamera_cs_b200 (the B200 cubed-sphere MHD
step and ionosphere solve).

The shared library is built in place (``make -C gamera_cube_b200``).  It is
loaded on first use of ``gamera_cube_b200.lib`` (so the ctypes struct mirrors
in ``abi`` and the case descriptions in ``cases`` can be imported without
it), and that first use raises if the library is missing: there is no CPU
fallback.
"""
import ctypes as C
import os

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "libgamera_cs_b200.so")


def _load(path=None):
    path = path or LIBRARY_PATH
    if not os.path.exists(path):
        raise ImportError(
            "libgamera_cs_b200.so is not built (run make -C gamera_cube_b200); "
            "the CUDA library is required, there is no CPU fallback")
    lib = C.CDLL(path, mode=os.RTLD_LOCAL | getattr(os, "RTLD_NOW", 2))
    P = C.POINTER
    c_sz3 = C.c_size_t * 3
    sig = {
        "gamera_cs_advance_six": (C.c_int, [P(abi.Grid), P(abi.Storage), c_sz3,
                                            C.c_size_t, C.c_double, C.c_double,
                                            P(abi.AdvanceOptions)]),
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
        "gamera_cs_halo_valid_state": (C.c_int, [P(C.c_double)]),
        "gcs_context_create": (C.c_void_p, [P(abi.Grid), c_sz3, C.c_size_t]),
        "gcs_context_destroy": (None, [C.c_void_p]),
        "gcs_last_error": (C.c_char_p, []),
        "gcs_context_error": (C.c_char_p, [C.c_void_p]),
        "gcs_context_upload_background": (C.c_int, [C.c_void_p,
                                                    P(abi.BackgroundField)]),
        "gcs_context_upload_state": (C.c_int, [C.c_void_p, P(abi.Storage)]),
        "gcs_context_download_state": (C.c_int, [C.c_void_p, P(abi.Storage),
                                                 C.c_int]),
        "gcs_context_step": (C.c_int, [C.c_void_p, P(abi.AdvanceOptions),
                                       C.c_double, C.c_double]),
        "gcs_context_timestep": (C.c_int, [C.c_void_p, P(abi.TimestepOptions),
                                           P(C.c_double)]),
        "gcs_context_run": (C.c_int, [C.c_void_p, P(abi.AdvanceOptions),
                                      P(abi.TimestepOptions), C.c_double,
                                      C.c_int, C.c_int]),
        "gcs_context_sync": (C.c_int, [C.c_void_p]),
        "gcs_context_params": (C.c_int, [C.c_void_p, P(C.c_double),
                                         P(C.c_double), P(C.c_double),
                                         P(C.c_int)]),
        "gcs_context_set_params": (C.c_int, [C.c_void_p, C.c_double, C.c_double,
                                             C.c_double, C.c_int]),
        "gcs_context_failure": (C.c_int, [C.c_void_p] + [P(C.c_int)] * 5),
        "gcs_context_reset_failure": (C.c_int, [C.c_void_p]),
        "gcs_context_stream": (C.c_size_t, [C.c_void_p]),
        "gcs_context_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
        "gcs_context_set_flux_staging": (C.c_int, [C.c_void_p, C.c_int]),
        "gcs_context_stage_times": (C.c_int, [C.c_void_p, P(C.c_double),
                                              P(C.c_longlong), C.c_int]),
        "gcs_stage_name": (C.c_char_p, [C.c_int]),
        "gcs_context_device_bytes": (C.c_size_t, [C.c_void_p]),
        "gcs_halo_plan_context": (C.c_void_p, [C.c_void_p]),
        "gcs_context_set_resident": (C.c_int, [C.c_void_p, C.c_int]),
        "gcs_context_create_case": (C.c_void_p, [C.c_int, C.c_size_t, C.c_size_t,
                                                 C.c_ulonglong]),
        "gcs_case_options": (C.c_int, [C.c_int, P(abi.AdvanceOptions),
                                       P(abi.TimestepOptions)]),
        "gcs_context_dims": (C.c_int, [C.c_void_p, P(C.c_size_t),
                                       P(C.c_size_t)]),
        "gcs_context_advance_host": (C.c_int, [C.c_void_p, P(abi.Storage),
                                               P(abi.AdvanceOptions), C.c_double,
                                               C.c_double]),
        "gcs_context_debug_array": (C.c_int, [C.c_void_p, C.c_int, C.c_int,
                                              C.c_int, C.c_int, P(C.c_double),
                                              C.c_size_t]),
        "gamera_mi_apply_constant_pedersen": (
            C.c_int, [P(abi.MiSolverConfig), P(C.c_double), P(C.c_double)]),
        "gamera_mi_solve_constant_pedersen": (
            C.c_int, [P(abi.MiSolverConfig), P(C.c_double), P(C.c_double),
                      P(abi.MiSolverStats)]),
        "gamera_mi_apply_conductance_tensor": (
            C.c_int, [P(abi.MiSolverConfig), P(C.c_double), P(C.c_double),
                      P(C.c_double), P(C.c_double)]),
        "gamera_mi_solve_conductance_tensor": (
            C.c_int, [P(abi.MiSolverConfig), P(C.c_double), P(C.c_double),
                      P(C.c_double), P(C.c_double), P(abi.MiSolverStats)]),
        "gcs_mi_tensor_plan_create": (C.c_int, [P(abi.MiSolverConfig), P(C.c_void_p)]),
        "gcs_mi_tensor_plan_destroy": (None, [C.c_void_p]),
        "gcs_mi_tensor_plan_buffers": (C.c_int, [C.c_void_p] + [P(C.c_void_p)] * 4),
        "gcs_mi_tensor_plan_upload": (C.c_int, [C.c_void_p] + [P(C.c_double)] * 4),
        "gcs_mi_tensor_solve_async": (C.c_int, [C.c_void_p, C.c_void_p]),
        "gcs_mi_tensor_plan_set_ordering": (C.c_int, [C.c_void_p, C.c_int]),
        "gcs_mi_tensor_plan_set_schedule": (C.c_int, [C.c_void_p, C.c_int]),
        "gcs_mi_tensor_plan_schedule": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
        "gcs_mi_tensor_results": (C.c_int, [C.c_void_p, P(abi.MiSolverStats),
                                            P(C.c_int)]),
        "gcs_mi_plan_create": (C.c_int, [P(abi.MiSolverConfig), C.c_int,
                                         P(C.c_void_p)]),
        "gcs_mi_plan_destroy": (None, [C.c_void_p]),
        "gcs_mi_plan_info": (C.c_int, [C.c_void_p, P(C.c_int), P(C.c_int),
                                       P(C.c_size_t)]),
        "gcs_mi_plan_buffers": (C.c_int, [C.c_void_p, P(C.c_void_p),
                                          P(C.c_void_p)]),
        "gcs_mi_solve_constant_pedersen_async": (
            C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "gcs_mi_plan_results": (C.c_int, [C.c_void_p, P(abi.MiSolverStats),
                                          P(C.c_int)]),
        "gcs_mi_net_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_uint,
                                        P(C.c_void_p)]),
        "gcs_mi_net_destroy": (None, [C.c_void_p]),
        "gcs_mi_net_info": (C.c_int, [C.c_void_p] + [P(C.c_int)] * 4),
        "gcs_mi_net_get_params": (C.c_int, [C.c_void_p, P(C.c_float), C.c_int, C.c_int]),
        "gcs_mi_net_set_params": (C.c_int, [C.c_void_p, P(C.c_float), C.c_int]),
        "gcs_mi_net_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
        "gcs_mi_net_train_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                            C.c_float, C.c_int, P(C.c_float)]),
        "gcs_mi_solve_conductance_tensor_learned": (
            C.c_int, [C.c_void_p, C.c_int, P(abi.MiSolverConfig)] + [P(C.c_double)] * 4 +
            [P(abi.MiSolverStats), P(C.c_int)]),
        "gcs_mi_learned_apply": (C.c_int, [C.c_void_p, C.c_int, C.c_int,
                                           P(abi.MiSolverConfig)] + [P(C.c_double)] * 4),
    }
    sig["gcs_context_set_precision"] = (C.c_int, [C.c_void_p, C.c_int])
    sig["gcs_context_precision"] = (C.c_int, [C.c_void_p])
    sig["gcs_context_set_bulk_threshold"] = (C.c_int, [C.c_void_p, C.c_double])
    sig["gcs_context_bulk_split"] = (C.c_int, [C.c_void_p])
    c_sz3p = P(C.c_size_t)
    for name in ("gamera_cs_fill_tangential_cell_halos", "gamera_cs_fill_magnetic_face_halos",
                 "gamera_cs_sync_edge_emf"):
        sig[name] = (C.c_int, [P(abi.Grid), P(abi.Storage), c_sz3p, C.c_size_t])
    for name in ("gamera_cs_fill_radial_outflow_cells", "gamera_cs_sync_magnetic_face_flux",
                 "gamera_cs_sync_mhd_face_fluxes"):
        sig[name] = (C.c_int, [P(abi.Storage), c_sz3p, C.c_size_t])
    sig["gamera_cs_fill_radial_outflow_cells_face"] = (
        C.c_int, [P(abi.Storage), c_sz3p, C.c_size_t, C.c_int])
    for name in ("gamera_cs_fill_tangential_cell_halos_planned_face",
                 "gamera_cs_fill_magnetic_face_halos_planned_face"):
        sig[name] = (C.c_int, [C.c_void_p, P(abi.Grid), P(abi.Storage), C.c_int])
    sig["gamera_cs_edge_sync_plan_create"] = (C.c_int, [P(abi.Grid), c_sz3p, C.c_size_t,
                                                        P(C.c_void_p)])
    sig["gamera_cs_edge_sync_plan_destroy"] = (None, [C.c_void_p])
    sig["gamera_cs_sync_edge_emf_planned"] = (C.c_int, [C.c_void_p, P(abi.Storage)])
    sig.update(abi.mi_dipole_signatures())
    sig.update(abi.ensemble_signatures())
    sig["gcs_context_set_mi_coupling"] = (C.c_int, [C.c_void_p, C.c_void_p, C.c_int])
    sig["gcs_context_time"] = (C.c_int, [C.c_void_p, P(C.c_double)])
    sig["gcs_mi_plan_create_pedersen"] = (C.c_int, [P(abi.MiSolverConfig), P(C.c_double),
                                                    C.c_int, P(C.c_void_p)])
    sig["gcs_mi_solve_pedersen_pcg"] = (C.c_int, [P(abi.MiSolverConfig), P(C.c_double),
                                                  P(C.c_double), P(C.c_double),
                                                  P(abi.MiSolverStats)])
    sig["gcs_context_mi_dipole_create"] = (
        C.c_int, [C.c_void_p, P(abi.EarthStartup), P(abi.MiDipoleConfig),
                  P(C.c_void_p)])
    return abi.bind(lib, sig)


_lib = None


def __getattr__(name):
    # the library is loaded by the first access to gamera_cube_b200.lib
    global _lib
    if name == "lib":
        if _lib is None:
            _lib = _load()
        return _lib
    raise AttributeError("module %r has no attribute %r" % (__name__, name))


__all__ = ["abi", "lib", "LIBRARY_PATH"]
