"""ctypes mirrors of the reference GAMERA-Cube C data types.

Layout-identical to include/gamera_cs_types.h (and therefore to the
reference headers cited there); used by the Python host interface and the
tests to hand reference-layout host arrays to the C-ABI library.
"""
import ctypes as C

import numpy as np

FACE_COUNT = 6
FLUX_COUNT = 5


class Vec3(C.Structure):
    _fields_ = [("value", C.c_double * 3)]


class FaceGeometry(C.Structure):
    _fields_ = [("area", C.c_double), ("area_vector", Vec3), ("centroid", Vec3),
                ("normal", Vec3), ("tangent1", Vec3), ("tangent2", Vec3)]


class CellGeometry(C.Structure):
    _fields_ = [("volume", C.c_double), ("centroid", Vec3),
                ("face", (FaceGeometry * 2) * 3), ("cfl_length", C.c_double * 3)]


class EdgeGeometry(C.Structure):
    _fields_ = [("length", C.c_double), ("normal", Vec3), ("tangent1", Vec3),
                ("tangent2", Vec3)]


class FaceGrid(C.Structure):
    _fields_ = [("extent", C.c_size_t * 3), ("value", C.POINTER(FaceGeometry))]


class EdgeGrid(C.Structure):
    _fields_ = [("extent", C.c_size_t * 3), ("value", C.POINTER(EdgeGeometry)),
                ("valid", C.POINTER(C.c_ubyte))]


class Grid(C.Structure):
    _fields_ = [("cell_extent", C.c_size_t * 3), ("vertex_extent", C.c_size_t * 3),
                ("vertex", C.POINTER(Vec3)), ("cell", C.POINTER(CellGeometry)),
                ("face", FaceGrid * 3), ("edge", EdgeGrid * 3)]


class Storage(C.Structure):
    _fields_ = [
        ("cell_extent", C.c_size_t * 3),
        ("face_extent", (C.c_size_t * 3) * 3),
        ("edge_extent", (C.c_size_t * 3) * 3),
        ("conserved", C.POINTER(C.c_double)),
        ("old_conserved", C.POINTER(C.c_double)),
        ("predicted_conserved", C.POINTER(C.c_double)),
        ("cell_magnetic", C.POINTER(Vec3)),
        ("old_cell_magnetic", C.POINTER(Vec3)),
        ("predicted_cell_magnetic", C.POINTER(Vec3)),
        ("face_flux", C.POINTER(C.c_double) * 3),
        ("old_face_flux", C.POINTER(C.c_double) * 3),
        ("predicted_face_flux", C.POINTER(C.c_double) * 3),
        ("edge_emf", C.POINTER(C.c_double) * 3),
        ("fluid_face_flux", C.POINTER(C.c_double) * 3),
        ("maxwell_face_flux", C.POINTER(Vec3) * 3),
        ("hydro_rate", C.POINTER(C.c_double)),
        ("maxwell_rate", C.POINTER(Vec3)),
        ("emergency_diffusion_face_count", C.c_size_t),
        ("emergency_diffusion_max_interface_speed", C.c_double),
        ("inner_wall_clamped_face_count", C.c_size_t * 2),
        ("inner_wall_positive_mass_max", C.c_double * 2),
        ("inner_wall_positive_energy_max", C.c_double * 2),
        ("inner_wall_fluid_momentum_max", C.c_double * 2),
        ("inner_wall_maxwell_momentum_max", C.c_double * 2),
        ("inner_wall_density_max", C.c_double * 2),
        ("inner_wall_pressure_max", C.c_double * 2),
        ("inner_wall_pressure_gradient_max", C.c_double * 2),
        ("inner_wall_speed_max", C.c_double * 2),
        ("inner_wall_residual_magnetic_max", C.c_double * 2),
        ("inner_wall_residual_magnetic_location", Vec3 * 2),
        ("inner_wall_lowlat_pressure_max", C.c_double * 2),
        ("inner_wall_lowlat_pressure_gradient_max", C.c_double * 2),
        ("inner_wall_lowlat_speed_max", C.c_double * 2),
        ("inner_wall_lowlat_residual_magnetic_max", C.c_double * 2),
    ]


class SweepOptions(C.Structure):
    _fields_ = [("gamma", C.c_double), ("density_floor", C.c_double),
                ("pressure_floor", C.c_double), ("pdm_coefficient", C.c_double),
                ("hydro_hogs_coefficient", C.c_double),
                ("magnetic_hogs_coefficient", C.c_double),
                ("light_speed", C.c_double), ("use_mhd", C.c_bool),
                ("use_hogs", C.c_bool), ("use_boris", C.c_bool),
                ("use_background", C.c_bool)]


class BackgroundField(C.Structure):
    _fields_ = [("cell_magnetic", C.POINTER(Vec3)),
                ("face_magnetic", C.POINTER(Vec3) * 3),
                ("face_flux", C.POINTER(C.c_double) * 3),
                ("edge_magnetic", C.POINTER(Vec3) * 3),
                ("cell_force", C.POINTER(Vec3))]


class EmfOptions(C.Structure):
    _fields_ = [("density_floor", C.c_double), ("pdm_coefficient", C.c_double),
                ("diffusion_coefficient", C.c_double), ("light_speed", C.c_double),
                ("cfl", C.c_double), ("dt", C.c_double), ("use_boris", C.c_bool),
                ("use_background", C.c_bool)]


class UpdateOptions(C.Structure):
    _fields_ = [("gamma", C.c_double), ("density_floor", C.c_double),
                ("pressure_floor", C.c_double), ("light_speed", C.c_double),
                ("use_mhd", C.c_bool), ("use_boris", C.c_bool),
                ("use_background", C.c_bool)]


class TimestepOptions(C.Structure):
    _fields_ = [("gamma", C.c_double), ("density_floor", C.c_double),
                ("pressure_floor", C.c_double), ("cfl", C.c_double),
                ("light_speed", C.c_double), ("use_mhd", C.c_bool),
                ("use_boris", C.c_bool), ("use_background", C.c_bool)]


class AdvanceOptions(C.Structure):
    _fields_ = [("stress", SweepOptions), ("emf", EmfOptions),
                ("update", UpdateOptions), ("cell_source", C.c_void_p),
                ("source_context", C.c_void_p), ("indexed_cell_source", C.c_void_p),
                ("indexed_source_context", C.c_void_p), ("source_time", C.c_double),
                ("fluid_flux_sync", C.c_void_p), ("fluid_flux_context", C.c_void_p),
                ("edge_emf_sync", C.c_void_p), ("edge_emf_context", C.c_void_p)]


class MiSolverConfig(C.Structure):
    _fields_ = [("longitude_count", C.c_size_t), ("colatitude_count", C.c_size_t),
                ("maximum_colatitude", C.c_double),
                ("ionosphere_radius_m", C.c_double),
                ("pedersen_siemens", C.c_double), ("hall_siemens", C.c_double),
                ("low_latitude_potential_v", C.c_double), ("hemisphere", C.c_int),
                ("maximum_iterations", C.c_int), ("relative_tolerance", C.c_double),
                ("absolute_tolerance", C.c_double)]


class MiSolverStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("initial_residual", C.c_double),
                ("final_residual", C.c_double), ("converged", C.c_int)]


def _view(ptr, count):
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_double)), shape=(count,))


def storage_arrays(storage):
    """numpy views (no copy) of the arrays of one gamera_no_storage."""
    ce = tuple(storage.cell_extent)
    ncell = ce[0] * ce[1] * ce[2]
    out = {
        "conserved": _view(storage.conserved, 5 * ncell).reshape(ce + (5,)),
        "old_conserved": _view(storage.old_conserved, 5 * ncell).reshape(ce + (5,)),
        "predicted_conserved":
            _view(storage.predicted_conserved, 5 * ncell).reshape(ce + (5,)),
        "cell_magnetic": _view(storage.cell_magnetic, 3 * ncell).reshape(ce + (3,)),
        "old_cell_magnetic":
            _view(storage.old_cell_magnetic, 3 * ncell).reshape(ce + (3,)),
        "predicted_cell_magnetic":
            _view(storage.predicted_cell_magnetic, 3 * ncell).reshape(ce + (3,)),
    }
    for d in range(3):
        fe = tuple(storage.face_extent[d])
        ee = tuple(storage.edge_extent[d])
        nf = fe[0] * fe[1] * fe[2]
        ne = ee[0] * ee[1] * ee[2]
        out["face_flux%d" % d] = _view(storage.face_flux[d], nf).reshape(fe)
        out["old_face_flux%d" % d] = _view(storage.old_face_flux[d], nf).reshape(fe)
        out["predicted_face_flux%d" % d] = \
            _view(storage.predicted_face_flux[d], nf).reshape(fe)
        out["fluid_face_flux%d" % d] = \
            _view(storage.fluid_face_flux[d], 5 * nf).reshape(fe + (5,))
        out["maxwell_face_flux%d" % d] = \
            _view(storage.maxwell_face_flux[d], 3 * nf).reshape(fe + (3,))
        out["edge_emf%d" % d] = _view(storage.edge_emf[d], ne).reshape(ee)
    return out


class Dipole(C.Structure):
    _fields_ = [("moment", Vec3)]


class EarthStartup(C.Structure):
    """cubedsphere/cubedsphere_earth_startup.h:10-24"""
    _fields_ = [("inner_radius", C.c_double), ("density", C.c_double),
                ("speed", C.c_double), ("mach", C.c_double), ("gamma", C.c_double),
                ("ambient_density", C.c_double), ("ambient_pressure", C.c_double),
                ("front_x", C.c_double), ("front_width", C.c_double),
                ("cut_radius", C.c_double), ("cut_length", C.c_double),
                ("imf", Vec3), ("dipole", Dipole)]


class MiDipoleConfig(C.Structure):
    """cubedsphere/cubedsphere_mi_dipole.h:16-28"""
    _fields_ = [("azimuth_points", C.c_size_t), ("colatitude_points", C.c_size_t),
                ("current_shell", C.c_size_t), ("ionosphere_radius_re", C.c_double),
                ("pedersen_siemens", C.c_double), ("coupling_interval_s", C.c_double),
                ("length_norm_m", C.c_double), ("speed_norm_m_s", C.c_double),
                ("mass_density_norm_kg_m3", C.c_double),
                ("maximum_iterations", C.c_int), ("relative_tolerance", C.c_double)]


class MiAnalysisView(C.Structure):
    """cubedsphere/cubedsphere_mi_dipole.h:32-39"""
    _fields_ = [("azimuth_points", C.c_size_t), ("colatitude_points", C.c_size_t),
                ("shell_j_cells", C.c_size_t), ("shell_k_cells", C.c_size_t),
                ("maximum_colatitude_rad", C.c_double), ("epoch_s", C.c_double),
                ("sample_radius_re", C.c_double), ("pedersen_siemens", C.c_double),
                ("fac_parallel_a_m2", C.POINTER(C.c_double) * 2),
                ("potential_v", C.POINTER(C.c_double) * 2)]


class SolarWindState(C.Structure):
    """nonorthogonal/src/solar_wind.h:17-22"""
    _fields_ = [("density", C.c_double), ("pressure", C.c_double),
                ("velocity", C.c_double * 3), ("magnetic", C.c_double * 3)]


class SolarWindSeries(C.Structure):
    """nonorthogonal/src/solar_wind.h:24-35"""
    _fields_ = [("count", C.c_size_t), ("time", C.POINTER(C.c_double)),
                ("state", C.POINTER(SolarWindState)), ("reference", C.c_double * 3),
                ("time_offset", C.c_double), ("by_coefficient", C.c_double),
                ("bz_coefficient", C.c_double), ("bx_offset", C.c_double),
                ("enforce_bx_relation", C.c_int), ("linear_interpolation", C.c_int)]


class EarthBoundary(C.Structure):
    """cubedsphere/cubedsphere_earth_boundary.h:13-24"""
    _fields_ = [("startup", C.POINTER(EarthStartup)), ("wind", C.POINTER(SolarWindSeries)),
                ("background", C.POINTER(BackgroundField)), ("mi", C.c_void_p),
                ("density_floor", C.c_double), ("pressure_floor", C.c_double),
                ("step_time", C.c_double), ("step_dt", C.c_double), ("cfl", C.c_double),
                ("strict_inner_gas_wall", C.c_int)]


class WindDriver(C.Structure):
    """gcs_wind_driver: upstream n (cm^-3), Vx (km/s), T (K), IMF Bz (nT)."""
    _fields_ = [("density_cm3", C.c_double), ("velocity_x_kms", C.c_double),
                ("temperature_k", C.c_double), ("bz_nt", C.c_double)]


class PressureControl(C.Structure):
    """gcs_pressure_control: the arguments of gamera_no_apply_pressure_control
    after dt (nonorthogonal_step.h:26-32)."""
    _fields_ = [("gamma", C.c_double), ("density_floor", C.c_double),
                ("pressure_floor", C.c_double), ("light_speed", C.c_double),
                ("low_density_threshold", C.c_double),
                ("low_density_sound_speed", C.c_double)]


class EnsembleConfig(C.Structure):
    """gcs_ensemble_config."""
    _fields_ = [("count", C.c_int), ("nr", C.POINTER(C.c_size_t)),
                ("n", C.POINTER(C.c_size_t)), ("drivers", C.POINTER(WindDriver)),
                ("seed", C.c_ulonglong), ("fp32_bulk", C.c_int),
                ("autotune_repetitions", C.c_int), ("dt_fraction", C.c_double)]


def ensemble_signatures():
    P = C.POINTER
    sig = {
        "gcs_context_create_wind": (C.c_void_p, [C.c_size_t, C.c_size_t, C.c_ulonglong,
                                                 P(WindDriver)]),
        "gcs_tile_limit": (C.c_int, [C.c_int]),
        "gcs_context_set_tile": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
        "gcs_context_tile": (C.c_int, [C.c_void_p, C.c_int, P(C.c_int), P(C.c_int)]),
        "gcs_context_autotune": (C.c_int, [C.c_void_p, P(AdvanceOptions),
                                           P(TimestepOptions), C.c_int, P(C.c_double),
                                           P(C.c_double)]),
        "gcs_ensemble_draw": (C.c_int, [C.c_ulonglong, C.c_int, P(C.c_size_t),
                                        P(WindDriver)]),
        "gcs_ensemble_estimate_bytes": (C.c_double, [C.c_int, P(C.c_size_t),
                                                     P(C.c_size_t), C.c_int]),
        "gcs_ensemble_create": (C.c_void_p, [P(EnsembleConfig)]),
        "gcs_ensemble_destroy": (None, [C.c_void_p]),
        "gcs_ensemble_count": (C.c_int, [C.c_void_p]),
        "gcs_ensemble_run_context": (C.c_void_p, [C.c_void_p, C.c_int]),
        "gcs_ensemble_grid_owner": (C.c_int, [C.c_void_p, C.c_int]),
        "gcs_ensemble_advance": (C.c_int, [C.c_void_p, C.c_int]),
        "gcs_ensemble_sync": (C.c_int, [C.c_void_p, P(C.c_int)]),
        "gcs_ensemble_stream": (C.c_size_t, [C.c_void_p]),
        "gcs_ensemble_device_bytes": (C.c_size_t, [C.c_void_p]),
        "gcs_ensemble_graph_info": (C.c_int, [C.c_void_p, P(C.c_int), P(C.c_int)]),
        "gcs_earth_create": (C.c_int, [C.c_void_p, P(Grid), P(EarthBoundary),
                                       P(C.c_void_p)]),
        "gcs_earth_create_case": (C.c_int, [C.c_void_p, P(EarthBoundary), P(C.c_void_p)]),
        "gcs_earth_set_wind": (C.c_int, [C.c_void_p, P(SolarWindSeries)]),
        "gcs_earth_destroy": (None, [C.c_void_p]),
        "gcs_earth_device_bytes": (C.c_size_t, [C.c_void_p]),
        "gcs_earth_copy_layers": (C.c_size_t, [C.c_void_p, C.c_void_p, C.c_size_t]),
        "gcs_context_step_earth": (C.c_int, [C.c_void_p, C.c_void_p, P(AdvanceOptions),
                                             C.c_double, C.c_double, C.c_double,
                                             C.c_double]),
        "gcs_context_run_earth": (C.c_int, [C.c_void_p, C.c_void_p, P(AdvanceOptions),
                                            P(TimestepOptions), C.c_double, C.c_int,
                                            C.c_int]),
    }
    sig.update(earth_callback_signatures())
    sig.update({
        "gcs_analysis_frame_floats": (C.c_size_t, [C.c_void_p]),
        "gcs_context_analysis_frame": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p,
                                                 C.c_void_p]),
        "gcs_context_write_analysis": (C.c_int, [C.c_void_p, C.c_char_p, C.c_long, C.c_long,
                                                 C.c_double, C.c_double, C.c_double,
                                                 P(Grid)]),
        "gcs_context_pressure_control": (C.c_int, [C.c_void_p, P(Grid), C.c_double,
                                                   P(PressureControl), P(C.c_size_t),
                                                   P(C.c_size_t), P(C.c_double),
                                                   P(C.c_double)]),
        "gcs_context_set_pressure_control": (C.c_int, [C.c_void_p, P(Grid),
                                                       P(PressureControl)]),
        "gcs_context_pressure_control_stats": (C.c_int, [C.c_void_p, P(C.c_size_t),
                                                         P(C.c_size_t), P(C.c_double),
                                                         P(C.c_double), C.c_int]),
    })
    return sig


def earth_callback_signatures():
    """The reference's Earth radial-boundary callbacks (same in the reference
    library and in this one)."""
    P = C.POINTER
    c_sz3 = C.c_size_t * 3
    return {
        "gamera_cs_earth_fill_radial_ghosts": (
            C.c_int, [P(Grid), P(Storage), c_sz3, C.c_size_t, C.c_double, C.c_double,
                      C.c_void_p]),
        "gamera_cs_earth_fill_radial_ghosts_face": (
            C.c_int, [P(Grid), P(Storage), c_sz3, C.c_size_t, C.c_double, C.c_double,
                      C.c_void_p, C.c_int]),
        "gamera_cs_earth_inner_fluid_flux": (
            C.c_int, [P(Storage), P(Grid), c_sz3, c_sz3, C.c_void_p]),
        "gamera_cs_earth_no_mi_emf": (
            C.c_int, [P(Storage), P(Grid), c_sz3, c_sz3, C.c_void_p]),
    }


def mi_dipole_signatures():
    """ctypes signatures of the cubedsphere_mi_dipole.h entry points, shared
    by this library and the reference build."""
    P = C.POINTER
    return {
        "gamera_cs_mi_dipole_create": (C.c_int, [P(Grid), P(Storage),
                                                 P(BackgroundField), P(EarthStartup),
                                                 P(C.c_size_t), C.c_size_t,
                                                 P(MiDipoleConfig), P(C.c_void_p)]),
        "gamera_cs_mi_dipole_destroy": (None, [C.c_void_p]),
        "gamera_cs_mi_dipole_create_potential_view": (
            C.c_int, [P(EarthStartup), P(MiDipoleConfig), P(C.c_void_p)]),
        "gamera_cs_mi_dipole_export_potential": (
            C.c_int, [C.c_void_p, P(C.c_double), C.c_size_t, P(C.c_double),
                      P(C.c_double)]),
        "gamera_cs_mi_dipole_import_potential": (
            C.c_int, [C.c_void_p, P(C.c_double), C.c_size_t, C.c_double, C.c_double]),
        "gamera_cs_mi_dipole_maybe_update": (C.c_int, [C.c_void_p, C.c_double]),
        "gamera_cs_mi_dipole_update_due": (C.c_int, [C.c_void_p, C.c_double]),
        "gamera_cs_mi_dipole_ready": (C.c_int, [C.c_void_p]),
        "gamera_cs_mi_dipole_potential": (C.c_int, [C.c_void_p, Vec3, P(C.c_double)]),
        "gamera_cs_mi_dipole_apply_inner_emf": (C.c_int, [C.c_void_p, P(Storage),
                                                          P(Grid), C.c_size_t]),
        "gamera_cs_mi_dipole_ghost_velocity": (C.c_int, [C.c_void_p, Vec3, Vec3,
                                                         P(Vec3)]),
        "gamera_cs_mi_dipole_stats": (C.c_int, [C.c_void_p, P(C.c_double),
                                                P(C.c_double), P(C.c_double),
                                                P(C.c_double), P(MiSolverStats)]),
        "gamera_cs_mi_dipole_analysis_view": (C.c_int, [C.c_void_p, P(MiAnalysisView)]),
        "gamera_cs_mi_dipole_export_shell_current": (
            C.c_int, [C.c_void_p, P(C.c_double), P(C.c_double), P(C.c_double),
                      C.c_size_t]),
        "gamera_cs_mi_dipole_write_csv": (C.c_int, [C.c_void_p, C.c_char_p]),
        "gamera_cs_mi_dipole_write_shell_current_csv": (C.c_int, [C.c_void_p,
                                                                  C.c_char_p]),
    }


def bind(lib, signatures):
    for name, (res, args) in signatures.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib
