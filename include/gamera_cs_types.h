/*
 * Plain-C data types of the GAMERA-Cube cubed-sphere MHD interface.
 *
 * These declarations are layout-identical to the reference types so that a
 * caller compiled against the reference headers can hand its host arrays to
 * this library unchanged.  Each type cites the reference declaration it
 * mirrors (paths inside the GAMERA-Cube project).  Index convention of every
 * array: (i * extent[1] + j) * extent[2] + k, k contiguous, i radial
 * (nonorthogonal/src/nonorthogonal/nonorthogonal_grid.c:7-10).
 */
#ifndef GAMERA_CS_TYPES_H
#define GAMERA_CS_TYPES_H

#include <stddef.h>
#include <stdint.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* nonorthogonal_geometry.h:10-17 */
enum {
  GAMERA_NO_I = 0,
  GAMERA_NO_J = 1,
  GAMERA_NO_K = 2,
  GAMERA_NO_DIM = 3,
  GAMERA_NO_LOWER = 0,
  GAMERA_NO_UPPER = 1
};

/* nonorthogonal_flux.h:12-19 */
enum {
  GAMERA_NO_FLUX_DENSITY = 0,
  GAMERA_NO_FLUX_MOMENTUM_X,
  GAMERA_NO_FLUX_MOMENTUM_Y,
  GAMERA_NO_FLUX_MOMENTUM_Z,
  GAMERA_NO_FLUX_ENERGY,
  GAMERA_NO_FLUX_COUNT
};

/* cubedsphere/cubedsphere_mesh.h:14-30 */
enum {
  GAMERA_CS_POS_X = 0,
  GAMERA_CS_NEG_X,
  GAMERA_CS_POS_Y,
  GAMERA_CS_NEG_Y,
  GAMERA_CS_POS_Z,
  GAMERA_CS_NEG_Z,
  GAMERA_CS_FACE_COUNT
};
enum {
  GAMERA_CS_A_LOWER = 0,
  GAMERA_CS_A_UPPER,
  GAMERA_CS_B_LOWER,
  GAMERA_CS_B_UPPER,
  GAMERA_CS_EDGE_COUNT
};

/* nonorthogonal_geometry.h:19-21 */
typedef struct {
  double value[GAMERA_NO_DIM];
} gamera_no_vec3;

/* nonorthogonal_geometry.h:23-30 */
typedef struct {
  double area;
  gamera_no_vec3 area_vector;
  gamera_no_vec3 centroid;
  gamera_no_vec3 normal;
  gamera_no_vec3 tangent1;
  gamera_no_vec3 tangent2;
} gamera_no_face_geometry;

/* nonorthogonal_geometry.h:32-37 */
typedef struct {
  double volume;
  gamera_no_vec3 centroid;
  gamera_no_face_geometry face[GAMERA_NO_DIM][2];
  double cfl_length[GAMERA_NO_DIM];
} gamera_no_cell_geometry;

/* nonorthogonal_geometry.h:39-44 */
typedef struct {
  double length;
  gamera_no_vec3 normal;
  gamera_no_vec3 tangent1;
  gamera_no_vec3 tangent2;
} gamera_no_edge_geometry;

/* nonorthogonal_grid.h:12-30 */
typedef struct {
  size_t extent[3];
  gamera_no_face_geometry *value;
} gamera_no_face_grid;

typedef struct {
  size_t extent[3];
  gamera_no_edge_geometry *value;
  unsigned char *valid;
} gamera_no_edge_grid;

typedef struct {
  size_t cell_extent[3];
  size_t vertex_extent[3];
  gamera_no_vec3 *vertex;
  gamera_no_cell_geometry *cell;
  gamera_no_face_grid face[3];
  gamera_no_edge_grid edge[3];
} gamera_no_grid;

/* nonorthogonal_flux.h:21-25 */
typedef struct {
  double density;
  gamera_no_vec3 velocity;
  double pressure;
} gamera_no_primitive;

/* nonorthogonal_storage.h:12-47 */
typedef struct {
  size_t cell_extent[3];
  size_t face_extent[3][3];
  size_t edge_extent[3][3];
  double *conserved;
  double *old_conserved;
  double *predicted_conserved;
  gamera_no_vec3 *cell_magnetic;
  gamera_no_vec3 *old_cell_magnetic;
  gamera_no_vec3 *predicted_cell_magnetic;
  double *face_flux[3];
  double *old_face_flux[3];
  double *predicted_face_flux[3];
  double *edge_emf[3];
  double *fluid_face_flux[3];
  gamera_no_vec3 *maxwell_face_flux[3];
  double *hydro_rate;
  gamera_no_vec3 *maxwell_rate;
  size_t emergency_diffusion_face_count;
  double emergency_diffusion_max_interface_speed;
  size_t inner_wall_clamped_face_count[2];
  double inner_wall_positive_mass_max[2];
  double inner_wall_positive_energy_max[2];
  double inner_wall_fluid_momentum_max[2];
  double inner_wall_maxwell_momentum_max[2];
  double inner_wall_density_max[2];
  double inner_wall_pressure_max[2];
  double inner_wall_pressure_gradient_max[2];
  double inner_wall_speed_max[2];
  double inner_wall_residual_magnetic_max[2];
  gamera_no_vec3 inner_wall_residual_magnetic_location[2];
  double inner_wall_lowlat_pressure_max[2];
  double inner_wall_lowlat_pressure_gradient_max[2];
  double inner_wall_lowlat_speed_max[2];
  double inner_wall_lowlat_residual_magnetic_max[2];
} gamera_no_storage;

/* nonorthogonal_sweep.h:13-25 */
typedef struct {
  double gamma;
  double density_floor;
  double pressure_floor;
  double pdm_coefficient;
  double hydro_hogs_coefficient;
  double magnetic_hogs_coefficient;
  double light_speed;
  bool use_mhd;
  bool use_hogs;
  bool use_boris;
  bool use_background;
} gamera_no_sweep_options;

/* nonorthogonal_sweep.h:32-38 */
typedef struct {
  const gamera_no_vec3 *cell_magnetic;
  const gamera_no_vec3 *face_magnetic[3];
  const double *face_flux[3];
  const gamera_no_vec3 *edge_magnetic[3];
  const gamera_no_vec3 *cell_force;
} gamera_no_background_field;

/* nonorthogonal_sweep.h:40-49 */
typedef struct {
  double density_floor;
  double pdm_coefficient;
  double diffusion_coefficient;
  double light_speed;
  double cfl;
  double dt;
  bool use_boris;
  bool use_background;
} gamera_no_emf_options;

/* nonorthogonal_step.h:57-65 */
typedef struct {
  double gamma;
  double density_floor;
  double pressure_floor;
  double light_speed;
  bool use_mhd;
  bool use_boris;
  bool use_background;
} gamera_no_update_options;

/* nonorthogonal_step.h:67-76 */
typedef struct {
  double gamma;
  double density_floor;
  double pressure_floor;
  double cfl;
  double light_speed;
  bool use_mhd;
  bool use_boris;
  bool use_background;
} gamera_no_timestep_options;

/* nonorthogonal_advance.h:11-52 */
typedef struct {
  gamera_no_sweep_options stress;
  gamera_no_emf_options emf;
  gamera_no_update_options update;
  int (*cell_source)(gamera_no_vec3 point,
                     const double predicted[GAMERA_NO_FLUX_COUNT],
                     double time, void *context,
                     double rate[GAMERA_NO_FLUX_COUNT]);
  void *source_context;
  int (*indexed_cell_source)(
      size_t cell, gamera_no_vec3 point,
      const double predicted[GAMERA_NO_FLUX_COUNT], double time,
      void *context, double rate[GAMERA_NO_FLUX_COUNT]);
  void *indexed_source_context;
  double source_time;
  int (*fluid_flux_sync)(gamera_no_storage *storage,
                         const gamera_no_grid *grid,
                         const size_t active_lower[3],
                         const size_t active_upper[3], void *context);
  void *fluid_flux_context;
  int (*edge_emf_sync)(gamera_no_storage *storage,
                       const gamera_no_grid *grid,
                       const size_t active_lower[3],
                       const size_t active_upper[3], void *context);
  void *edge_emf_context;
} gamera_no_advance_options;

/* cubedsphere/cubedsphere_step.h:27-31 */
typedef int (*gamera_cs_radial_boundary_function)(
    const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
    gamera_no_storage storage[GAMERA_CS_FACE_COUNT],
    const size_t active[3], size_t ghost, double current_time,
    double previous_time, void *context);

/* nonorthogonal/src/nonorthogonal/nonorthogonal_mi.h:12-15 */
enum {
  GAMERA_MI_NORTH = -1,
  GAMERA_MI_SOUTH = 1
};

/* nonorthogonal_mi.h:45-57 */
typedef struct {
  size_t longitude_count;
  size_t colatitude_count;
  double maximum_colatitude;
  double ionosphere_radius_m;
  double pedersen_siemens;
  double hall_siemens;
  double low_latitude_potential_v;
  int hemisphere;
  int maximum_iterations;
  double relative_tolerance;
  double absolute_tolerance;
} gamera_mi_solver_config;

/* nonorthogonal_mi.h:59-64 */
typedef struct {
  int iterations;
  double initial_residual;
  double final_residual;
  int converged;
} gamera_mi_solver_stats;

/* nonorthogonal/src/nonorthogonal/nonorthogonal_background.h:42-45 */
typedef struct {
  gamera_no_vec3 moment;
} gamera_no_dipole;

/* cubedsphere/cubedsphere_earth_startup.h:10-24 */
typedef struct {
  double inner_radius;
  double density;
  double speed;
  double mach;
  double gamma;
  double ambient_density;
  double ambient_pressure;
  double front_x;
  double front_width;
  double cut_radius;
  double cut_length;
  gamera_no_vec3 imf;
  gamera_no_dipole dipole;
} gamera_cs_earth_startup;

/* cubedsphere/cubedsphere_mi_dipole.h:16-28 */
typedef struct gamera_cs_mi_dipole_config {
  size_t azimuth_points;
  size_t colatitude_points;
  size_t current_shell; /* zero-based active radial cell */
  double ionosphere_radius_re;
  double pedersen_siemens;
  double coupling_interval_s;
  double length_norm_m;
  double speed_norm_m_s;
  double mass_density_norm_kg_m3;
  int maximum_iterations;
  double relative_tolerance;
} gamera_cs_mi_dipole_config;

/* cubedsphere/cubedsphere_mi_dipole.h:32-39 */
typedef struct {
  size_t azimuth_points, colatitude_points;
  size_t shell_j_cells, shell_k_cells;
  double maximum_colatitude_rad, epoch_s, sample_radius_re;
  double pedersen_siemens;
  const double *fac_parallel_a_m2[2];
  const double *potential_v[2];
} gamera_cs_mi_analysis_view;

/* nonorthogonal/src/solar_wind.h:10-15 */
enum {
  GAMERA_WIND_X = 0,
  GAMERA_WIND_Y = 1,
  GAMERA_WIND_Z = 2,
  GAMERA_WIND_DIM = 3
};

/* nonorthogonal/src/solar_wind.h:17-22 */
typedef struct {
  double density;
  double pressure;
  double velocity[GAMERA_WIND_DIM];
  double magnetic[GAMERA_WIND_DIM];
} gamera_solar_wind_state;

/* nonorthogonal/src/solar_wind.h:24-35 */
typedef struct {
  size_t count;
  double *time;
  gamera_solar_wind_state *state;
  double reference[GAMERA_WIND_DIM];
  double time_offset;
  double by_coefficient;
  double bz_coefficient;
  double bx_offset;
  int enforce_bx_relation;
  int linear_interpolation;
} gamera_solar_wind_series;

struct gamera_cs_mi_dipole;

/* cubedsphere/cubedsphere_earth_boundary.h:13-24 */
typedef struct {
  const gamera_cs_earth_startup *startup;
  const gamera_solar_wind_series *wind;
  const gamera_no_background_field *background; /* six faces */
  const struct gamera_cs_mi_dipole *mi;          /* NULL: no-MI wall */
  double density_floor;
  double pressure_floor;
  double step_time;
  double step_dt;
  double cfl;
  int strict_inner_gas_wall;
} gamera_cs_earth_boundary;

#ifdef __cplusplus
}
#endif

#endif
