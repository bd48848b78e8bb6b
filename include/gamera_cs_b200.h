/*
 * libgamera_cs_b200 — B200 (sm_100a) implementation of the GAMERA-Cube
 * six-face cubed-sphere MHD step and ionosphere potential solve.
 *
 * Part 1 declares drop-in replacements for the reference C entry points:
 * same names, signatures, argument meaning and return convention (0 ok,
 * -1 error; state may be partially updated on error).  Each cites the
 * reference declaration it replaces.  All six faces are kept resident on
 * the current CUDA device; host arrays in the reference layout are uploaded
 * before and downloaded after every call unless a context is put into
 * resident mode (Part 2).
 *
 * Part 2 is the device-resident context API used by callers that keep the
 * state on the GPU between steps (benchmarks, multi-step drivers).  It has
 * no counterpart in the reference.
 */
#ifndef GAMERA_CS_B200_H
#define GAMERA_CS_B200_H

#include <stddef.h>
#include <stdint.h>

#include "gamera_cs_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- Part 1 */

/* cubedsphere/cubedsphere_halo.h:12.  Here the plan also owns the device
 * copy of the grid, its derived constants and the device state. */
typedef struct gamera_cs_halo_plan gamera_cs_halo_plan;

/* cubedsphere/cubedsphere_step.h:16-21 */
int gamera_cs_advance_six(const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
                          gamera_no_storage storage[GAMERA_CS_FACE_COUNT],
                          const size_t active[3], size_t ghost,
                          double predictor_ratio, double dt,
                          const gamera_no_advance_options *options);

/* cubedsphere/cubedsphere_step.h:33-40 */
int gamera_cs_advance_six_with_boundary(
    const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
    gamera_no_storage storage[GAMERA_CS_FACE_COUNT], const size_t active[3],
    size_t ghost, double predictor_ratio, double dt,
    const gamera_no_advance_options *options,
    gamera_cs_radial_boundary_function radial_boundary, double current_time,
    double previous_time, void *boundary_context);

/* cubedsphere/cubedsphere_step.h:46-54 */
int gamera_cs_advance_six_with_background(
    const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
    gamera_no_storage storage[GAMERA_CS_FACE_COUNT], const size_t active[3],
    size_t ghost, double predictor_ratio, double dt,
    const gamera_no_advance_options *options,
    const gamera_no_background_field background[GAMERA_CS_FACE_COUNT],
    gamera_cs_radial_boundary_function radial_boundary, double current_time,
    double previous_time, void *boundary_context);

/* cubedsphere/cubedsphere_step.h:58-67 */
int gamera_cs_advance_six_with_background_planned(
    const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
    gamera_no_storage storage[GAMERA_CS_FACE_COUNT], const size_t active[3],
    size_t ghost, double predictor_ratio, double dt,
    const gamera_no_advance_options *options,
    const gamera_no_background_field background[GAMERA_CS_FACE_COUNT],
    const gamera_cs_halo_plan *halo_plan,
    gamera_cs_radial_boundary_function radial_boundary, double current_time,
    double previous_time, void *boundary_context);

/* cubedsphere/cubedsphere_halo.h:37-40 */
int gamera_cs_halo_plan_create(const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
                               const size_t active[3], size_t ghost,
                               gamera_cs_halo_plan **out);
void gamera_cs_halo_plan_destroy(gamera_cs_halo_plan *plan);

/* cubedsphere/cubedsphere_halo.h:46-53 */
int gamera_cs_fill_tangential_cell_halos_planned(
    const gamera_cs_halo_plan *plan,
    const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
    gamera_no_storage storage[GAMERA_CS_FACE_COUNT]);
int gamera_cs_fill_magnetic_face_halos_planned(
    const gamera_cs_halo_plan *plan,
    const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
    gamera_no_storage storage[GAMERA_CS_FACE_COUNT]);

/* cubedsphere/cubedsphere_halo.h:32 */
int gamera_cs_halo_valid_state(const double state[GAMERA_NO_FLUX_COUNT]);

/* cubedsphere/cubedsphere_halo.h:52-59: as the planned fills, writing only
 * the receiver face's host arrays. */
int gamera_cs_fill_tangential_cell_halos_planned_face(
    const gamera_cs_halo_plan *plan,
    const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
    gamera_no_storage storage[GAMERA_CS_FACE_COUNT], int receiver);
int gamera_cs_fill_magnetic_face_halos_planned_face(
    const gamera_cs_halo_plan *plan,
    const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
    gamera_no_storage storage[GAMERA_CS_FACE_COUNT], int receiver);
/* cubedsphere/cubedsphere_halo.h:68-71, :84-87: unplanned fills; the device
 * plan of the grid is built on first use and shared with the step. */
int gamera_cs_fill_tangential_cell_halos(const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
                                         gamera_no_storage storage[GAMERA_CS_FACE_COUNT],
                                         const size_t active[3], size_t ghost);
int gamera_cs_fill_magnetic_face_halos(const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
                                       gamera_no_storage storage[GAMERA_CS_FACE_COUNT],
                                       const size_t active[3], size_t ghost);
/* cubedsphere/cubedsphere_halo.h:74-79 */
int gamera_cs_fill_radial_outflow_cells(gamera_no_storage storage[GAMERA_CS_FACE_COUNT],
                                        const size_t active[3], size_t ghost);
int gamera_cs_fill_radial_outflow_cells_face(
    gamera_no_storage storage[GAMERA_CS_FACE_COUNT], const size_t active[3],
    size_t ghost, int receiver);

/* cubedsphere/cubedsphere_interface.h:13-37: seam syncs of the face fluxes
 * and the signed edge-EMF means (the edge-sync plan is the device context
 * of the grid). */
int gamera_cs_sync_magnetic_face_flux(gamera_no_storage storage[GAMERA_CS_FACE_COUNT],
                                      const size_t active[3], size_t ghost);
int gamera_cs_sync_mhd_face_fluxes(gamera_no_storage storage[GAMERA_CS_FACE_COUNT],
                                   const size_t active[3], size_t ghost);
int gamera_cs_sync_edge_emf(const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
                            gamera_no_storage storage[GAMERA_CS_FACE_COUNT],
                            const size_t active[3], size_t ghost);
typedef struct gamera_cs_edge_sync_plan gamera_cs_edge_sync_plan;
int gamera_cs_edge_sync_plan_create(const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
                                    const size_t active[3], size_t ghost,
                                    gamera_cs_edge_sync_plan **out);
void gamera_cs_edge_sync_plan_destroy(gamera_cs_edge_sync_plan *plan);
int gamera_cs_sync_edge_emf_planned(const gamera_cs_edge_sync_plan *plan,
                                    gamera_no_storage storage[GAMERA_CS_FACE_COUNT]);

/* Ionosphere potential solves, host arrays in the reference layout
 * (theta-major, longitude contiguous), synchronous.  The constant-Pedersen
 * solve runs on the GPU; its stats count the GPU's own iterations (dot
 * products are summed in a fixed parallel order, so the iteration count may
 * differ from the CPU solver's by a few and the potential agrees to the
 * solver tolerance).  The apply functions are bitwise the reference's.
 * nonorthogonal/src/nonorthogonal/nonorthogonal_mi.h:70-72 */
int gamera_mi_apply_constant_pedersen(const gamera_mi_solver_config *config,
                                      const double *potential_v, double *result);
/* nonorthogonal_mi.h:81-83 */
int gamera_mi_solve_constant_pedersen(const gamera_mi_solver_config *config,
                                      const double *fac_a_m2, double *potential_v,
                                      gamera_mi_solver_stats *stats);
/* nonorthogonal_mi.h:95-98 */
int gamera_mi_apply_conductance_tensor(const gamera_mi_solver_config *config,
                                       const double *pedersen, const double *hall,
                                       const double *potential_v, double *result);
/* nonorthogonal_mi.h:99-102.  SSOR-BiCGStab on one GPU CTA: the SSOR
 * sweeps run as row wavefronts with the reference's per-point arithmetic;
 * at most 512 interior colatitude rows. */
int gamera_mi_solve_conductance_tensor(const gamera_mi_solver_config *config,
                                       const double *fac_a_m2, const double *pedersen,
                                       const double *hall, double *potential_v,
                                       gamera_mi_solver_stats *stats);

/* Magnetosphere-ionosphere coupling, cubedsphere/cubedsphere_mi_dipole.h.
 * The FAC curl, polar sampling and both potential solves of an update run
 * on the GPU holding the MHD state (the context of `grid`, shared with the
 * step calls); the potential, FAC and solver stats are then held on the
 * host, where the lookups below read them.  Potentials agree with the
 * reference to the solver tolerance (see gamera_mi_solve_constant_pedersen). */
typedef struct gamera_cs_mi_dipole gamera_cs_mi_dipole;
/* cubedsphere_mi_dipole.h:40-41 */
int gamera_cs_mi_dipole_analysis_view(const gamera_cs_mi_dipole *state,
                                      gamera_cs_mi_analysis_view *view);
/* cubedsphere_mi_dipole.h:44-46 */
int gamera_cs_mi_dipole_export_shell_current(const gamera_cs_mi_dipole *state,
                                             double *jparallel_a_m2, double *mlat_deg,
                                             double *phi_deg, size_t count);
/* cubedsphere_mi_dipole.h:51-57 */
int gamera_cs_mi_dipole_create(const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
                               gamera_no_storage storage[GAMERA_CS_FACE_COUNT],
                               const gamera_no_background_field background[GAMERA_CS_FACE_COUNT],
                               const gamera_cs_earth_startup *startup,
                               const size_t active[3], size_t ghost,
                               const gamera_cs_mi_dipole_config *config,
                               gamera_cs_mi_dipole **result);
/* cubedsphere_mi_dipole.h:58 */
void gamera_cs_mi_dipole_destroy(gamera_cs_mi_dipole *state);
/* cubedsphere_mi_dipole.h:62-65 */
int gamera_cs_mi_dipole_create_potential_view(const gamera_cs_earth_startup *startup,
                                              const gamera_cs_mi_dipole_config *config,
                                              gamera_cs_mi_dipole **result);
/* cubedsphere_mi_dipole.h:66-71 */
int gamera_cs_mi_dipole_export_potential(const gamera_cs_mi_dipole *state, double *values,
                                         size_t count, double *epoch_s,
                                         double *next_update_s);
int gamera_cs_mi_dipole_import_potential(gamera_cs_mi_dipole *state, const double *values,
                                         size_t count, double epoch_s,
                                         double next_update_s);
/* cubedsphere_mi_dipole.h:75-80 */
int gamera_cs_mi_dipole_maybe_update(gamera_cs_mi_dipole *state, double time_code);
int gamera_cs_mi_dipole_update_due(const gamera_cs_mi_dipole *state, double time_code);
int gamera_cs_mi_dipole_ready(const gamera_cs_mi_dipole *state);
/* cubedsphere_mi_dipole.h:81-88 */
int gamera_cs_mi_dipole_potential(const gamera_cs_mi_dipole *state, gamera_no_vec3 point,
                                  double *potential_v);
int gamera_cs_mi_dipole_apply_inner_emf(const gamera_cs_mi_dipole *state,
                                        gamera_no_storage *storage,
                                        const gamera_no_grid *grid, size_t wall_i);
int gamera_cs_mi_dipole_ghost_velocity(const gamera_cs_mi_dipole *state,
                                       gamera_no_vec3 point,
                                       gamera_no_vec3 source_velocity,
                                       gamera_no_vec3 *ghost_velocity);
/* cubedsphere_mi_dipole.h:89-98 */
int gamera_cs_mi_dipole_write_csv(const gamera_cs_mi_dipole *state, const char *prefix);
int gamera_cs_mi_dipole_write_shell_current_csv(const gamera_cs_mi_dipole *state,
                                                const char *prefix);
int gamera_cs_mi_dipole_stats(const gamera_cs_mi_dipole *state, double *fac_min,
                              double *fac_max, double *potential_min_v,
                              double *potential_max_v, gamera_mi_solver_stats solve[2]);

/* ---------------------------------------------------------------- Part 2 */

typedef struct gcs_context gcs_context;

/* Stage codes reported by gcs_context_failure (first failing stage). */
enum {
  GCS_STAGE_NONE = 0,
  GCS_STAGE_PREDICT = 1,
  GCS_STAGE_RECOVER_PREDICT = 2,
  GCS_STAGE_RECONSTRUCT = 3,
  GCS_STAGE_KINETIC_FLUID = 4,
  GCS_STAGE_KINETIC_MAXWELL = 5,
  GCS_STAGE_EMERGENCY = 6,
  GCS_STAGE_EDGE_GEOMETRY = 7,
  GCS_STAGE_EDGE_VELOCITY = 8,
  GCS_STAGE_TRANSVERSE = 9,
  GCS_STAGE_EDGE_DENSITY = 10,
  GCS_STAGE_EDGE_EMF = 11,
  GCS_STAGE_UPDATE = 12,
  GCS_STAGE_RECOVER_UPDATE = 13,
  GCS_STAGE_RECOVER_FINAL = 14,
  GCS_STAGE_TIMESTEP = 15,
  GCS_STAGE_HOST = 16,
  GCS_STAGE_SOLVE_EDGE = 17,
  GCS_STAGE_OPTIONS = 18,
  GCS_STAGE_PRESSURE_CONTROL = 19,
  GCS_STAGE_TILE_COPY = 20,
  GCS_STAGE_MI_COUPLING = 21
};

/* Build a device context from a host grid in the reference layout
 * (all six faces; active[1] == active[2] >= 9; ghost == 4).  Returns NULL on
 * failure; gcs_last_error() then describes it. */
gcs_context *gcs_context_create(const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
                                const size_t active[3], size_t ghost);
void gcs_context_destroy(gcs_context *ctx);
const char *gcs_last_error(void);

/* Build a case directly in device memory (no host grid): kind 0 uniform MHD
 * state (r in [2, 2.5]), 1 radial MHD shock (r in [2, 3]), 2 solar wind
 * with aligned dipole B0 and seeded +-1% density noise (log-stretched r in
 * [2.5, 30] R_E), 3 the wind with a 20% density pulse; nr radial and n
 * angular active cells per face, 4 ghosts.  Same inputs as the oracle's
 * case set up to device-libm rounding. */
gcs_context *gcs_context_create_case(int kind, size_t nr, size_t n,
                                     unsigned long long seed);
/* Step, CFL and driver options of a case kind. */
int gcs_case_options(int kind, gamera_no_advance_options *options,
                     gamera_no_timestep_options *timestep);
int gcs_context_dims(const gcs_context *ctx, size_t active[3], size_t *ghost);
/* Diagnostics: copy one device geometry/background node array of one face
 * (nodes_per_face = (nr+9)(n+9)^2 doubles, padded node index) to out. */
int gcs_context_debug_array(gcs_context *ctx, int which, int face, int d, int q,
                            double *out, size_t capacity);
/* The drop-in step of gamera_cs_advance_six_with_background_planned on
 * host storage (state uploaded before, downloaded after the step) for a
 * context built by gcs_context_create_case, which owns its grid and
 * background. */
int gcs_context_advance_host(gcs_context *ctx,
                             gamera_no_storage storage[GAMERA_CS_FACE_COUNT],
                             const gamera_no_advance_options *options,
                             double predictor_ratio, double dt);
const char *gcs_context_error(const gcs_context *ctx);

int gcs_context_upload_background(
    gcs_context *ctx,
    const gamera_no_background_field background[GAMERA_CS_FACE_COUNT]);
int gcs_context_upload_state(gcs_context *ctx,
                             const gamera_no_storage storage[GAMERA_CS_FACE_COUNT]);
/* include_scratch != 0 also downloads predicted arrays, fluid/Maxwell face
 * fluxes and edge EMFs of the last step. */
int gcs_context_download_state(gcs_context *ctx,
                               gamera_no_storage storage[GAMERA_CS_FACE_COUNT],
                               int include_scratch);

/* One step on the device-resident state (no host transfers); same stage
 * order and options as gamera_cs_advance_six_with_background_planned with
 * outflow radial ghosts and no callbacks. */
int gcs_context_step(gcs_context *ctx, const gamera_no_advance_options *options,
                     double predictor_ratio, double dt);

/* Minimum CFL step over the active cells of all faces
 * (nonorthogonal_step.c:449-525, reduced over the six faces). */
int gcs_context_timestep(gcs_context *ctx,
                         const gamera_no_timestep_options *options,
                         double *dt);

/* Driver loop on the device: before the first call the step size is
 * dt_fraction * timestep; each step then sets
 * dt = min(dt_fraction * cfl_min, 1.25 dt_prev) and the predictor ratio
 * 0.5 dt / dt_prev on the device.  use_graph != 0 replays one captured
 * CUDA graph per step.  Does not synchronise; call gcs_context_sync. */
int gcs_context_run(gcs_context *ctx, const gamera_no_advance_options *options,
                    const gamera_no_timestep_options *timestep,
                    double dt_fraction, int steps, int use_graph);
int gcs_context_sync(gcs_context *ctx);
/* Simulation time (code units) of the state in the device driver loop: the
 * sum of the time steps gcs_context_run has taken. */
int gcs_context_time(gcs_context *ctx, double *time);
int gcs_context_params(gcs_context *ctx, double *dt, double *ratio,
                       double *cfl_min, int *steps);
int gcs_context_set_params(gcs_context *ctx, double dt, double ratio,
                           double dt_prev, int steps);
/* First failure since the last reset; returns the stage code (0 = none). */
int gcs_context_failure(gcs_context *ctx, int *dir, int *face, int *i, int *j,
                        int *k);
int gcs_context_reset_failure(gcs_context *ctx);
/* The CUDA stream (cudaStream_t) every kernel of this context runs on. */
uintptr_t gcs_context_stream(gcs_context *ctx);
/* Profiling: record CUDA events around each stage of every step. */
int gcs_context_set_profiling(gcs_context *ctx, int on);
/* Flux sweeps with the Up7 stencil cells staged in shared memory by TMA
 * (on = 1) or read per face from global memory (on = 0, the default, the
 * faster of the two on B200); the two give the same fluxes bit for bit. */
int gcs_context_set_flux_staging(gcs_context *ctx, int on);
/* Accumulated device milliseconds and launch counts per stage since
 * profiling was switched on; returns the number of stages written. */
int gcs_context_stage_times(gcs_context *ctx, double *ms, long long *calls,
                            int capacity);
const char *gcs_stage_name(int stage_slot);
size_t gcs_context_device_bytes(const gcs_context *ctx);
/* Allocation-free CFL time step.  No counterpart in the reference: an
 * addition for callers that cannot call cudaMalloc when they need the step
 * (device arrays owned by another allocator or runtime, or a driver that
 * forbids device allocation after start-up).  Inputs are caller-owned
 * DEVICE arrays in the reference layout (cells: gamera_no_cell_geometry per
 * cell; conserved: 5 doubles per cell; cell and background B: one vec3 per
 * cell, NULL where the options do not use them); the minimum over the
 * active box of the reference cell step (the quantity
 * gamera_no_local_timestep computes) is returned in *local_dt on the host.
 * No device memory is allocated or freed: the reduction uses a static
 * device array of gcs_noalloc_scratch_bytes() bytes (about 768 KiB) that
 * every GPU loading this library holds until exit.  At most 16,777,216
 * active cells per call; larger boxes are rejected with -1 and a message in
 * gcs_noalloc_last_error().  Every call looks up the array's device
 * address in the current context (an address kept from before a
 * cudaDeviceReset would be stale), so make calls outside stream capture.
 * Under CUDA's default lazy module loading the array is loaded onto a
 * device by the first call there: a caller that must fix its footprint at
 * start-up makes one call then (or sets CUDA_MODULE_LOADING=EAGER); later
 * calls change the device footprint by nothing.  Calls share the array:
 * calls that overlap on the GPU race and must be serialised.  A failed
 * kernel launch returns -1.  Runs on the default stream and returns after
 * the result is on the host. */
int gcs_local_timestep_noalloc(const size_t cell_extent[3],
                               const gamera_no_cell_geometry *cells,
                               const double *conserved,
                               const gamera_no_vec3 *cell_magnetic,
                               const gamera_no_vec3 *background_cell_magnetic,
                               const size_t active_lower[3],
                               const size_t active_upper[3],
                               const gamera_no_timestep_options *options,
                               double *local_dt);
const char *gcs_noalloc_last_error(void);
size_t gcs_noalloc_scratch_bytes(void);

/* Resident mode: the device copy stays authoritative between drop-in calls
 * made with the same storage pointer; gcs_context_download_state copies it
 * back explicitly. */
gcs_context *gcs_halo_plan_context(gamera_cs_halo_plan *plan);
int gcs_context_set_resident(gcs_context *ctx, int on);

/* FP32-bulk precision variant (no reference counterpart).  With fp32_bulk
 * set, the flux, face-velocity and edge-EMF sweeps compute in FP32 from
 * FP32 copies of the metric, background, cell primitives and face fields
 * (outside the strong-dipole layers, below) and store FP64 results; the
 * conserved state, face B flux, predictor, B recovery, CT and cell update
 * stay FP64, so div B stays at FP64 round-off.  The FP32 copies (108
 * floats per node) are allocated and converted on first use and follow
 * later background uploads.  Host callbacks need the FP64 path. */
int gcs_context_set_precision(gcs_context *ctx, int fp32_bulk);
int gcs_context_precision(const gcs_context *ctx);
/* Radial layers whose largest cell |B0| exceeds b0_threshold (code units,
 * default 8), and every layer inside them, keep the FP64 sweeps in the
 * FP32-bulk path: there the residual field is small against the dipole and
 * FP32 rounding of the B0 cross terms of the Maxwell stress and EMF would
 * dominate their differences.  gcs_context_bulk_split returns the first
 * FP32 radial layer (cell index, ghosts included). */
int gcs_context_set_bulk_threshold(gcs_context *ctx, double b0_threshold);
int gcs_context_bulk_split(const gcs_context *ctx);

/* The reference's Earth radial-boundary callbacks
 * (cubedsphere/cubedsphere_earth_boundary.h:26-52), same signatures and
 * results.  Passed to the drop-in step (radial_boundary =
 * gamera_cs_earth_fill_radial_ghosts with options->fluid_flux_sync =
 * gamera_cs_earth_inner_fluid_flux, options->edge_emf_sync =
 * gamera_cs_earth_no_mi_emf and the same boundary as both contexts), they
 * run as device kernels inside the step with no host round trip, a ready
 * MI coupling included (its potential copied to the device each step);
 * called directly they work on host storage (the radial fill through the
 * grid's device context). */
int gamera_cs_earth_fill_radial_ghosts(const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
                                       gamera_no_storage storage[GAMERA_CS_FACE_COUNT],
                                       const size_t active[3], size_t ghost,
                                       double current_time, double previous_time,
                                       void *context);
int gamera_cs_earth_fill_radial_ghosts_face(const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
                                            gamera_no_storage storage[GAMERA_CS_FACE_COUNT],
                                            const size_t active[3], size_t ghost,
                                            double current_time, double previous_time,
                                            void *context, int face);
int gamera_cs_earth_inner_fluid_flux(gamera_no_storage *storage, const gamera_no_grid *grid,
                                     const size_t lower[3], const size_t upper[3],
                                     void *context);
int gamera_cs_earth_no_mi_emf(gamera_no_storage *storage, const gamera_no_grid *grid,
                              const size_t lower[3], const size_t upper[3], void *context);

/* Device Earth radial boundary (no-MI wall) of a context made from a host
 * grid: the reference callbacks gamera_cs_earth_fill_radial_ghosts
 * (radial ghost cells and faces of the state and old state at both shells,
 * cell B recovered, cubedsphere_earth_boundary.c:27-212),
 * gamera_cs_earth_inner_fluid_flux (:259-266) and gamera_cs_earth_no_mi_emf
 * (:298-451) as kernels at the reference step's callback positions.
 * gcs_earth_create copies the boundary layers' geometry from `grid`, the
 * outer faces' B0 flux from boundary->background and the monitor series
 * boundary->wind to the device; with boundary->mi set, each step uses its
 * potential while it is ready (MI-coupled wall: E x B drift ghost velocity,
 * inner-shell EMF from the potential). */
typedef struct gcs_earth gcs_earth;
int gcs_earth_create(gcs_context *ctx, const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
                     const gamera_cs_earth_boundary *boundary, gcs_earth **earth);
/* The same for a device-built wind case (gcs_context_create_case kind 2/3,
 * gcs_context_create_wind): the boundary layers' geometry is rebuilt on the
 * device and the outer faces' B0 flux taken from the context's background
 * (boundary->background may be NULL). */
int gcs_earth_create_case(gcs_context *ctx, const gamera_cs_earth_boundary *boundary,
                          gcs_earth **earth);
/* Replace the monitor time series (e.g. a longer one). */
int gcs_earth_set_wind(gcs_earth *earth, const gamera_solar_wind_series *wind);
void gcs_earth_destroy(gcs_earth *earth);
size_t gcs_earth_device_bytes(const gcs_earth *earth);
/* Diagnostics: copy the boundary-layer geometry (cell centroids; per face
 * family outer ghost-face centroids, area vectors, B0 flux; per edge family
 * midpoints, directions, lengths; edge validity bytes; node-plane layout of
 * 2g, g and 5 layers per face) to `host` when capacity suffices; returns
 * its size in bytes. */
size_t gcs_earth_copy_layers(const gcs_earth *earth, void *host, size_t capacity);
/* One step on the device-resident state with the device Earth boundary:
 * gamera_cs_advance_six_with_background_planned(..., radial_boundary =
 * gamera_cs_earth_fill_radial_ghosts, current_time, previous_time,
 * boundary) with options->fluid_flux_sync = gamera_cs_earth_inner_fluid_flux
 * and options->edge_emf_sync = gamera_cs_earth_no_mi_emf, the boundary's
 * step_time = current_time and step_dt = dt as the reference driver sets
 * them (test_cubedsphere_dipole_background.c:667-668).  Callbacks in
 * `options` are not called. */
int gcs_context_step_earth(gcs_context *ctx, gcs_earth *earth,
                           const gamera_no_advance_options *options,
                           double predictor_ratio, double dt, double current_time,
                           double previous_time);
/* The driver loop of gcs_context_run with the device Earth boundary: its
 * times come from the device step parameters (current time t, previous
 * t - dt_prev or t on the first step, EMF at t + dt/2), so with use_graph
 * each step is one CUDA graph launch and needs no host synchronisation.
 * The simulation time starts at 0 with the context's first driver step.
 * The MI potential (boundary->mi at creation) is the one current at the
 * call. */
int gcs_context_run_earth(gcs_context *ctx, gcs_earth *earth,
                          const gamera_no_advance_options *options,
                          const gamera_no_timestep_options *timestep, double dt_fraction,
                          int steps, int use_graph);

/* Post-step pressure control of the Earth drivers
 * (nonorthogonal/src/nonorthogonal/nonorthogonal_step.h:26-32
 * gamera_no_apply_pressure_control, called after each step by
 * cubedsphere/tests/test_cubedsphere_mpi_earth_tile.c:459-481 with gamma,
 * 1e-6, 1e-8, 10, 1e-3, 1e-7).  The arguments after dt, same meaning. */
typedef struct gcs_pressure_control {
  double gamma;
  double density_floor;
  double pressure_floor;
  double light_speed;
  double low_density_threshold;
  double low_density_sound_speed;
} gcs_pressure_control;
/* gamera_no_apply_pressure_control over the active cells of all six faces
 * of a device-resident state, on the device: counts summed over the faces,
 * maxima over them.  The dipole line lengths come from `grid` (the host
 * grid of the context) or, for a device-built case, grid NULL, from its
 * device-built centroids; computed on the first call and kept.  -1 on an
 * invalid argument or a failed cell, as the reference (other cells
 * updated). */
int gcs_context_pressure_control(gcs_context *ctx, const gamera_no_grid *grid, double dt,
                                 const gcs_pressure_control *config,
                                 size_t *low_density_cell_count,
                                 size_t *high_sound_speed_cell_count,
                                 double *maximum_sound_speed, double *maximum_pressure);
/* Run the pressure control after every step of the device driver loop
 * (gcs_context_run, gcs_context_run_earth; inside the step's CUDA graph,
 * dt from the step parameters, the next CFL step from the controlled
 * state); config NULL turns it off.  Counts accumulate over the steps and
 * maxima are taken over them until read with reset; a failed cell fails
 * the step (stage "pressure_control"). */
int gcs_context_set_pressure_control(gcs_context *ctx, const gamera_no_grid *grid,
                                     const gcs_pressure_control *config);
/* Counters of the driver-loop pressure control; 0, 1 when a cell failed,
 * -1 on error.  reset != 0 zeroes them (stream-ordered). */
int gcs_context_pressure_control_stats(gcs_context *ctx, size_t *low_density_cell_count,
                                       size_t *high_sound_speed_cell_count,
                                       double *maximum_sound_speed, double *maximum_pressure,
                                       int reset);

/* Analysis output (cubedsphere/cubedsphere_analysis_hdf5.c:299-355,
 * cubedsphere/docs/OUTPUT_DATA_MODEL.md).  The frame of a face is float32
 * [8][nr][n][n]: rho, p, vx, vy, vz (primitives with floors 1e-12 and the
 * given gamma) and Bx, By, Bz (residual plus cell B0 where the context has a
 * background) over the active cells; six faces in order.  Computed on the
 * device into `device_out` (gcs_analysis_frame_floats floats) and/or
 * copied to `host_out`.  Fails on an invalid state or a non-finite field,
 * as the reference writer does. */
size_t gcs_analysis_frame_floats(const gcs_context *ctx);
int gcs_context_analysis_frame(gcs_context *ctx, double gamma, float *device_out,
                               float *host_out);
/* The reference's per-face file set in `directory` with raw little-endian
 * datasets and JSON metadata in place of HDF5: analysis_grid_p<f>.json with
 * .coordinates.f64 [3][nr][n][n] and .vertices.f64 [3][nr+1][n+1][n+1]
 * (written when absent; from `grid`, or rebuilt on the device for a
 * device-built case when grid is NULL), and analysis_p<f>_<sequence:06>.json
 * with .state.f32 (the frame) and the reference's metadata datasets. */
int gcs_context_write_analysis(gcs_context *ctx, const char *directory, long sequence,
                               long step, double time_code, double time_seconds,
                               double gamma, const gamera_no_grid *grid);

/* Upstream solar wind of a wind run (no reference counterpart; the
 * reference driver fixes it at n = 5 cm^-3, V = -400 km/s, T = 1e5 K,
 * Bz = -5 nT, test_cubedsphere_dipole_background.c:282-294): density
 * (proton cm^-3, before the seeded +-1% noise), Vx (km/s), proton
 * temperature (K), IMF Bz (nT). */
typedef struct gcs_wind_driver {
  double density_cm3;
  double velocity_x_kms;
  double temperature_k;
  double bz_nt;
} gcs_wind_driver;

/* The wind case (gcs_context_create_case kind 2: log-stretched r in
 * [2.5, 30] R_E, aligned dipole, seeded +-1% density noise) with the given
 * upstream driver. */
gcs_context *gcs_context_create_wind(size_t nr, size_t n, unsigned long long seed,
                                     const gcs_wind_driver *driver);

/* Launch tiles (no reference counterpart).  A kernel family's thread block
 * is a tile of bx consecutive points of the flattened (j, k) plane of a
 * radial layer times by radial layers; bx * by must be a multiple of 32 and
 * at most gcs_tile_limit(family).  Tiles change speed, never results.
 * Defaults: 64 x 1 for the flux and edge-EMF sweeps, 128 x 1 otherwise. */
enum {
  GCS_TILE_PREDICT = 0,
  GCS_TILE_FLUX = 1,
  GCS_TILE_FACE_VELOCITY = 2,
  GCS_TILE_EDGE_EMF = 3,
  GCS_TILE_CT = 4,
  GCS_TILE_UPDATE = 5,
  GCS_TILE_RECOVER = 6,
  GCS_TILE_FAMILIES = 7
};
int gcs_tile_limit(int family);
int gcs_context_set_tile(gcs_context *ctx, int family, int bx, int by);
int gcs_context_tile(const gcs_context *ctx, int family, int *bx, int *by);
/* Autotuner: for the predictor, flux, face-velocity, edge-EMF and
 * recovery/CFL families, times every candidate tile (`repetitions`
 * launches each, CUDA events on the context stream) on the context's
 * current state and keeps the fastest.  These kernels write only per-step
 * scratch, so the state is unchanged; CT and the cell update keep their
 * tile.  best_ms / default_ms (nullable, GCS_TILE_FAMILIES entries, 0 for
 * untuned families) receive the chosen and the default tile's ms per
 * launch sequence.  Needs a context with a background (wind case). */
int gcs_context_autotune(gcs_context *ctx, const gamera_no_advance_options *options,
                         const gamera_no_timestep_options *timestep, int repetitions,
                         double best_ms[GCS_TILE_FAMILIES],
                         double default_ms[GCS_TILE_FAMILIES]);

/* Ensembles (no reference counterpart): independent wind runs of uneven
 * resolution and different drivers advanced together, one CUDA graph per
 * ensemble step, each run with its own device time step
 * (dt = min(dt_fraction * CFL step, 1.25 dt_prev), as gcs_context_run) and
 * failure status.  Runs of equal (nr, n) share the grid (geometry,
 * background, plans, FP32 metric, per-step scratch) of the first run of
 * that size and own only their state; they run one after another inside
 * the step, runs of different sizes concurrently.  Run i uses the noise
 * seed `seed + i` and the options of gcs_case_options(2). */
typedef struct gcs_ensemble gcs_ensemble;
typedef struct gcs_ensemble_config {
  int count;
  const size_t *nr;                 /* radial active cells per run */
  const size_t *n;                  /* angular active cells per run */
  const gcs_wind_driver *drivers;   /* one per run */
  unsigned long long seed;
  int fp32_bulk;                    /* FP32-bulk sweeps for every run */
  int autotune_repetitions;         /* 0: default tiles; else tune each grid */
  double dt_fraction;               /* 0.5 in the reference driver */
} gcs_ensemble_config;
/* Seeded draw of `count` runs: angular size from {48, 64, 96, 128} (the
 * radial size is the caller's; 2n in the ensemble benchmark) and drivers
 * uniform in Bz [-10, 5] nT, Vx [-800, -300] km/s, n [1, 20] cm^-3,
 * T [5e4, 2e5] K.  Either output may be NULL. */
int gcs_ensemble_draw(unsigned long long seed, int count, size_t *n,
                      gcs_wind_driver *drivers);
/* Device bytes an ensemble of these sizes needs (host arithmetic). */
double gcs_ensemble_estimate_bytes(int count, const size_t *nr, const size_t *n,
                                   int fp32_bulk);
/* NULL on failure (gcs_last_error(); also when the estimate exceeds the
 * free device memory). */
gcs_ensemble *gcs_ensemble_create(const gcs_ensemble_config *config);
void gcs_ensemble_destroy(gcs_ensemble *ensemble);
int gcs_ensemble_count(const gcs_ensemble *ensemble);
/* Run i's context (borrowed; for state downloads, parameters, failures). */
gcs_context *gcs_ensemble_run_context(gcs_ensemble *ensemble, int run);
/* Index of the run whose grid run i uses (i itself for the first run of a
 * size). */
int gcs_ensemble_grid_owner(const gcs_ensemble *ensemble, int run);
/* Enqueue `steps` ensemble steps (graph launches) on the ensemble stream;
 * the first call sets every run's first step size and captures the graph.
 * Does not synchronise. */
int gcs_ensemble_advance(gcs_ensemble *ensemble, int steps);
/* Wait, then check every run's status; *failed_run = first failed run or
 * -1. */
int gcs_ensemble_sync(gcs_ensemble *ensemble, int *failed_run);
uintptr_t gcs_ensemble_stream(gcs_ensemble *ensemble);
size_t gcs_ensemble_device_bytes(const gcs_ensemble *ensemble);
/* Nodes of the captured step graph and number of distinct grids. */
int gcs_ensemble_graph_info(const gcs_ensemble *ensemble, int *nodes, int *grids);

/* Device-resident ionosphere solves (no reference counterpart).  A plan
 * holds `count` independent systems on one polar grid (for example the two
 * hemispheres, configs differing in `hemisphere`); one solve launch runs
 * them concurrently, one thread-block cluster each, entirely on chip.
 * Arrays are count x colatitude_count x longitude_count doubles in device
 * memory; NULL selects the plan's own buffers (gcs_mi_plan_buffers).  The
 * launch is asynchronous on `stream` (a cudaStream_t, NULL = default);
 * gcs_mi_plan_results waits for it and returns per-system stats and status
 * (0 converged, 1 not converged, 2 non-finite FAC: potential untouched).
 * Grids up to about 100,000 unknowns per system are supported; larger ones
 * fail at plan creation.  maximum_iterations is clamped to 1,048,576. */
typedef struct gcs_mi_plan gcs_mi_plan;
/* Device buffers of the tensor solve for one configuration (no reference
 * counterpart): fill the plan's buffers (gcs_mi_tensor_plan_buffers:
 * FAC, Pedersen, Hall, initial potential, nt x np each), launch, read the
 * stats and status (0 converged, 1 not converged, 2 non-finite FAC). */
typedef struct gcs_mi_tensor_plan gcs_mi_tensor_plan;
int gcs_mi_tensor_plan_create(const gamera_mi_solver_config *config,
                              gcs_mi_tensor_plan **plan);
void gcs_mi_tensor_plan_destroy(gcs_mi_tensor_plan *plan);
int gcs_mi_tensor_plan_buffers(gcs_mi_tensor_plan *plan, double **fac, double **pedersen,
                               double **hall, double **potential);
int gcs_mi_tensor_plan_upload(gcs_mi_tensor_plan *plan, const double *fac,
                              const double *pedersen, const double *hall,
                              const double *potential);
int gcs_mi_tensor_solve_async(gcs_mi_tensor_plan *plan, void *stream);
/* Ordering of the SSOR preconditioner (no reference counterpart): 0 the
 * reference's row-by-row sweeps (default; one warp advances a wavefront),
 * 1 the same splitting with the unknowns ordered by colour (pole; (row +
 * longitude) parity off the seam column; row parity on it), each colour
 * swept by the whole cluster at once.  Both solve to the configured
 * tolerance; the iteration counts differ. */
int gcs_mi_tensor_plan_set_ordering(gcs_mi_tensor_plan *plan, int colored);
/* Schedule of the row-by-row sweeps (no reference counterpart): 1 the band
 * pipeline (available where each CTA of the cluster gets at most 32
 * interior rows and the band's coefficients fit in shared memory; the
 * default on grids of fewer than 17 longitudes), each CTA sweeping its band
 * of rows and passing its edge row to the next CTA; 0 one warp advancing
 * the whole wavefront (the default elsewhere).  Both compute the same
 * preconditioner with the same operations and give identical results.  -1
 * when the plan has no band schedule.  gcs_mi_tensor_plan_schedule returns
 * 1 (band, with the rows per band and the band count), 0 (one warp) or -1. */
int gcs_mi_tensor_plan_set_schedule(gcs_mi_tensor_plan *plan, int banded);
int gcs_mi_tensor_plan_schedule(const gcs_mi_tensor_plan *plan, int *rows_per_band,
                                int *bands);
int gcs_mi_tensor_results(gcs_mi_tensor_plan *plan, gamera_mi_solver_stats *stats,
                          int *status);
/* Ionosphere coupling of a device-built case (gcs_context_create_case with
 * a background): as gamera_cs_mi_dipole_create, with the state, geometry
 * and B0 taken from the context; the shell must lie within the innermost
 * four active layers (current_shell <= 2).  No reference counterpart. */
int gcs_context_mi_dipole_create(gcs_context *ctx, const gamera_cs_earth_startup *startup,
                                 const gamera_cs_mi_dipole_config *config,
                                 gamera_cs_mi_dipole **result);
/* The coupling update inside the device driver loop (gcs_context_run,
 * gcs_context_run_earth): before every step the step's CUDA graph
 * evaluates the coupling's cadence on the device and, when it is due, runs
 * the FAC kernels and both hemisphere solves, with no host round trip.
 * every_steps = 0 keeps the reference's rule on the simulation time of the
 * state (cubedsphere_mi_dipole.c:372-378, gamera_cs_mi_dipole_maybe_update
 * with the driver's time); every_steps = n updates before every n-th step
 * (and before the first).  A failed update fails the step (stage
 * GCS_STAGE_MI_COUPLING).  An Earth boundary with this coupling as its MI
 * wall reads the potential on the device.  The coupling's host entry points
 * see the device's state after the run.  The caller does not also call
 * gamera_cs_mi_dipole_maybe_update for steps run this way.  mi = NULL
 * detaches.  No reference counterpart. */
int gcs_context_set_mi_coupling(gcs_context *ctx, gamera_cs_mi_dipole *mi, int every_steps);
int gcs_mi_plan_create(const gamera_mi_solver_config *configs, int count,
                       gcs_mi_plan **plan);
/* Plain PCG on the variable-Pedersen, Hall-free operator.  No reference
 * counterpart: the reference solves the conductance tensor by SSOR-BiCGStab
 * (gamera_mi_solve_conductance_tensor); with Hall = 0 and a single pole
 * conductance (pedersen row 0 uniform) that operator is symmetric positive
 * definite, and this is Jacobi-preconditioned CG on it: the five-point
 * stencil of nonorthogonal_mi.c:744-865 with Hall = 0, the reference
 * tensor solve's right-hand side and residual norm
 * (nonorthogonal_mi.c:1000-1044, :415-431), true-residual check at
 * convergence and every 1024 iterations.  pedersen: count * nt * np values
 * (row 0 = pole).  The plan solves through gcs_mi_solve_constant_pedersen_async
 * and reports through gcs_mi_plan_results like a constant-Pedersen plan. */
int gcs_mi_plan_create_pedersen(const gamera_mi_solver_config *configs,
                                const double *pedersen, int count, gcs_mi_plan **plan);
/* The same solve on host arrays, synchronous (0 converged, -1 otherwise). */
int gcs_mi_solve_pedersen_pcg(const gamera_mi_solver_config *config, const double *fac_a_m2,
                              const double *pedersen, double *potential_v,
                              gamera_mi_solver_stats *stats);
void gcs_mi_plan_destroy(gcs_mi_plan *plan);
int gcs_mi_plan_info(const gcs_mi_plan *plan, int *cluster_ctas,
                     int *threads_per_cta, size_t *shared_bytes);
int gcs_mi_plan_buffers(gcs_mi_plan *plan, double **fac, double **potential);
int gcs_mi_solve_constant_pedersen_async(gcs_mi_plan *plan, const double *fac,
                                         double *potential, void *stream);
int gcs_mi_plan_results(gcs_mi_plan *plan, gamera_mi_solver_stats *stats,
                        int *status);

/* Learned preconditioner of the conductance-tensor ionosphere solve (no
 * reference counterpart): a four-level convolutional network on the polar
 * grid (interior rows x longitudes, padded to H0 x W0: gcs_mi_net_info), BF16
 * weights and activations with FP32 accumulation on the tensor cores.
 * Inputs [B][4][H0][W0] and outputs / targets [B][H0][W0] are FP32 device
 * arrays.  Parameters are exchanged packed: per convolution and output
 * channel, 9 x input-channel weights then the bias (gradients = 1 returns
 * the gradients of the last training step instead). */
typedef struct gcs_mi_net gcs_mi_net;
int gcs_mi_net_create(int interior_rows, int longitudes, int max_batch, unsigned seed,
                      gcs_mi_net **net);
void gcs_mi_net_destroy(gcs_mi_net *net);
int gcs_mi_net_info(const gcs_mi_net *net, int *H0, int *W0, int *params,
                    int *in_channels);
int gcs_mi_net_get_params(gcs_mi_net *net, float *params, int count, int gradients);
int gcs_mi_net_set_params(gcs_mi_net *net, const float *params, int count);
int gcs_mi_net_forward(gcs_mi_net *net, const float *inputs, int batch, float *outputs);
/* Loss sum over valid points of (output - target)^2 / (batch x rows x
 * longitudes) and its gradients; update != 0 applies one Adam step. */
int gcs_mi_net_train_step(gcs_mi_net *net, const float *inputs, const float *targets,
                          int batch, float learning_rate, int update, float *loss);
/* The conductance-tensor solve (arguments, validation and result as
 * gamera_mi_solve_conductance_tensor, nonorthogonal_mi.h:96-102) by flexible
 * GMRES(40) on the reduced system, its rows scaled so that the residual
 * 2-norm is the reference's residual norm, left-preconditioned by a linear
 * L and right-preconditioned by a flexible N.  Method 0: L the two-level
 * step (a coarse correction on ring means -- one value per colatitude ring
 * and the pole -- two damped Jacobi steps, the coarse correction again) and
 * N the network (net, built for interior_rows = colatitude_count - 2 and
 * longitudes = longitude_count); 1: L Jacobi, N the identity; 2: L the
 * two-level step, N the identity.  Convergence is judged on the FP64 true
 * residual against the reference's target at every restart.  If
 * maximum_iterations pass without convergence, the reference algorithm
 * continues from the iterate and *fallback is set to 1.  No reference
 * counterpart. */
int gcs_mi_solve_conductance_tensor_learned(gcs_mi_net *net, int method,
                                            const gamera_mi_solver_config *config,
                                            const double *fac_a_m2, const double *pedersen,
                                            const double *hall, double *potential_v,
                                            gamera_mi_solver_stats *stats, int *fallback);
/* One application of the learned solve's scaled operator (what = 1), its
 * left preconditioner L (what = 0) or its right preconditioner N (what = 2)
 * for `method` to a host vector of the reduced
 * system (1 + (colatitude_count - 2) longitude_count doubles), for checking
 * them against a CPU restatement.  No reference counterpart. */
int gcs_mi_learned_apply(gcs_mi_net *net, int method, int what,
                         const gamera_mi_solver_config *config, const double *pedersen,
                         const double *hall, const double *v, double *y);

#ifdef __cplusplus
}
#endif

#endif
