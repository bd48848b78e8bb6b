/*
 * CPU restatement of the GAMERA-Cube cubed-sphere hot path (test oracle).
 *
 * TEST INFRASTRUCTURE: plain C99 restatement, operating on the reference
 * data layout (include/gamera_cs_types.h), of the reference algorithms that
 * the CUDA library replaces, plus the case set-up they need.  It exists to
 * check the CUDA library; the library never links or calls it.  Each
 * function cites the reference file:line it restates, keeps the reference's
 * operation order, and is checked bit for bit against the reference itself
 * (tests/test_oracle.py) and against the committed golden vectors
 * (tests/golden/).
 */
#ifndef GCS_ORACLE_H
#define GCS_ORACLE_H

#include "gamera_cs_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gcso_case gcso_case;
typedef struct gcso_halo_plan gcso_halo_plan;
typedef struct gcso_edge_plan gcso_edge_plan;

/* Background field arrays owned by the oracle (the dipole B0 of
 * nonorthogonal_background.c:273-442). */
typedef struct {
  gamera_no_background_field field;
  gamera_no_vec3 *cell_magnetic;
  gamera_no_vec3 *face_magnetic[3];
  double *face_flux[3];
  gamera_no_vec3 *edge_magnetic[3];
  gamera_no_vec3 *cell_force;
} gcso_background;

int gcso_generate_vertices(int face, const size_t active[3], size_t ghost,
                           double r_inner, double r_outer, double stretch,
                           gamera_no_vec3 *vertices);
int gcso_grid_create(const size_t cell_extent[3], const gamera_no_vec3 *v,
                     gamera_no_grid *grid);
void gcso_grid_destroy(gamera_no_grid *grid);
int gcso_calibrate_face_frames(gamera_no_grid *grid);
int gcso_storage_create(const size_t cell_extent[3], gamera_no_storage *s);
void gcso_storage_destroy(gamera_no_storage *s);
int gcso_background_create(const gamera_no_grid *grid, gamera_no_vec3 moment,
                           gcso_background *bg);
void gcso_background_destroy(gcso_background *bg);

int gcso_halo_plan_create(const gamera_no_grid grid[6], const size_t active[3],
                          size_t ghost, gcso_halo_plan **out);
void gcso_halo_plan_destroy(gcso_halo_plan *plan);
int gcso_edge_plan_create(const size_t active[3], size_t ghost,
                          gcso_edge_plan **out);
void gcso_edge_plan_destroy(gcso_edge_plan *plan);

int gcso_fill_cell_halos(const gcso_halo_plan *p, gamera_no_storage st[6]);
int gcso_fill_face_halos(const gcso_halo_plan *p, const gamera_no_grid grid[6],
                         gamera_no_storage st[6]);
int gcso_fill_radial_outflow(gamera_no_storage st[6], const size_t act[3], size_t g);
int gcso_sync_faces(gamera_no_storage st[6], const size_t act[3], size_t g,
                    int magnetic);
int gcso_sync_edges(const gcso_edge_plan *p, gamera_no_storage st[6]);
int gcso_advance_six(const gamera_no_grid grid[6], gamera_no_storage storage[6],
                     const size_t active[3], size_t ghost, double ratio,
                     double dt, const gamera_no_advance_options *options,
                     const gamera_no_background_field background[6],
                     const gcso_halo_plan *halo, const gcso_edge_plan *edges);
int gcso_local_timestep(const gamera_no_grid *grid, const double *conserved,
                        const gamera_no_vec3 *cell_magnetic,
                        const size_t lower[3], const size_t upper[3],
                        const gamera_no_timestep_options *options,
                        const gamera_no_vec3 *background_cell, double *dt);

int gcso_apply_pressure_control(gamera_no_storage *storage, const gamera_no_grid *grid,
                                const size_t lower[3], const size_t upper[3], double dt,
                                double gamma, double density_floor, double pressure_floor,
                                double light_speed, double low_density_threshold,
                                double low_density_sound_speed, size_t *low_count,
                                size_t *hot_count, double *max_sound, double *max_pressure);

int gcso_mi_apply_constant_pedersen(const gamera_mi_solver_config *config,
                                    const double *potential, double *result);
int gcso_mi_solve_constant_pedersen(const gamera_mi_solver_config *config,
                                    const double *fac, double *potential,
                                    gamera_mi_solver_stats *stats);
int gcso_mi_apply_conductance_tensor(const gamera_mi_solver_config *config,
                                     const double *pedersen,
                                     const double *hall,
                                     const double *potential, double *result);
int gcso_mi_solve_pedersen_pcg(const gamera_mi_solver_config *config, const double *fac,
                               const double *pedersen, double *potential,
                               gamera_mi_solver_stats *stats);
int gcso_mi_solve_conductance_tensor(const gamera_mi_solver_config *config,
                                     const double *fac, const double *pedersen,
                                     const double *hall, double *potential,
                                     gamera_mi_solver_stats *stats);

/* Cases (oracle/cases_common.h): kind, active radial/angular cells (0 =
 * default), noise seed. */
gcso_case *gcso_case_create(int kind, size_t nr, size_t n,
                            unsigned long long seed);
/* The wind case with an explicit upstream driver (n cm^-3, Vx km/s, T K,
 * Bz nT). */
gcso_case *gcso_case_create_driven(size_t nr, size_t n, unsigned long long seed,
                                   double density_cm3, double vx_kms,
                                   double temperature_k, double bz_nt);
void gcso_case_destroy(gcso_case *c);
gamera_no_grid *gcso_case_grid(gcso_case *c);
gamera_no_storage *gcso_case_storage(gcso_case *c);
gamera_no_background_field *gcso_case_background(gcso_case *c);
gamera_no_advance_options *gcso_case_options(gcso_case *c);
gamera_no_timestep_options *gcso_case_timestep_options(gcso_case *c);
const size_t *gcso_case_active(gcso_case *c);
size_t gcso_case_ghost(gcso_case *c);
double gcso_case_default_dt(gcso_case *c);
double gcso_case_default_ratio(gcso_case *c);
int gcso_case_local_timestep(gcso_case *c, double *dt);
int gcso_case_step(gcso_case *c, double ratio, double dt);
int gcso_case_copy_storage(gcso_case *dst, const gcso_case *src);

#ifdef __cplusplus
}
#endif

#endif
