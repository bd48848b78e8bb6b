/*
 * Test-infrastructure harness linked into oracle/_ref/libgamera_ref.so.
 *
 * This file is this repository's own code.  It builds six-face cubed-sphere
 * cases exclusively through the reference GAMERA-Cube public setup API
 * (vertex generation, grid/storage/background creation, initialisation) and
 * advances them with the reference's own step, so that the tests can compare
 * the CUDA library against the unmodified reference on identical inputs.
 * It is never linked into, or called by, the product library.
 *
 * Case kinds:
 *   FX_UNIFORM  uniform MHD state on 5x9x9 faces, r in [2, 2.5]
 *               (cubedsphere/tests/test_cubedsphere_six_mhd.c:9-62)
 *   FX_SHOCK    radial MHD shock on 12x9x9 faces, r in [2, 3]
 *               (cubedsphere/tests/test_cubedsphere_mhd_shock.c:112-170)
 *   FX_WIND     uniform solar wind n=5, V=(-400,0,0) km/s, T=1e5 K, IMF
 *               Bz=-5 nT, aligned 3.1e-5 T dipole B0, +-1% seeded density
 *               noise, log-stretched r in [2.5, 30] R_E, Earth-driver options
 *               (cubedsphere/tests/test_cubedsphere_dipole_background.c:
 *               282-294, 405-444; nonorthogonal_radial_map.c:152-156)
 *   FX_PULSE    FX_WIND with V=-450 km/s and a 20% sinusoidal density pulse
 *               of wavelength 10 R_E.
 */
#include "cubedsphere_halo.h"
#include "cubedsphere_interface.h"
#include "cubedsphere_mi_dipole.h"
#include "cubedsphere_step.h"
#include "nonorthogonal_background.h"
#include "nonorthogonal_initialization.h"
#include "nonorthogonal_state.h"
#include "nonorthogonal_step.h"

#include "cases_common.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { FX_UNIFORM = CASE_UNIFORM, FX_SHOCK = CASE_SHOCK, FX_WIND = CASE_WIND,
       FX_PULSE = CASE_PULSE };

typedef struct {
  int kind;
  size_t active[3];
  size_t ghost;
  gamera_no_grid grid[GAMERA_CS_FACE_COUNT];
  gamera_no_storage storage[GAMERA_CS_FACE_COUNT];
  gamera_no_background_data owned[GAMERA_CS_FACE_COUNT];
  gamera_no_background_field background[GAMERA_CS_FACE_COUNT];
  int use_background;
  gamera_no_advance_options options;
  gamera_no_timestep_options timestep;
  gamera_cs_halo_plan *plan;
  double dt;
  double ratio;
  /* wind parameters */
  double wind_density, wind_speed, wind_pressure, pulse_amplitude;
  double pulse_wavelength;
  gamera_no_vec3 imf;
  unsigned long long seed;
} fx_case;

double fx_magnetic_norm_tesla(void) { return case_magnetic_norm_tesla(); }

double fx_noise(unsigned long long seed, int face, size_t cell) {
  return case_noise(seed, face, cell);
}

static int uniform_potential(gamera_no_vec3 point, void *context,
                             gamera_no_vec3 *potential) {
  const gamera_no_vec3 *b = (const gamera_no_vec3 *)context;
  potential->value[0] = 0.5 * (b->value[1] * point.value[2] -
                               b->value[2] * point.value[1]);
  potential->value[1] = 0.5 * (b->value[2] * point.value[0] -
                               b->value[0] * point.value[2]);
  potential->value[2] = 0.5 * (b->value[0] * point.value[1] -
                               b->value[1] * point.value[0]);
  return 0;
}

void fx_destroy(fx_case *c) {
  if (c == NULL) return;
  gamera_cs_halo_plan_destroy(c->plan);
  for (int f = 0; f < GAMERA_CS_FACE_COUNT; ++f) {
    if (c->use_background) gamera_no_background_destroy(&c->owned[f]);
    gamera_no_storage_destroy(&c->storage[f]);
    gamera_no_grid_destroy(&c->grid[f]);
  }
  free(c);
}

static void set_uniform_flux(fx_case *c, int f, gamera_no_vec3 b) {
  for (int d = 0; d < 3; ++d) {
    const size_t count = gamera_no_element_count3(c->grid[f].face[d].extent);
    for (size_t n = 0; n < count; ++n) {
      const gamera_no_vec3 a = c->grid[f].face[d].value[n].area_vector;
      double flux = 0.0;
      for (int m = 0; m < 3; ++m) flux += b.value[m] * a.value[m];
      c->storage[f].face_flux[d][n] = flux;
      c->storage[f].old_face_flux[d][n] = flux;
    }
  }
}

/* nr, n: active radial and angular cells (0 selects the case default). */
fx_case *fx_create(int kind, size_t nr, size_t n, unsigned long long seed) {
  fx_case *c = calloc(1, sizeof(*c));
  if (c == NULL) return NULL;
  c->kind = kind;
  c->ghost = 4;
  c->seed = seed;
  const double gamma = 5.0 / 3.0;
  if (kind == FX_UNIFORM) {
    c->active[0] = nr ? nr : 5; c->active[1] = c->active[2] = n ? n : 9;
  } else if (kind == FX_SHOCK) {
    c->active[0] = nr ? nr : 12; c->active[1] = c->active[2] = n ? n : 9;
  } else if (kind == FX_WIND || kind == FX_PULSE) {
    c->active[0] = nr ? nr : 48; c->active[1] = c->active[2] = n ? n : 32;
  } else {
    free(c);
    return NULL;
  }
  const size_t g = c->ghost;
  const size_t extent[3] = {c->active[0] + 2 * g, c->active[1] + 2 * g,
                            c->active[2] + 2 * g};
  const size_t vextent[3] = {extent[0] + 1, extent[1] + 1, extent[2] + 1};
  gamera_no_radial_map map;
  const int wind = kind == FX_WIND || kind == FX_PULSE;
  if (wind && gamera_no_radial_map_init(
                  &map, GAMERA_NO_RADIAL_MAP_LEGACY_EXPONENTIAL, 2.5, 30.0,
                  log(12.0)) != 0) {
    free(c);
    return NULL;
  }
  gamera_no_dipole dipole = {{{0.0, 0.0, CASE_DIPOLE_MOMENT}}};
  c->use_background = wind;
  const double bnorm = fx_magnetic_norm_tesla();
  if (wind) {
    c->wind_density = 5.0;
    c->wind_speed = kind == FX_PULSE ? -4.5 : -4.0;
    /* n k T / (rho_norm u_norm^2), protons only, T = 1e5 K. */
    c->wind_pressure = case_wind_pressure();
    c->imf = (gamera_no_vec3){{0.0, 0.0, -5.0e-9 / bnorm}};
    c->pulse_amplitude = kind == FX_PULSE ? 0.2 : 0.0;
    c->pulse_wavelength = 10.0;
  }
  for (int f = 0; f < GAMERA_CS_FACE_COUNT; ++f) {
    gamera_no_vec3 *v = calloc(gamera_no_element_count3(vextent), sizeof(*v));
    int bad = v == NULL;
    if (!bad) {
      if (kind == FX_UNIFORM)
        bad = gamera_cs_generate_vertices(f, c->active, g, 2.0, 2.5, v) != 0;
      else if (kind == FX_SHOCK)
        bad = gamera_cs_generate_vertices(f, c->active, g, 2.0, 3.0, v) != 0;
      else
        bad = gamera_cs_generate_vertices_radial_map(f, c->active, g, &map,
                                                     v) != 0;
    }
    bad = bad || gamera_no_grid_create(extent, v, &c->grid[f]) != 0 ||
          gamera_cs_calibrate_face_frames(&c->grid[f]) != 0 ||
          gamera_no_storage_create(extent, &c->storage[f]) != 0;
    free(v);
    if (bad) { fx_destroy(c); return NULL; }
    if (wind) {
      if (gamera_no_background_create(&c->grid[f], gamera_no_dipole_field,
                                      &dipole, &c->owned[f]) != 0) {
        c->use_background = 0;
        fx_destroy(c);
        return NULL;
      }
      c->background[f] = c->owned[f].field;
    }
    const size_t cells = gamera_no_element_count3(extent);
    gamera_no_storage *s = &c->storage[f];
    for (size_t cell = 0; cell < cells; ++cell) {
      gamera_no_primitive p;
      if (kind == FX_UNIFORM) {
        p = (gamera_no_primitive){1.2, {{0.23, -0.17, 0.09}}, 0.74};
      } else if (kind == FX_SHOCK) {
        const gamera_no_vec3 x = c->grid[f].cell[cell].centroid;
        const double r = sqrt(x.value[0] * x.value[0] +
                              x.value[1] * x.value[1] +
                              x.value[2] * x.value[2]);
        p = r < 2.5 ? (gamera_no_primitive){1.0, {{0.0, 0.0, 0.0}}, 1.0}
                    : (gamera_no_primitive){0.125, {{0.0, 0.0, 0.0}}, 0.1};
      } else {
        const gamera_no_vec3 x = c->grid[f].cell[cell].centroid;
        const double rho = case_wind_density(kind, seed, f, cell, x.value[0]);
        p = (gamera_no_primitive){rho, {{c->wind_speed, 0.0, 0.0}},
                                  c->wind_pressure};
      }
      const double floor = wind ? 1e-6 : 1e-12;
      const double pfloor = wind ? 1e-8 : 1e-12;
      if (gamera_no_primitive_to_conserved(&p, gamma, floor, pfloor,
              &s->conserved[cell * GAMERA_NO_FLUX_COUNT]) != 0) {
        fx_destroy(c);
        return NULL;
      }
    }
    if (kind == FX_UNIFORM || kind == FX_SHOCK) {
      const gamera_no_vec3 b = kind == FX_UNIFORM
          ? (gamera_no_vec3){{0.38, -0.21, 0.16}}
          : (gamera_no_vec3){{0.1, 0.08, -0.03}};
      for (size_t cell = 0; cell < cells; ++cell) s->cell_magnetic[cell] = b;
      set_uniform_flux(c, f, b);
    } else if (gamera_no_initialize_flux_from_vector_potential(
                   &c->grid[f], s, uniform_potential, &c->imf) != 0) {
      fx_destroy(c);
      return NULL;
    }
    if (gamera_no_save_current_as_old(s) != 0) { fx_destroy(c); return NULL; }
  }
  if (kind == FX_UNIFORM) {
    c->options = (gamera_no_advance_options){
        .stress = {gamma, 1e-12, 1e-12, 1.0, 0.0, 0.0, 100.0,
                   true, false, false, false},
        .emf = {1e-12, 1.0, 0.0, 100.0, 0.8, 0.01, false, false},
        .update = {gamma, 1e-12, 1e-12, 100.0, true, false, false},
        .source_time = 0.0};
    c->timestep = (gamera_no_timestep_options){gamma, 1e-12, 1e-12, 0.8,
                                               100.0, true, false, false};
    c->dt = 0.01;
    c->ratio = 0.5;
  } else if (kind == FX_SHOCK) {
    c->options = (gamera_no_advance_options){
        .stress = {gamma, 1e-12, 1e-12, 1.0, 0.25, 0.25, 100.0,
                   true, true, false, false},
        .emf = {1e-12, 1.0, 0.5, 100.0, 0.3, 0.001, false, false},
        .update = {gamma, 1e-12, 1e-12, 100.0, true, false, false},
        .source_time = 0.0};
    c->timestep = (gamera_no_timestep_options){gamma, 1e-12, 1e-12, 0.3,
                                               100.0, true, false, false};
    c->dt = 0.001;
    c->ratio = 0.5;
  } else {
    c->options = (gamera_no_advance_options){
        .stress = {gamma, 1e-6, 1e-8, 1.0, 0.25, 0.25, 10.0,
                   true, true, true, true},
        .emf = {1e-6, 1.0, 0.5, 10.0, 0.3, 0.0, true, true},
        .update = {gamma, 1e-6, 1e-8, 10.0, true, true, true},
        .source_time = 0.0};
    c->timestep = (gamera_no_timestep_options){gamma, 1e-6, 1e-8, 0.3,
                                               10.0, true, true, true};
    c->ratio = 0.0;
    c->dt = 0.0;
  }
  if (gamera_cs_halo_plan_create(c->grid, c->active, c->ghost, &c->plan) != 0) {
    fx_destroy(c);
    return NULL;
  }
  return c;
}

gamera_no_grid *fx_grid(fx_case *c) { return c->grid; }
gamera_no_storage *fx_storage(fx_case *c) { return c->storage; }
gamera_no_background_field *fx_background(fx_case *c) {
  return c->use_background ? c->background : NULL;
}
gamera_no_advance_options *fx_options(fx_case *c) { return &c->options; }
gamera_no_timestep_options *fx_timestep_options(fx_case *c) {
  return &c->timestep;
}
gamera_cs_halo_plan *fx_plan(fx_case *c) { return c->plan; }
const size_t *fx_active(fx_case *c) { return c->active; }
size_t fx_ghost(fx_case *c) { return c->ghost; }
double fx_default_dt(fx_case *c) { return c->dt; }
double fx_default_ratio(fx_case *c) { return c->ratio; }

/* Minimum reference CFL step over the six faces
 * (test_cubedsphere_dipole_background.c:593-616 without the 0.5 factor). */
int fx_local_timestep(fx_case *c, double *dt) {
  const size_t lower[3] = {c->ghost, c->ghost, c->ghost};
  const size_t upper[3] = {c->ghost + c->active[0], c->ghost + c->active[1],
                           c->ghost + c->active[2]};
  double smallest = INFINITY;
  for (int f = 0; f < GAMERA_CS_FACE_COUNT; ++f) {
    double local;
    if (gamera_no_local_timestep(
            &c->grid[f], c->storage[f].conserved, c->storage[f].cell_magnetic,
            lower, upper, &c->timestep,
            c->use_background ? c->owned[f].cell_magnetic : NULL,
            &local) != 0)
      return -1;
    smallest = fmin(smallest, local);
  }
  *dt = smallest;
  return 0;
}

/* One reference step with the reference planned halo and no radial
 * callback (outflow radial ghosts). */
int fx_step(fx_case *c, double ratio, double dt) {
  return gamera_cs_advance_six_with_background_planned(
      c->grid, c->storage, c->active, c->ghost, ratio, dt, &c->options,
      c->use_background ? c->background : NULL, c->plan, NULL, 0.0, 0.0,
      NULL);
}

/* Copy every storage array of src into dst (same kind and size). */
int fx_copy_storage(fx_case *dst, const fx_case *src) {
  for (int f = 0; f < GAMERA_CS_FACE_COUNT; ++f) {
    const gamera_no_storage *a = &src->storage[f];
    gamera_no_storage *b = &dst->storage[f];
    const size_t cells = gamera_no_element_count3(a->cell_extent);
    if (cells != gamera_no_element_count3(b->cell_extent)) return -1;
    memcpy(b->conserved, a->conserved, cells * 5 * sizeof(double));
    memcpy(b->old_conserved, a->old_conserved, cells * 5 * sizeof(double));
    memcpy(b->predicted_conserved, a->predicted_conserved,
           cells * 5 * sizeof(double));
    memcpy(b->cell_magnetic, a->cell_magnetic, cells * sizeof(gamera_no_vec3));
    memcpy(b->old_cell_magnetic, a->old_cell_magnetic,
           cells * sizeof(gamera_no_vec3));
    memcpy(b->predicted_cell_magnetic, a->predicted_cell_magnetic,
           cells * sizeof(gamera_no_vec3));
    memcpy(b->hydro_rate, a->hydro_rate, cells * 5 * sizeof(double));
    memcpy(b->maxwell_rate, a->maxwell_rate, cells * sizeof(gamera_no_vec3));
    for (int d = 0; d < 3; ++d) {
      const size_t faces = gamera_no_element_count3(a->face_extent[d]);
      const size_t edges = gamera_no_element_count3(a->edge_extent[d]);
      memcpy(b->face_flux[d], a->face_flux[d], faces * sizeof(double));
      memcpy(b->old_face_flux[d], a->old_face_flux[d], faces * sizeof(double));
      memcpy(b->predicted_face_flux[d], a->predicted_face_flux[d],
             faces * sizeof(double));
      memcpy(b->fluid_face_flux[d], a->fluid_face_flux[d],
             faces * 5 * sizeof(double));
      memcpy(b->maxwell_face_flux[d], a->maxwell_face_flux[d],
             faces * sizeof(gamera_no_vec3));
      memcpy(b->edge_emf[d], a->edge_emf[d], edges * sizeof(double));
    }
  }
  return 0;
}

/* Ionosphere coupling on a fixture case.  fx_set_mi_field puts the analytic
 * residual field of the reference MI shell test
 * (cubedsphere/tests/test_cubedsphere_mi_shell.c:54-66) on every active cell
 * of both time levels; fx_mi_create builds the reference coupling on the
 * case through gamera_cs_mi_dipole_create. */
int fx_set_mi_field(fx_case *c) {
  for (int f = 0; f < GAMERA_CS_FACE_COUNT; ++f) {
    const size_t *e = c->grid[f].cell_extent;
    for (size_t i = c->ghost; i < c->ghost + c->active[0]; ++i)
      for (size_t j = c->ghost; j < c->ghost + c->active[1]; ++j)
        for (size_t k = c->ghost; k < c->ghost + c->active[2]; ++k) {
          const size_t cell = gamera_no_index3(e, i, j, k);
          const gamera_no_vec3 p = c->grid[f].cell[cell].centroid;
          const double r2 = p.value[0] * p.value[0] + p.value[1] * p.value[1] +
                            p.value[2] * p.value[2];
          const gamera_no_vec3 b = {{0.03 * p.value[1] / r2, -0.02 * p.value[0] / r2,
                                     0.01 * p.value[0] * p.value[2] / r2}};
          c->storage[f].cell_magnetic[cell] = b;
          c->storage[f].old_cell_magnetic[cell] = b;
        }
  }
  return 0;
}

gamera_cs_mi_dipole *fx_mi_create(fx_case *c, const gamera_cs_earth_startup *startup,
                                  const gamera_cs_mi_dipole_config *config) {
  gamera_cs_mi_dipole *mi = NULL;
  if (!c->use_background ||
      gamera_cs_mi_dipole_create(c->grid, c->storage, c->background, startup,
                                 c->active, c->ghost, config, &mi) != 0)
    return NULL;
  return mi;
}
