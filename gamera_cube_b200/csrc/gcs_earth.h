// Device form of the reference's Earth radial boundary callbacks
// (cubedsphere/cubedsphere_earth_boundary.c) for the no-MI wall: radial
// ghost states at both shells, the inner mass/energy flux trap and the
// wind-driven outer / zero inner tangential EMF, as kernels run at the
// reference step's callback positions (gcs_earth.cu).
#pragma once

#include "gcs_kernels.cuh"
#include "gamera_cs_types.h"
#include "gcs_mi_lookup.cuh"

struct gcs_earth;

namespace gcs {

// Monitor time series of the solar wind (nonorthogonal/src/solar_wind.h),
// states as 8 doubles: density, pressure, velocity[3], magnetic[3].
struct WindDev {
  int count;
  int linear;
  const double *time;
  const double *state;
  double reference[3];
  double time_offset, by, bz;
};

// Geometry of the radial boundary layers on the node plane of a face
// (N1 x N2 per layer, six faces):
//   cells: 2g layers, i = l (inner, l < g) or outer + l - g;
//   outer ghost faces of family d: g layers, i = outer + (d == 0) + l;
//   edges of family d: 5 layers, i = g (l = 0) or outer - 3 + (l - 1).
struct EarthDev {
  const double *cell_cen[3];
  const double *face_cen[3][3], *face_av[3][3], *face_bg[3];
  const double *edge_mid[3][3], *edge_nrm[3][3], *edge_len[3];
  const unsigned char *edge_valid[3];
  // edge end points on the inner shell (i = g), edge families 1 and 2
  const double *inner_a[2][3], *inner_b[2][3];
  WindDev wind;
  double gamma, rho_floor, p_floor, cfl;
  int strict_wall;
  // ready MI coupling: inner ghost velocity from the E x B drift and the
  // inner-shell EMF from the mapped potential (device copy in mil.pot)
  int mi;
  MiLookup mil;
  double mi_potential_norm;
};

// Times of one step with the device Earth boundary: the radial fill at
// (current, previous) time, the EMF at step_time + step_dt / 2.
// With device_times the times are read from the context's step parameters
// instead (driver mode): current = time, previous = time - dt_prev (time on
// the first step), step time = time, step dt = dt, as the reference driver
// sets them (test_cubedsphere_dipole_background.c:655-692).
struct EarthStep {
  const EarthDev *dev;
  double current_time, previous_time, step_time, step_dt;
  int device_times;
};

void launch_earth_radial(const Ctx &X, const EarthStep &es, cudaStream_t s);
void launch_earth_trap(const Ctx &X, cudaStream_t s);
void launch_earth_emf(const Ctx &X, const EarthStep &es, cudaStream_t s);

struct Context;
// The device boundary the drop-in step and the host entry points use for
// (context, boundary): created on first use, its wind series, floors, CFL
// and wall flag refreshed from `b` on every call.  NULL on failure.
// With allow_mi a ready MI coupling is accepted (the host entry points
// then set the inner ghost velocities themselves).
gcs_earth *earth_for(Context &C, const gamera_no_grid grid[kFaces],
                     const gamera_cs_earth_boundary *b, bool allow_mi);
// Drop the boundaries cached for a context being destroyed.
void earth_forget(const Context &C);

}  // namespace gcs

// The C handle (gamera_cs_b200.h): device arrays of one context's boundary.
struct gcs_earth {
  gcs::Context *C = nullptr;
  gcs::EarthDev dev{};
  void *pool = nullptr;          // geometry of the boundary layers
  void *wind_pool = nullptr;     // monitor time series
  size_t pool_bytes = 0;
  const gamera_cs_mi_dipole *mi = nullptr;  // coupling named at creation
  double *mi_pot = nullptr;      // device copy of its potential, 2 x nt x np
  size_t mi_count = 0;
};

namespace gcs {
// Point the device boundary at the MI coupling's current potential (copied
// to the device) when it is ready; plain wall otherwise.
int earth_sync_mi(gcs_earth *e, const gamera_cs_mi_dipole *mi);
}  // namespace gcs
