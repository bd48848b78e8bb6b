// Host-side owner of one six-face device run: device arrays, plans, stream,
// optional CUDA graph of the driver step, and the state transfers between
// the caller's reference-layout host arrays and the device node layout.
#pragma once

#include <vector>

#include <cstdio>

#include "gamera_cs_types.h"
#include "gcs_kernels.cuh"
#include "gcs_topology.h"

struct gamera_cs_mi_dipole;

namespace gcs {

enum ArrayKind {
  kArrU, kArrUo, kArrUp, kArrB, kArrBo, kArrBp,
  kArrP, kArrPo, kArrPp, kArrF, kArrM, kArrE
};

// Wind states of the case kinds 2 and 3, and of an explicit upstream
// driver (n in cm^-3, Vx in km/s, T in K, Bz in nT) (gcs_build.cu).
WindInit case_wind(int kind);
WindInit driven_wind(double density_cm3, double velocity_x_kms, double temperature_k,
                     double bz_nt);

// Arguments of the post-step pressure control (nonorthogonal_step.h:26-32).
struct PressureControl {
  double gamma, density_floor, pressure_floor, light_speed, low_density_threshold,
      low_density_sound_speed;
};

struct Context {
  Ctx X;
  cudaStream_t stream = nullptr;
  void *pool = nullptr;
  size_t pool_bytes = 0;
  void *bg_pool = nullptr;
  size_t bg_bytes = 0;
  void *plans = nullptr;
  size_t plans_bytes = 0;
  void *staging = nullptr;
  size_t staging_bytes = 0;
  void *staging_host = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  unsigned long long graph_key = 0;
  int bg_uploaded = 0;
  const void *bg_key[kFaces][11] = {};
  const gamera_no_cell_geometry *grid_cell[kFaces] = {};
  const gamera_no_face_geometry *grid_face[kFaces][3] = {};
  // device state belongs to this host storage (resident mode)
  const gamera_no_storage *resident_storage = nullptr;
  int resident = 0;
  DevStatus host_status{};
  char error[256] = {0};
  // Geometry of the innermost radial layers of a device-built case (cell
  // centroids of layers [0, win_layers), vertices of [0, win_layers + 1)),
  // kept for the ionosphere-coupling plans; empty for host-grid contexts.
  int win_layers = 0;
  std::vector<gamera_no_vec3> win_centroid[kFaces];
  std::vector<gamera_no_vec3> win_vertex[kFaces];
  // Post-step pressure control of the driver loop (gcs_pressure.cu): the
  // dipole line length of every active cell and the device counters.
  PressureControl pc{};
  int pc_on = 0;
  double *pc_dipole = nullptr;
  void *pc_stats = nullptr;
  // ionosphere coupling updated inside the driver loop's step graph
  // (gcs_context_set_mi_coupling), or null
  ::gamera_cs_mi_dipole *mi_graph = nullptr;
  // per-stage timing (profiling mode)
  int profiling = 0;
  double stage_ms[16] = {0};
  long long stage_calls[16] = {0};

  ~Context();
  int init(const gamera_no_grid grid[kFaces], const size_t active[3],
           size_t ghost);
  // Build a case (kind, sizes, seed) directly on the device
  // (gcs_build.cu); no host grid is involved.
  int init_case(int kind, size_t nr, size_t n, unsigned long long seed,
                const WindInit *driver = nullptr);
  // Active centroids and vertices of one face of a device-built case
  // (gcs_build.cu).
  int face_coordinates(int f, std::vector<double> &centroids, std::vector<double> &vertices);
  int kind_shock = 0;   // device-built radial shock case (r in [2, 3])
  // Radial boundary-layer geometry of a device-built wind case for the
  // device Earth boundary (gcs_build.cu).
  int build_earth_layers(const EarthLayers &L);
  // A wind run on the grid of `o` with its own state (gcs_build.cu).
  int init_member(Context &o, unsigned long long seed, const WindInit &w);
  // Non-null for a run sharing the grid of another context; only the state
  // arrays, params, status and stream are this context's.
  Context *owner = nullptr;
  int allocate(const size_t active[3], size_t ghost);
  int init_topology(const size_t active[3], size_t ghost);
  int allocate_background();
  // FP32-bulk sweeps on (1) or off (0); the FP32 arrays are allocated and
  // the metric and background converted on first use (gcs_setup.cu).
  int enable_bulk(int on);
  void *bulk_pool = nullptr;
  size_t bulk_bytes = 0;
  int bulk_bg_dirty = 0;   // background uploaded since its FP32 copies
  double bulk_b0_threshold = 8.0;   // |B0| above which a layer stays FP64
  int set_bulk_split(double b0_threshold);
  int derive();
  int build_plans(const HaloGeometry &geo);
  void release();
  int upload_background(const gamera_no_background_field bg[kFaces]);
  bool background_matches(const gamera_no_background_field bg[kFaces]) const;
  int transfer_array(int f, int kind, int dir, bool upload, double *host);
  int upload_state(const gamera_no_storage st[kFaces]);
  int download_state(gamera_no_storage st[kFaces], int scratch);
  void reset_status_async();
  int read_status(DevStatus *out);
  void set_error(const char *what, const char *where);
  bool grid_matches(const gamera_no_grid grid[kFaces]) const {
    for (int f = 0; f < kFaces; ++f) {
      if (grid[f].cell != grid_cell[f]) return false;
      for (int d = 0; d < 3; ++d)
        if (grid[f].face[d].value != grid_face[f][d]) return false;
    }
    return true;
  }
};

// gcs_mi_dipole.cu: the coupling update inside the driver loop's step
int mi_launch_in_step(::gamera_cs_mi_dipole *s, cudaStream_t st);
int mi_before_run(::gamera_cs_mi_dipole *s);
void mi_after_run(::gamera_cs_mi_dipole *s);
const double *mi_graph_potential(const ::gamera_cs_mi_dipole *s, const Context *C);

// gcs_pressure.cu
int pressure_prepare(Context &C, const gamera_no_grid *grid);
int pressure_reset_async(Context &C);
// cfl set (the driver loop): dt from the step parameters, failures into the
// step status, and the CFL step of the controlled state reduced with it.
void launch_pressure_control(Context &C, const PressureControl &pc, double dt,
                             const Opts *cfl, cudaStream_t s);

}  // namespace gcs

// The C handle of a context (gamera_cs_b200.h).
struct gcs_context {
  gcs::Context c;
  std::vector<cudaEvent_t> events;   // profiling: 2 per recorded stage
  std::vector<int> event_slot;
};
