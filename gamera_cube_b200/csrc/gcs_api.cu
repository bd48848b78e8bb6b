// extern "C" entry points: the reference drop-in functions and the
// device-resident context API declared in include/gamera_cs_b200.h.
#include "gamera_cs_b200.h"
#include "gcs_context.h"
#include "gcs_earth.h"

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <array>
#include <map>
#include <mutex>
#include <new>
#include <vector>

struct gamera_cs_halo_plan {
  gcs_context *ctx;
};

struct gamera_cs_edge_sync_plan {
  gcs_context *ctx;
};

namespace {

thread_local char g_last_error[256] = "";

void set_last(const char *msg) {
  snprintf(g_last_error, sizeof(g_last_error), "%s", msg);
}

// cubedsphere/cubedsphere_step.c:8-11
bool same_value(double a, double b) {
  const double scale = fmax(1.0, fmax(fabs(a), fabs(b)));
  return std::isfinite(a) && std::isfinite(b) && fabs(a - b) <= 8e-15 * scale;
}

// Stage names of the MHD_FAILURE line.  The three B recoveries (predictor,
// update, final) keep separate codes in gcs_context_failure but print the
// reference's one name for its recovery, recover_B (nonorthogonal_step.c:351).
const char *kStageNames[] = {
    "none",           "predict",         "recover_B",       "reconstruct_face",
    "kinetic_fluid",  "kinetic_maxwell", "emergency",       "edge_geometry",
    "edge_velocity",  "transverse_field", "edge_density",   "compute_edge_emf",
    "boris_after_hydro", "recover_B",    "recover_B",       "timestep",
    "host_callback",  "solve_edge_field", "options",        "pressure_control",
    "tile_copy",      "mi_coupling"};

// Option checks of the reference step and of each stage it calls
// (cubedsphere_step.c:23-47, nonorthogonal_sweep.c:48-62, 209-221,
// nonorthogonal_step.c:421-429).
bool make_opts(const gamera_no_advance_options *o, bool have_background,
               gcs::Opts *out) {
  if (o == nullptr) return false;
  const gamera_no_sweep_options &s = o->stress;
  const gamera_no_emf_options &e = o->emf;
  const gamera_no_update_options &u = o->update;
  if (o->cell_source != nullptr || o->indexed_cell_source != nullptr ||
      u.use_background != s.use_background ||
      u.use_background != e.use_background ||
      (u.use_background && !have_background) || !std::isfinite(o->source_time) ||
      !same_value(s.gamma, u.gamma) ||
      !same_value(s.density_floor, u.density_floor) ||
      !same_value(s.pressure_floor, u.pressure_floor) ||
      !same_value(e.density_floor, u.density_floor) ||
      s.use_mhd != u.use_mhd || s.use_boris != u.use_boris ||
      e.use_boris != u.use_boris ||
      (u.use_boris &&
       (!same_value(s.light_speed, u.light_speed) ||
        !same_value(e.light_speed, u.light_speed))))
    return false;
  // sweep options
  if (!std::isfinite(s.gamma) || s.gamma <= 1.0 ||
      !std::isfinite(s.density_floor) || s.density_floor <= 0.0 ||
      !std::isfinite(s.pressure_floor) || s.pressure_floor <= 0.0 ||
      !std::isfinite(s.pdm_coefficient) || s.pdm_coefficient < 0.0 ||
      !std::isfinite(s.hydro_hogs_coefficient) || s.hydro_hogs_coefficient < 0.0 ||
      !std::isfinite(s.magnetic_hogs_coefficient) ||
      s.magnetic_hogs_coefficient < 0.0 ||
      (s.use_boris && !(std::isfinite(s.light_speed) && s.light_speed > DBL_MIN)))
    return false;
  // update options
  if (!std::isfinite(u.gamma) || u.gamma <= 1.0 ||
      !std::isfinite(u.density_floor) || u.density_floor <= 0.0 ||
      !std::isfinite(u.pressure_floor) || u.pressure_floor <= 0.0 ||
      (u.use_boris && !(std::isfinite(u.light_speed) && u.light_speed > DBL_MIN)))
    return false;
  // emf options (dt is checked per call)
  if (u.use_mhd &&
      (!std::isfinite(e.density_floor) || e.density_floor <= 0.0 ||
       !std::isfinite(e.pdm_coefficient) || e.pdm_coefficient < 0.0 ||
       !std::isfinite(e.diffusion_coefficient) || !std::isfinite(e.cfl) ||
       e.cfl < 0.0 ||
       (e.use_boris && !(std::isfinite(e.light_speed) && e.light_speed > DBL_MIN))))
    return false;
  gcs::Opts &O = *out;
  std::memset(&O, 0, sizeof(O));
  O.s_gamma = s.gamma;
  O.s_rho_floor = s.density_floor;
  O.s_p_floor = s.pressure_floor;
  O.pdm = s.pdm_coefficient;
  O.hogs_h = s.hydro_hogs_coefficient;
  O.hogs_m = s.magnetic_hogs_coefficient;
  O.s_c = s.light_speed;
  O.s_mhd = s.use_mhd;
  O.hogs = s.use_hogs;
  O.s_boris = s.use_boris;
  O.s_bg = s.use_background;
  O.e_rho_floor = e.density_floor;
  O.e_pdm = e.pdm_coefficient;
  O.e_diff = e.diffusion_coefficient;
  O.e_c = e.light_speed;
  O.e_cfl = e.cfl;
  O.e_boris = e.use_boris;
  O.e_bg = e.use_background;
  O.u_gamma = u.gamma;
  O.u_rho_floor = u.density_floor;
  O.u_p_floor = u.pressure_floor;
  O.u_c = u.light_speed;
  O.u_mhd = u.use_mhd;
  O.u_boris = u.use_boris;
  O.u_bg = u.use_background;
  // time-step options default to the update group
  O.t_gamma = u.gamma;
  O.t_rho_floor = u.density_floor;
  O.t_p_floor = u.pressure_floor;
  O.t_c = u.light_speed;
  O.t_cfl = 0.3;
  O.t_mhd = u.use_mhd;
  O.t_boris = u.use_boris;
  O.t_bg = u.use_background;
  O.dt_fraction = 0.5;
  return true;
}

bool set_timestep_opts(const gamera_no_timestep_options *t, gcs::Opts *O) {
  if (t == nullptr || !std::isfinite(t->gamma) || t->gamma <= 1.0 ||
      !std::isfinite(t->density_floor) || t->density_floor <= 0.0 ||
      !std::isfinite(t->pressure_floor) || t->pressure_floor <= 0.0 ||
      !std::isfinite(t->cfl) || t->cfl <= 0.0 ||
      (t->use_boris && !(std::isfinite(t->light_speed) && t->light_speed > DBL_MIN)))
    return false;
  O->t_gamma = t->gamma;
  O->t_rho_floor = t->density_floor;
  O->t_p_floor = t->pressure_floor;
  O->t_cfl = t->cfl;
  O->t_c = t->light_speed;
  O->t_mhd = t->use_mhd;
  O->t_boris = t->use_boris;
  O->t_bg = t->use_background;
  return true;
}

enum Slot {
  kSlotSeamPhi = 0, kSlotHalo, kSlotPredict, kSlotFlux, kSlotSeamFlux,
  kSlotEmf, kSlotEdgeSync, kSlotUpdate, kSlotSeamPhiFinal, kSlotRecover,
  kSlotDt, kSlotMi, kSlotCount
};
const char *kSlotNames[kSlotCount] = {
    "seam_sync_phi", "halo", "predict", "flux", "seam_sync_flux",
    "edge_emf", "edge_sync", "ct_update", "seam_sync_phi_final",
    "recover_cfl", "next_dt", "mi_coupling"};

struct Marker {
  gcs_context *ctx;
  cudaEvent_t last = nullptr;
  void begin() {
    if (!ctx->c.profiling) return;
    cudaEventCreate(&last);
    cudaEventRecord(last, ctx->c.stream);
  }
  void mark(int slot) {
    if (!ctx->c.profiling) return;
    cudaEvent_t ev;
    cudaEventCreate(&ev);
    cudaEventRecord(ev, ctx->c.stream);
    ctx->events.push_back(last);
    ctx->events.push_back(ev);
    ctx->event_slot.push_back(slot);
    last = ev;
  }
};

// Host-callback hooks of the reference step, run between device stages.
struct Hooks {
  const gamera_no_grid *grid;
  gamera_no_storage *storage;
  const size_t *active;
  size_t ghost;
  gamera_cs_radial_boundary_function radial;
  double t, tprev;
  void *radial_ctx;
  const gamera_no_advance_options *options;
};

int transfer_fluxes(gcs::Context &C, gamera_no_storage *st, bool upload) {
  for (int f = 0; f < gcs::kFaces; ++f)
    for (int d = 0; d < 3; ++d)
      if (C.transfer_array(f, gcs::kArrF, d, upload, st[f].fluid_face_flux[d]) ||
          C.transfer_array(f, gcs::kArrM, d, upload,
                           (double *)st[f].maxwell_face_flux[d]))
        return -1;
  return 0;
}

int transfer_emf(gcs::Context &C, gamera_no_storage *st, bool upload) {
  for (int f = 0; f < gcs::kFaces; ++f)
    for (int d = 0; d < 3; ++d)
      if (C.transfer_array(f, gcs::kArrE, d, upload, st[f].edge_emf[d]))
        return -1;
  return 0;
}

bool device_failed(gcs::Context &C) {
  gcs::DevStatus s;
  if (C.read_status(&s) != 0) return true;
  C.host_status = s;
  return s.first != 0;
}

// The stage sequence of one step (cubedsphere_step.c:48-152).  With hooks,
// host callbacks run at their reference positions on downloaded arrays.
int run_step(gcs_context *ctx, const gcs::Opts &O, int driver_mode,
             const Hooks *hk, const gcs::EarthStep *es = nullptr) {
  gcs::Context &C = ctx->c;
  if (hk && C.X.bulk &&
      (hk->radial || hk->options->fluid_flux_sync || hk->options->edge_emf_sync)) {
    C.set_error("host callbacks need the FP64 path", "step");
    return -1;
  }
  const gcs::Ctx &X = C.X;
  cudaStream_t s = C.stream;
  const bool post_control = driver_mode && C.pc_on;
  Marker mk{ctx};
  mk.begin();
  if (driver_mode && C.mi_graph != nullptr) {
    // the ionosphere coupling on its device-side cadence, before the step
    // (test_cubedsphere_dipole_background.c:631)
    if (gcs::mi_launch_in_step(C.mi_graph, s) != 0) return -1;
    mk.mark(kSlotMi);
  }
  gcs::launch_seam_sync(X, 1, s);
  mk.mark(kSlotSeamPhi);
  gcs::launch_halo(X, s);
  if (es) gcs::launch_earth_radial(X, *es, s);
  mk.mark(kSlotHalo);
  const size_t lower[3] = {hk ? hk->ghost : 0, hk ? hk->ghost : 0,
                           hk ? hk->ghost : 0};
  size_t upper[3] = {0, 0, 0};
  if (hk)
    for (int a = 0; a < 3; ++a) upper[a] = hk->ghost + hk->active[a];
  if (hk && hk->radial) {
    if (device_failed(C) || C.download_state(hk->storage, 0) != 0) return -1;
    if (hk->radial(hk->grid, hk->storage, hk->active, hk->ghost, hk->t,
                   hk->tprev, hk->radial_ctx) != 0)
      return -1;
    if (C.upload_state(hk->storage) != 0) return -1;
  }
  gcs::launch_predict(X, O, s);
  mk.mark(kSlotPredict);
  gcs::launch_flux(X, O, s);
  mk.mark(kSlotFlux);
  gcs::launch_seam_sync(X, 0, s);
  if (es) gcs::launch_earth_trap(X, s);
  mk.mark(kSlotSeamFlux);
  if (hk && hk->options->fluid_flux_sync) {
    if (device_failed(C) || transfer_fluxes(C, hk->storage, false) != 0)
      return -1;
    for (int f = 0; f < gcs::kFaces; ++f)
      if (hk->options->fluid_flux_sync(&hk->storage[f], &hk->grid[f], lower,
                                       upper, hk->options->fluid_flux_context))
        return -1;
    if (transfer_fluxes(C, hk->storage, true) != 0) return -1;
  }
  if (O.u_mhd) {
    gcs::launch_emf(X, O, s);
    if (es) gcs::launch_earth_emf(X, *es, s);
    mk.mark(kSlotEmf);
    if (hk && hk->options->edge_emf_sync) {
      if (device_failed(C) || transfer_emf(C, hk->storage, false) != 0)
        return -1;
      for (int f = 0; f < gcs::kFaces; ++f)
        if (hk->options->edge_emf_sync(&hk->storage[f], &hk->grid[f], lower,
                                       upper, hk->options->edge_emf_context))
          return -1;
      if (transfer_emf(C, hk->storage, true) != 0) return -1;
    }
    gcs::launch_edge_sync(X, s);
    mk.mark(kSlotEdgeSync);
  }
  gcs::launch_update(X, O, s);
  mk.mark(kSlotUpdate);
  if (O.u_mhd) {
    gcs::launch_seam_sync(X, 1, s);
    mk.mark(kSlotSeamPhiFinal);
    gcs::launch_recover(X, O, driver_mode && !post_control, s);
    mk.mark(kSlotRecover);
  }
  if (post_control) {
    // the Earth drivers' post-step pressure control with this step's dt,
    // fused with the CFL reduction of the controlled state
    gcs::launch_pressure_control(C, C.pc, 0.0, &O, s);
  }
  if (driver_mode) {
    gcs::launch_count_step(X, s);
    gcs::launch_next_dt(X, O.dt_fraction, s);
    mk.mark(kSlotDt);
  }
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

void report_failure(gcs::Context &C) {
  const unsigned long long v = C.host_status.first;
  const int stage = (int)(v >> 56) & 0xff;
  const char *rank = getenv("PMI_RANK");
  if (!rank) rank = getenv("SLURM_PROCID");
  fprintf(stderr,
          "MHD_FAILURE rank=%s stage=%s direction=%d face=%d local=%d,%d,%d\n",
          rank ? rank : "unknown",
          stage < (int)(sizeof(kStageNames) / sizeof(kStageNames[0]))
              ? kStageNames[stage] : "unknown",
          (int)(v >> 52) & 0xf, (int)(v >> 48) & 0xf, (int)(v >> 32) & 0xffff,
          (int)(v >> 16) & 0xffff, (int)v & 0xffff);
}

std::mutex g_registry_mutex;
std::map<const void *, gcs_context *> g_registry;

gcs_context *create_context(const gamera_no_grid grid[6], const size_t active[3],
                            size_t ghost) {
  if (grid == nullptr || active == nullptr) {
    set_last("null argument");
    return nullptr;
  }
  gcs_context *ctx = new (std::nothrow) gcs_context;
  if (!ctx) {
    set_last("out of host memory");
    return nullptr;
  }
  if (ctx->c.init(grid, active, ghost) != 0) {
    set_last(ctx->c.error);
    delete ctx;
    return nullptr;
  }
  return ctx;
}

gcs_context *context_for(const gamera_no_grid grid[6], const size_t active[3],
                         size_t ghost) {
  std::lock_guard<std::mutex> lock(g_registry_mutex);
  auto it = g_registry.find(grid[0].cell);
  if (it != g_registry.end() && it->second->c.grid_matches(grid)) return it->second;
  gcs_context *ctx = create_context(grid, active, ghost);
  if (ctx) g_registry[grid[0].cell] = ctx;
  return ctx;
}

int drop_in_step(gcs_context *ctx, const gamera_no_grid grid[6],
                 gamera_no_storage storage[6], const size_t active[3],
                 size_t ghost, double ratio, double dt,
                 const gamera_no_advance_options *options,
                 const gamera_no_background_field background[6],
                 gamera_cs_radial_boundary_function radial, double t,
                 double tprev, void *radial_ctx) {
  // grid == nullptr: a context built on the device (gcs_context_create_case)
  // with its own background; host callbacks are then not available.
  if (ctx == nullptr || storage == nullptr || active == nullptr ||
      options == nullptr || ghost < 4 || !std::isfinite(dt) || dt <= 0.0 ||
      (radial != nullptr && (!std::isfinite(t) || !std::isfinite(tprev))) ||
      !std::isfinite(ratio) || active[1] != active[2])
    return -1;
  gcs::Context &C = ctx->c;
  if ((grid != nullptr && !C.grid_matches(grid)) ||
      (grid == nullptr && (radial || options->fluid_flux_sync ||
                           options->edge_emf_sync)) ||
      (size_t)C.X.D.nr != active[0] || (size_t)C.X.D.n != active[1] ||
      (size_t)C.X.D.g != ghost)
    return -1;
  gcs::Opts O;
  const bool own_bg = grid == nullptr && C.bg_uploaded;
  if (!make_opts(options, background != nullptr || own_bg, &O)) return -1;
  if (O.u_mhd && !(std::isfinite(dt) && dt > DBL_MIN)) return -1;
  if (O.u_bg && !own_bg) {
    for (int f = 0; f < 6; ++f)
      for (int d = 0; d < 3; ++d)
        if (background[f].face_magnetic[d] == nullptr ||
            background[f].face_flux[d] == nullptr ||
            (O.u_mhd && background[f].edge_magnetic[d] == nullptr))
          return -1;
    if (!C.background_matches(background)) {
      if (C.upload_background(background) != 0) return -1;
      C.bulk_bg_dirty = 1;
    }
  }
  if (C.X.bulk && C.bulk_bg_dirty && C.enable_bulk(1) != 0) return -1;
  if (!(C.resident && C.resident_storage == storage)) {
    if (C.upload_state(storage) != 0) return -1;
  }
  C.resident_storage = storage;
  gcs::StepParams p;
  std::memset(&p, 0, sizeof(p));
  p.dt = dt;
  p.ratio = ratio;
  if (cudaMemcpyAsync(C.X.params, &p, sizeof(p), cudaMemcpyHostToDevice,
                      C.stream) != cudaSuccess)
    return -1;
  C.reset_status_async();
  // The reference's Earth callbacks of this library run as device kernels
  // inside the step, with no host round trip.
  const gamera_cs_earth_boundary *eb = nullptr;
  if (grid != nullptr && radial == gamera_cs_earth_fill_radial_ghosts &&
      options->fluid_flux_sync == gamera_cs_earth_inner_fluid_flux &&
      options->edge_emf_sync == gamera_cs_earth_no_mi_emf &&
      options->edge_emf_context == radial_ctx && radial_ctx != nullptr)
    eb = (const gamera_cs_earth_boundary *)radial_ctx;
  int rc;
  if (eb != nullptr) {
    // the reference's EMF callback fails on these (cubedsphere_earth_boundary.c:388-389)
    if (!std::isfinite(eb->step_time) || !(eb->step_dt > 0.0)) return -1;
    gcs_earth *earth = gcs::earth_for(C, grid, eb, true);
    if (earth == nullptr) return -1;
    const gcs::EarthStep es{&earth->dev, t, tprev, eb->step_time, eb->step_dt, 0};
    rc = run_step(ctx, O, 0, nullptr, &es);
  } else {
    Hooks hk{grid, storage, active, ghost, radial, t, tprev, radial_ctx, options};
    const bool hooks = radial || options->fluid_flux_sync || options->edge_emf_sync;
    rc = run_step(ctx, O, 0, hooks ? &hk : nullptr);
  }
  const bool fail = device_failed(C);
  if (fail) report_failure(C);
  // Emergency-diffusion statistics accumulate in the caller's storage.
  for (int f = 0; f < 6; ++f) {
    storage[f].emergency_diffusion_face_count += C.host_status.emergency_count[f];
    double mx;
    std::memcpy(&mx, &C.host_status.emergency_max_bits[f], sizeof(mx));
    storage[f].emergency_diffusion_max_interface_speed =
        fmax(storage[f].emergency_diffusion_max_interface_speed, mx);
  }
  if (!C.resident && C.download_state(storage, 0) != 0) return -1;
  return (rc != 0 || fail) ? -1 : 0;
}

// ---- stand-alone halo and seam entry points -------------------------------

// Downloads of one face (receiver >= 0) or all faces.
int download_arrays(gcs::Context &C, gamera_no_storage *st, const int *kinds, int nk,
                    int receiver) {
  for (int f = 0; f < gcs::kFaces; ++f) {
    if (receiver >= 0 && f != receiver) continue;
    for (int q = 0; q < nk; ++q) {
      const int kind = kinds[q];
      int dirs = (kind == gcs::kArrP || kind == gcs::kArrPo || kind == gcs::kArrF ||
                  kind == gcs::kArrM || kind == gcs::kArrE) ? 3 : 1;
      for (int d = 0; d < dirs; ++d) {
        double *host = nullptr;
        switch (kind) {
          case gcs::kArrU: host = st[f].conserved; break;
          case gcs::kArrUo: host = st[f].old_conserved; break;
          case gcs::kArrB: host = (double *)st[f].cell_magnetic; break;
          case gcs::kArrBo: host = (double *)st[f].old_cell_magnetic; break;
          case gcs::kArrP: host = st[f].face_flux[d]; break;
          case gcs::kArrPo: host = st[f].old_face_flux[d]; break;
          case gcs::kArrF: host = st[f].fluid_face_flux[d]; break;
          case gcs::kArrM: host = (double *)st[f].maxwell_face_flux[d]; break;
          case gcs::kArrE: host = st[f].edge_emf[d]; break;
          default: return -1;
        }
        if (C.transfer_array(f, kind, d, false, host) != 0) return -1;
      }
    }
  }
  return 0;
}

int upload_arrays(gcs::Context &C, gamera_no_storage *st, const int *kinds, int nk) {
  for (int f = 0; f < gcs::kFaces; ++f)
    for (int q = 0; q < nk; ++q) {
      const int kind = kinds[q];
      int dirs = (kind == gcs::kArrP || kind == gcs::kArrPo || kind == gcs::kArrF ||
                  kind == gcs::kArrM || kind == gcs::kArrE) ? 3 : 1;
      for (int d = 0; d < dirs; ++d) {
        double *host = nullptr;
        switch (kind) {
          case gcs::kArrU: host = st[f].conserved; break;
          case gcs::kArrUo: host = st[f].old_conserved; break;
          case gcs::kArrB: host = (double *)st[f].cell_magnetic; break;
          case gcs::kArrBo: host = (double *)st[f].old_cell_magnetic; break;
          case gcs::kArrP: host = st[f].face_flux[d]; break;
          case gcs::kArrPo: host = st[f].old_face_flux[d]; break;
          case gcs::kArrF: host = st[f].fluid_face_flux[d]; break;
          case gcs::kArrM: host = (double *)st[f].maxwell_face_flux[d]; break;
          case gcs::kArrE: host = st[f].edge_emf[d]; break;
          default: return -1;
        }
        if (C.transfer_array(f, kind, d, true, host) != 0) return -1;
      }
    }
  return 0;
}

const int kCellArrays[4] = {gcs::kArrU, gcs::kArrUo, gcs::kArrB, gcs::kArrBo};
const int kFaceArrays[2] = {gcs::kArrP, gcs::kArrPo};

bool dims_match(const gcs::Context &C, const size_t active[3], size_t ghost) {
  return active && (size_t)C.X.D.nr == active[0] && (size_t)C.X.D.n == active[1] &&
         (size_t)C.X.D.n == active[2] && (size_t)C.X.D.g == ghost;
}

bool storage_matches(const gcs::Context &C, const gamera_no_storage *st) {
  for (int f = 0; f < gcs::kFaces; ++f)
    if (st[f].cell_extent[0] != (size_t)C.X.D.E0 ||
        st[f].cell_extent[1] != (size_t)C.X.D.E1 ||
        st[f].cell_extent[2] != (size_t)C.X.D.E2)
      return false;
  return true;
}

int cell_halos(gcs::Context &C, gamera_no_storage *st, int receiver) {
  if (upload_arrays(C, st, kCellArrays, 4) != 0) return -1;
  C.reset_status_async();
  gcs::launch_halo_cells_only(C.X, C.stream);
  if (cudaStreamSynchronize(C.stream) != cudaSuccess) return -1;
  return download_arrays(C, st, kCellArrays, 4, receiver);
}

int face_halos(gcs::Context &C, gamera_no_storage *st, int receiver) {
  const int kinds[6] = {gcs::kArrB, gcs::kArrBo, gcs::kArrP, gcs::kArrPo};
  if (upload_arrays(C, st, kinds, 4) != 0) return -1;
  C.reset_status_async();
  gcs::launch_halo_faces_only(C.X, C.stream);
  if (cudaStreamSynchronize(C.stream) != cudaSuccess) return -1;
  return download_arrays(C, st, kFaceArrays, 2, receiver);
}

// Contexts without a grid (state arrays, seams and edge groups only) for
// the entry points that take storage alone, one per active extent.
std::mutex g_topo_mutex;
std::map<std::array<size_t, 4>, gcs_context *> g_topo;

gcs_context *topology_context(const size_t active[3], size_t ghost) {
  if (!active) return nullptr;
  std::lock_guard<std::mutex> lock(g_topo_mutex);
  const std::array<size_t, 4> key{active[0], active[1], active[2], ghost};
  auto it = g_topo.find(key);
  if (it != g_topo.end()) return it->second;
  gcs_context *ctx = new (std::nothrow) gcs_context;
  if (!ctx) return nullptr;
  if (ctx->c.init_topology(active, ghost) != 0) {
    set_last(ctx->c.error);
    delete ctx;
    return nullptr;
  }
  g_topo[key] = ctx;
  return ctx;
}

int radial_outflow(gamera_no_storage storage[6], const size_t active[3], size_t ghost,
                   int receiver) {
  if (!storage || !active || ghost < 4 || active[0] == 0) return -1;
  gcs_context *ctx = topology_context(active, ghost);
  if (!ctx || !storage_matches(ctx->c, storage)) return -1;
  gcs::Context &C = ctx->c;
  if (upload_arrays(C, storage, kCellArrays, 4) != 0) return -1;
  gcs::launch_radial_outflow_all(C.X, C.stream);
  if (cudaStreamSynchronize(C.stream) != cudaSuccess) return -1;
  return download_arrays(C, storage, kCellArrays, 4, receiver);
}

}  // namespace

namespace gcs {
void set_api_error(const char *msg) { set_last(msg); }
Context *context_for_grid(const gamera_no_grid grid[6], const size_t active[3],
                          size_t ghost) {
  gcs_context *ctx = context_for(grid, active, ghost);
  return ctx ? &ctx->c : nullptr;
}
Context *context_of(gcs_context *ctx) { return ctx ? &ctx->c : nullptr; }
bool driver_opts(const gamera_no_advance_options *options,
                 const gamera_no_timestep_options *t, double fraction, Opts *O) {
  if (!std::isfinite(fraction) || fraction <= 0.0) return false;
  if (!make_opts(options, true, O) || !set_timestep_opts(t, O)) return false;
  O->dt_fraction = fraction;
  return true;
}
int enqueue_driver_step(gcs_context *ctx, const Opts &O) {
  return run_step(ctx, O, 1, nullptr);
}
}  // namespace gcs

extern "C" {

// ------------------------------------------------------------------ Part 1

int gamera_cs_advance_six_with_background_planned(
    const gamera_no_grid grid[6], gamera_no_storage storage[6],
    const size_t active[3], size_t ghost, double predictor_ratio, double dt,
    const gamera_no_advance_options *options,
    const gamera_no_background_field background[6],
    const gamera_cs_halo_plan *halo_plan,
    gamera_cs_radial_boundary_function radial_boundary, double current_time,
    double previous_time, void *boundary_context) {
  if (grid == nullptr || active == nullptr) return -1;
  gcs_context *ctx = halo_plan ? halo_plan->ctx : context_for(grid, active, ghost);
  return drop_in_step(ctx, grid, storage, active, ghost, predictor_ratio, dt,
                      options, background, radial_boundary, current_time,
                      previous_time, boundary_context);
}

int gamera_cs_advance_six_with_background(
    const gamera_no_grid grid[6], gamera_no_storage storage[6],
    const size_t active[3], size_t ghost, double predictor_ratio, double dt,
    const gamera_no_advance_options *options,
    const gamera_no_background_field background[6],
    gamera_cs_radial_boundary_function radial_boundary, double current_time,
    double previous_time, void *boundary_context) {
  return gamera_cs_advance_six_with_background_planned(
      grid, storage, active, ghost, predictor_ratio, dt, options, background,
      nullptr, radial_boundary, current_time, previous_time, boundary_context);
}

int gamera_cs_advance_six_with_boundary(
    const gamera_no_grid grid[6], gamera_no_storage storage[6],
    const size_t active[3], size_t ghost, double predictor_ratio, double dt,
    const gamera_no_advance_options *options,
    gamera_cs_radial_boundary_function radial_boundary, double current_time,
    double previous_time, void *boundary_context) {
  return gamera_cs_advance_six_with_background(
      grid, storage, active, ghost, predictor_ratio, dt, options, nullptr,
      radial_boundary, current_time, previous_time, boundary_context);
}

int gamera_cs_advance_six(const gamera_no_grid grid[6],
                          gamera_no_storage storage[6], const size_t active[3],
                          size_t ghost, double predictor_ratio, double dt,
                          const gamera_no_advance_options *options) {
  return gamera_cs_advance_six_with_boundary(grid, storage, active, ghost,
                                             predictor_ratio, dt, options,
                                             nullptr, 0.0, 0.0, nullptr);
}

int gamera_cs_halo_plan_create(const gamera_no_grid grid[6],
                               const size_t active[3], size_t ghost,
                               gamera_cs_halo_plan **out) {
  if (out == nullptr) return -1;
  *out = nullptr;
  gcs_context *ctx = create_context(grid, active, ghost);
  if (!ctx) return -1;
  gamera_cs_halo_plan *plan = new (std::nothrow) gamera_cs_halo_plan;
  if (!plan) {
    delete ctx;
    return -1;
  }
  plan->ctx = ctx;
  *out = plan;
  return 0;
}

void gamera_cs_halo_plan_destroy(gamera_cs_halo_plan *plan) {
  if (!plan) return;
  delete plan->ctx;
  delete plan;
}

int gamera_cs_fill_tangential_cell_halos_planned(const gamera_cs_halo_plan *plan,
                                                 const gamera_no_grid grid[6],
                                                 gamera_no_storage storage[6]) {
  if (!plan || !grid || !storage || !plan->ctx->c.grid_matches(grid)) return -1;
  gcs::Context &C = plan->ctx->c;
  if (C.upload_state(storage) != 0) return -1;
  C.reset_status_async();
  gcs::launch_halo_cells_only(C.X, C.stream);
  if (cudaStreamSynchronize(C.stream) != cudaSuccess) return -1;
  return C.download_state(storage, 0);
}

int gamera_cs_fill_magnetic_face_halos_planned(const gamera_cs_halo_plan *plan,
                                               const gamera_no_grid grid[6],
                                               gamera_no_storage storage[6]) {
  if (!plan || !grid || !storage || !plan->ctx->c.grid_matches(grid)) return -1;
  gcs::Context &C = plan->ctx->c;
  if (C.upload_state(storage) != 0) return -1;
  C.reset_status_async();
  gcs::launch_halo_faces_only(C.X, C.stream);
  if (cudaStreamSynchronize(C.stream) != cudaSuccess) return -1;
  return C.download_state(storage, 0);
}

// cubedsphere_halo.c:103-115 (a scalar predicate; no device work)
int gamera_cs_halo_valid_state(const double state[5]) {
  const double rho = state[0];
  if (!std::isfinite(rho) || rho <= 0.0) return 0;
  double m2 = 0.0;
  for (int d = 0; d < 3; ++d) {
    const double m = state[1 + d];
    if (!std::isfinite(m)) return 0;
    m2 += m * m;
  }
  return std::isfinite(state[4]) && state[4] > 0.5 * m2 / rho;
}

// cubedsphere_halo.h:52-59
int gamera_cs_fill_tangential_cell_halos_planned_face(const gamera_cs_halo_plan *plan,
                                                      const gamera_no_grid grid[6],
                                                      gamera_no_storage storage[6],
                                                      int receiver) {
  if (!plan || !grid || !storage || receiver < 0 || receiver >= 6 ||
      !plan->ctx->c.grid_matches(grid))
    return -1;
  return cell_halos(plan->ctx->c, storage, receiver);
}

int gamera_cs_fill_magnetic_face_halos_planned_face(const gamera_cs_halo_plan *plan,
                                                    const gamera_no_grid grid[6],
                                                    gamera_no_storage storage[6],
                                                    int receiver) {
  if (!plan || !grid || !storage || receiver < 0 || receiver >= 6 ||
      !plan->ctx->c.grid_matches(grid))
    return -1;
  return face_halos(plan->ctx->c, storage, receiver);
}

// cubedsphere_halo.h:68-71 (the device plan of the grid is built on first use)
int gamera_cs_fill_tangential_cell_halos(const gamera_no_grid grid[6],
                                         gamera_no_storage storage[6],
                                         const size_t active[3], size_t ghost) {
  if (!grid || !storage || !active) return -1;
  gcs_context *ctx = context_for(grid, active, ghost);
  if (!ctx || !dims_match(ctx->c, active, ghost) || !storage_matches(ctx->c, storage))
    return -1;
  return cell_halos(ctx->c, storage, -1);
}

// cubedsphere_halo.h:84-87
int gamera_cs_fill_magnetic_face_halos(const gamera_no_grid grid[6],
                                       gamera_no_storage storage[6],
                                       const size_t active[3], size_t ghost) {
  if (!grid || !storage || !active) return -1;
  gcs_context *ctx = context_for(grid, active, ghost);
  if (!ctx || !dims_match(ctx->c, active, ghost) || !storage_matches(ctx->c, storage))
    return -1;
  return face_halos(ctx->c, storage, -1);
}

// cubedsphere_halo.h:74-79
int gamera_cs_fill_radial_outflow_cells(gamera_no_storage storage[6],
                                        const size_t active[3], size_t ghost) {
  return radial_outflow(storage, active, ghost, -1);
}

int gamera_cs_fill_radial_outflow_cells_face(gamera_no_storage storage[6],
                                             const size_t active[3], size_t ghost,
                                             int receiver) {
  if (receiver < 0 || receiver >= 6) return -1;
  return radial_outflow(storage, active, ghost, receiver);
}

// cubedsphere_interface.h:13-18
int gamera_cs_sync_magnetic_face_flux(gamera_no_storage storage[6],
                                      const size_t active[3], size_t ghost) {
  if (!storage || !active) return -1;
  gcs_context *ctx = topology_context(active, ghost);
  if (!ctx || !storage_matches(ctx->c, storage)) return -1;
  gcs::Context &C = ctx->c;
  if (upload_arrays(C, storage, kFaceArrays, 2) != 0) return -1;
  C.reset_status_async();
  gcs::launch_seam_sync(C.X, 1, C.stream);
  if (cudaStreamSynchronize(C.stream) != cudaSuccess) return -1;
  return download_arrays(C, storage, kFaceArrays, 2, -1);
}

int gamera_cs_sync_mhd_face_fluxes(gamera_no_storage storage[6], const size_t active[3],
                                   size_t ghost) {
  if (!storage || !active) return -1;
  gcs_context *ctx = topology_context(active, ghost);
  if (!ctx || !storage_matches(ctx->c, storage)) return -1;
  gcs::Context &C = ctx->c;
  const int kinds[2] = {gcs::kArrF, gcs::kArrM};
  if (upload_arrays(C, storage, kinds, 2) != 0) return -1;
  C.reset_status_async();
  gcs::launch_seam_sync(C.X, 0, C.stream);
  if (cudaStreamSynchronize(C.stream) != cudaSuccess) return -1;
  return download_arrays(C, storage, kinds, 2, -1);
}

// cubedsphere_interface.h:22-25 and the plan of :29-37 (the plan is the
// context of the grid; the edge groups are its immutable edge identities)
int gamera_cs_sync_edge_emf(const gamera_no_grid grid[6], gamera_no_storage storage[6],
                            const size_t active[3], size_t ghost) {
  if (!grid || !storage || !active) return -1;
  gcs_context *ctx = context_for(grid, active, ghost);
  if (!ctx || !dims_match(ctx->c, active, ghost) || !storage_matches(ctx->c, storage))
    return -1;
  gcs::Context &C = ctx->c;
  const int kinds[1] = {gcs::kArrE};
  if (upload_arrays(C, storage, kinds, 1) != 0) return -1;
  C.reset_status_async();
  gcs::launch_edge_sync(C.X, C.stream);
  if (cudaStreamSynchronize(C.stream) != cudaSuccess) return -1;
  return download_arrays(C, storage, kinds, 1, -1);
}

int gamera_cs_edge_sync_plan_create(const gamera_no_grid grid[6], const size_t active[3],
                                    size_t ghost, gamera_cs_edge_sync_plan **out) {
  if (!out) return -1;
  *out = nullptr;
  if (!grid || !active) return -1;
  gcs_context *ctx = context_for(grid, active, ghost);
  if (!ctx || !dims_match(ctx->c, active, ghost)) return -1;
  *out = new (std::nothrow) gamera_cs_edge_sync_plan{ctx};
  return *out ? 0 : -1;
}

void gamera_cs_edge_sync_plan_destroy(gamera_cs_edge_sync_plan *plan) { delete plan; }

int gamera_cs_sync_edge_emf_planned(const gamera_cs_edge_sync_plan *plan,
                                    gamera_no_storage storage[6]) {
  if (!plan || !storage || !storage_matches(plan->ctx->c, storage)) return -1;
  gcs::Context &C = plan->ctx->c;
  const int kinds[1] = {gcs::kArrE};
  if (upload_arrays(C, storage, kinds, 1) != 0) return -1;
  C.reset_status_async();
  gcs::launch_edge_sync(C.X, C.stream);
  if (cudaStreamSynchronize(C.stream) != cudaSuccess) return -1;
  return download_arrays(C, storage, kinds, 1, -1);
}

// ------------------------------------------------------------------ Part 2

gcs_context *gcs_context_create(const gamera_no_grid grid[6],
                                const size_t active[3], size_t ghost) {
  return create_context(grid, active, ghost);
}

gcs_context *gcs_context_create_case(int kind, size_t nr, size_t n,
                                     unsigned long long seed) {
  gcs_context *ctx = new (std::nothrow) gcs_context;
  if (!ctx) {
    set_last("out of host memory");
    return nullptr;
  }
  if (ctx->c.init_case(kind, nr, n, seed) != 0) {
    set_last(ctx->c.error);
    delete ctx;
    return nullptr;
  }
  return ctx;
}

int gcs_case_options(int kind, gamera_no_advance_options *o,
                     gamera_no_timestep_options *t) {
  if (!o || !t || kind < 0 || kind > 3) return -1;
  const double g = 5.0 / 3.0;
  std::memset(o, 0, sizeof(*o));
  std::memset(t, 0, sizeof(*t));
  if (kind == 0) {
    o->stress = {g, 1e-12, 1e-12, 1.0, 0.0, 0.0, 100.0, true, false, false, false};
    o->emf = {1e-12, 1.0, 0.0, 100.0, 0.8, 0.01, false, false};
    o->update = {g, 1e-12, 1e-12, 100.0, true, false, false};
    *t = {g, 1e-12, 1e-12, 0.8, 100.0, true, false, false};
  } else if (kind == 1) {
    o->stress = {g, 1e-12, 1e-12, 1.0, 0.25, 0.25, 100.0, true, true, false, false};
    o->emf = {1e-12, 1.0, 0.5, 100.0, 0.3, 0.001, false, false};
    o->update = {g, 1e-12, 1e-12, 100.0, true, false, false};
    *t = {g, 1e-12, 1e-12, 0.3, 100.0, true, false, false};
  } else {
    // Earth driver options (test_cubedsphere_dipole_background.c:405-444)
    o->stress = {g, 1e-6, 1e-8, 1.0, 0.25, 0.25, 10.0, true, true, true, true};
    o->emf = {1e-6, 1.0, 0.5, 10.0, 0.3, 0.0, true, true};
    o->update = {g, 1e-6, 1e-8, 10.0, true, true, true};
    *t = {g, 1e-6, 1e-8, 0.3, 10.0, true, true, true};
  }
  return 0;
}

int gcs_context_advance_host(gcs_context *ctx, gamera_no_storage storage[6],
                             const gamera_no_advance_options *options,
                             double predictor_ratio, double dt) {
  if (!ctx) return -1;
  const size_t active[3] = {(size_t)ctx->c.X.D.nr, (size_t)ctx->c.X.D.n,
                            (size_t)ctx->c.X.D.n};
  return drop_in_step(ctx, nullptr, storage, active, (size_t)ctx->c.X.D.g,
                      predictor_ratio, dt, options, nullptr, nullptr, 0.0, 0.0,
                      nullptr);
}

// Copy one device node array (nodes_per_face doubles of face `face`) to the
// host, for diagnostics and set-up tests.  which: 0 volume, 1 area[d],
// 2 face normal[d][q], 3 face t1[d][q], 4 face t2[d][q], 5 B0 cell[q],
// 6 B0 force[q], 7 face B0[d][q], 8 face B0 normal[d], 9 edge B0.t1[d],
// 10 edge B0.t2[d], 11 central8 volume[d], 12 edge length[d],
// 13 recovery map column q (0..17).
int gcs_context_debug_array(gcs_context *ctx, int which, int face, int d, int q,
                            double *out, size_t capacity) {
  if (!ctx || !out || face < 0 || face >= 6 || d < 0 || d > 2) return -1;
  gcs::Context &C = ctx->c;
  const long long nn = C.X.D.Nn;
  if ((long long)capacity < nn) return -1;
  const gcs::DevGeom &G = C.X.G;
  const gcs::DevBg &B = C.X.BG;
  const double *src = nullptr;
  const bool bgok = C.bg_pool != nullptr;
  switch (which) {
    case 0: src = G.vol; break;
    case 1: src = G.area[d]; break;
    case 2: src = G.fn[d][q % 3]; break;
    case 3: src = G.ft1[d][q % 3]; break;
    case 4: src = G.ft2[d][q % 3]; break;
    case 5: src = bgok ? B.b0[q % 3] : nullptr; break;
    case 6: src = bgok ? B.force[q % 3] : nullptr; break;
    case 7: src = bgok ? B.fb0[d][q % 3] : nullptr; break;
    case 8: src = bgok ? B.fb0n[d] : nullptr; break;
    case 9: src = bgok ? B.eb0t1[d] : nullptr; break;
    case 10: src = bgok ? B.eb0t2[d] : nullptr; break;
    case 11: src = G.iv[d]; break;
    case 12: src = G.elen[d]; break;
    case 13: src = G.rec[q % 18]; break;
    default: return -1;
  }
  if (!src) return -1;
  if (cudaMemcpyAsync(out, src + face * nn, nn * sizeof(double),
                      cudaMemcpyDeviceToHost, C.stream) != cudaSuccess ||
      cudaStreamSynchronize(C.stream) != cudaSuccess)
    return -1;
  return 0;
}

int gcs_context_dims(const gcs_context *ctx, size_t active[3], size_t *ghost) {
  if (!ctx || !active || !ghost) return -1;
  active[0] = (size_t)ctx->c.X.D.nr;
  active[1] = active[2] = (size_t)ctx->c.X.D.n;
  *ghost = (size_t)ctx->c.X.D.g;
  return 0;
}

void gcs_context_destroy(gcs_context *ctx) {
  if (!ctx) return;
  gcs::earth_forget(ctx->c);
  for (cudaEvent_t e : ctx->events) cudaEventDestroy(e);
  delete ctx;
}

const char *gcs_last_error(void) { return g_last_error; }
const char *gcs_context_error(const gcs_context *ctx) {
  return ctx ? ctx->c.error : g_last_error;
}

int gcs_context_upload_background(gcs_context *ctx,
                                  const gamera_no_background_field bg[6]) {
  if (!ctx || !bg) return -1;
  ctx->c.bulk_bg_dirty = 1;
  if (ctx->c.upload_background(bg) != 0) return -1;
  return ctx->c.X.bulk ? ctx->c.enable_bulk(1) : 0;
}

int gcs_context_upload_state(gcs_context *ctx, const gamera_no_storage st[6]) {
  if (!ctx || !st) return -1;
  return ctx->c.upload_state(st);
}

int gcs_context_download_state(gcs_context *ctx, gamera_no_storage st[6],
                               int scratch) {
  if (!ctx || !st) return -1;
  return ctx->c.download_state(st, scratch);
}

int gcs_context_step(gcs_context *ctx, const gamera_no_advance_options *options,
                     double ratio, double dt) {
  if (!ctx || !std::isfinite(dt) || dt <= 0.0 || !std::isfinite(ratio)) return -1;
  gcs::Opts O;
  if (!make_opts(options, ctx->c.bg_uploaded != 0, &O)) return -1;
  gcs::Context &C = ctx->c;
  gcs::StepParams p;
  std::memset(&p, 0, sizeof(p));
  p.dt = dt;
  p.ratio = ratio;
  if (cudaMemcpyAsync(C.X.params, &p, sizeof(p), cudaMemcpyHostToDevice,
                      C.stream) != cudaSuccess)
    return -1;
  C.reset_status_async();
  const int rc = run_step(ctx, O, 0, nullptr);
  const bool fail = device_failed(C);
  if (fail) report_failure(C);
  return (rc != 0 || fail) ? -1 : 0;
}

int gcs_context_step_earth(gcs_context *ctx, gcs_earth *earth,
                           const gamera_no_advance_options *options,
                           double ratio, double dt, double current_time,
                           double previous_time) {
  if (!ctx || !earth || earth->C != &ctx->c || !options) return -1;
  if (!std::isfinite(current_time) || !std::isfinite(previous_time) || !(dt > 0.0) ||
      !std::isfinite(dt)) {
    set_last("invalid step times");
    return -1;
  }
  gcs::Opts O;
  if (!make_opts(options, ctx->c.bg_uploaded != 0, &O)) return -1;
  gcs::Context &C = ctx->c;
  gcs::StepParams p;
  std::memset(&p, 0, sizeof(p));
  p.dt = dt;
  p.ratio = ratio;
  if (cudaMemcpyAsync(C.X.params, &p, sizeof(p), cudaMemcpyHostToDevice,
                      C.stream) != cudaSuccess)
    return -1;
  C.reset_status_async();
  if (gcs::earth_sync_mi(earth, earth->mi) != 0) return -1;
  // the reference driver sets step_time = current time, step_dt = dt
  // (test_cubedsphere_dipole_background.c:667-668)
  const gcs::EarthStep es{&earth->dev, current_time, previous_time, current_time, dt, 0};
  const int rc = run_step(ctx, O, 0, nullptr, &es);
  const bool fail = device_failed(C);
  if (fail) report_failure(C);
  return (rc != 0 || fail) ? -1 : 0;
}

int gcs_context_timestep(gcs_context *ctx, const gamera_no_timestep_options *t,
                         double *dt) {
  if (!ctx || !dt) return -1;
  gcs::Opts O;
  std::memset(&O, 0, sizeof(O));
  if (!set_timestep_opts(t, &O)) return -1;
  if (O.t_bg && !ctx->c.bg_uploaded) return -1;
  gcs::Context &C = ctx->c;
  C.reset_status_async();
  gcs::launch_timestep(C.X, O, C.stream);
  if (device_failed(C)) return -1;
  double v;
  std::memcpy(&v, &C.host_status.cfl_min_bits, sizeof(v));
  *dt = v;
  return 0;
}

}  // extern "C"

namespace {

// The driver loop of gcs_context_run, optionally with the device Earth
// boundary in driver mode (times from the step parameters).
int context_run(gcs_context *ctx, const gamera_no_advance_options *options,
                const gamera_no_timestep_options *t, double fraction, int steps,
                int use_graph, const gcs::EarthStep *es) {
  if (!ctx || steps < 0 || !std::isfinite(fraction) || fraction <= 0.0) return -1;
  gcs::Opts O;
  if (!make_opts(options, ctx->c.bg_uploaded != 0, &O) ||
      !set_timestep_opts(t, &O))
    return -1;
  O.dt_fraction = fraction;
  gcs::Context &C = ctx->c;
  if (C.mi_graph != nullptr && gcs::mi_before_run(C.mi_graph) != 0) return -1;
  gcs::StepParams p;
  if (cudaMemcpyAsync(&p, C.X.params, sizeof(p), cudaMemcpyDeviceToHost,
                      C.stream) != cudaSuccess ||
      cudaStreamSynchronize(C.stream) != cudaSuccess)
    return -1;
  if (p.step == 0 && p.dt == 0.0) {
    // first step: dt = fraction * CFL step of the initial state, ratio 0
    double local;
    if (gcs_context_timestep(ctx, t, &local) != 0) return -1;
    std::memset(&p, 0, sizeof(p));
    p.dt = fraction * local;
    p.ratio = 0.0;
    if (cudaMemcpyAsync(C.X.params, &p, sizeof(p), cudaMemcpyHostToDevice,
                        C.stream) != cudaSuccess)
      return -1;
    C.reset_status_async();
  }
  if (use_graph && !C.profiling) {
    unsigned long long key = 1469598103934665603ULL;
    const unsigned char *b = (const unsigned char *)&O;
    for (size_t q = 0; q < sizeof(O); ++q) key = (key ^ b[q]) * 1099511628211ULL;
    key = (key ^ (unsigned long long)C.X.bulk) * 1099511628211ULL;
    key = (key ^ (unsigned long long)(0x5354ULL + C.X.flux_staged)) * 1099511628211ULL;
    key = (key ^ (unsigned long long)(uintptr_t)C.mi_graph) * 1099511628211ULL;
    if (es) {
      const unsigned char *e = (const unsigned char *)es->dev;
      for (size_t q = 0; q < sizeof(*es->dev); ++q) key = (key ^ e[q]) * 1099511628211ULL;
      key = (key ^ 0x45415254ULL) * 1099511628211ULL;
    }
    for (int f = 0; f < gcs::kTileFamilies; ++f)
      key = (key ^ (unsigned long long)(C.X.tile[f].bx * 64 + C.X.tile[f].by)) *
            1099511628211ULL;
    if (C.pc_on) {
      const unsigned char *pb = (const unsigned char *)&C.pc;
      for (size_t q = 0; q < sizeof(C.pc); ++q) key = (key ^ pb[q]) * 1099511628211ULL;
      key = (key ^ 0x50524553ULL) * 1099511628211ULL;
    }
    if (!C.graph_exec || C.graph_key != key) {
      if (C.graph_exec) cudaGraphExecDestroy(C.graph_exec);
      C.graph_exec = nullptr;
      cudaGraph_t graph;
      if (cudaStreamBeginCapture(C.stream, cudaStreamCaptureModeThreadLocal) !=
          cudaSuccess)
        return -1;
      run_step(ctx, O, 1, nullptr, es);
      if (cudaStreamEndCapture(C.stream, &graph) != cudaSuccess) return -1;
      const cudaError_t ie = cudaGraphInstantiate(&C.graph_exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ie != cudaSuccess) return -1;
      C.graph_key = key;
    }
    for (int q = 0; q < steps; ++q)
      if (cudaGraphLaunch(C.graph_exec, C.stream) != cudaSuccess) {
        if (C.mi_graph != nullptr) gcs::mi_after_run(C.mi_graph);
        return -1;
      }
  } else {
    for (int q = 0; q < steps; ++q)
      if (run_step(ctx, O, 1, nullptr, es) != 0) {
        if (C.mi_graph != nullptr) gcs::mi_after_run(C.mi_graph);
        return -1;
      }
  }
  if (C.mi_graph != nullptr) gcs::mi_after_run(C.mi_graph);
  return 0;
}

}  // namespace

extern "C" {

int gcs_context_run(gcs_context *ctx, const gamera_no_advance_options *options,
                    const gamera_no_timestep_options *t, double fraction,
                    int steps, int use_graph) {
  return context_run(ctx, options, t, fraction, steps, use_graph, nullptr);
}

int gcs_context_run_earth(gcs_context *ctx, gcs_earth *earth,
                          const gamera_no_advance_options *options,
                          const gamera_no_timestep_options *t, double fraction,
                          int steps, int use_graph) {
  if (!ctx || !earth || earth->C != &ctx->c) return -1;
  if (gcs::earth_sync_mi(earth, earth->mi) != 0) return -1;
  const gcs::EarthStep es{&earth->dev, 0.0, 0.0, 0.0, 0.0, 1};
  return context_run(ctx, options, t, fraction, steps, use_graph, &es);
}

int gcs_context_sync(gcs_context *ctx) {
  if (!ctx) return -1;
  if (cudaStreamSynchronize(ctx->c.stream) != cudaSuccess) return -1;
  gcs::DevStatus s;
  if (ctx->c.read_status(&s) != 0) return -1;
  ctx->c.host_status = s;
  if (s.first) {
    report_failure(ctx->c);
    return -1;
  }
  return 0;
}

int gcs_context_time(gcs_context *ctx, double *time) {
  if (!ctx || !time) return -1;
  gcs::StepParams p;
  if (cudaMemcpyAsync(&p, ctx->c.X.params, sizeof(p), cudaMemcpyDeviceToHost,
                      ctx->c.stream) != cudaSuccess ||
      cudaStreamSynchronize(ctx->c.stream) != cudaSuccess)
    return -1;
  *time = p.time;
  return 0;
}

int gcs_context_params(gcs_context *ctx, double *dt, double *ratio,
                       double *cfl_min, int *steps) {
  if (!ctx) return -1;
  gcs::StepParams p;
  if (cudaMemcpyAsync(&p, ctx->c.X.params, sizeof(p), cudaMemcpyDeviceToHost,
                      ctx->c.stream) != cudaSuccess ||
      cudaStreamSynchronize(ctx->c.stream) != cudaSuccess)
    return -1;
  if (dt) *dt = p.dt;
  if (ratio) *ratio = p.ratio;
  if (cfl_min) *cfl_min = p.cfl_min;
  if (steps) *steps = p.step;
  return 0;
}

int gcs_context_set_params(gcs_context *ctx, double dt, double ratio,
                           double dt_prev, int steps) {
  if (!ctx) return -1;
  gcs::StepParams p;
  std::memset(&p, 0, sizeof(p));
  p.dt = dt;
  p.ratio = ratio;
  p.dt_prev = dt_prev;
  p.step = steps;
  if (cudaMemcpyAsync(ctx->c.X.params, &p, sizeof(p), cudaMemcpyHostToDevice,
                      ctx->c.stream) != cudaSuccess ||
      cudaStreamSynchronize(ctx->c.stream) != cudaSuccess)
    return -1;
  return 0;
}

int gcs_context_failure(gcs_context *ctx, int *dir, int *face, int *i, int *j,
                        int *k) {
  if (!ctx) return -1;
  gcs::DevStatus s;
  if (ctx->c.read_status(&s) != 0) return -1;
  const unsigned long long v = s.first;
  if (dir) *dir = (int)(v >> 52) & 0xf;
  if (face) *face = (int)(v >> 48) & 0xf;
  if (i) *i = (int)(v >> 32) & 0xffff;
  if (j) *j = (int)(v >> 16) & 0xffff;
  if (k) *k = (int)v & 0xffff;
  return (int)(v >> 56) & 0xff;
}

int gcs_context_reset_failure(gcs_context *ctx) {
  if (!ctx) return -1;
  ctx->c.reset_status_async();
  return cudaStreamSynchronize(ctx->c.stream) == cudaSuccess ? 0 : -1;
}

uintptr_t gcs_context_stream(gcs_context *ctx) {
  return ctx ? (uintptr_t)ctx->c.stream : 0;
}

int gcs_context_set_flux_staging(gcs_context *ctx, int on) {
  if (!ctx || (on != 0 && on != 1)) return -1;
  ctx->c.X.flux_staged = on;
  return 0;
}

int gcs_context_set_profiling(gcs_context *ctx, int on) {
  if (!ctx) return -1;
  ctx->c.profiling = on;
  return 0;
}

int gcs_context_stage_times(gcs_context *ctx, double *ms, long long *calls,
                            int capacity) {
  if (!ctx) return -1;
  if (cudaStreamSynchronize(ctx->c.stream) != cudaSuccess) return -1;
  for (size_t q = 0; q < ctx->event_slot.size(); ++q) {
    float t = 0.0f;
    cudaEventElapsedTime(&t, ctx->events[2 * q], ctx->events[2 * q + 1]);
    const int slot = ctx->event_slot[q];
    ctx->c.stage_ms[slot] += t;
    ctx->c.stage_calls[slot] += 1;
  }
  // events are chained (end of one = start of the next): destroy each once
  std::vector<cudaEvent_t> uniq;
  for (size_t q = 0; q < ctx->events.size(); ++q) {
    bool seen = false;
    for (cudaEvent_t e : uniq)
      if (e == ctx->events[q]) { seen = true; break; }
    if (!seen) uniq.push_back(ctx->events[q]);
  }
  for (cudaEvent_t e : uniq) cudaEventDestroy(e);
  ctx->events.clear();
  ctx->event_slot.clear();
  const int n = capacity < kSlotCount ? capacity : kSlotCount;
  for (int q = 0; q < n; ++q) {
    if (ms) ms[q] = ctx->c.stage_ms[q];
    if (calls) calls[q] = ctx->c.stage_calls[q];
  }
  return n;
}

const char *gcs_stage_name(int slot) {
  return slot >= 0 && slot < kSlotCount ? kSlotNames[slot] : "";
}

size_t gcs_context_device_bytes(const gcs_context *ctx) {
  if (!ctx) return 0;
  return ctx->c.pool_bytes + ctx->c.bg_bytes + ctx->c.plans_bytes +
         ctx->c.staging_bytes;
}

gcs_context *gcs_halo_plan_context(gamera_cs_halo_plan *plan) {
  return plan ? plan->ctx : nullptr;
}

int gcs_context_set_resident(gcs_context *ctx, int on) {
  if (!ctx) return -1;
  ctx->c.resident = on;
  if (!on) ctx->c.resident_storage = nullptr;
  return 0;
}

int gcs_context_set_precision(gcs_context *ctx, int fp32_bulk) {
  if (!ctx) {
    set_last("null context");
    return -1;
  }
  if (ctx->c.enable_bulk(fp32_bulk ? 1 : 0) != 0) {
    set_last(ctx->c.error);
    return -1;
  }
  return 0;
}

int gcs_context_precision(const gcs_context *ctx) { return ctx ? ctx->c.X.bulk : -1; }

int gcs_context_set_bulk_threshold(gcs_context *ctx, double b0_threshold) {
  if (!ctx || !std::isfinite(b0_threshold) || b0_threshold < 0.0) {
    set_last("invalid threshold");
    return -1;
  }
  if (ctx->c.set_bulk_split(b0_threshold) != 0) {
    set_last(ctx->c.error);
    return -1;
  }
  return 0;
}

int gcs_context_bulk_split(const gcs_context *ctx) {
  return ctx ? ctx->c.X.bulk_split : -1;
}

}  // extern "C"
