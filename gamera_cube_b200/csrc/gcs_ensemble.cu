// Batched ensembles of uneven-resolution solar-wind runs (no reference
// counterpart) and the launch-tile autotuner.
//
// An ensemble is a list of wind runs, each with its own angular size
// (radial = the caller's choice, 2n for the seeded draw), upstream driver
// and noise seed.  Runs of equal size share one grid: the first of a size
// is a full device-built case (geometry, background, halo/seam/edge plans,
// FP32 metric copies, per-step scratch); every further run of that size
// owns only the state that lives from step to step (22 doubles per node
// against about 250 for a full case), which is what lets sixteen runs of up
// to 6 x 128 x 128 x 256 cells fit in one GPU's HBM.  One ensemble step is
// one CUDA graph: one branch per grid size, the runs of a size in sequence
// inside it (they share the scratch arrays), each run with its own device
// time step, predictor ratio and failure status, exactly the step
// gcs_context_run replays for a single run.
//
// The autotuner times the tile candidates of each kernel family (threads
// along the flattened (j, k) plane x radial layers per block) on a run's
// own state and keeps the fastest per family and grid size.  It times only
// the families whose kernels write nothing but per-step scratch (predictor,
// flux sweeps, face velocities, edge EMFs, the CFL reduction), so tuning
// leaves the state untouched; CT and the cell update keep their default
// tile.
#include "gcs_context.h"
#include "gcs_error.h"
#include "gamera_cs_b200.h"

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

namespace {

using gcs::Tile;

// Tile candidates (bx, by); each family keeps those within its limit.
constexpr Tile kCandidates[] = {{128, 1}, {64, 2}, {32, 4}, {96, 1}, {64, 1},
                                {256, 1}, {128, 2}, {64, 4}, {32, 8}};

bool tile_ok(int family, int bx, int by) {
  if (family < 0 || family >= gcs::kTileFamilies || bx < 1 || by < 1) return false;
  const int t = bx * by;
  return t % 32 == 0 && t <= gcs::kTileMaxThreads[family] && by <= 64;
}

bool tuned_family(int f) {
  return f == gcs::kTilePredict || f == gcs::kTileFlux || f == gcs::kTileFaceVelocity ||
         f == gcs::kTileEdgeEmf || f == gcs::kTileRecover;
}

void launch_family(const gcs::Ctx &X, const gcs::Opts &O, int family, cudaStream_t s) {
  switch (family) {
    case gcs::kTilePredict: gcs::launch_predict(X, O, s); break;
    case gcs::kTileFlux: gcs::launch_flux(X, O, s); break;
    case gcs::kTileFaceVelocity: gcs::launch_face_velocities(X, O, s); break;
    case gcs::kTileEdgeEmf: gcs::launch_edge_emfs(X, O, s); break;
    case gcs::kTileRecover: gcs::launch_timestep(X, O, s); break;
    default: break;
  }
}

uint64_t mix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}

// Device bytes of a full wind case and of a run sharing its grid, per the
// allocations of Context::allocate, allocate_background, enable_bulk,
// init_member and the staging buffer (plans excluded: a few MB).
void case_bytes(size_t nr, size_t n, int bulk, double *full, double *member) {
  const double nodes = 6.0 * (double)(nr + 9) * (double)(n + 9) * (double)(n + 9);
  const double cells = (double)(nr + 8) * (double)(n + 8) * (double)(n + 8);
  *full = nodes * (176.0 * 8.0 + 4.0 + 24.0 * 8.0 + (bulk ? 108.0 * 4.0 : 0.0)) +
          cells * (double)sizeof(gamera_no_cell_geometry);
  *member = nodes * 22.0 * 8.0;
}

}  // namespace

struct gcs_ensemble {
  std::vector<gcs_context *> runs;
  std::vector<int> owner;        // run index whose grid each run uses
  std::vector<int> prev;         // previous run on the same grid, -1 first
  std::vector<cudaEvent_t> done;
  gcs::Opts O{};
  gamera_no_advance_options options{};
  gamera_no_timestep_options timestep{};
  double fraction = 0.5;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;
  cudaGraphExec_t exec = nullptr;
  size_t nodes = 0;
  int grids = 0;
  int started = 0;
  ~gcs_ensemble() {
    if (exec) cudaGraphExecDestroy(exec);
    for (cudaEvent_t e : done)
      if (e) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    // runs on a shared grid first: they borrow their owner's arrays
    for (size_t i = 0; i < runs.size(); ++i)
      if (runs[i] && owner[i] != (int)i) delete runs[i];
    for (size_t i = 0; i < runs.size(); ++i)
      if (runs[i] && owner[i] == (int)i) delete runs[i];
    if (stream) cudaStreamDestroy(stream);
  }
};

extern "C" {

gcs_context *gcs_context_create_wind(size_t nr, size_t n, unsigned long long seed,
                                     const gcs_wind_driver *driver) {
  if (!driver || !std::isfinite(driver->density_cm3) || driver->density_cm3 <= 0.0 ||
      !std::isfinite(driver->velocity_x_kms) || !std::isfinite(driver->temperature_k) ||
      driver->temperature_k <= 0.0 || !std::isfinite(driver->bz_nt)) {
    gcs::set_api_error("invalid wind driver");
    return nullptr;
  }
  gcs_context *ctx = new (std::nothrow) gcs_context;
  if (!ctx) {
    gcs::set_api_error("out of host memory");
    return nullptr;
  }
  const gcs::WindInit w = gcs::driven_wind(driver->density_cm3, driver->velocity_x_kms,
                                           driver->temperature_k, driver->bz_nt);
  if (ctx->c.init_case(2, nr, n, seed, &w) != 0) {
    gcs::set_api_error(ctx->c.error);
    delete ctx;
    return nullptr;
  }
  return ctx;
}

int gcs_tile_limit(int family) {
  return family >= 0 && family < gcs::kTileFamilies ? gcs::kTileMaxThreads[family] : -1;
}

int gcs_context_set_tile(gcs_context *ctx, int family, int bx, int by) {
  if (!ctx || !tile_ok(family, bx, by)) {
    gcs::set_api_error("invalid tile");
    return -1;
  }
  ctx->c.X.tile[family] = Tile{bx, by};
  return 0;
}

int gcs_context_tile(const gcs_context *ctx, int family, int *bx, int *by) {
  if (!ctx || family < 0 || family >= gcs::kTileFamilies) return -1;
  if (bx) *bx = ctx->c.X.tile[family].bx;
  if (by) *by = ctx->c.X.tile[family].by;
  return 0;
}

int gcs_context_autotune(gcs_context *ctx, const gamera_no_advance_options *options,
                         const gamera_no_timestep_options *timestep, int repetitions,
                         double best_ms[GCS_TILE_FAMILIES],
                         double default_ms[GCS_TILE_FAMILIES]) {
  gcs::Opts O;
  if (!ctx || repetitions < 1 || !ctx->c.bg_uploaded ||
      !gcs::driver_opts(options, timestep, 0.5, &O)) {
    gcs::set_api_error("invalid autotune arguments");
    return -1;
  }
  gcs::Context &C = ctx->c;
  Tile keep[gcs::kTileFamilies];
  for (int f = 0; f < gcs::kTileFamilies; ++f) keep[f] = C.X.tile[f];
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
      cudaStreamSynchronize(C.stream) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    gcs::set_api_error("autotune: CUDA error");
    return -1;
  }
  C.reset_status_async();
  int rc = 0;
  for (int f = 0; f < gcs::kTileFamilies && rc == 0; ++f) {
    if (best_ms) best_ms[f] = 0.0;
    if (default_ms) default_ms[f] = 0.0;
    if (!tuned_family(f)) continue;
    double best = DBL_MAX;
    Tile pick = keep[f];
    const Tile def = gcs::Ctx{}.tile[f];
    for (const Tile &t : kCandidates) {
      if (!tile_ok(f, t.bx, t.by)) continue;
      C.X.tile[f] = t;
      launch_family(C.X, O, f, C.stream);   // warm-up
      cudaEventRecord(e0, C.stream);
      for (int r = 0; r < repetitions; ++r) launch_family(C.X, O, f, C.stream);
      cudaEventRecord(e1, C.stream);
      float ms = 0.0f;
      if (cudaEventSynchronize(e1) != cudaSuccess ||
          cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
        rc = -1;
        break;
      }
      const double per = (double)ms / repetitions;
      if (t.bx == def.bx && t.by == def.by && default_ms) default_ms[f] = per;
      if (per < best) {
        best = per;
        pick = t;
      }
    }
    C.X.tile[f] = pick;
    if (best_ms && best < DBL_MAX) best_ms[f] = best;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  gcs::DevStatus s;
  if (rc != 0 || C.read_status(&s) != 0 || s.first != 0) {
    // a kernel failed on this state: the timings mean nothing
    for (int f = 0; f < gcs::kTileFamilies; ++f) C.X.tile[f] = keep[f];
    C.reset_status_async();
    cudaStreamSynchronize(C.stream);
    gcs::set_api_error("autotune: a kernel failed on the current state");
    return -1;
  }
  // the CFL reduction left its minimum in the status: clear it
  C.reset_status_async();
  return cudaStreamSynchronize(C.stream) == cudaSuccess ? 0 : -1;
}

int gcs_ensemble_draw(unsigned long long seed, int count, size_t *n,
                      gcs_wind_driver *drivers) {
  if (count < 1 || (!n && !drivers)) return -1;
  static const size_t kSizes[4] = {48, 64, 96, 128};
  uint64_t s = mix64((uint64_t)seed ^ 0x656e73656d626c65ULL);
  auto uniform = [&]() {
    s = mix64(s);
    return (double)(s >> 11) * 0x1.0p-53;
  };
  for (int i = 0; i < count; ++i) {
    s = mix64(s);
    const size_t size = kSizes[s >> 62];
    const double bz = -10.0 + 15.0 * uniform();
    const double vx = -800.0 + 500.0 * uniform();
    const double dn = 1.0 + 19.0 * uniform();
    const double tk = 5.0e4 + 1.5e5 * uniform();
    if (n) n[i] = size;
    if (drivers) drivers[i] = gcs_wind_driver{dn, vx, tk, bz};
  }
  return 0;
}

double gcs_ensemble_estimate_bytes(int count, const size_t *nr, const size_t *n,
                                   int fp32_bulk) {
  if (count < 1 || !nr || !n) return -1.0;
  double total = 0.0;
  for (int i = 0; i < count; ++i) {
    bool first = true;
    for (int j = 0; j < i; ++j)
      if (nr[j] == nr[i] && n[j] == n[i]) first = false;
    double full, member;
    case_bytes(nr[i], n[i], fp32_bulk, &full, &member);
    total += first ? full : member;
  }
  return total;
}

gcs_ensemble *gcs_ensemble_create(const gcs_ensemble_config *cfg) {
  if (!cfg || cfg->count < 1 || !cfg->nr || !cfg->n || !cfg->drivers ||
      !std::isfinite(cfg->dt_fraction) || cfg->dt_fraction <= 0.0 ||
      cfg->autotune_repetitions < 0) {
    gcs::set_api_error("invalid ensemble configuration");
    return nullptr;
  }
  const int count = cfg->count;
  for (int i = 0; i < count; ++i) {
    const gcs_wind_driver &d = cfg->drivers[i];
    if (!std::isfinite(d.density_cm3) || d.density_cm3 <= 0.0 ||
        !std::isfinite(d.velocity_x_kms) || !std::isfinite(d.temperature_k) ||
        d.temperature_k <= 0.0 || !std::isfinite(d.bz_nt)) {
      gcs::set_api_error("invalid wind driver");
      return nullptr;
    }
  }
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
    gcs::set_api_error("no CUDA device");
    return nullptr;
  }
  const double need = gcs_ensemble_estimate_bytes(count, cfg->nr, cfg->n, cfg->fp32_bulk);
  if (need > (double)free_b - 2.0e9) {
    char msg[160];
    snprintf(msg, sizeof(msg), "ensemble needs about %.1f GB of device memory, %.1f GB free",
             need * 1e-9, free_b * 1e-9);
    gcs::set_api_error(msg);
    return nullptr;
  }
  gcs_ensemble *E = new (std::nothrow) gcs_ensemble;
  if (!E) {
    gcs::set_api_error("out of host memory");
    return nullptr;
  }
  gcs_case_options(2, &E->options, &E->timestep);
  E->fraction = cfg->dt_fraction;
  if (!gcs::driver_opts(&E->options, &E->timestep, E->fraction, &E->O)) {
    delete E;
    gcs::set_api_error("invalid wind options");
    return nullptr;
  }
  E->runs.assign(count, nullptr);
  E->owner.assign(count, -1);
  E->prev.assign(count, -1);
  E->done.assign(count, nullptr);
  auto fail = [&](const char *msg) -> gcs_ensemble * {
    gcs::set_api_error(msg);
    delete E;
    return nullptr;
  };
  for (int i = 0; i < count; ++i) {
    const gcs_wind_driver &d = cfg->drivers[i];
    const unsigned long long seed = cfg->seed + (unsigned long long)i;
    int o = -1;
    for (int j = 0; j < i; ++j)
      if (E->owner[j] == j && cfg->nr[j] == cfg->nr[i] && cfg->n[j] == cfg->n[i]) o = j;
    gcs_context *ctx = new (std::nothrow) gcs_context;
    if (!ctx) return fail("out of host memory");
    const gcs::WindInit w =
        gcs::driven_wind(d.density_cm3, d.velocity_x_kms, d.temperature_k, d.bz_nt);
    int rc;
    if (o < 0) {
      rc = ctx->c.init_case(2, cfg->nr[i], cfg->n[i], seed, &w);
      if (rc == 0 && cfg->fp32_bulk) rc = ctx->c.enable_bulk(1);
      E->owner[i] = i;
      ++E->grids;
    } else {
      rc = ctx->c.init_member(E->runs[o]->c, seed, w);
      if (rc == 0 && cfg->fp32_bulk) rc = ctx->c.enable_bulk(1);
      E->owner[i] = o;
      int p = o;
      for (int j = o + 1; j < i; ++j)
        if (E->owner[j] == o) p = j;
      E->prev[i] = p;
    }
    E->runs[i] = ctx;
    if (rc != 0) {
      char msg[300];
      snprintf(msg, sizeof(msg), "run %d: %s", i, ctx->c.error);
      return fail(msg);
    }
    if (cudaEventCreateWithFlags(&E->done[i], cudaEventDisableTiming) != cudaSuccess)
      return fail("cannot create events");
  }
  // tiles: tuned on each grid's first run, shared by the runs on that grid
  if (cfg->autotune_repetitions > 0) {
    for (int i = 0; i < count; ++i) {
      if (E->owner[i] != i) continue;
      if (gcs_context_autotune(E->runs[i], &E->options, &E->timestep,
                               cfg->autotune_repetitions, nullptr, nullptr) != 0)
        return fail("autotune failed");
    }
    for (int i = 0; i < count; ++i)
      if (E->owner[i] != i)
        for (int f = 0; f < gcs::kTileFamilies; ++f)
          E->runs[i]->c.X.tile[f] = E->runs[E->owner[i]]->c.X.tile[f];
  }
  if (cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&E->fork, cudaEventDisableTiming) != cudaSuccess)
    return fail("cannot create the ensemble stream");
  return E;
}

void gcs_ensemble_destroy(gcs_ensemble *E) { delete E; }

int gcs_ensemble_count(const gcs_ensemble *E) { return E ? (int)E->runs.size() : -1; }

gcs_context *gcs_ensemble_run_context(gcs_ensemble *E, int run) {
  if (!E || run < 0 || run >= (int)E->runs.size()) return nullptr;
  return E->runs[run];
}

int gcs_ensemble_grid_owner(const gcs_ensemble *E, int run) {
  if (!E || run < 0 || run >= (int)E->runs.size()) return -1;
  return E->owner[run];
}

uintptr_t gcs_ensemble_stream(gcs_ensemble *E) { return E ? (uintptr_t)E->stream : 0; }

size_t gcs_ensemble_device_bytes(const gcs_ensemble *E) {
  if (!E) return 0;
  size_t b = 0;
  for (size_t i = 0; i < E->runs.size(); ++i) {
    const gcs::Context &c = E->runs[i]->c;
    b += c.pool_bytes + c.bg_bytes + c.plans_bytes + c.staging_bytes + c.bulk_bytes;
  }
  return b;
}

static int ensemble_capture(gcs_ensemble *E) {
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(E->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return -1;
  int rc = cudaEventRecord(E->fork, E->stream) == cudaSuccess ? 0 : -1;
  const int count = (int)E->runs.size();
  for (int i = 0; i < count && rc == 0; ++i) {
    gcs::Context &C = E->runs[i]->c;
    const cudaEvent_t after = E->prev[i] < 0 ? E->fork : E->done[E->prev[i]];
    if (cudaStreamWaitEvent(C.stream, after, 0) != cudaSuccess ||
        gcs::enqueue_driver_step(E->runs[i], E->O) != 0 ||
        cudaEventRecord(E->done[i], C.stream) != cudaSuccess)
      rc = -1;
  }
  // join every run's stream back into the capturing stream
  for (int i = 0; i < count && rc == 0; ++i)
    if (cudaStreamWaitEvent(E->stream, E->done[i], 0) != cudaSuccess) rc = -1;
  const cudaError_t ee = cudaStreamEndCapture(E->stream, &g);
  if (rc != 0 || ee != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return -1;
  }
  cudaGraphGetNodes(g, nullptr, &E->nodes);
  const cudaError_t ie = cudaGraphInstantiate(&E->exec, g, 0);
  cudaGraphDestroy(g);
  return ie == cudaSuccess ? 0 : -1;
}

int gcs_ensemble_advance(gcs_ensemble *E, int steps) {
  if (!E || steps < 0) return -1;
  if (!E->started) {
    // each run's first step size: dt_fraction x its own CFL step
    for (size_t i = 0; i < E->runs.size(); ++i)
      if (gcs_context_run(E->runs[i], &E->options, &E->timestep, E->fraction, 0, 0) != 0) {
        gcs::set_api_error("initial time step failed");
        return -1;
      }
    for (size_t i = 0; i < E->runs.size(); ++i)
      if (cudaStreamSynchronize(E->runs[i]->c.stream) != cudaSuccess) return -1;
    if (ensemble_capture(E) != 0) {
      gcs::set_api_error("ensemble graph capture failed");
      return -1;
    }
    E->started = 1;
  }
  for (int s = 0; s < steps; ++s)
    if (cudaGraphLaunch(E->exec, E->stream) != cudaSuccess) return -1;
  return 0;
}

int gcs_ensemble_sync(gcs_ensemble *E, int *failed_run) {
  if (failed_run) *failed_run = -1;
  if (!E || cudaStreamSynchronize(E->stream) != cudaSuccess) return -1;
  for (size_t i = 0; i < E->runs.size(); ++i) {
    if (gcs_context_sync(E->runs[i]) != 0) {
      if (failed_run) *failed_run = (int)i;
      return -1;
    }
  }
  return 0;
}

int gcs_ensemble_graph_info(const gcs_ensemble *E, int *nodes, int *grids) {
  if (!E) return -1;
  if (nodes) *nodes = (int)E->nodes;
  if (grids) *grids = E->grids;
  return 0;
}

}  // extern "C"
