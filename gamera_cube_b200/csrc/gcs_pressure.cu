// Post-step pressure control of the Earth drivers
// (nonorthogonal/src/nonorthogonal/nonorthogonal_step.c:74-171, called after
// each step by cubedsphere/tests/test_cubedsphere_mpi_earth_tile.c:459-481):
// over the active cells, cells at or below a density threshold get the
// pressure of a fixed sound speed (not below the pressure floor), and cells
// whose sound speed exceeds 1.5 c relax towards the pressure of sound speed
// 1.5 c over the bounce time L / c_s of their dipole line, L = r^3 / (x^2 +
// y^2) at the cell centroid.  Counts of both kinds and the maximum sound
// speed and pressure (after the low-density reset, before the relaxation)
// are summed over the cells.
//
// One thread per active cell of all six faces; the dipole line length of
// every active cell is computed once on the host from the centroids and
// kept on the device.  Compiled without FMA contraction, so every cell
// changes bit for bit as in the reference.
#include "gcs_context.h"
#include "gcs_error.h"
#include "gamera_cs_b200.h"

#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "gcs_kernel_util.cuh"
#include "gcs_physics.cuh"

namespace gcs {
namespace {

struct PcStats {
  unsigned long long low, hot, max_sound_bits, max_pressure_bits;
  int failed, pad;
};

__device__ inline unsigned long long warp_sum(unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ inline unsigned long long warp_max(unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}

// CFL candidate of one active cell (nonorthogonal_step.c:449-525, the same
// arithmetic as the recovery kernel's fused CFL reduction): false when the
// reference fails the cell.
__device__ inline bool cfl_candidate(const double u[5], const double bn[3], const double *b0,
                                     double cflmin, const Opts &O, double *cand) {
  Prim p;
  if (cons_to_prim(u, O.t_gamma, O.t_rho_floor, O.t_p_floor, &p)) return false;
  const double cs = sqrt(O.t_gamma * p.p / p.rho);
  double va = 0.0;
  if (O.t_mhd) {
    double bx = bn[0], by = bn[1], bz = bn[2];
    if (b0) {
      bx = bn[0] + b0[0];
      by = bn[1] + b0[1];
      bz = bn[2] + b0[2];
    }
    double s2 = 0.0;
    s2 += bx * bx;
    s2 += by * by;
    s2 += bz * bz;
    va = sqrt(s2) / sqrt(p.rho);
    if (O.t_boris) va = O.t_c * va / hypot(O.t_c, va);
  }
  double v2 = 0.0;
  v2 += p.vx * p.vx;
  v2 += p.vy * p.vy;
  v2 += p.vz * p.vz;
  const double speed = sqrt(v2) + hypot(cs, va);
  const double c0 = O.t_cfl * cflmin / speed;
  if (!isfinite(c0) || c0 <= 0.0) return false;
  *cand = c0;
  return true;
}

// nonorthogonal_step.c:95-152, one thread per active cell; dt from the step
// parameters when prm is set (the device driver loop), else `dt`.  In the
// driver loop (with_cfl) the kernel also reduces the CFL step of the
// controlled state into the status word, the next step's dt.
__global__ void __launch_bounds__(256) k_pressure_control(
    Dims D, DevState S, DevGeom G, DevBg BG, Opts O, const double *dipole_l,
    PressureControl pc, double dt, const StepParams *prm, PcStats *out, DevStatus *status,
    int with_cfl) {
  const int count = D.nr * D.n * D.n;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int f = blockIdx.y;
  unsigned long long low = 0, hot = 0, smax = 0, pmax = 0;
  double cand = DBL_MAX;
  if (t < count) {
    const int nn = D.n * D.n;
    const int i = t / nn;
    const int j = (t - i * nn) / D.n;
    const int k = t - i * nn - j * D.n;
    const long long c = f * D.Nn + D.node(D.g + i, D.g + j, D.g + k);
    if (prm) dt = prm->dt;
    double u[5];
    for (int m = 0; m < 5; ++m) u[m] = S.U[m][c];
    Prim p;
    bool bad = cons_to_prim(u, pc.gamma, pc.density_floor, pc.pressure_floor, &p) != 0;
    if (!bad) {
      bool changed = false;
      if (p.rho <= pc.low_density_threshold) {
        p.p = fmax(pc.pressure_floor,
                   p.rho * pc.low_density_sound_speed * pc.low_density_sound_speed / pc.gamma);
        low = 1;
        changed = true;
      }
      const double sound = sqrt(pc.gamma * p.p / p.rho);
      // fmax with the running maxima (0 at the start): NaN and values not
      // above 0 never raise them; positive doubles order as their bits
      if (sound > 0.0) smax = (unsigned long long)__double_as_longlong(sound);
      if (p.p > 0.0) pmax = (unsigned long long)__double_as_longlong(p.p);
      if (sound > 1.5 * pc.light_speed) {
        const double L = dipole_l[(long long)f * count + t];
        if (isnan(L)) {
          bad = true;   // centroid on the axis: the reference skips the cell
        } else {
          const double target = p.rho * (1.5 * pc.light_speed) * (1.5 * pc.light_speed) / pc.gamma;
          const double bounce = L / sound;
          p.p -= (dt / bounce) * (p.p - target);
          hot = 1;
          changed = true;
        }
      }
      if (!bad && changed) {
        double w[5];
        if (prim_to_cons(p, pc.gamma, pc.density_floor, pc.pressure_floor, w) != 0) {
          bad = true;
        } else {
          for (int m = 0; m < 5; ++m) {
            S.U[m][c] = w[m];
            u[m] = w[m];
          }
        }
      }
    }
    if (bad) {
      atomicOr(&out->failed, 1);
      if (status) fail(status, kStagePressureControl, 0, f, D.g + i, D.g + j, D.g + k);
    }
    if (with_cfl) {
      // the cell as stored now: controlled, or unchanged
      const double bn[3] = {S.B[0][c], S.B[1][c], S.B[2][c]};
      double b0[3];
      if (O.t_bg)
        for (int m = 0; m < 3; ++m) b0[m] = BG.b0[m][c];
      if (!cfl_candidate(u, bn, O.t_bg ? b0 : nullptr, G.cflmin[c], O, &cand)) {
        cand = DBL_MAX;
        fail(status, kStageTimestep, 0, f, D.g + i, D.g + j, D.g + k);
      }
    }
  }
  low = warp_sum(low);
  hot = warp_sum(hot);
  smax = warp_max(smax);
  pmax = warp_max(pmax);
  if (with_cfl)
    for (int o = 16; o > 0; o >>= 1) cand = fmin(cand, __shfl_xor_sync(0xffffffffu, cand, o));
  if ((threadIdx.x & 31) == 0) {
    if (low) atomicAdd(&out->low, low);
    if (hot) atomicAdd(&out->hot, hot);
    if (smax) atomicMax(&out->max_sound_bits, smax);
    if (pmax) atomicMax(&out->max_pressure_bits, pmax);
    // positive doubles order as unsigned 64-bit integers
    if (with_cfl && cand < DBL_MAX)
      atomicMin(&status->cfl_min_bits, (unsigned long long)__double_as_longlong(cand));
  }
}

// nonorthogonal_step.c:119-129: L = r r^2 / (x^2 + y^2), NaN where the
// reference fails the cell (r^2 not > 0, or x^2 + y^2 not above DBL_MIN).
double dipole_length(const gamera_no_vec3 &x) {
  const double r2 = x.value[0] * x.value[0] + x.value[1] * x.value[1] + x.value[2] * x.value[2];
  const double c2 = x.value[0] * x.value[0] + x.value[1] * x.value[1];
  if (!(r2 > 0.0) || !(c2 > DBL_MIN)) return NAN;
  return sqrt(r2) * r2 / c2;
}

bool valid(const PressureControl &pc) {
  return pc.gamma > 1.0 && pc.density_floor > 0.0 && pc.pressure_floor > 0.0 &&
         pc.light_speed > 0.0 && pc.low_density_threshold > 0.0 &&
         pc.low_density_sound_speed >= 0.0;
}

}  // namespace

// Dipole line lengths of the active cells, from `grid` or, for a
// device-built case, from its centroids rebuilt on the device.
int pressure_prepare(Context &C, const gamera_no_grid *grid) {
  if (C.pc_dipole && C.pc_stats) return 0;
  const Dims &D = C.X.D;
  const size_t count = (size_t)D.nr * D.n * D.n;
  std::vector<double> L((size_t)kFaces * count);
  for (int f = 0; f < kFaces; ++f) {
    if (grid) {
      for (int i = 0; i < D.nr; ++i)
        for (int j = 0; j < D.n; ++j)
          for (int k = 0; k < D.n; ++k) {
            const size_t cell = ((size_t)(i + D.g) * D.E1 + j + D.g) * D.E2 + k + D.g;
            L[f * count + ((size_t)i * D.n + j) * D.n + k] =
                dipole_length(grid[f].cell[cell].centroid);
          }
    } else {
      std::vector<double> cen, vert;
      if (C.face_coordinates(f, cen, vert) != 0) {
        C.set_error("pass the host grid for this context", "pressure control");
        return -1;
      }
      for (size_t q = 0; q < count; ++q) {
        const gamera_no_vec3 x = {{cen[q], cen[count + q], cen[2 * count + q]}};
        L[f * count + q] = dipole_length(x);
      }
    }
  }
  void *p = nullptr;
  if (cudaMalloc(&p, L.size() * sizeof(double) + sizeof(PcStats)) != cudaSuccess) {
    C.set_error("cannot allocate the pressure-control arrays", "pressure control");
    return -1;
  }
  if (cudaMemcpy(p, L.data(), L.size() * sizeof(double), cudaMemcpyHostToDevice) !=
      cudaSuccess) {
    cudaFree(p);
    C.set_error("cannot upload the dipole lengths", "pressure control");
    return -1;
  }
  C.pc_dipole = (double *)p;
  C.pc_stats = (char *)p + L.size() * sizeof(double);
  return 0;
}

int pressure_reset_async(Context &C) {
  return cudaMemsetAsync(C.pc_stats, 0, sizeof(PcStats), C.stream) == cudaSuccess ? 0 : -1;
}

void launch_pressure_control(Context &C, const PressureControl &pc, double dt,
                             const Opts *cfl, cudaStream_t s) {
  const Dims &D = C.X.D;
  const long long count = (long long)D.nr * D.n * D.n;
  const Opts none{};
  k_pressure_control<<<dim3((unsigned)((count + 255) / 256), kFaces), 256, 0, s>>>(
      D, C.X.S, C.X.G, C.X.BG, cfl ? *cfl : none, C.pc_dipole, pc, dt,
      cfl ? C.X.params : nullptr, (PcStats *)C.pc_stats, cfl ? C.X.status : nullptr,
      cfl ? 1 : 0);
}

int pressure_read(Context &C, size_t *low, size_t *hot, double *max_sound,
                  double *max_pressure, int *failed) {
  PcStats h{};
  if (cudaMemcpyAsync(&h, C.pc_stats, sizeof(h), cudaMemcpyDeviceToHost, C.stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(C.stream) != cudaSuccess)
    return -1;
  if (low) *low = (size_t)h.low;
  if (hot) *hot = (size_t)h.hot;
  if (max_sound) memcpy(max_sound, &h.max_sound_bits, sizeof(double));
  if (max_pressure) memcpy(max_pressure, &h.max_pressure_bits, sizeof(double));
  if (failed) *failed = h.failed;
  return 0;
}

bool pressure_valid(const PressureControl &pc) { return valid(pc); }

}  // namespace gcs

extern "C" {

int gcs_context_pressure_control(gcs_context *ctx, const gamera_no_grid *grid, double dt,
                                 const gcs_pressure_control *config,
                                 size_t *low_density_cell_count,
                                 size_t *high_sound_speed_cell_count,
                                 double *maximum_sound_speed, double *maximum_pressure) {
  if (!ctx || !config || !(dt > 0.0)) return -1;
  const gcs::PressureControl pc{config->gamma, config->density_floor, config->pressure_floor,
                                config->light_speed, config->low_density_threshold,
                                config->low_density_sound_speed};
  if (!gcs::pressure_valid(pc)) return -1;
  gcs::Context &C = ctx->c;
  if (gcs::pressure_prepare(C, grid) != 0 || gcs::pressure_reset_async(C) != 0) return -1;
  gcs::launch_pressure_control(C, pc, dt, nullptr, C.stream);
  if (cudaGetLastError() != cudaSuccess) return -1;
  int failed = 0;
  if (gcs::pressure_read(C, low_density_cell_count, high_sound_speed_cell_count,
                         maximum_sound_speed, maximum_pressure, &failed) != 0)
    return -1;
  return failed ? -1 : 0;
}

int gcs_context_set_pressure_control(gcs_context *ctx, const gamera_no_grid *grid,
                                     const gcs_pressure_control *config) {
  if (!ctx) return -1;
  gcs::Context &C = ctx->c;
  if (!config) {
    C.pc_on = 0;
    return 0;
  }
  const gcs::PressureControl pc{config->gamma, config->density_floor, config->pressure_floor,
                                config->light_speed, config->low_density_threshold,
                                config->low_density_sound_speed};
  if (!gcs::pressure_valid(pc)) return -1;
  if (gcs::pressure_prepare(C, grid) != 0 || gcs::pressure_reset_async(C) != 0) return -1;
  C.pc = pc;
  C.pc_on = 1;
  return 0;
}

int gcs_context_pressure_control_stats(gcs_context *ctx, size_t *low_density_cell_count,
                                       size_t *high_sound_speed_cell_count,
                                       double *maximum_sound_speed, double *maximum_pressure,
                                       int reset) {
  if (!ctx || !ctx->c.pc_stats) return -1;
  gcs::Context &C = ctx->c;
  int failed = 0;
  if (gcs::pressure_read(C, low_density_cell_count, high_sound_speed_cell_count,
                         maximum_sound_speed, maximum_pressure, &failed) != 0)
    return -1;
  if (reset && gcs::pressure_reset_async(C) != 0) return -1;
  return failed ? 1 : 0;
}

}  // extern "C"
