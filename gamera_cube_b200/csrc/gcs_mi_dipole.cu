// Aligned-dipole magnetosphere-ionosphere coupling of the six-face cube
// (cubedsphere/cubedsphere_mi_dipole.c).
//
// An update (gamera_cs_mi_dipole_maybe_update) runs entirely on the device
// holding the MHD state:
//   1. k_shell_field: the residual cell B of the three radial layers around
//      the sample shell, with a one-cell angular fringe interpolated
//      bilinearly from the physical donor face (:223-265);
//   2. k_shell_current: the Stokes curl of that field on every physical
//      shell cell (nonorthogonal_mi.c:43-166) recovered with the cube's
//      calibrated face-flux map, projected on B0 and mapped to the
//      ionosphere: FAC = (J . B0)/|B0| * dipole ratio * J_norm (:266-290);
//   3. k_shell_fringe: the scalar FAC fringe from the owning face (:291-332);
//   4. k_polar_sample: bilinear samples of the shell FAC on the two polar
//      grids (:344-370, :393-413);
//   5. the two constant-Pedersen solves, one thread-block cluster each
//      (gcs_mi.cu), warm-started from the held potential (:414-429).
// Every index, weight and dipole factor of steps 1-4 depends only on the
// grid and is computed once on the host when the coupling is created.  The
// potential and FAC are then copied to the host, where the reference-layout
// entry points (potential lookup, wall EMF, ghost E x B drift, statistics,
// CSV and analysis views) read them.
//
// Cadence on the device.  Attached to its context's driver loop
// (gcs_context_set_mi_coupling), the update runs inside the step's CUDA
// graph: k_mi_due evaluates the reference's rule (cubedsphere_mi_dipole.c:
// 372-378, 430-435) from the step parameters' simulation time, or every
// n-th step, and sets a gate that every kernel of the update, the cluster
// solve included, reads first; k_mi_check turns a non-finite FAC or an
// unconverged solve into a step failure.  The host copies of potential,
// FAC, statistics and cadence are then refreshed on the next host access.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "gamera_cs_b200.h"
#include "gcs_context.h"
#include "gcs_error.h"
#include "gcs_topology.h"
#include "gcs_mi_lookup.cuh"
#include "gcs_kernel_util.cuh"

using gcs::set_api_error;

namespace gcs {
// gcs_mi.cu: gated, array-bound solve plans
int mi_plan_gate(gcs_mi_plan *p, const int *gate, const double *fac, double *pot);
const int *mi_plan_status(const gcs_mi_plan *p);
int mi_plan_launch(gcs_mi_plan *p, cudaStream_t stream);
}  // namespace gcs

namespace {

constexpr int kHemispheres = 2;

// Device-side cadence of one coupling (the host's ready / epoch /
// next-update state, mirrored) and the gate of the current update.
struct MiCadence {
  double next_update_s, epoch_s;
  double length_norm_m, speed_norm_m_s;   // code time -> seconds, as the host
  double interval_s;     // coupling interval
  int ready, due;        // due: the gate every kernel of an update reads
  int every;             // > 0: every n-th step; 0: the reference's time rule
  int pad;
};

struct FringeB {      // one fringe cell of the shell field
  double wx, wy;
  int donor;          // donor face
  int j0, k0;         // active-relative donor corner
  int pad;
};

struct FringeFac {    // one fringe entry of the shell FAC
  double wx, wy;
  int donor;
  int lower;          // donor shell index of the lower corner
};

struct Sample {       // one polar grid node
  double wx, wy;
  int face;           // -1: beyond the sampled colatitude, FAC = 0
  int index;          // shell index of the lower corner
};

struct EdgeG {        // edge direction and length
  double n[3];
  double len;
};

// Device view of one coupling.
struct MiDev {
  int n, g, shell_i, S;          // S = n + 2 (shell stride)
  long long Nn;                  // nodes per face
  int N1, N2;                    // node strides
  double jnorm;
  double *field;                 // 6 x 3 layers x S^2 x 3 components
  const FringeB *fringe_b;       // 6 x 3 x S^2 (donor < 0: interior copy)
  const EdgeG *edges;            // 6 x 5 sets x (n+1)^2
  const double *ratio;           // 6 x n^2 dipole ratio per shell cell
  const double *b0;              // 6 x n^2 x 3 background B of the shell cells
  double *shell_fac;             // 6 x S^2
  const FringeFac *fringe_fac;   // 6 x S^2 (donor < 0: physical)
  const Sample *samples;         // 2 x nt x np
  double *fac;                   // 2 x nt x np
  int polar_count;               // nt x np
  int *status;                   // nonzero: update failed
};

__device__ inline long long node(const MiDev &M, int i, int j, int k) {
  return ((long long)i * M.N1 + j) * M.N2 + k;
}

// Shell field at absolute (layer i, j, k) of face f; layer i in
// [shell_i - 1, shell_i + 1], j, k in [g - 1, g + n].
__device__ inline const double *field_at(const MiDev &M, int f, int i, int j, int k) {
  const int l = i - (M.shell_i - 1);
  return M.field + ((((size_t)f * 3 + l) * M.S + (j - M.g + 1)) * M.S +
                    (k - M.g + 1)) * 3;
}

struct FieldPtrs {
  const double *b[3];            // residual cell B per component
};

__global__ void k_shell_field(FieldPtrs B, MiDev M, const int *gate) {
  if (*gate == 0) return;
  const long long per = 3LL * M.S * M.S;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 6 * per) return;
  const int f = (int)(t / per);
  const long long r = t - f * per;
  const int l = (int)(r / ((long long)M.S * M.S));
  const int jj = (int)((r / M.S) % M.S), kk = (int)(r % M.S);
  const int radial = M.shell_i - 1 + l;
  const FringeB &P = M.fringe_b[t];
  double v[3] = {0.0, 0.0, 0.0};
  if (P.donor < 0) {
    const long long c = f * M.Nn + node(M, radial, M.g - 1 + jj, M.g - 1 + kk);
    for (int a = 0; a < 3; ++a) v[a] = B.b[a][c];
  } else {
    // cubedsphere_mi_dipole.c:246-262, donor taps in (dj, dk) order
    for (int dj = 0; dj < 2; ++dj)
      for (int dk = 0; dk < 2; ++dk) {
        const long long c = P.donor * M.Nn +
                            node(M, radial, M.g + P.j0 + dj, M.g + P.k0 + dk);
        const double w = (dj == 0 ? 1.0 - P.wx : P.wx) * (dk == 0 ? 1.0 - P.wy : P.wy);
        for (int a = 0; a < 3; ++a) v[a] += w * B.b[a][c];
      }
  }
  double *out = M.field + t * 3;
  for (int a = 0; a < 3; ++a) out[a] = v[a];
}

// Edge sets: 0 I-edges at the shell layer, 1/2 J-edges at the shell layer
// and the one above, 3/4 K-edges at the shell layer and the one above.
__device__ inline const EdgeG &edge_at(const MiDev &M, int f, int set, int j, int k) {
  const int m = M.n + 1;
  return M.edges[(((size_t)f * 5 + set) * m + (j - M.g)) * m + (k - M.g)];
}

// Line integral of the 4-cell average along one edge
// (nonorthogonal_mi.c:43-103).
__device__ double edge_integral(const MiDev &M, int f, int dir, int i, int j, int k) {
  int c[4][3] = {{i, j, k}, {i, j, k}, {i, j, k}, {i, j, k}};
  int set;
  if (dir == 0) {
    --c[1][1]; --c[2][2]; --c[3][1]; --c[3][2];
    set = 0;
  } else if (dir == 1) {
    --c[1][0]; --c[2][2]; --c[3][0]; --c[3][2];
    set = i == M.shell_i ? 1 : 2;
  } else {
    --c[1][0]; --c[2][1]; --c[3][0]; --c[3][1];
    set = i == M.shell_i ? 3 : 4;
  }
  double avg[3] = {0.0, 0.0, 0.0};
  for (int p = 0; p < 4; ++p) {
    const double *b = field_at(M, f, c[p][0], c[p][1], c[p][2]);
    for (int a = 0; a < 3; ++a) avg[a] += 0.25 * b[a];
  }
  const EdgeG &e = edge_at(M, f, set, j, k);
  double d = 0.0;
  for (int a = 0; a < 3; ++a) d += avg[a] * e.n[a];
  return d * e.len;
}

__global__ void k_shell_current(gcs::DevGeom G, MiDev M, const int *gate) {
  if (*gate == 0) return;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per = (long long)M.n * M.n;
  if (t >= 6 * per) return;
  const int f = (int)(t / per);
  const int jj = (int)((t - f * per) / M.n), kk = (int)((t - f * per) % M.n);
  const int i = M.shell_i, j = M.g + jj, k = M.g + kk;
  auto E = [&](int dir, int a, int b, int c) { return edge_integral(M, f, dir, a, b, c); };
  // face circulations (nonorthogonal_mi.c:105-138), order i-lo, i-hi, ...
  double phi[6];
  phi[0] = E(1, i, j, k) + E(2, i, j + 1, k) - E(1, i, j, k + 1) - E(2, i, j, k);
  phi[1] = E(1, i + 1, j, k) + E(2, i + 1, j + 1, k) - E(1, i + 1, j, k + 1) -
           E(2, i + 1, j, k);
  phi[2] = E(2, i, j, k) + E(0, i, j, k + 1) - E(2, i + 1, j, k) - E(0, i, j, k);
  phi[3] = E(2, i, j + 1, k) + E(0, i, j + 1, k + 1) - E(2, i + 1, j + 1, k) -
           E(0, i, j + 1, k);
  phi[4] = E(0, i, j, k) + E(1, i + 1, j, k) - E(0, i, j + 1, k) - E(1, i, j, k);
  phi[5] = E(0, i, j, k + 1) + E(1, i + 1, j, k + 1) - E(0, i, j + 1, k + 1) -
           E(1, i, j, k + 1);
  const long long c = f * M.Nn + node(M, i, j, k);
  double J[3];
  bool ok = true;
  for (int q = 0; q < 6; ++q) ok = ok && isfinite(phi[q]);
  if (ok && G.cell_ok[c]) {
    for (int r = 0; r < 3; ++r) {
      double s = 0.0;
      for (int col = 0; col < 6; ++col) s += G.rec[r * 6 + col][c] * phi[col];
      J[r] = s;
    }
  } else {
    ok = false;
  }
  // cubedsphere_mi_dipole.c:272-287 (its dot has no leading zero)
  const double bx = M.b0[3 * t], by = M.b0[3 * t + 1], bz = M.b0[3 * t + 2];
  const double bmag = sqrt(bx * bx + by * by + bz * bz);
  double fac = NAN;
  if (ok && bmag > 0.0)
    fac = (J[0] * bx + J[1] * by + J[2] * bz) / bmag * M.ratio[t] * M.jnorm;
  if (!isfinite(fac)) atomicExch(M.status, 1);
  M.shell_fac[(size_t)f * M.S * M.S + (size_t)(jj + 1) * M.S + kk + 1] = fac;
}

__global__ void k_shell_fringe(MiDev M, const int *gate) {
  if (*gate == 0) return;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per = (long long)M.S * M.S;
  if (t >= 6 * per) return;
  const FringeFac &P = M.fringe_fac[t];
  if (P.donor < 0) return;
  // cubedsphere_mi_dipole.c:322-329
  const double *src = M.shell_fac + (size_t)P.donor * per;
  const double low = (1.0 - P.wy) * src[P.lower] + P.wy * src[P.lower + 1];
  const double high = (1.0 - P.wy) * src[P.lower + M.S] + P.wy * src[P.lower + M.S + 1];
  const double fac = (1.0 - P.wx) * low + P.wx * high;
  if (!isfinite(fac)) atomicExch(M.status, 1);
  M.shell_fac[t] = fac;
}

__global__ void k_polar_sample(MiDev M, const int *gate) {
  if (*gate == 0) return;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)kHemispheres * M.polar_count) return;
  const Sample &P = M.samples[t];
  if (P.face < 0) {
    M.fac[t] = 0.0;
    return;
  }
  // cubedsphere_mi_dipole.c:362-369
  const double *src = M.shell_fac + (size_t)P.face * M.S * M.S;
  const double lower = (1.0 - P.wy) * src[P.index] + P.wy * src[P.index + 1];
  const double upper = (1.0 - P.wy) * src[P.index + M.S] + P.wy * src[P.index + M.S + 1];
  const double v = (1.0 - P.wx) * lower + P.wx * upper;
  if (!isfinite(v)) atomicExch(M.status, 1);
  M.fac[t] = v;
}

// An update requested by the host: open the gate, clear the FAC status.
__global__ void k_open_gate(MiCadence *c, int *status) {
  c->due = 1;
  *status = 0;
}

// The cadence of an update inside the step graph, before the step:
// the reference's rule on the simulation time of the state (seconds
// = code time x time_scale), or every n-th step.  A due update advances the
// cadence as the host does after an update (the step fails if the update
// does, so the advance is never seen without it).
__global__ void k_mi_due(const gcs::StepParams *prm, MiCadence *c, int *status,
                         const gcs::DevStatus *st) {
  if (gcs::failed(st)) {
    c->due = 0;
    return;
  }
  const double time_s = prm->time * c->length_norm_m / c->speed_norm_m_s;
  int due;
  if (c->every > 0)
    due = !c->ready || prm->step % c->every == 0;
  else
    due = !c->ready || time_s + 1e-10 >= c->next_update_s;
  c->due = due;
  if (!due) return;
  *status = 0;
  c->ready = 1;
  c->epoch_s = time_s;
  if (c->every == 0) {
    do {
      c->next_update_s += c->interval_s;
    } while (c->next_update_s <= time_s + 1e-10);
  }
}

// A failed update inside the step graph fails the step.
__global__ void k_mi_check(const MiCadence *c, const int *fac_status,
                           const int *solve_status, gcs::DevStatus *st) {
  if (c->due == 0) return;
  if (*fac_status != 0 || solve_status[0] != 0 || solve_status[1] != 0)
    gcs::fail(st, gcs::kStageMiCoupling, 0, 0, 0, 0, 0);
}

double vdot(const gamera_no_vec3 &a, const gamera_no_vec3 &b) {
  return a.value[0] * b.value[0] + a.value[1] * b.value[1] + a.value[2] * b.value[2];
}
double vmag(const gamera_no_vec3 &a) { return sqrt(vdot(a, a)); }

// nonorthogonal_mi.c:168-180
double mapped_colatitude(double th, double r, double ri) {
  return gcs::mi_mapped_colatitude(th, r, ri);
}

// nonorthogonal_mi.c:182-195
double dipole_field_ratio(double th, double r, double ri) {
  const double thi = mapped_colatitude(th, r, ri);
  if (!std::isfinite(thi)) return NAN;
  const double rr = r / ri;
  return rr * rr * rr * sqrt(1.0 + 3.0 * pow(cos(thi), 2.0)) /
         sqrt(1.0 + 3.0 * pow(cos(th), 2.0));
}

// cubedsphere_mi_dipole.c:37-52
bool valid_config(const gamera_cs_mi_dipole_config *c) {
  return c != nullptr && c->azimuth_points >= 8U && c->colatitude_points >= 3U &&
         c->current_shell < 64U && std::isfinite(c->ionosphere_radius_re) &&
         c->ionosphere_radius_re > 0.0 && std::isfinite(c->pedersen_siemens) &&
         c->pedersen_siemens > 0.0 && std::isfinite(c->coupling_interval_s) &&
         c->coupling_interval_s > 0.0 && std::isfinite(c->length_norm_m) &&
         c->length_norm_m > 0.0 && std::isfinite(c->speed_norm_m_s) &&
         c->speed_norm_m_s > 0.0 && std::isfinite(c->mass_density_norm_kg_m3) &&
         c->mass_density_norm_kg_m3 > 0.0 && c->maximum_iterations > 0 &&
         std::isfinite(c->relative_tolerance) && c->relative_tolerance > 0.0;
}

// Host view of the grid geometry the plans need: the reference-layout grid
// of a host-grid context, or the innermost layers kept by a device-built
// one.
struct GeomView {
  const gamera_no_grid *grid = nullptr;
  const gcs::Context *ctx = nullptr;
  int E1 = 0, E2 = 0, win_layers = 0;
  gamera_no_vec3 centroid(int f, int i, int j, int k) const {
    if (grid) return grid[f].cell[((size_t)i * E1 + j) * E2 + k].centroid;
    return ctx->win_centroid[f][((size_t)i * E1 + j) * E2 + k];
  }
  gamera_no_vec3 vertex(int f, int i, int j, int k) const {
    if (grid)
      return grid[f].vertex[((size_t)i * (E1 + 1) + j) * (E2 + 1) + k];
    return ctx->win_vertex[f][((size_t)i * (E1 + 1) + j) * (E2 + 1) + k];
  }
  // Edge direction and length (nonorthogonal_geometry.c:245-262).
  bool edge(int f, int d, int i, int j, int k, EdgeG *out) const {
    if (grid) {
      const size_t *ex = grid[f].edge[d].extent;
      const size_t idx = ((size_t)i * ex[1] + j) * ex[2] + k;
      if (!grid[f].edge[d].valid[idx]) return false;
      const gamera_no_edge_geometry &e = grid[f].edge[d].value[idx];
      for (int a = 0; a < 3; ++a) out->n[a] = e.normal.value[a];
      out->len = e.length;
      return true;
    }
    int end[3] = {i, j, k};
    ++end[d];
    const gamera_no_vec3 a = vertex(f, i, j, k), b = vertex(f, end[0], end[1], end[2]);
    double v[3], n2 = 0.0;
    for (int q = 0; q < 3; ++q) {
      v[q] = b.value[q] - a.value[q];
      n2 += v[q] * v[q];
    }
    const double len = sqrt(n2);
    if (!std::isfinite(len) || len <= DBL_MIN) return false;
    for (int q = 0; q < 3; ++q) out->n[q] = v[q] * (1.0 / len);
    out->len = len;
    return true;
  }
};

}  // namespace

struct gamera_cs_mi_dipole {
  gamera_cs_earth_startup startup{};
  gamera_cs_mi_dipole_config config{};
  size_t active[3] = {0, 0, 0};
  size_t ghost = 0;
  int np = 0, nt = 0, S = 0;
  double sample_radius_re = 0.0, maximum_colatitude = 0.0;
  double sample_maximum_colatitude = 0.0, magnetic_norm_t = 0.0;
  double potential_norm_v = 0.0, current_norm_a_m2 = 0.0;
  double next_update_s = 0.0, epoch_s = 0.0;
  int ready = 0;
  // binding to the MHD state (null for a potential view)
  gcs::Context *ctx = nullptr;
  gamera_no_storage *storage = nullptr;  // host storage of a host-grid context
  std::vector<gamera_no_vec3> shell_centroid;  // 6 x n x n
  std::vector<gamera_no_vec3> shell_b0;        // 6 x n x n
  std::vector<double> shell_ratio;             // 6 x n x n dipole ratio
  // device
  void *pool = nullptr;
  MiDev dev{};
  gcs_mi_plan *solver = nullptr;
  double *d_pot = nullptr;  // 2 x nt x np (warm start)
  MiCadence *d_cad = nullptr;  // device cadence and update gate
  int every = 0;               // cadence of the in-graph update (0: time rule)
  int in_graph = 0;            // attached to its context's driver loop
  int stale = 0;               // host copies older than the device's
  int push = 0;                // host cadence newer than the device's
  // host copies of the last solved state
  std::vector<double> fac[kHemispheres], pot[kHemispheres];
  std::vector<double> host_shell_fac;  // 6 x S^2
  gamera_mi_solver_stats solve[kHemispheres] = {};
};

namespace {

// Lookup parameters of a coupling with its host copy of the potential.
gcs::MiLookup lookup_of(const gamera_cs_mi_dipole *s) {
  gcs::MiLookup L;
  L.np = s->np;
  L.nt = s->nt;
  L.maximum_colatitude = s->maximum_colatitude;
  L.ionosphere_radius_re = s->config.ionosphere_radius_re;
  L.length_norm_m = s->config.length_norm_m;
  L.speed_norm_m_s = s->config.speed_norm_m_s;
  L.magnetic_norm_t = s->magnetic_norm_t;
  L.pot[0] = s->pot[0].data();
  L.pot[1] = s->pot[1].data();
  L.startup = s->startup;
  return L;
}

bool cuda_ok(cudaError_t e, const char *what);

// Host copies (cadence, potential, FAC, statistics) from the device after
// updates that ran inside the step graph.
int sync_host(const gamera_cs_mi_dipole *cs) {
  gamera_cs_mi_dipole *s = const_cast<gamera_cs_mi_dipole *>(cs);
  if (s == nullptr || !s->stale || s->ctx == nullptr) return 0;
  s->stale = 0;
  MiCadence c;
  if (!cuda_ok(cudaStreamSynchronize(s->ctx->stream), "MI coupling") ||
      !cuda_ok(cudaMemcpy(&c, s->d_cad, sizeof(c), cudaMemcpyDeviceToHost), "cudaMemcpy"))
    return -1;
  s->ready = c.ready;
  s->epoch_s = c.epoch_s;
  s->next_update_s = c.next_update_s;
  if (!c.ready) return 0;
  const size_t count = (size_t)s->np * s->nt;
  for (int h = 0; h < kHemispheres; ++h)
    if (!cuda_ok(cudaMemcpy(s->pot[h].data(), s->d_pot + h * count, count * sizeof(double),
                            cudaMemcpyDeviceToHost), "cudaMemcpy") ||
        !cuda_ok(cudaMemcpy(s->fac[h].data(), s->dev.fac + h * count,
                            count * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy"))
      return -1;
  if (!cuda_ok(cudaMemcpy(s->host_shell_fac.data(), s->dev.shell_fac,
                          s->host_shell_fac.size() * sizeof(double),
                          cudaMemcpyDeviceToHost), "cudaMemcpy"))
    return -1;
  return gcs_mi_plan_results(s->solver, s->solve, nullptr);
}

// The device cadence from the host's, before a step graph runs.
int push_cadence(gamera_cs_mi_dipole *s) {
  if (!s->push || s->d_cad == nullptr) return 0;
  MiCadence c{};
  c.next_update_s = s->next_update_s;
  c.epoch_s = s->epoch_s;
  c.length_norm_m = s->config.length_norm_m;
  c.speed_norm_m_s = s->config.speed_norm_m_s;
  c.interval_s = s->config.coupling_interval_s;
  c.ready = s->ready;
  c.due = 0;
  c.every = s->every;
  if (!cuda_ok(cudaStreamSynchronize(s->ctx->stream), "MI coupling") ||
      !cuda_ok(cudaMemcpy(s->d_cad, &c, sizeof(c), cudaMemcpyHostToDevice), "cudaMemcpy"))
    return -1;
  s->push = 0;
  return 0;
}

void destroy_state(gamera_cs_mi_dipole *s) {
  if (!s) return;
  if (s->ctx != nullptr && s->ctx->mi_graph == s) s->ctx->mi_graph = nullptr;
  if (s->solver) gcs_mi_plan_destroy(s->solver);
  cudaFree(s->pool);
  delete s;
}

// cubedsphere_mi_dipole.c:54-77
int init_view(gamera_cs_mi_dipole *s, const gamera_cs_earth_startup *startup,
              const gamera_cs_mi_dipole_config *config) {
  if (startup == nullptr || !valid_config(config) ||
      !(config->ionosphere_radius_re < startup->inner_radius) ||
      config->azimuth_points > SIZE_MAX / config->colatitude_points)
    return -1;
  s->startup = *startup;
  s->config = *config;
  s->np = (int)config->azimuth_points;
  s->nt = (int)config->colatitude_points;
  s->maximum_colatitude = asin(sqrt(config->ionosphere_radius_re / startup->inner_radius));
  const double mu0 = 4.0e-7 * acos(-1.0);
  s->magnetic_norm_t = config->speed_norm_m_s * sqrt(mu0 * config->mass_density_norm_kg_m3);
  s->current_norm_a_m2 = s->magnetic_norm_t / (mu0 * config->length_norm_m);
  s->potential_norm_v = config->speed_norm_m_s * s->magnetic_norm_t * config->length_norm_m;
  if (!(s->potential_norm_v > 0.0) || !std::isfinite(s->maximum_colatitude)) return -1;
  const size_t count = config->azimuth_points * config->colatitude_points;
  for (int h = 0; h < kHemispheres; ++h) {
    s->pot[h].assign(count, 0.0);
    s->fac[h].assign(count, 0.0);
  }
  return 0;
}

bool cuda_ok(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return true;
  char msg[256];
  snprintf(msg, sizeof(msg), "%s: %s", what, cudaGetErrorString(e));
  set_api_error(msg);
  return false;
}

// Plans and device buffers of a coupling bound to context C.
int build_coupling(gamera_cs_mi_dipole *s, gcs::Context &C, const GeomView &G,
                   const gamera_no_background_field *background) {
  const gcs::Dims &D = C.X.D;
  const int n = D.n, g = D.g, S = n + 2;
  const int shell_i = g + (int)s->config.current_shell;
  const double qp = 0.25 * acos(-1.0);
  s->S = S;
  // sample radius: mean centroid radius of the physical shell cells
  double radius_sum = 0.0;
  size_t radius_count = 0;
  s->shell_centroid.resize((size_t)6 * n * n);
  s->shell_b0.resize((size_t)6 * n * n);
  for (int f = 0; f < 6; ++f)
    for (int j = g; j < g + n; ++j)
      for (int k = g; k < g + n; ++k) {
        const gamera_no_vec3 c = G.centroid(f, shell_i, j, k);
        s->shell_centroid[((size_t)f * n + (j - g)) * n + (k - g)] = c;
        radius_sum += vmag(c);
        ++radius_count;
      }
  s->sample_radius_re = radius_sum / (double)radius_count;
  s->sample_maximum_colatitude =
      asin(sqrt(s->config.ionosphere_radius_re / s->sample_radius_re));
  if (!std::isfinite(s->sample_radius_re) ||
      !(s->sample_radius_re > s->startup.inner_radius)) {
    set_api_error("MI sample shell is not outside the inner radius");
    return -1;
  }
  // shell B0 (host background or the device copy)
  if (background) {
    for (int f = 0; f < 6; ++f)
      for (int j = 0; j < n; ++j)
        for (int k = 0; k < n; ++k)
          s->shell_b0[((size_t)f * n + j) * n + k] =
              background[f].cell_magnetic[((size_t)shell_i * D.E1 + g + j) * D.E2 + g + k];
  } else {
    std::vector<double> tmp(n);
    for (int f = 0; f < 6; ++f)
      for (int a = 0; a < 3; ++a)
        for (int j = 0; j < n; ++j) {
          const long long c = f * D.Nn + D.node(shell_i, g + j, g);
          if (!cuda_ok(cudaMemcpy(tmp.data(), C.X.BG.b0[a] + c, n * sizeof(double),
                                  cudaMemcpyDeviceToHost),
                       "cudaMemcpy"))
            return -1;
          for (int k = 0; k < n; ++k)
            s->shell_b0[((size_t)f * n + j) * n + k].value[a] = tmp[k];
        }
  }
  // fringe of the shell field (cubedsphere_mi_dipole.c:228-262)
  std::vector<FringeB> fb((size_t)6 * 3 * S * S);
  for (int f = 0; f < 6; ++f)
    for (int l = 0; l < 3; ++l)
      for (int jj = 0; jj < S; ++jj)
        for (int kk = 0; kk < S; ++kk) {
          FringeB &P = fb[(((size_t)f * 3 + l) * S + jj) * S + kk];
          P = FringeB{0.0, 0.0, -1, 0, 0, 0};
          if (jj > 0 && jj <= n && kk > 0 && kk <= n) continue;
          const gamera_no_vec3 c = G.centroid(f, shell_i - 1 + l, g - 1 + jj, g - 1 + kk);
          int donor;
          double a, b;
          if (gcs::topo::inverse(c.value, &donor, &a, &b) != 0 || donor == f) {
            set_api_error("MI fringe donor not found");
            return -1;
          }
          const double x = (a + qp) * (double)n / (2.0 * qp) - 0.5;
          const double y = (b + qp) * (double)n / (2.0 * qp) - 0.5;
          const int j0 = (int)(size_t)fmax(0.0, fmin((double)n - 2.0, floor(x)));
          const int k0 = (int)(size_t)fmax(0.0, fmin((double)n - 2.0, floor(y)));
          P = FringeB{x - (double)j0, y - (double)k0, donor, j0, k0, 0};
        }
  // edges of the curl: I at the shell layer, J and K at it and above
  const int m = n + 1;
  std::vector<EdgeG> eg((size_t)6 * 5 * m * m, EdgeG{{0.0, 0.0, 0.0}, 0.0});
  for (int f = 0; f < 6; ++f)
    for (int set = 0; set < 5; ++set) {
      const int d = set == 0 ? 0 : (set <= 2 ? 1 : 2);
      const int li = (set == 2 || set == 4) ? shell_i + 1 : shell_i;
      const int jmax = d == 1 ? n - 1 : n, kmax = d == 2 ? n - 1 : n;
      for (int jj = 0; jj <= jmax; ++jj)
        for (int kk = 0; kk <= kmax; ++kk)
          if (!G.edge(f, d, li, g + jj, g + kk,
                      &eg[(((size_t)f * 5 + set) * m + jj) * m + kk])) {
            set_api_error("invalid edge in the MI shell");
            return -1;
          }
    }
  // dipole ratio per shell cell (cubedsphere_mi_dipole.c:276-283)
  std::vector<double> ratio((size_t)6 * n * n);
  for (size_t q = 0; q < ratio.size(); ++q) {
    const gamera_no_vec3 &p = s->shell_centroid[q];
    const double r = vmag(p);
    if (!(r > 0.0)) {
      set_api_error("MI shell centroid at the origin");
      return -1;
    }
    const double th = acos(fmin(1.0, fabs(p.value[2]) / r));
    ratio[q] = dipole_field_ratio(th, r, s->config.ionosphere_radius_re);
  }
  // FAC fringe (cubedsphere_mi_dipole.c:298-331)
  std::vector<FringeFac> ff((size_t)6 * S * S);
  for (int f = 0; f < 6; ++f)
    for (int jj = 0; jj < S; ++jj)
      for (int kk = 0; kk < S; ++kk) {
        FringeFac &P = ff[((size_t)f * S + jj) * S + kk];
        P = FringeFac{0.0, 0.0, -1, 0};
        if (jj > 0 && jj <= n && kk > 0 && kk <= n) continue;
        const gamera_no_vec3 c = G.centroid(f, shell_i, g - 1 + jj, g - 1 + kk);
        int donor;
        double a, b;
        if (gcs::topo::inverse(c.value, &donor, &a, &b) != 0 || donor == f) {
          set_api_error("MI FAC fringe donor not found");
          return -1;
        }
        const double x = (a + qp) * (double)n / (2.0 * qp) - 0.5;
        const double y = (b + qp) * (double)n / (2.0 * qp) - 0.5;
        const int j0 = (int)(size_t)fmax(0.0, fmin((double)n - 2.0, floor(x)));
        const int k0 = (int)(size_t)fmax(0.0, fmin((double)n - 2.0, floor(y)));
        P = FringeFac{x - (double)j0, y - (double)k0, donor, (j0 + 1) * S + k0 + 1};
      }
  // polar samples (cubedsphere_mi_dipole.c:344-370, :393-413)
  const int np = s->np, nt = s->nt;
  std::vector<Sample> smp((size_t)kHemispheres * nt * np);
  const double dtheta = s->maximum_colatitude / (double)(nt - 1);
  const double dphi = 2.0 * acos(-1.0) / (double)np;
  for (int h = 0; h < kHemispheres; ++h) {
    const double sign = h == 0 ? 1.0 : -1.0;
    for (int t = 0; t < nt; ++t) {
      const double th_i = (double)t * dtheta;
      const bool zero = th_i > s->sample_maximum_colatitude + 4e-14;
      const double arg = fmin(1.0, sin(th_i) * sqrt(s->sample_radius_re /
                                                    s->config.ionosphere_radius_re));
      const double th = asin(arg);
      for (int p = 0; p < np; ++p) {
        Sample &P = smp[((size_t)h * nt + t) * np + p];
        P = Sample{0.0, 0.0, -1, 0};
        if (zero) continue;
        const double phi = (double)p * dphi;
        const double pt[3] = {s->sample_radius_re * sin(th) * cos(phi),
                              s->sample_radius_re * sin(th) * sin(phi),
                              sign * s->sample_radius_re * cos(th)};
        int face;
        double a, b;
        if (gcs::topo::inverse(pt, &face, &a, &b) != 0) {
          set_api_error("MI polar sample outside the cube");
          return -1;
        }
        const double scale = (double)n / (2.0 * qp);
        const double x = (a + qp) * scale - 0.5, y = (b + qp) * scale - 0.5;
        const long j = (long)floor(x), k = (long)floor(y);
        if (j < -1L || k < -1L || j >= (long)n || k >= (long)n) {
          set_api_error("MI polar sample outside the shell");
          return -1;
        }
        P = Sample{x - (double)j, y - (double)k, face, (int)((j + 1) * S + (k + 1))};
      }
    }
  }
  // device pool
  const size_t nfield = (size_t)6 * 3 * S * S * 3, nfac = (size_t)6 * S * S;
  const size_t npolar = (size_t)kHemispheres * nt * np;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += (bytes + 255) / 256 * 256;
    return o;
  };
  const size_t o_field = take(nfield * sizeof(double));
  const size_t o_fb = take(fb.size() * sizeof(FringeB));
  const size_t o_eg = take(eg.size() * sizeof(EdgeG));
  const size_t o_ratio = take(ratio.size() * sizeof(double));
  const size_t o_b0 = take(s->shell_b0.size() * sizeof(gamera_no_vec3));
  const size_t o_sfac = take(nfac * sizeof(double));
  const size_t o_ff = take(ff.size() * sizeof(FringeFac));
  const size_t o_smp = take(smp.size() * sizeof(Sample));
  const size_t o_fac = take(npolar * sizeof(double));
  const size_t o_pot = take(npolar * sizeof(double));
  const size_t o_status = take(sizeof(int));
  const size_t o_cad = take(sizeof(MiCadence));
  if (!cuda_ok(cudaMalloc(&s->pool, off), "cudaMalloc")) return -1;
  char *base = (char *)s->pool;
  if (!cuda_ok(cudaMemset(s->pool, 0, off), "cudaMemset") ||
      !cuda_ok(cudaMemcpy(base + o_fb, fb.data(), fb.size() * sizeof(FringeB),
                          cudaMemcpyHostToDevice), "cudaMemcpy") ||
      !cuda_ok(cudaMemcpy(base + o_eg, eg.data(), eg.size() * sizeof(EdgeG),
                          cudaMemcpyHostToDevice), "cudaMemcpy") ||
      !cuda_ok(cudaMemcpy(base + o_ratio, ratio.data(), ratio.size() * sizeof(double),
                          cudaMemcpyHostToDevice), "cudaMemcpy") ||
      !cuda_ok(cudaMemcpy(base + o_b0, s->shell_b0.data(),
                          s->shell_b0.size() * sizeof(gamera_no_vec3),
                          cudaMemcpyHostToDevice), "cudaMemcpy") ||
      !cuda_ok(cudaMemcpy(base + o_ff, ff.data(), ff.size() * sizeof(FringeFac),
                          cudaMemcpyHostToDevice), "cudaMemcpy") ||
      !cuda_ok(cudaMemcpy(base + o_smp, smp.data(), smp.size() * sizeof(Sample),
                          cudaMemcpyHostToDevice), "cudaMemcpy"))
    return -1;
  MiDev &M = s->dev;
  M.n = n;
  M.g = g;
  M.shell_i = shell_i;
  M.S = S;
  M.Nn = D.Nn;
  M.N1 = D.N1;
  M.N2 = D.N2;
  M.jnorm = s->current_norm_a_m2;
  M.field = (double *)(base + o_field);
  M.fringe_b = (const FringeB *)(base + o_fb);
  M.edges = (const EdgeG *)(base + o_eg);
  M.ratio = (const double *)(base + o_ratio);
  M.b0 = (const double *)(base + o_b0);
  s->shell_ratio = ratio;
  M.shell_fac = (double *)(base + o_sfac);
  M.fringe_fac = (const FringeFac *)(base + o_ff);
  M.samples = (const Sample *)(base + o_smp);
  M.fac = (double *)(base + o_fac);
  M.polar_count = nt * np;
  M.status = (int *)(base + o_status);
  s->d_pot = (double *)(base + o_pot);
  s->d_cad = (MiCadence *)(base + o_cad);
  // the two hemisphere solves (cubedsphere_mi_dipole.c:414-424)
  gamera_mi_solver_config sc[kHemispheres];
  for (int h = 0; h < kHemispheres; ++h) {
    gamera_mi_solver_config &c = sc[h];
    c.longitude_count = (size_t)np;
    c.colatitude_count = (size_t)nt;
    c.maximum_colatitude = s->maximum_colatitude;
    c.ionosphere_radius_m = s->config.ionosphere_radius_re * s->config.length_norm_m;
    c.pedersen_siemens = s->config.pedersen_siemens;
    c.hall_siemens = 0.0;
    c.low_latitude_potential_v = 0.0;
    c.hemisphere = h == 0 ? GAMERA_MI_NORTH : GAMERA_MI_SOUTH;
    c.maximum_iterations = s->config.maximum_iterations;
    c.relative_tolerance = s->config.relative_tolerance;
    c.absolute_tolerance = 0.0;
  }
  if (gcs_mi_plan_create(sc, kHemispheres, &s->solver) != 0) return -1;
  // every solve of this coupling is gated by its cadence and bound to its
  // FAC and potential arrays
  if (gcs::mi_plan_gate(s->solver, &s->d_cad->due, M.fac, s->d_pot) != 0) return -1;
  s->host_shell_fac.assign(nfac, 0.0);
  s->push = 1;
  return 0;
}

// One coupling update on the device (cubedsphere_mi_dipole.c:223-332,
// :386-429); results copied to the host copies.
int run_update(gamera_cs_mi_dipole *s) {
  gcs::Context &C = *s->ctx;
  cudaStream_t st = C.stream;
  if (s->storage && !C.resident) {
    // the host storage is authoritative between drop-in calls: refresh B
    for (int f = 0; f < 6; ++f)
      if (C.transfer_array(f, gcs::kArrB, 0, true,
                           (double *)s->storage[f].cell_magnetic) != 0)
        return -1;
  }
  MiDev &M = s->dev;
  const int bs = 128;
  const long long nf = 6LL * 3 * M.S * M.S, nc = 6LL * M.n * M.n, ns = 6LL * M.S * M.S;
  const long long np = (long long)kHemispheres * M.polar_count;
  const FieldPtrs bp{{C.X.S.B[0], C.X.S.B[1], C.X.S.B[2]}};
  const int *gate = &s->d_cad->due;
  k_open_gate<<<1, 1, 0, st>>>(s->d_cad, M.status);
  k_shell_field<<<(unsigned)((nf + bs - 1) / bs), bs, 0, st>>>(bp, M, gate);
  k_shell_current<<<(unsigned)((nc + bs - 1) / bs), bs, 0, st>>>(C.X.G, M, gate);
  k_shell_fringe<<<(unsigned)((ns + bs - 1) / bs), bs, 0, st>>>(M, gate);
  k_polar_sample<<<(unsigned)((np + bs - 1) / bs), bs, 0, st>>>(M, gate);
  bool ok = cuda_ok(cudaGetLastError(), "MI coupling launch");
  int status = 0;
  ok = ok && cuda_ok(cudaMemcpyAsync(&status, M.status, sizeof(int),
                                     cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync") &&
       cuda_ok(cudaStreamSynchronize(st), "MI coupling");
  if (!ok) return -1;
  if (status != 0) {
    set_api_error("non-finite field-aligned current on the MI shell");
    return -1;
  }
  if (gcs_mi_solve_constant_pedersen_async(s->solver, M.fac, s->d_pot, st) != 0) return -1;
  int solve_status[kHemispheres] = {2, 2};
  if (gcs_mi_plan_results(s->solver, s->solve, solve_status) != 0) return -1;
  const size_t count = (size_t)s->np * s->nt;
  for (int h = 0; h < kHemispheres; ++h) {
    if (!cuda_ok(cudaMemcpy(s->pot[h].data(), s->d_pot + h * count,
                            count * sizeof(double), cudaMemcpyDeviceToHost),
                 "cudaMemcpy") ||
        !cuda_ok(cudaMemcpy(s->fac[h].data(), M.fac + h * count, count * sizeof(double),
                            cudaMemcpyDeviceToHost),
                 "cudaMemcpy"))
      return -1;
  }
  if (!cuda_ok(cudaMemcpy(s->host_shell_fac.data(), M.shell_fac,
                          s->host_shell_fac.size() * sizeof(double),
                          cudaMemcpyDeviceToHost),
               "cudaMemcpy"))
    return -1;
  for (int h = 0; h < kHemispheres; ++h)
    if (solve_status[h] != 0 || !s->solve[h].converged) {
      set_api_error("MI potential solve did not converge");
      return -1;
    }
  return 0;
}

// J_parallel of a physical shell cell (A/m^2, before the dipole mapping):
// the device shell FAC of the last update divided by the cell's dipole ratio.
double shell_jparallel(const gamera_cs_mi_dipole *s, int f, int j, int k) {
  const size_t q = ((size_t)f * s->active[1] + j) * s->active[2] + k;
  return s->host_shell_fac[((size_t)f * s->S + j + 1) * s->S + k + 1] / s->shell_ratio[q];
}

}  // namespace

extern "C" {

int gamera_cs_mi_dipole_create(const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
                               gamera_no_storage storage[GAMERA_CS_FACE_COUNT],
                               const gamera_no_background_field background[GAMERA_CS_FACE_COUNT],
                               const gamera_cs_earth_startup *startup,
                               const size_t active[3], size_t ghost,
                               const gamera_cs_mi_dipole_config *config,
                               gamera_cs_mi_dipole **result) {
  if (result == nullptr) return -1;
  *result = nullptr;
  if (grid == nullptr || storage == nullptr || background == nullptr ||
      startup == nullptr || active == nullptr || ghost < 4U || active[0] < 3U ||
      active[1] < 8U || active[1] != active[2] || !valid_config(config) ||
      config->current_shell + 1U >= active[0] ||
      !(config->ionosphere_radius_re < startup->inner_radius) ||
      config->azimuth_points > SIZE_MAX / config->colatitude_points) {
    set_api_error("invalid MI coupling arguments");
    return -1;
  }
  gcs::Context *C = gcs::context_for_grid(grid, active, ghost);
  if (!C) return -1;
  gamera_cs_mi_dipole *s = new gamera_cs_mi_dipole();
  GeomView G;
  G.grid = grid;
  G.E1 = C->X.D.E1;
  G.E2 = C->X.D.E2;
  if (init_view(s, startup, config) != 0) {
    set_api_error("invalid MI coupling configuration");
    destroy_state(s);
    return -1;
  }
  s->ctx = C;
  s->storage = storage;
  memcpy(s->active, active, sizeof(s->active));
  s->ghost = ghost;
  if (build_coupling(s, *C, G, background) != 0) {
    destroy_state(s);
    return -1;
  }
  *result = s;
  return 0;
}

int gcs_context_mi_dipole_create(gcs_context *ctx, const gamera_cs_earth_startup *startup,
                                 const gamera_cs_mi_dipole_config *config,
                                 gamera_cs_mi_dipole **result) {
  if (result == nullptr) return -1;
  *result = nullptr;
  gcs::Context *C = gcs::context_of(ctx);
  if (C == nullptr || startup == nullptr || !valid_config(config)) {
    set_api_error("invalid MI coupling arguments");
    return -1;
  }
  const gcs::Dims &D = C->X.D;
  if (C->win_layers == 0 || D.nr < 3 || D.n < 8 ||
      (int)config->current_shell + 1 >= D.nr ||
      D.g + (int)config->current_shell + 2 > C->win_layers ||
      !(config->ionosphere_radius_re < startup->inner_radius) || C->X.BG.b0[0] == nullptr) {
    set_api_error("MI coupling needs a device-built case with a background "
                  "and a shell within the innermost four active layers");
    return -1;
  }
  gamera_cs_mi_dipole *s = new gamera_cs_mi_dipole();
  if (init_view(s, startup, config) != 0) {
    set_api_error("invalid MI coupling configuration");
    destroy_state(s);
    return -1;
  }
  GeomView G;
  G.ctx = C;
  G.E1 = D.E1;
  G.E2 = D.E2;
  G.win_layers = C->win_layers;
  s->ctx = C;
  s->active[0] = (size_t)D.nr;
  s->active[1] = s->active[2] = (size_t)D.n;
  s->ghost = (size_t)D.g;
  if (build_coupling(s, *C, G, nullptr) != 0) {
    destroy_state(s);
    return -1;
  }
  *result = s;
  return 0;
}

void gamera_cs_mi_dipole_destroy(gamera_cs_mi_dipole *state) { destroy_state(state); }

int gamera_cs_mi_dipole_create_potential_view(const gamera_cs_earth_startup *startup,
                                              const gamera_cs_mi_dipole_config *config,
                                              gamera_cs_mi_dipole **result) {
  if (result == nullptr) return -1;
  *result = nullptr;
  gamera_cs_mi_dipole *s = new gamera_cs_mi_dipole();
  if (init_view(s, startup, config) != 0) {
    destroy_state(s);
    return -1;
  }
  *result = s;
  return 0;
}

}  // extern "C"

namespace gcs {
bool mi_lookup(const gamera_cs_mi_dipole *s, MiLookup *L, double *potential_norm_v) {
  if (s == nullptr || sync_host(s) != 0 || !s->ready) return false;
  *L = lookup_of(s);
  *potential_norm_v = s->potential_norm_v;
  return true;
}
}  // namespace gcs

extern "C" {

int gamera_cs_mi_dipole_ready(const gamera_cs_mi_dipole *s) {
  if (s != nullptr && sync_host(s) != 0) return 0;
  return s != nullptr && s->ready;
}

// cubedsphere_mi_dipole.c:372-378
int gamera_cs_mi_dipole_update_due(const gamera_cs_mi_dipole *s, double time_code) {
  if (s == nullptr || !std::isfinite(time_code) || time_code < 0.0) return -1;
  if (sync_host(s) != 0) return -1;
  const double time_s = time_code * s->config.length_norm_m / s->config.speed_norm_m_s;
  return !s->ready || time_s + 1e-10 >= s->next_update_s;
}

// cubedsphere_mi_dipole.c:380-436
int gamera_cs_mi_dipole_maybe_update(gamera_cs_mi_dipole *s, double time_code) {
  const int due = gamera_cs_mi_dipole_update_due(s, time_code);
  if (due <= 0) return due;
  if (s->ctx == nullptr) return -1;
  const double time_s = time_code * s->config.length_norm_m / s->config.speed_norm_m_s;
  if (run_update(s) != 0) return -1;
  s->ready = 1;
  s->epoch_s = time_s;
  do {
    s->next_update_s += s->config.coupling_interval_s;
  } while (s->next_update_s <= time_s + 1e-10);
  s->push = 1;
  return 1;
}

int gamera_cs_mi_dipole_export_potential(const gamera_cs_mi_dipole *s, double *values,
                                         size_t count, double *epoch_s,
                                         double *next_update_s) {
  if (!gamera_cs_mi_dipole_ready(s) || values == nullptr || epoch_s == nullptr ||
      next_update_s == nullptr)
    return -1;
  const size_t per = (size_t)s->np * s->nt;
  if (count != kHemispheres * per) return -1;
  for (int h = 0; h < kHemispheres; ++h)
    memcpy(values + h * per, s->pot[h].data(), per * sizeof(double));
  *epoch_s = s->epoch_s;
  *next_update_s = s->next_update_s;
  return 0;
}

int gamera_cs_mi_dipole_import_potential(gamera_cs_mi_dipole *s, const double *values,
                                         size_t count, double epoch_s,
                                         double next_update_s) {
  if (s == nullptr || values == nullptr || !std::isfinite(epoch_s) ||
      !std::isfinite(next_update_s) || epoch_s < 0.0 || next_update_s <= epoch_s ||
      sync_host(s) != 0)
    return -1;
  const size_t per = (size_t)s->np * s->nt;
  if (count != kHemispheres * per) return -1;
  for (size_t q = 0; q < count; ++q)
    if (!std::isfinite(values[q])) return -1;
  for (int h = 0; h < kHemispheres; ++h)
    memcpy(s->pot[h].data(), values + h * per, per * sizeof(double));
  if (s->d_pot &&
      !cuda_ok(cudaMemcpy(s->d_pot, values, count * sizeof(double), cudaMemcpyHostToDevice),
               "cudaMemcpy"))
    return -1;
  s->epoch_s = epoch_s;
  s->next_update_s = next_update_s;
  s->ready = 1;
  s->push = 1;
  return 0;
}

// cubedsphere_mi_dipole.c:442-476
int gamera_cs_mi_dipole_potential(const gamera_cs_mi_dipole *s, gamera_no_vec3 point,
                                  double *potential_v) {
  if (!gamera_cs_mi_dipole_ready(s) || potential_v == nullptr) return -1;
  return gcs::mi_potential(lookup_of(s), point, potential_v);
}

// cubedsphere_mi_dipole.c:478-503
int gamera_cs_mi_dipole_apply_inner_emf(const gamera_cs_mi_dipole *s,
                                        gamera_no_storage *storage,
                                        const gamera_no_grid *grid, size_t wall_i) {
  if (!gamera_cs_mi_dipole_ready(s) || storage == nullptr || grid == nullptr) return -1;
  for (int d = 1; d <= 2; ++d)
    for (size_t j = 0; j < grid->edge[d].extent[1]; ++j)
      for (size_t k = 0; k < grid->edge[d].extent[2]; ++k) {
        const size_t *ex = grid->edge[d].extent;
        const size_t edge = (wall_i * ex[1] + j) * ex[2] + k;
        if (!grid->edge[d].valid[edge]) continue;
        size_t end[3] = {wall_i, j, k};
        ++end[d];
        const size_t *vx = grid->vertex_extent;
        const gamera_no_vec3 a = grid->vertex[(wall_i * vx[1] + j) * vx[2] + k];
        const gamera_no_vec3 b = grid->vertex[(end[0] * vx[1] + end[1]) * vx[2] + end[2]];
        double pa, pb;
        if (gamera_cs_mi_dipole_potential(s, a, &pa) != 0 ||
            gamera_cs_mi_dipole_potential(s, b, &pb) != 0)
          return -1;
        storage->edge_emf[d][edge] = -(pb - pa) / s->potential_norm_v;
      }
  return 0;
}

// cubedsphere_mi_dipole.c:505-543 with nonorthogonal_mi.c:20-41
int gamera_cs_mi_dipole_ghost_velocity(const gamera_cs_mi_dipole *s, gamera_no_vec3 point,
                                       gamera_no_vec3 source_velocity,
                                       gamera_no_vec3 *ghost_velocity) {
  if (!gamera_cs_mi_dipole_ready(s) || ghost_velocity == nullptr) return -1;
  return gcs::mi_ghost_velocity(lookup_of(s), point, source_velocity, ghost_velocity);
}

// cubedsphere_mi_dipole.c:545-570
int gamera_cs_mi_dipole_stats(const gamera_cs_mi_dipole *s, double *fac_min,
                              double *fac_max, double *potential_min_v,
                              double *potential_max_v, gamera_mi_solver_stats solve[2]) {
  if (!gamera_cs_mi_dipole_ready(s) || fac_min == nullptr || fac_max == nullptr ||
      potential_min_v == nullptr || potential_max_v == nullptr || solve == nullptr)
    return -1;
  *fac_min = INFINITY;
  *fac_max = -INFINITY;
  *potential_min_v = INFINITY;
  *potential_max_v = -INFINITY;
  for (int h = 0; h < kHemispheres; ++h) {
    solve[h] = s->solve[h];
    for (size_t q = 0; q < s->fac[h].size(); ++q) {
      *fac_min = fmin(*fac_min, s->fac[h][q]);
      *fac_max = fmax(*fac_max, s->fac[h][q]);
      *potential_min_v = fmin(*potential_min_v, s->pot[h][q]);
      *potential_max_v = fmax(*potential_max_v, s->pot[h][q]);
    }
  }
  return 0;
}

// cubedsphere_mi_dipole.c:572-590
int gamera_cs_mi_dipole_analysis_view(const gamera_cs_mi_dipole *s,
                                      gamera_cs_mi_analysis_view *view) {
  if (!gamera_cs_mi_dipole_ready(s) || view == nullptr || s->ctx == nullptr) return -1;
  view->azimuth_points = (size_t)s->np;
  view->colatitude_points = (size_t)s->nt;
  view->shell_j_cells = s->active[1];
  view->shell_k_cells = s->active[2];
  view->maximum_colatitude_rad = s->maximum_colatitude;
  view->epoch_s = s->epoch_s;
  view->sample_radius_re = s->sample_radius_re;
  view->pedersen_siemens = s->config.pedersen_siemens;
  for (int h = 0; h < kHemispheres; ++h) {
    view->fac_parallel_a_m2[h] = s->fac[h].data();
    view->potential_v[h] = s->pot[h].data();
  }
  return 0;
}

// cubedsphere_mi_dipole.c:592-618
int gamera_cs_mi_dipole_export_shell_current(const gamera_cs_mi_dipole *s,
                                             double *jparallel_a_m2, double *mlat_deg,
                                             double *phi_deg, size_t count) {
  if (!gamera_cs_mi_dipole_ready(s) || s->ctx == nullptr || !jparallel_a_m2 ||
      !mlat_deg || !phi_deg || count != 6 * s->active[1] * s->active[2])
    return -1;
  const double pi = acos(-1.0);
  for (int f = 0; f < 6; ++f)
    for (size_t j = 0; j < s->active[1]; ++j)
      for (size_t k = 0; k < s->active[2]; ++k) {
        const size_t q = ((size_t)f * s->active[1] + j) * s->active[2] + k;
        const gamera_no_vec3 &p = s->shell_centroid[q];
        const double r = vmag(p);
        if (!(r > 0.0)) return -1;
        double phi = atan2(p.value[1], p.value[0]) * 180.0 / pi;
        if (phi < 0.0) phi += 360.0;
        mlat_deg[q] = asin(p.value[2] / r) * 180.0 / pi;
        phi_deg[q] = phi;
        jparallel_a_m2[q] = shell_jparallel(s, f, (int)j, (int)k);
      }
  return 0;
}

// cubedsphere_mi_dipole.c:620-651
int gamera_cs_mi_dipole_write_csv(const gamera_cs_mi_dipole *s, const char *prefix) {
  if (!gamera_cs_mi_dipole_ready(s) || prefix == nullptr) return -1;
  if (strlen(prefix) > 4000U) return -1;
  char name[4096];
  const size_t np = (size_t)s->np, nt = (size_t)s->nt;
  for (int h = 0; h < kHemispheres; ++h) {
    if (snprintf(name, sizeof(name), "%s.mi_%s.csv", prefix, h == 0 ? "north" : "south") >=
        (int)sizeof(name))
      return -1;
    FILE *file = fopen(name, "w");
    if (file == nullptr) return -1;
    fputs("time_s,hemisphere,theta_deg,phi_deg,fac_A_m2,potential_V\n", file);
    for (size_t t = 0; t < nt; ++t)
      for (size_t p = 0; p < np; ++p) {
        const size_t q = t * np + p;
        fprintf(file, "%.17g,%s,%.17g,%.17g,%.17g,%.17g\n", s->epoch_s,
                h == 0 ? "north" : "south",
                s->maximum_colatitude * (double)t / (double)(nt - 1U) * 180.0 / acos(-1.0),
                360.0 * (double)p / (double)np, s->fac[h][q], s->pot[h][q]);
      }
    if (fclose(file) != 0) return -1;
  }
  return 0;
}

// cubedsphere_mi_dipole.c:653-689
int gamera_cs_mi_dipole_write_shell_current_csv(const gamera_cs_mi_dipole *s,
                                                const char *prefix) {
  if (!gamera_cs_mi_dipole_ready(s) || prefix == nullptr || s->ctx == nullptr) return -1;
  char path[4096];
  if (snprintf(path, sizeof(path), "%s.shell_j.csv", prefix) >= (int)sizeof(path)) return -1;
  FILE *file = fopen(path, "w");
  if (file == nullptr) return -1;
  fputs("face,j,k,mlat_deg,phi_deg,jparallel_A_m2\n", file);
  const double pi = acos(-1.0);
  for (int f = 0; f < 6; ++f)
    for (size_t j = 0; j < s->active[1]; ++j)
      for (size_t k = 0; k < s->active[2]; ++k) {
        const gamera_no_vec3 &p = s->shell_centroid[((size_t)f * s->active[1] + j) *
                                                        s->active[2] + k];
        const double r = vmag(p);
        double phi = atan2(p.value[1], p.value[0]) * 180.0 / pi;
        if (phi < 0.0) phi += 360.0;
        fprintf(file, "%d,%zu,%zu,%.17g,%.17g,%.17g\n", f, j, k,
                asin(p.value[2] / r) * 180.0 / pi, phi, shell_jparallel(s, f, (int)j, (int)k));
      }
  return fclose(file) == 0 ? 0 : -1;
}

}  // extern "C"

namespace gcs {

// The coupling update inside a step of the device driver loop, before the
// step: cadence, gated FAC kernels and solve, failure check.
int mi_launch_in_step(gamera_cs_mi_dipole *s, cudaStream_t st) {
  Context &C = *s->ctx;
  MiDev &M = s->dev;
  const int bs = 128;
  const long long nf = 6LL * 3 * M.S * M.S, nc = 6LL * M.n * M.n, ns = 6LL * M.S * M.S;
  const long long np = (long long)kHemispheres * M.polar_count;
  const FieldPtrs bp{{C.X.S.B[0], C.X.S.B[1], C.X.S.B[2]}};
  const int *gate = &s->d_cad->due;
  k_mi_due<<<1, 1, 0, st>>>(C.X.params, s->d_cad, M.status, C.X.status);
  k_shell_field<<<(unsigned)((nf + bs - 1) / bs), bs, 0, st>>>(bp, M, gate);
  k_shell_current<<<(unsigned)((nc + bs - 1) / bs), bs, 0, st>>>(C.X.G, M, gate);
  k_shell_fringe<<<(unsigned)((ns + bs - 1) / bs), bs, 0, st>>>(M, gate);
  k_polar_sample<<<(unsigned)((np + bs - 1) / bs), bs, 0, st>>>(M, gate);
  if (mi_plan_launch(s->solver, st) != 0) return -1;
  k_mi_check<<<1, 1, 0, st>>>(s->d_cad, M.status, mi_plan_status(s->solver), C.X.status);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

// Before a driver-loop run: the device cadence takes the host's changes.
int mi_before_run(gamera_cs_mi_dipole *s) { return push_cadence(s); }

// After a driver-loop run: the host copies are refreshed on next access.
void mi_after_run(gamera_cs_mi_dipole *s) { s->stale = 1; }

// The device potential of a coupling updated inside context C's step graph
// (the Earth boundary reads it directly), else null.
const double *mi_graph_potential(const gamera_cs_mi_dipole *s, const Context *C) {
  return s != nullptr && s->in_graph && s->ctx == C && C->mi_graph == s ? s->d_pot
                                                                        : nullptr;
}

// Lookup parameters of a coupling updated inside context C's step graph,
// with the potential pointing at its device copy: every step's update runs
// before the step reads it, so the wall uses the coupling from the first
// step on.
bool mi_lookup_device(const gamera_cs_mi_dipole *s, const Context *C, MiLookup *L,
                      double *potential_norm_v) {
  const double *d = mi_graph_potential(s, C);
  if (d == nullptr) return false;
  *L = lookup_of(s);
  L->pot[0] = d;
  L->pot[1] = d + (size_t)s->np * s->nt;
  *potential_norm_v = s->potential_norm_v;
  return true;
}

}  // namespace gcs

extern "C" {

int gcs_context_set_mi_coupling(gcs_context *ctx, gamera_cs_mi_dipole *mi,
                                int every_steps) {
  gcs::Context *C = gcs::context_of(ctx);
  if (C == nullptr || every_steps < 0) {
    set_api_error("invalid MI coupling attachment");
    return -1;
  }
  if (C->mi_graph != nullptr) {
    gamera_cs_mi_dipole *old = C->mi_graph;
    if (sync_host(old) != 0) return -1;
    old->in_graph = 0;
    C->mi_graph = nullptr;
  }
  if (mi == nullptr) return 0;
  if (mi->ctx != C || mi->d_cad == nullptr) {
    set_api_error("the MI coupling belongs to another context");
    return -1;
  }
  if (sync_host(mi) != 0) return -1;
  mi->every = every_steps;
  mi->in_graph = 1;
  mi->push = 1;
  if (push_cadence(mi) != 0) return -1;
  C->mi_graph = mi;
  return 0;
}

}  // extern "C"
