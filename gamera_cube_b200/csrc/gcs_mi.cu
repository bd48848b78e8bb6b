// Ionosphere potential solves on the polar cap
// (nonorthogonal/src/nonorthogonal/nonorthogonal_mi.c).
//
// Constant Pedersen conductance (the solve the cube's MI coupling calls,
// cubedsphere/cubedsphere_mi_dipole.c:414-429): the reduced symmetric system
// of nonorthogonal_mi.c:305-431 -- one pole unknown plus sin(theta)-weighted
// interior rows -- solved by Jacobi-preconditioned CG with the reference's
// iteration rules (:433-609): the recurrence residual norm is tested every
// iteration, and at convergence or every 1024 iterations the true residual
// rhs - A x is recomputed and the iteration restarted from it.
//
// One thread-block cluster solves one system and keeps it on chip for the
// whole solve.  CTA c of the cluster owns a contiguous band of colatitude
// rows; the search direction lives in the CTA's shared memory (neighbours
// read the adjacent row of the band through distributed shared memory), the
// solution and residual live in registers, and every dot product is a
// block reduction followed by one cluster barrier and a fixed-order sum of
// the CTAs' partials, so all CTAs see bit-identical scalars and take the
// same branches.  Several systems (the two hemispheres) are independent
// clusters of one launch.  HBM is touched only to load the inputs and store
// the potential.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "gamera_cs_b200.h"
#include "gcs_error.h"

namespace cg = cooperative_groups;

struct gcs_mi_plan;

namespace gcs {
namespace mi {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxCluster = 16;
constexpr int kPortableCluster = 8;
constexpr int kSlots = 4;       // rotating cluster-reduction slots
constexpr int kSlotWidth = 4;   // values per reduction
constexpr int kTruePeriod = 1024;
// One launch runs at most this many iterations (about two seconds on a
// B200 at the largest supported grid); larger maximum_iterations are
// clamped.
constexpr int kMaxIterations = 1 << 20;

// Constants of one interior colatitude row i (1 <= i <= nt-2), computed on
// the host with the reference's formulas (nonorthogonal_mi.c:235-244,
// :346-357, :464-478).
struct Row {
  double w;      // sin(theta): row weight of the reduced system
  double lo;     // theta_coefficient at theta - dtheta/2
  double up;     // theta_coefficient at theta + dtheta/2
  double lon;    // longitude coefficient
  double rdg;    // 1 / (w (lo + up + 2 lon)): Jacobi preconditioner
  double rw;     // 1 / w: residual norm of the unweighted row
  double inc;    // dipole cos(inclination)
  double extra;  // (w up) low on the last interior row, else 0
};

struct System {
  int np, nt;
  int max_iter;
  int pad;
  double pe;        // pole edge coefficient (nonorthogonal_mi.c:324-334)
  double neg_r2;    // -R^2
  double low;       // low-latitude Dirichlet potential
  double abs_tol, rel_tol;
  const Row *rows;  // nt - 2 rows
  const double *fac;
  double *pot;
  gamera_mi_solver_stats *stats;
  int *status;      // 0 converged, 1 not converged, 2 non-finite FAC
};

__device__ __forceinline__ double warp_sum(double v) {
  // xor butterfly: every lane ends with the same value (a + b == b + a)
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum of N values over the CTA; every thread receives the same result.
template <int N>
__device__ __forceinline__ void block_sum(double (&v)[N], double *wbuf) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < N; ++q) {
    v[q] = warp_sum(v[q]);
    if (lane == 0) wbuf[warp * N + q] = v[q];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < N; ++q) {
    double a = 0.0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) a += wbuf[w * N + q];
    v[q] = a;
  }
}

// Sum of each CTA's N values over the cluster, in rank order.  The cluster
// barrier also publishes every shared-memory write made before it.
template <int N>
__device__ __forceinline__ void cluster_sum(cg::cluster_group &cl, double (&v)[N],
                                            double *slots, int &ctr, int csize) {
  const int slot = ctr & (kSlots - 1);
  ++ctr;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < N; ++q) slots[slot * kSlotWidth + q] = v[q];
  }
  cl.sync();
#pragma unroll
  for (int q = 0; q < N; ++q) v[q] = 0.0;
  for (int c = 0; c < csize; ++c) {
    const double *rs = cl.map_shared_rank(slots, c);
#pragma unroll
    for (int q = 0; q < N; ++q) v[q] += rs[slot * kSlotWidth + q];
  }
}

struct Band {
  int ra, nrow;            // first interior row (0-based) and row count
  const double *up;        // neighbour band above (rank - 1), or null
  const double *dn;        // neighbour band below (rank + 1), or null
  int up_last;             // offset of the above band's last row
};

// Reduced operator row (nonorthogonal_mi.c:394-409), evaluated in the
// reference's order.  s holds this band's rows; pole is the pole value.
__device__ __forceinline__ double apply_row(const double *s, const Band &b,
                                            const Row &rw, int np, int R,
                                            int l, int j, int p, double pole) {
  const double c = s[p];
  const double sm = j == 0 ? s[p + np - 1] : s[p - 1];
  const double sp = j == np - 1 ? s[p - np + 1] : s[p + 1];
  double lv, uv;
  if (l > 0) lv = s[p - np];
  else lv = b.ra == 0 ? pole : b.up[b.up_last + j];
  if (l < b.nrow - 1) uv = s[p + np];
  else uv = b.ra + b.nrow == R ? 0.0 : b.dn[j];
  return rw.w * (rw.lo * (c - lv) + rw.up * (c - uv) +
                 rw.lon * (2.0 * c - sm - sp));
}

// Walks the points p = t, t + kThreads, ... of a band of nrow rows of np
// longitudes, keeping (row, longitude) of p without a division per point.
struct Walk {
  int l0, j0, dl, dj;
  __device__ Walk(int t, int np) {
    l0 = t / np;
    j0 = t - l0 * np;
    dl = kThreads / np;
    dj = kThreads - dl * np;
  }
};
#define GCS_MI_FOR_POINTS(W, P, np)                                     \
  for (int p = threadIdx.x, l = (W).l0, j = (W).j0; p < (P);            \
       p += kThreads, l += (W).dl + ((j + (W).dj) >= (np) ? 1 : 0),     \
           j = (j + (W).dj) >= (np) ? j + (W).dj - (np) : j + (W).dj)

__global__ void __launch_bounds__(kThreads, 1)
    k_pcg(const System *systems, int csize) {
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const System S = systems[blockIdx.x / csize];
  const int np = S.np, R = S.nt - 2;
  const int t = threadIdx.x;

  extern __shared__ __align__(16) double dyn[];
  __shared__ double wbuf[kWarps * kSlotWidth];
  __shared__ double slots[kSlots * kSlotWidth];
  __shared__ double pole_s;

  Band b;
  b.ra = (int)((long long)rank * R / csize);
  const int rb = (int)((long long)(rank + 1) * R / csize);
  b.nrow = rb - b.ra;
  const int P = b.nrow * np;
  const size_t stride = (size_t)((R + csize - 1) / csize) * np;
  double *s = dyn;               // search direction (read by neighbours)
  double *xs = dyn + stride;     // solution
  double *rs = dyn + 2 * stride; // residual
  double *as = dyn + 3 * stride; // A s
  Row *rt = reinterpret_cast<Row *>(dyn + 4 * stride);
  b.up = nullptr;
  b.dn = nullptr;
  b.up_last = 0;
  if (rank > 0) {
    b.up = cl.map_shared_rank(s, rank - 1);
    const int ra_up = (int)((long long)(rank - 1) * R / csize);
    b.up_last = (b.ra - ra_up - 1) * np;
  }
  if (rank + 1 < csize) b.dn = cl.map_shared_rank(s, rank + 1);
  for (int l = t; l < b.nrow; l += kThreads) rt[l] = S.rows[b.ra + l];
  const bool lead = rank == 0;
  const double dnp = (double)np;
  const double ps = dnp * S.pe;  // pole diagonal and pole residual scale
  const Walk W(t, np);
  int ctr = 0;

  // Initial guess (nonorthogonal_mi.c:487-501): the pole mean of the finite
  // pole-row entries, zero for non-finite interior entries.
  double x0 = 0.0, r0 = 0.0;
  if (lead) {
    double pm[1] = {0.0};
    for (int j = t; j < np; j += kThreads) {
      const double v = S.pot[j];
      if (isfinite(v)) pm[0] += v / dnp;
    }
    block_sum<1>(pm, wbuf);
    x0 = pm[0];
  }
  GCS_MI_FOR_POINTS(W, P, np) {
    const double v = S.pot[(size_t)(b.ra + l + 1) * np + j];
    const double xv = isfinite(v) ? v : 0.0;
    xs[p] = xv;
    s[p] = xv;
  }
  if (lead && t == 0) pole_s = x0;
  cl.sync();

  // True residual of x (held in s): r = rhs - A x, its unweighted norm, the
  // rhs norm and a count of non-finite FAC (nonorthogonal_mi.c:462-513).
  auto true_residual = [&](double (&out)[3]) {
    double v[4] = {0.0, 0.0, 0.0, 0.0};  // norm^2, rhs^2, bad, ring
    const double pole = lead ? pole_s : 0.0;
    GCS_MI_FOR_POINTS(W, P, np) {
      const Row &rw = rt[l];
      const double f = S.fac[(size_t)(b.ra + l + 1) * np + j];
      const double u = S.neg_r2 * f * rw.inc;
      const double rhs = rw.w * u + rw.extra;
      const double ax = apply_row(s, b, rw, np, R, l, j, p, pole);
      const double r = rhs - ax;
      rs[p] = r;
      const double q = r * rw.rw;
      v[0] += q * q;
      v[1] += u * u;
      v[2] += isfinite(f) ? 0.0 : 1.0;
      if (b.ra + l == 0) v[3] += s[p];
    }
    block_sum<4>(v, wbuf);
    if (lead) {
      const double ax0 = S.pe * (dnp * pole - v[3]);
      r0 = 0.0 - ax0;
      const double pr = r0 / ps;
      v[0] += dnp * pr * pr;
      v[1] += dnp * S.low * S.low;
    }
    out[0] = v[0];
    out[1] = v[1];
    out[2] = v[2];
    cluster_sum<3>(cl, out, slots, ctr, csize);
  };

  // z = M^-1 r, s = z, rho = r . z
  auto restart = [&]() -> double {
    double v[1] = {0.0};
    GCS_MI_FOR_POINTS(W, P, np) {
      const double r = rs[p];
      const double z = r * rt[l].rdg;
      s[p] = z;
      v[0] += r * z;
    }
    block_sum<1>(v, wbuf);
    if (lead) {
      const double z0 = r0 / ps;
      v[0] += r0 * z0;
      if (t == 0) pole_s = z0;
    }
    cluster_sum<1>(cl, v, slots, ctr, csize);
    return v[0];
  };

  double tr[3];
  true_residual(tr);
  const double initial = sqrt(fmax(0.0, tr[0]));
  const double target =
      fmax(S.abs_tol, S.rel_tol * fmax(sqrt(fmax(0.0, tr[1])), 1.0));
  const bool bad = tr[2] > 0.0;
  double final_res = initial;
  int iters = 0;
  int conv = initial <= target;
  const int max_iter = S.max_iter < kMaxIterations ? S.max_iter : kMaxIterations;

  if (!bad && !conv) {
    double rho = restart();
    for (int it = 1; it <= max_iter; ++it) {
      if (!isfinite(rho) || rho <= DBL_MIN) break;
      // A s and s . A s
      double v[2] = {0.0, 0.0};  // s.As, first-ring sum of s
      const double pole = lead ? pole_s : 0.0;
      GCS_MI_FOR_POINTS(W, P, np) {
        const double a = apply_row(s, b, rt[l], np, R, l, j, p, pole);
        as[p] = a;
        v[0] += s[p] * a;
        if (b.ra + l == 0) v[1] += s[p];
      }
      block_sum<2>(v, wbuf);
      double As0 = 0.0;
      double den[1] = {v[0]};
      if (lead) {
        As0 = S.pe * (dnp * pole - v[1]);
        den[0] += pole * As0;
      }
      cluster_sum<1>(cl, den, slots, ctr, csize);
      if (!isfinite(den[0]) || den[0] <= DBL_MIN) break;
      const double alpha = rho / den[0];
      // x += alpha s, r -= alpha A s; residual norm and r . M^-1 r
      double w2[2] = {0.0, 0.0};
      GCS_MI_FOR_POINTS(W, P, np) {
        const Row &rw = rt[l];
        xs[p] += alpha * s[p];
        const double r = rs[p] - alpha * as[p];
        rs[p] = r;
        const double q = r * rw.rw;
        w2[0] += q * q;
        w2[1] += r * (r * rw.rdg);
      }
      block_sum<2>(w2, wbuf);
      if (lead) {
        x0 += alpha * pole;
        r0 -= alpha * As0;
        const double pr = r0 / ps;
        w2[0] += dnp * pr * pr;
        w2[1] += r0 * (r0 / ps);
      }
      cluster_sum<2>(cl, w2, slots, ctr, csize);
      final_res = sqrt(fmax(0.0, w2[0]));
      iters = it;
      if (final_res <= target || it % kTruePeriod == 0) {
        // Verify with the true residual (nonorthogonal_mi.c:562-582).
        GCS_MI_FOR_POINTS(W, P, np) { s[p] = xs[p]; }
        if (lead && t == 0) pole_s = x0;
        cl.sync();
        true_residual(tr);
        final_res = sqrt(fmax(0.0, tr[0]));
        if (final_res <= target) {
          conv = 1;
          break;
        }
        rho = restart();
        continue;
      }
      const double rho_new = w2[1];
      if (!isfinite(rho_new) || rho_new <= DBL_MIN) break;
      const double beta = rho_new / rho;
      GCS_MI_FOR_POINTS(W, P, np) { s[p] = rs[p] * rt[l].rdg + beta * s[p]; }
      if (lead && t == 0) pole_s = r0 / ps + beta * pole;
      rho = rho_new;
      cl.sync();
    }
  }

  if (bad) {
    if (lead && t == 0) *S.status = 2;
    cl.sync();  // no CTA leaves while a peer may still read its slots
    return;
  }
  // Expand the reduced solution (nonorthogonal_mi.c:595-605).
  GCS_MI_FOR_POINTS(W, P, np) { S.pot[(size_t)(b.ra + l + 1) * np + j] = xs[p]; }
  if (lead)
    for (int j = t; j < np; j += kThreads) S.pot[j] = x0;
  if (rb == R)
    for (int j = t; j < np; j += kThreads) S.pot[(size_t)(S.nt - 1) * np + j] = S.low;
  if (lead && t == 0) {
    *S.stats = gamera_mi_solver_stats{iters, initial, final_res, conv};
    *S.status = conv ? 0 : 1;
  }
  cl.sync();  // no CTA leaves while a peer may still read its shared memory
}

// ---------------------------------------------------------------- apply
// Full-layout operators of nonorthogonal_mi.c:248-287 and :658-732, one
// thread per node; the pole-row mean is summed by one thread in the
// reference's order so the result is bitwise the reference's.

__global__ void k_ring_mean(const double *p, int np, double *mean) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double m = 0.0;
    for (int j = 0; j < np; ++j) m += p[np + j] / (double)np;
    *mean = m;
  }
}

__global__ void k_apply_constant(const double *p, double *r, const Row *rows,
                                 const double *mean, int np, int nt) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)np * nt) return;
  const int i = (int)(q / np), j = (int)(q - (long long)i * np);
  if (i == 0) {
    r[q] = p[q] - *mean;
    return;
  }
  if (i == nt - 1) {
    r[q] = p[q];
    return;
  }
  const Row rw = rows[i - 1];
  const int jm = j == 0 ? np - 1 : j - 1, jp = j + 1 == np ? 0 : j + 1;
  const double c = p[q];
  r[q] = rw.lo * (c - p[q - np]) + rw.up * (c - p[q + np]) +
         rw.lon * (2.0 * c - p[(long long)i * np + jm] - p[(long long)i * np + jp]);
}

// Tensor rows: the theta metrics are per row; the conductances per node.
struct TensorRow {
  double s;          // sin(theta)
  double sl, il;     // sin and inclination^2 at theta - dtheta/2
  double su, iu;     // sin and inclination^2 at theta + dtheta/2
  double inc;        // dipole cos(inclination) of the row
};

__device__ __forceinline__ double f12(const double *hall, const TensorRow *tr,
                                      int np, int i, int j) {
  return -hall[(long long)i * np + j] / tr[i].inc;
}

__global__ void k_apply_tensor(const double *p, const double *sp, const double *sh,
                               double *r, const TensorRow *trow,
                               const double *mean, int np, int nt, double dth,
                               double dph) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)np * nt) return;
  const int i = (int)(q / np), j = (int)(q - (long long)i * np);
  if (i == 0) {
    r[q] = p[q] - *mean;
    return;
  }
  if (i == nt - 1) {
    r[q] = p[q];
    return;
  }
  const TensorRow &T = trow[i];
  const int jm = j == 0 ? np - 1 : j - 1, jp = j + 1 == np ? 0 : j + 1;
  const long long ci = q, cl = (long long)(i - 1) * np + j,
                  cu = (long long)(i + 1) * np + j, cm = (long long)i * np + jm,
                  cp = (long long)i * np + jp;
  const double sine = T.s;
  const double lower = T.sl * 0.5 * (sp[ci] + sp[cl]) / (T.il * sine * dth * dth);
  const double upper = T.su * 0.5 * (sp[ci] + sp[cu]) / (T.iu * sine * dth * dth);
  const double ll = 0.5 * (sp[ci] + sp[cm]) / (sine * sine * dph * dph);
  const double lu = 0.5 * (sp[ci] + sp[cp]) / (sine * sine * dph * dph);
  const double ped = lower * (p[ci] - p[cl]) + upper * (p[ci] - p[cu]) +
                     ll * (p[ci] - p[cm]) + lu * (p[ci] - p[cp]);
  const double dft = (f12(sh, trow, np, i + 1, j) - f12(sh, trow, np, i - 1, j)) /
                     (2.0 * dth);
  const double dfp = (f12(sh, trow, np, i, jp) - f12(sh, trow, np, i, jm)) /
                     (2.0 * dph);
  const double dpt = (p[cu] - p[cl]) / (2.0 * dth);
  const double dpp = (p[cp] - p[cm]) / (2.0 * dph);
  r[q] = ped + (-dft * dpp + dfp * dpt) / sine;
}

// ---------------------------------------------------------------- host

// nonorthogonal_mi.c:197-207
double cos_inclination(double theta, int hemisphere) {
  if (!std::isfinite(theta) || theta < 0.0 || theta > 0.5 * acos(-1.0) ||
      (hemisphere != GAMERA_MI_NORTH && hemisphere != GAMERA_MI_SOUTH))
    return NAN;
  const double c = cos(theta);
  return (double)hemisphere * 2.0 * c / sqrt(1.0 + 3.0 * c * c);
}

// nonorthogonal_mi.c:209-228
bool valid_config(const gamera_mi_solver_config *c) {
  return c != nullptr && c->longitude_count >= 4U && c->colatitude_count >= 3U &&
         std::isfinite(c->maximum_colatitude) && c->maximum_colatitude > 0.0 &&
         c->maximum_colatitude <= 0.5 * acos(-1.0) &&
         std::isfinite(c->ionosphere_radius_m) && c->ionosphere_radius_m > 0.0 &&
         std::isfinite(c->pedersen_siemens) && c->pedersen_siemens > 0.0 &&
         c->hall_siemens == 0.0 && std::isfinite(c->low_latitude_potential_v) &&
         (c->hemisphere == GAMERA_MI_NORTH || c->hemisphere == GAMERA_MI_SOUTH) &&
         c->maximum_iterations > 0 && std::isfinite(c->relative_tolerance) &&
         c->relative_tolerance > 0.0 && std::isfinite(c->absolute_tolerance) &&
         c->absolute_tolerance >= 0.0;
}

// nonorthogonal_mi.c:611-641 (configuration part; the conductance arrays
// are checked on the device copy)
bool valid_tensor_config(const gamera_mi_solver_config *c) {
  return c != nullptr && c->longitude_count >= 4U && c->colatitude_count >= 3U &&
         std::isfinite(c->maximum_colatitude) && c->maximum_colatitude > 0.0 &&
         c->maximum_colatitude <= 0.5 * acos(-1.0) &&
         std::isfinite(c->ionosphere_radius_m) && c->ionosphere_radius_m > 0.0 &&
         std::isfinite(c->low_latitude_potential_v) &&
         !(fabs(c->low_latitude_potential_v) > DBL_MIN) &&
         (c->hemisphere == GAMERA_MI_NORTH || c->hemisphere == GAMERA_MI_SOUTH) &&
         c->maximum_iterations > 0 && std::isfinite(c->relative_tolerance) &&
         c->relative_tolerance > 0.0 && std::isfinite(c->absolute_tolerance) &&
         c->absolute_tolerance >= 0.0 &&
         c->longitude_count <= SIZE_MAX / c->colatitude_count;
}

// nonorthogonal_mi.c:235-244
double theta_coefficient(const gamera_mi_solver_config *c, double th_half,
                         double th_center, double dth) {
  const double co = cos(th_half);
  const double ci2 = 4.0 * co * co / (1.0 + 3.0 * co * co);
  return sin(th_half) * c->pedersen_siemens / (ci2 * sin(th_center) * dth * dth);
}

// nonorthogonal_mi.c:324-334
double pole_edge(const gamera_mi_solver_config *c) {
  const double dth = c->maximum_colatitude / (double)(c->colatitude_count - 1U);
  const double th = 0.5 * dth;
  const double co = cos(th);
  const double ci2 = 4.0 * co * co / (1.0 + 3.0 * co * co);
  return sin(th) * c->pedersen_siemens / (ci2 * dth * dth);
}

std::vector<Row> build_rows(const gamera_mi_solver_config *c) {
  const size_t np = c->longitude_count, nt = c->colatitude_count;
  const double dth = c->maximum_colatitude / (double)(nt - 1U);
  const double dph = 2.0 * acos(-1.0) / (double)np;
  std::vector<Row> rows(nt - 2U);
  for (size_t i = 1U; i + 1U < nt; ++i) {
    const double th = (double)i * dth;
    Row &r = rows[i - 1U];
    r.w = sin(th);
    r.lo = theta_coefficient(c, th - 0.5 * dth, th, dth);
    r.up = theta_coefficient(c, th + 0.5 * dth, th, dth);
    r.lon = c->pedersen_siemens / (sin(th) * sin(th) * dph * dph);
    r.rdg = 1.0 / (r.w * (r.lo + r.up + 2.0 * r.lon));
    r.rw = 1.0 / r.w;
    r.inc = cos_inclination(th, c->hemisphere);
    r.extra = i + 2U == nt ? r.w * r.up * c->low_latitude_potential_v : 0.0;
  }
  return rows;
}

std::vector<TensorRow> build_tensor_rows(const gamera_mi_solver_config *c) {
  const size_t nt = c->colatitude_count;
  const double dth = c->maximum_colatitude / (double)(nt - 1U);
  std::vector<TensorRow> rows(nt);
  for (size_t i = 0; i < nt; ++i) {
    const double th = (double)i * dth;
    const double lth = th - 0.5 * dth, uth = th + 0.5 * dth;
    auto inc2 = [](double a) {
      const double co = cos(a);
      return 4.0 * co * co / (1.0 + 3.0 * co * co);
    };
    rows[i].s = sin(th);
    rows[i].sl = sin(lth);
    rows[i].il = inc2(lth);
    rows[i].su = sin(uth);
    rows[i].iu = inc2(uth);
    rows[i].inc = cos_inclination(th, c->hemisphere);
  }
  return rows;
}

cudaError_t configure(int csize, size_t smem) {
  cudaError_t e = cudaFuncSetAttribute(k_pcg, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  if (csize > kPortableCluster)
    e = cudaFuncSetAttribute(k_pcg, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  return e;
}

cudaLaunchConfig_t launch_config(int csize, int count, size_t smem, cudaStream_t stream,
                                 cudaLaunchAttribute *attr) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(csize * count));
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)csize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

int max_clusters(int csize, size_t smem) {
  if (configure(csize, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = launch_config(csize, 1, smem, nullptr, attr);
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k_pcg, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

// Shared memory of a band of `rows` rows: four vectors plus the row table.
size_t band_smem(int rows, int np) {
  return 4 * (size_t)rows * np * sizeof(double) + (size_t)rows * sizeof(Row);
}

constexpr size_t kMaxSmem = 200 * 1024;

}  // namespace mi
}  // namespace gcs

using namespace gcs::mi;

struct gcs_mi_plan {
  int count = 0;
  int np = 0, nt = 0;
  int csize = 0;
  size_t smem = 0;
  std::vector<gamera_mi_solver_config> configs;
  Row *d_rows = nullptr;          // count * (nt - 2)
  System *d_sys = nullptr;        // count
  double *d_fac = nullptr;        // count * nt * np
  double *d_pot = nullptr;        // count * nt * np
  gamera_mi_solver_stats *d_stats = nullptr;
  int *d_status = nullptr;
  std::vector<System> host_sys;
  cudaStream_t stream = nullptr;  // stream of the last solve
};

namespace {

using gcs::set_api_error;

void plan_free(gcs_mi_plan *p) {
  if (!p) return;
  cudaFree(p->d_rows);
  cudaFree(p->d_sys);
  cudaFree(p->d_fac);
  cudaFree(p->d_pot);
  cudaFree(p->d_stats);
  cudaFree(p->d_status);
  delete p;
}

bool cuda_ok(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return true;
  char msg[256];
  snprintf(msg, sizeof(msg), "%s: %s", what, cudaGetErrorString(e));
  set_api_error(msg);
  return false;
}

// Cluster size: about 2048 unknowns per CTA, at most 16 CTAs (8 where the
// device cannot co-schedule 16), every CTA owning at least one row.
int choose_cluster(gcs_mi_plan *p) {
  const int R = p->nt - 2;
  const long long points = (long long)p->np * R;
  int want = (int)((points + 2047) / 2048);
  if (want < 1) want = 1;
  for (int limit : {kMaxCluster, kPortableCluster}) {
    const int top = limit < R ? limit : R;
    int csize = want < top ? want : top;
    for (; csize <= top; ++csize)
      if (band_smem((R + csize - 1) / csize, p->np) <= kMaxSmem) break;
    if (csize > top) continue;
    const size_t smem = band_smem((R + csize - 1) / csize, p->np);
    if (max_clusters(csize, smem) >= 1) {
      p->csize = csize;
      p->smem = smem;
      return 0;
    }
  }
  set_api_error("MI grid too large for the on-chip cluster solve");
  return -1;
}

gcs_mi_plan *plan_create(const gamera_mi_solver_config *configs, int count) {
  if (count < 1) {
    set_api_error("MI plan needs at least one system");
    return nullptr;
  }
  for (int s = 0; s < count; ++s) {
    if (!valid_config(&configs[s])) {
      set_api_error("invalid MI solver configuration");
      return nullptr;
    }
    if (configs[s].longitude_count != configs[0].longitude_count ||
        configs[s].colatitude_count != configs[0].colatitude_count) {
      set_api_error("MI plan systems must share one grid");
      return nullptr;
    }
  }
  if (configs[0].longitude_count > 65535U || configs[0].colatitude_count > 32768U) {
    set_api_error("MI grid too large for the on-chip cluster solve");
    return nullptr;
  }
  gcs_mi_plan *p = new gcs_mi_plan();
  p->count = count;
  p->np = (int)configs[0].longitude_count;
  p->nt = (int)configs[0].colatitude_count;
  p->configs.assign(configs, configs + count);
  if (choose_cluster(p) != 0) {
    plan_free(p);
    return nullptr;
  }
  const size_t R = (size_t)p->nt - 2U, nodes = (size_t)p->np * p->nt;
  if (!cuda_ok(cudaMalloc(&p->d_rows, count * R * sizeof(Row)), "cudaMalloc") ||
      !cuda_ok(cudaMalloc(&p->d_sys, count * sizeof(System)), "cudaMalloc") ||
      !cuda_ok(cudaMalloc(&p->d_fac, count * nodes * sizeof(double)), "cudaMalloc") ||
      !cuda_ok(cudaMalloc(&p->d_pot, count * nodes * sizeof(double)), "cudaMalloc") ||
      !cuda_ok(cudaMalloc(&p->d_stats, count * sizeof(gamera_mi_solver_stats)),
               "cudaMalloc") ||
      !cuda_ok(cudaMalloc(&p->d_status, count * sizeof(int)), "cudaMalloc")) {
    plan_free(p);
    return nullptr;
  }
  p->host_sys.resize(count);
  for (int s = 0; s < count; ++s) {
    const gamera_mi_solver_config *c = &configs[s];
    std::vector<Row> rows = build_rows(c);
    if (!cuda_ok(cudaMemcpy(p->d_rows + s * R, rows.data(), R * sizeof(Row),
                            cudaMemcpyHostToDevice),
                 "cudaMemcpy")) {
      plan_free(p);
      return nullptr;
    }
    System &S = p->host_sys[s];
    S.np = p->np;
    S.nt = p->nt;
    S.max_iter = c->maximum_iterations;
    S.pad = 0;
    S.pe = pole_edge(c);
    S.neg_r2 = -(c->ionosphere_radius_m * c->ionosphere_radius_m);
    S.low = c->low_latitude_potential_v;
    S.abs_tol = c->absolute_tolerance;
    S.rel_tol = c->relative_tolerance;
    S.rows = p->d_rows + s * R;
    S.fac = p->d_fac + s * nodes;
    S.pot = p->d_pot + s * nodes;
    S.stats = p->d_stats + s;
    S.status = p->d_status + s;
  }
  if (!cuda_ok(cudaMemcpy(p->d_sys, p->host_sys.data(), count * sizeof(System),
                          cudaMemcpyHostToDevice),
               "cudaMemcpy")) {
    plan_free(p);
    return nullptr;
  }
  return p;
}

// Points the plan's systems at caller arrays (count * nt * np each).
bool plan_bind(gcs_mi_plan *p, const double *fac, double *pot, cudaStream_t stream) {
  const size_t nodes = (size_t)p->np * p->nt;
  const double *f = fac ? fac : p->d_fac;
  double *q = pot ? pot : p->d_pot;
  bool changed = false;
  for (int s = 0; s < p->count; ++s) {
    if (p->host_sys[s].fac != f + s * nodes || p->host_sys[s].pot != q + s * nodes)
      changed = true;
    p->host_sys[s].fac = f + s * nodes;
    p->host_sys[s].pot = q + s * nodes;
  }
  if (!changed) return true;
  // Synchronous: the host table is reused by the next call.
  return cuda_ok(cudaMemcpyAsync(p->d_sys, p->host_sys.data(),
                                 p->count * sizeof(System), cudaMemcpyHostToDevice,
                                 stream),
                 "cudaMemcpyAsync") &&
         cuda_ok(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
}

int plan_launch(gcs_mi_plan *p, cudaStream_t stream) {
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = launch_config(p->csize, p->count, p->smem, stream, attr);
  const cudaError_t e = cudaLaunchKernelEx(&cfg, k_pcg, (const System *)p->d_sys,
                                           p->csize);
  p->stream = stream;
  return cuda_ok(e, "MI solve launch") ? 0 : -1;
}

std::mutex g_cache_mutex;
gcs_mi_plan *g_cache = nullptr;  // plan of the last drop-in call

gcs_mi_plan *cached_plan(const gamera_mi_solver_config *config) {
  if (g_cache && g_cache->count == 1 &&
      memcmp(&g_cache->configs[0], config, sizeof(*config)) == 0)
    return g_cache;
  gcs_mi_plan *p = plan_create(config, 1);
  if (!p) return nullptr;
  plan_free(g_cache);
  g_cache = p;
  return p;
}

}  // namespace

extern "C" {

int gcs_mi_plan_create(const gamera_mi_solver_config *configs, int count,
                       gcs_mi_plan **plan) {
  if (!configs || !plan) {
    set_api_error("null argument");
    return -1;
  }
  *plan = plan_create(configs, count);
  return *plan ? 0 : -1;
}

void gcs_mi_plan_destroy(gcs_mi_plan *plan) {
  if (plan) cudaStreamSynchronize(plan->stream);
  plan_free(plan);
}

int gcs_mi_plan_info(const gcs_mi_plan *plan, int *cluster_ctas, int *threads_per_cta,
                     size_t *shared_bytes) {
  if (!plan) return -1;
  if (cluster_ctas) *cluster_ctas = plan->csize;
  if (threads_per_cta) *threads_per_cta = kThreads;
  if (shared_bytes) *shared_bytes = plan->smem;
  return 0;
}

int gcs_mi_plan_buffers(gcs_mi_plan *plan, double **fac, double **potential) {
  if (!plan) return -1;
  if (fac) *fac = plan->d_fac;
  if (potential) *potential = plan->d_pot;
  return 0;
}

int gcs_mi_solve_constant_pedersen_async(gcs_mi_plan *plan, const double *fac,
                                         double *potential, void *stream) {
  if (!plan) {
    set_api_error("null MI plan");
    return -1;
  }
  cudaStream_t st = (cudaStream_t)stream;
  if (!plan_bind(plan, fac, potential, st)) return -1;
  return plan_launch(plan, st);
}

int gcs_mi_plan_results(gcs_mi_plan *plan, gamera_mi_solver_stats *stats, int *status) {
  if (!plan) return -1;
  if (!cuda_ok(cudaStreamSynchronize(plan->stream), "MI solve")) return -1;
  if (stats &&
      !cuda_ok(cudaMemcpy(stats, plan->d_stats, plan->count * sizeof(*stats),
                          cudaMemcpyDeviceToHost),
               "cudaMemcpy"))
    return -1;
  if (status &&
      !cuda_ok(cudaMemcpy(status, plan->d_status, plan->count * sizeof(int),
                          cudaMemcpyDeviceToHost),
               "cudaMemcpy"))
    return -1;
  return 0;
}

// Drop-in for nonorthogonal_mi.c:433 (host arrays, synchronous).
int gamera_mi_solve_constant_pedersen(const gamera_mi_solver_config *config,
                                      const double *fac_a_m2, double *potential_v,
                                      gamera_mi_solver_stats *stats) {
  if (!valid_config(config) || fac_a_m2 == nullptr || potential_v == nullptr) {
    set_api_error("invalid MI solver arguments");
    return -1;
  }
  const size_t np = config->longitude_count, nt = config->colatitude_count;
  if (np > (SIZE_MAX - 1U) / (nt - 2U)) return -1;
  std::lock_guard<std::mutex> lock(g_cache_mutex);
  gcs_mi_plan *p = cached_plan(config);
  if (!p) return -1;
  const size_t bytes = np * nt * sizeof(double);
  cudaStream_t st = nullptr;
  if (!plan_bind(p, nullptr, nullptr, st)) return -1;
  int status = 2;
  gamera_mi_solver_stats s = {};
  if (!cuda_ok(cudaMemcpyAsync(p->d_fac, fac_a_m2, bytes, cudaMemcpyHostToDevice, st),
               "cudaMemcpyAsync") ||
      !cuda_ok(cudaMemcpyAsync(p->d_pot, potential_v, bytes, cudaMemcpyHostToDevice,
                               st),
               "cudaMemcpyAsync") ||
      plan_launch(p, st) != 0 ||
      !cuda_ok(cudaMemcpyAsync(potential_v, p->d_pot, bytes, cudaMemcpyDeviceToHost,
                               st),
               "cudaMemcpyAsync") ||
      !cuda_ok(cudaMemcpyAsync(&s, p->d_stats, sizeof(s), cudaMemcpyDeviceToHost, st),
               "cudaMemcpyAsync") ||
      !cuda_ok(cudaMemcpyAsync(&status, p->d_status, sizeof(int),
                               cudaMemcpyDeviceToHost, st),
               "cudaMemcpyAsync") ||
      !cuda_ok(cudaStreamSynchronize(st), "MI solve"))
    return -1;
  if (status == 2) {
    set_api_error("non-finite field-aligned current");
    return -1;
  }
  if (stats) *stats = s;
  return status == 0 ? 0 : -1;
}

// Drop-in for nonorthogonal_mi.c:248 (host arrays, synchronous).
int gamera_mi_apply_constant_pedersen(const gamera_mi_solver_config *config,
                                      const double *potential_v, double *result) {
  if (!valid_config(config) || potential_v == nullptr || result == nullptr) {
    set_api_error("invalid MI apply arguments");
    return -1;
  }
  const int np = (int)config->longitude_count, nt = (int)config->colatitude_count;
  const size_t nodes = (size_t)np * nt;
  std::vector<Row> rows = build_rows(config);
  double *d = nullptr;
  Row *dr = nullptr;
  const size_t bytes = nodes * sizeof(double);
  int rc = -1;
  if (cuda_ok(cudaMalloc(&d, 2 * bytes + sizeof(double)), "cudaMalloc") &&
      cuda_ok(cudaMalloc(&dr, rows.size() * sizeof(Row)), "cudaMalloc") &&
      cuda_ok(cudaMemcpy(dr, rows.data(), rows.size() * sizeof(Row),
                         cudaMemcpyHostToDevice),
              "cudaMemcpy") &&
      cuda_ok(cudaMemcpy(d, potential_v, bytes, cudaMemcpyHostToDevice), "cudaMemcpy")) {
    double *mean = d + 2 * nodes;
    k_ring_mean<<<1, 32>>>(d, np, mean);
    k_apply_constant<<<(unsigned)((nodes + 255) / 256), 256>>>(d, d + nodes, dr, mean,
                                                               np, nt);
    if (cuda_ok(cudaGetLastError(), "MI apply launch") &&
        cuda_ok(cudaMemcpy(result, d + nodes, bytes, cudaMemcpyDeviceToHost),
                "cudaMemcpy"))
      rc = 0;
  }
  cudaFree(d);
  cudaFree(dr);
  return rc;
}

// Drop-in for nonorthogonal_mi.c:657 (host arrays, synchronous).
int gamera_mi_apply_conductance_tensor(const gamera_mi_solver_config *config,
                                       const double *pedersen, const double *hall,
                                       const double *potential_v, double *result) {
  if (!valid_tensor_config(config) || pedersen == nullptr || hall == nullptr ||
      potential_v == nullptr || result == nullptr) {
    set_api_error("invalid MI tensor apply arguments");
    return -1;
  }
  const int np = (int)config->longitude_count, nt = (int)config->colatitude_count;
  const size_t nodes = (size_t)np * nt;
  for (size_t q = 0; q < nodes; ++q)
    if (!std::isfinite(pedersen[q]) || !(pedersen[q] > 0.0) ||
        !std::isfinite(hall[q]) || hall[q] < 0.0) {
      set_api_error("invalid conductance");
      return -1;
    }
  std::vector<TensorRow> rows = build_tensor_rows(config);
  const double dth = config->maximum_colatitude / (double)(nt - 1);
  const double dph = 2.0 * acos(-1.0) / (double)np;
  double *d = nullptr;
  TensorRow *dr = nullptr;
  const size_t bytes = nodes * sizeof(double);
  int rc = -1;
  if (cuda_ok(cudaMalloc(&d, 4 * bytes + sizeof(double)), "cudaMalloc") &&
      cuda_ok(cudaMalloc(&dr, rows.size() * sizeof(TensorRow)), "cudaMalloc") &&
      cuda_ok(cudaMemcpy(dr, rows.data(), rows.size() * sizeof(TensorRow),
                         cudaMemcpyHostToDevice),
              "cudaMemcpy") &&
      cuda_ok(cudaMemcpy(d, potential_v, bytes, cudaMemcpyHostToDevice), "cudaMemcpy") &&
      cuda_ok(cudaMemcpy(d + nodes, pedersen, bytes, cudaMemcpyHostToDevice),
              "cudaMemcpy") &&
      cuda_ok(cudaMemcpy(d + 2 * nodes, hall, bytes, cudaMemcpyHostToDevice),
              "cudaMemcpy")) {
    double *mean = d + 4 * nodes;
    k_ring_mean<<<1, 32>>>(d, np, mean);
    k_apply_tensor<<<(unsigned)((nodes + 255) / 256), 256>>>(
        d, d + nodes, d + 2 * nodes, d + 3 * nodes, dr, mean, np, nt, dth, dph);
    if (cuda_ok(cudaGetLastError(), "MI apply launch") &&
        cuda_ok(cudaMemcpy(result, d + 3 * nodes, bytes, cudaMemcpyDeviceToHost),
                "cudaMemcpy"))
      rc = 0;
  }
  cudaFree(d);
  cudaFree(dr);
  return rc;
}

}  // extern "C"
