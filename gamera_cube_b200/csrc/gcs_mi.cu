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
  const int *gate;  // when set, the solve runs only where *gate != 0
  // Variable Pedersen conductance (Hall = 0) when coef is set (k_pcg only):
  // the five-point stencil of the conductance-tensor operator
  // (nonorthogonal_mi.c:776-865) per reduced unknown -- diagonal, lower,
  // upper, longitude lower, longitude upper, `unknowns` entries each -- the
  // pole edge coefficients and the pole diagonal; Jacobi on that diagonal.
  const double *coef;
  const double *pedge;
  double diag0;
  long long unknowns;
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
// Warp butterflies, then lane w of every warp takes warp w's partial and a
// second butterfly combines them: each warp runs the identical sequence of
// additions, so all threads hold bit-identical sums.
template <int N>
__device__ __forceinline__ void block_sum(double (&v)[N], double *wbuf) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q < N; ++q) {
    v[q] = warp_sum(v[q]);
    if (lane == 0) wbuf[warp * kSlotWidth + q] = v[q];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < N; ++q)
    v[q] = warp_sum(lane < nwarps ? wbuf[lane * kSlotWidth + q] : 0.0);
}

// Sum of each CTA's N values over the cluster, in rank order.  Thread c
// pushes this CTA's values into CTA c's slot table (a store into distributed
// shared memory, so no thread waits on a remote load); after the cluster
// barrier -- which also publishes every shared-memory write made before it
// -- lane c of every warp reads rank c's entry locally and a warp butterfly
// sums them, so all CTAs hold bit-identical sums.
template <int N>
__device__ __forceinline__ void cluster_sum(cg::cluster_group &cl, double (&v)[N],
                                            double *slots, int &ctr, int rank,
                                            int csize) {
  const int slot = ctr & (kSlots - 1);
  ++ctr;
  if ((int)threadIdx.x < csize) {
    double *dst = cl.map_shared_rank(slots, (int)threadIdx.x) +
                  (slot * kMaxCluster + rank) * kSlotWidth;
#pragma unroll
    for (int q = 0; q < N; ++q) dst[q] = v[q];
  }
  cl.sync();
  const int lane = threadIdx.x & 31;
  const double *src = slots + slot * kMaxCluster * kSlotWidth;
#pragma unroll
  for (int q = 0; q < N; ++q)
    v[q] = warp_sum(lane < csize ? src[lane * kSlotWidth + q] : 0.0);
}

// A CTA's band of rows plus copies of the adjacent rows of the neighbouring
// bands (hs: search direction, hz: preconditioned residual), kept current by
// the owners' pushes.
struct Band {
  int ra, nrow;        // first interior row (0-based) and row count
  bool top, bottom;    // band holds the first / the last interior row
  double *hs_up, *hz_up;   // row above the band (last row of rank - 1)
  double *hs_dn, *hz_dn;   // row below the band (first row of rank + 1)
  double *peer_up_hs, *peer_up_hz;  // rank - 1's hs_dn / hz_dn
  double *peer_dn_hs, *peer_dn_hz;  // rank + 1's hs_up / hz_up
};

// Reduced operator row (nonorthogonal_mi.c:394-409), evaluated in the
// reference's order.  s holds this band's rows; pole is the pole value.
__device__ __forceinline__ double apply_row(const double *s, const Band &b,
                                            const Row &rw, int np, int l, int j,
                                            int p, double pole) {
  const double c = s[p];
  const double sm = j == 0 ? s[p + np - 1] : s[p - 1];
  const double sp = j == np - 1 ? s[p - np + 1] : s[p + 1];
  double lv, uv;
  if (l > 0) lv = s[p - np];
  else lv = b.top ? pole : b.hs_up[j];
  if (l < b.nrow - 1) uv = s[p + np];
  else uv = b.bottom ? 0.0 : b.hs_dn[j];
  return rw.w * (rw.lo * (c - lv) + rw.up * (c - uv) +
                 rw.lon * (2.0 * c - sm - sp));
}

// Tensor-stencil row (nonorthogonal_mi.c:872-897, Hall = 0), evaluated in
// the reference's order; ci is the reduced index of the point.
__device__ __forceinline__ double apply_var(const double *s, const Band &b,
                                            const System &S, int np, int l, int j,
                                            int p, double pole, long long ci) {
  const long long n = S.unknowns;
  const double c = s[p];
  const double sm = j == 0 ? s[p + np - 1] : s[p - 1];
  const double sp = j == np - 1 ? s[p - np + 1] : s[p + 1];
  double lv, uv;
  if (l > 0) lv = s[p - np];
  else lv = b.top ? pole : b.hs_up[j];
  if (l < b.nrow - 1) uv = s[p + np];
  else uv = b.bottom ? 0.0 : b.hs_dn[j];
  return S.coef[ci] * c + S.coef[n + ci] * lv + S.coef[2 * n + ci] * uv +
         S.coef[3 * n + ci] * sm + S.coef[4 * n + ci] * sp;
}

// Sets s[p] of an owned point and pushes it to the neighbour whose halo
// row holds it.
__device__ __forceinline__ void set_s(double *s, const Band &b, int l, int j, int p,
                                      double v) {
  s[p] = v;
  if (l == 0 && !b.top) b.peer_up_hs[j] = v;
  if (l == b.nrow - 1 && !b.bottom) b.peer_dn_hs[j] = v;
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
  // a gated solve that is not due: every CTA of the cluster leaves here,
  // before any cluster barrier
  if (S.gate != nullptr && *S.gate == 0) return;
  const int np = S.np, R = S.nt - 2;
  const int t = threadIdx.x;

  extern __shared__ __align__(16) double dyn[];
  __shared__ double wbuf[32 * kSlotWidth];
  __shared__ double slots[kSlots * kMaxCluster * kSlotWidth];
  __shared__ double pole_s;

  Band b;
  b.ra = (int)((long long)rank * R / csize);
  const int rb = (int)((long long)(rank + 1) * R / csize);
  b.nrow = rb - b.ra;
  b.top = rank == 0;
  b.bottom = rank == csize - 1;
  const int P = b.nrow * np;
  const size_t stride = (size_t)((R + csize - 1) / csize) * np;
  double *s = dyn;               // search direction
  double *xs = dyn + stride;     // solution
  double *rs = dyn + 2 * stride; // residual
  double *as = dyn + 3 * stride; // A s
  b.hs_up = dyn + 4 * stride;
  b.hz_up = b.hs_up + np;
  b.hs_dn = b.hz_up + np;
  b.hz_dn = b.hs_dn + np;
  Row *rt = reinterpret_cast<Row *>(b.hz_dn + np);
  b.peer_up_hs = b.top ? nullptr : cl.map_shared_rank(b.hs_dn, rank - 1);
  b.peer_up_hz = b.top ? nullptr : cl.map_shared_rank(b.hz_dn, rank - 1);
  b.peer_dn_hs = b.bottom ? nullptr : cl.map_shared_rank(b.hs_up, rank + 1);
  b.peer_dn_hz = b.bottom ? nullptr : cl.map_shared_rank(b.hz_up, rank + 1);
  for (int l = t; l < b.nrow; l += kThreads) rt[l] = S.rows[b.ra + l];
  const bool lead = b.top;
  const double dnp = (double)np;
  const double ps = dnp * S.pe;  // pole diagonal and pole residual scale
  const bool var = S.coef != nullptr;
  const double pd = var ? S.diag0 : ps;  // pole diagonal of the Jacobi step
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
    set_s(s, b, l, j, p, xv);
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
      const double rhs = rw.w * u + (var ? 0.0 : rw.extra);
      const long long ci = 1 + (long long)(b.ra + l) * np + j;
      const double ax = var ? apply_var(s, b, S, np, l, j, p, pole, ci)
                            : apply_row(s, b, rw, np, l, j, p, pole);
      const double r = rhs - ax;
      rs[p] = r;
      const double q = r * rw.rw;
      v[0] += q * q;
      v[1] += u * u;
      v[2] += isfinite(f) ? 0.0 : 1.0;
      if (b.ra + l == 0) v[3] += var ? S.pedge[j] * s[p] : s[p];
    }
    block_sum<4>(v, wbuf);
    if (lead) {
      const double ax0 = var ? S.diag0 * pole - v[3] : S.pe * (dnp * pole - v[3]);
      r0 = 0.0 - ax0;
      const double pr = r0 / ps;
      v[0] += dnp * pr * pr;
      if (!var) v[1] += dnp * S.low * S.low;
    }
    out[0] = v[0];
    out[1] = v[1];
    out[2] = v[2];
    cluster_sum<3>(cl, out, slots, ctr, rank, csize);
  };

  // z = M^-1 r, s = z, rho = r . z
  auto restart = [&]() -> double {
    double v[1] = {0.0};
    GCS_MI_FOR_POINTS(W, P, np) {
      const double r = rs[p];
      const double z = var ? r / S.coef[1 + (long long)(b.ra + l) * np + j]
                           : r * rt[l].rdg;
      set_s(s, b, l, j, p, z);
      v[0] += r * z;
    }
    block_sum<1>(v, wbuf);
    if (lead) {
      const double z0 = r0 / pd;
      v[0] += r0 * z0;
      if (t == 0) pole_s = z0;
    }
    cluster_sum<1>(cl, v, slots, ctr, rank, csize);
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
        const double a = var ? apply_var(s, b, S, np, l, j, p, pole,
                                         1 + (long long)(b.ra + l) * np + j)
                             : apply_row(s, b, rt[l], np, l, j, p, pole);
        as[p] = a;
        v[0] += s[p] * a;
        if (b.ra + l == 0) v[1] += var ? S.pedge[j] * s[p] : s[p];
      }
      block_sum<2>(v, wbuf);
      double As0 = 0.0;
      double den[1] = {v[0]};
      if (lead) {
        As0 = var ? S.diag0 * pole - v[1] : S.pe * (dnp * pole - v[1]);
        den[0] += pole * As0;
      }
      cluster_sum<1>(cl, den, slots, ctr, rank, csize);
      if (!isfinite(den[0]) || den[0] <= DBL_MIN) break;
      const double alpha = rho / den[0];
      // x += alpha s, r -= alpha A s; residual norm and r . M^-1 r.  The
      // band's edge rows of z go to the neighbours, which then advance
      // their halo copies of s themselves.
      double w2[2] = {0.0, 0.0};
      GCS_MI_FOR_POINTS(W, P, np) {
        const Row &rw = rt[l];
        xs[p] += alpha * s[p];
        const double r = rs[p] - alpha * as[p];
        rs[p] = r;
        const double q = r * rw.rw;
        const double z = var ? r / S.coef[1 + (long long)(b.ra + l) * np + j] : r * rw.rdg;
        w2[0] += q * q;
        w2[1] += r * z;
        if (l == 0 && !b.top) b.peer_up_hz[j] = z;
        if (l == b.nrow - 1 && !b.bottom) b.peer_dn_hz[j] = z;
      }
      block_sum<2>(w2, wbuf);
      if (lead) {
        x0 += alpha * pole;
        r0 -= alpha * As0;
        const double pr = r0 / ps;
        w2[0] += dnp * pr * pr;
        w2[1] += r0 * (r0 / pd);
      }
      cluster_sum<2>(cl, w2, slots, ctr, rank, csize);
      final_res = sqrt(fmax(0.0, w2[0]));
      iters = it;
      if (final_res <= target || it % kTruePeriod == 0) {
        // Verify with the true residual (nonorthogonal_mi.c:562-582).
        GCS_MI_FOR_POINTS(W, P, np) { set_s(s, b, l, j, p, xs[p]); }
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
      if (var) {
        GCS_MI_FOR_POINTS(W, P, np) {
          s[p] = rs[p] / S.coef[1 + (long long)(b.ra + l) * np + j] + beta * s[p];
        }
      } else {
        GCS_MI_FOR_POINTS(W, P, np) { s[p] = rs[p] * rt[l].rdg + beta * s[p]; }
      }
      for (int j = t; j < np; j += kThreads) {
        if (!b.top) b.hs_up[j] = b.hz_up[j] + beta * b.hs_up[j];
        if (!b.bottom) b.hs_dn[j] = b.hz_dn[j] + beta * b.hs_dn[j];
      }
      if (lead && t == 0) pole_s = r0 / pd + beta * pole;
      rho = rho_new;
      __syncthreads();
    }
  }

  if (bad) {
    if (lead && t == 0) *S.status = 2;
    cl.sync();  // no CTA leaves while a peer may still write its memory
    return;
  }
  // Expand the reduced solution (nonorthogonal_mi.c:595-605).
  GCS_MI_FOR_POINTS(W, P, np) { S.pot[(size_t)(b.ra + l + 1) * np + j] = xs[p]; }
  if (lead)
    for (int j = t; j < np; j += kThreads) S.pot[j] = x0;
  if (b.bottom)
    for (int j = t; j < np; j += kThreads) S.pot[(size_t)(S.nt - 1) * np + j] = S.low;
  if (lead && t == 0) {
    *S.stats = gamera_mi_solver_stats{iters, initial, final_res, conv};
    *S.status = conv ? 0 : 1;
  }
  cl.sync();  // no CTA leaves while a peer may still write its memory
}

// ------------------------------------------------------- column kernel
// The same solve with one thread per longitude column of the band: thread
// j keeps the band's column of s, x, r and A s in registers (MR rows at
// most), takes the vertical stencil neighbours from its own registers and
// only the longitude neighbours from shared memory.  Used when the grid fits
// (np <= col_threads(MR), band rows <= MR); k_pcg serves the rest.

__host__ __device__ constexpr int col_threads(int mr) {
  return mr <= 4 ? 512 : (mr <= 12 ? 384 : 256);
}

template <int MR>
__global__ void __launch_bounds__(col_threads(MR), 1)
    k_pcg_col(const System *systems, int csize) {
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const System &S = systems[blockIdx.x / csize];
  if (S.gate != nullptr && *S.gate == 0) return;
  const int np = S.np, R = S.nt - 2;
  const int j = threadIdx.x;
  const bool on = j < np;
  const int jm = j == 0 ? np - 1 : j - 1;
  const int jp = j + 1 >= np ? 0 : j + 1;

  extern __shared__ __align__(16) double dyn[];
  __shared__ double wbuf[32 * kSlotWidth];
  __shared__ double slots[kSlots * kMaxCluster * kSlotWidth];
  __shared__ double pole_s;

  // halo rows: [0] s above, [np] z above, [2np] s below, [3np] z below
  const int ra = (int)((long long)rank * R / csize);
  const int nrow = (int)((long long)(rank + 1) * R / csize) - ra;
  const bool top = rank == 0, bottom = rank == csize - 1;
  double *ssm = dyn;                    // MR rows of s
  double *halo = dyn + (size_t)MR * np;
  Row *rt = reinterpret_cast<Row *>(halo + 4 * (size_t)np);
  // the neighbours' halo rows that this band's edge rows feed
  double *peer_up = top ? nullptr : cl.map_shared_rank(halo, rank - 1) + 2 * np + j;
  double *peer_dn = bottom ? nullptr : cl.map_shared_rank(halo, rank + 1) + j;
  for (int l = j; l < nrow; l += blockDim.x) rt[l] = S.rows[ra + l];
  const bool lead = top;
  const double dnp = (double)np;
  const double ps = dnp * S.pe;
  int ctr = 0;

  double sv[MR], xv[MR], rv[MR], av[MR];

  // s of row l := v, in registers, shared memory and the neighbours' halos
  auto put_s = [&](int l, double v) {
    sv[l] = v;
    ssm[l * np + j] = v;
    if (l == 0 && !top) peer_up[0] = v;
    if (l == nrow - 1 && !bottom) peer_dn[0] = v;
  };
  // A s of row l from the registers of the column (nonorthogonal_mi.c:394-409)
  auto stencil = [&](int l, const Row &rw, double pole) {
    const double c = sv[l];
    const double sm = ssm[l * np + jm];
    const double sp = ssm[l * np + jp];
    const double lv = l > 0 ? sv[l > 0 ? l - 1 : 0] : (top ? pole : halo[j]);
    const double uv = l < nrow - 1 ? sv[l + 1 < MR ? l + 1 : MR - 1]
                                   : (bottom ? 0.0 : halo[2 * np + j]);
    return rw.w * (rw.lo * (c - lv) + rw.up * (c - uv) +
                   rw.lon * (2.0 * c - sm - sp));
  };

  double x0 = 0.0, r0 = 0.0;
  if (lead) {
    double pm[1] = {0.0};
    for (int q = j; q < np; q += blockDim.x) {
      const double v = S.pot[q];
      if (isfinite(v)) pm[0] += v / dnp;
    }
    block_sum<1>(pm, wbuf);
    x0 = pm[0];
  }
#pragma unroll
  for (int l = 0; l < MR; ++l) {
    xv[l] = 0.0;
    rv[l] = 0.0;
    av[l] = 0.0;
    sv[l] = 0.0;
    if (l < nrow && on) {
      const double v = S.pot[(size_t)(ra + l + 1) * np + j];
      xv[l] = isfinite(v) ? v : 0.0;
      put_s(l, xv[l]);
    }
  }
  if (lead && j == 0) pole_s = x0;
  cl.sync();

  auto true_residual = [&](double (&out)[3]) {
    double v[4] = {0.0, 0.0, 0.0, 0.0};  // norm^2, rhs^2, bad, ring
    const double pole = lead ? pole_s : 0.0;
#pragma unroll
    for (int l = 0; l < MR; ++l) {
      if (l < nrow && on) {
        const Row rw = rt[l];
        const double f = S.fac[(size_t)(ra + l + 1) * np + j];
        const double u = S.neg_r2 * f * rw.inc;
        const double rhs = rw.w * u + rw.extra;
        rv[l] = rhs - stencil(l, rw, pole);
        const double q = rv[l] * rw.rw;
        v[0] += q * q;
        v[1] += u * u;
        v[2] += isfinite(f) ? 0.0 : 1.0;
        if (l == 0 && top) v[3] += sv[0];
      }
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
    cluster_sum<3>(cl, out, slots, ctr, rank, csize);
  };

  auto restart = [&]() -> double {
    double v[1] = {0.0};
#pragma unroll
    for (int l = 0; l < MR; ++l) {
      if (l < nrow && on) {
        const double z = rv[l] * rt[l].rdg;
        put_s(l, z);
        v[0] += rv[l] * z;
      }
    }
    block_sum<1>(v, wbuf);
    if (lead) {
      const double z0 = r0 / ps;
      v[0] += r0 * z0;
      if (j == 0) pole_s = z0;
    }
    cluster_sum<1>(cl, v, slots, ctr, rank, csize);
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
      double v[2] = {0.0, 0.0};  // s.As, first-ring sum of s
      const double pole = lead ? pole_s : 0.0;
#pragma unroll
      for (int l = 0; l < MR; ++l) {
        if (l < nrow && on) {
          av[l] = stencil(l, rt[l], pole);
          v[0] += sv[l] * av[l];
          if (l == 0 && top) v[1] += sv[0];
        }
      }
      block_sum<2>(v, wbuf);
      double As0 = 0.0;
      double den[1] = {v[0]};
      if (lead) {
        As0 = S.pe * (dnp * pole - v[1]);
        den[0] += pole * As0;
      }
      cluster_sum<1>(cl, den, slots, ctr, rank, csize);
      if (!isfinite(den[0]) || den[0] <= DBL_MIN) break;
      const double alpha = rho / den[0];
      double w2[2] = {0.0, 0.0};
#pragma unroll
      for (int l = 0; l < MR; ++l) {
        if (l < nrow && on) {
          const Row &rw = rt[l];
          xv[l] += alpha * sv[l];
          rv[l] -= alpha * av[l];
          const double q = rv[l] * rw.rw;
          const double z = rv[l] * rw.rdg;
          w2[0] += q * q;
          w2[1] += rv[l] * z;
          if (l == 0 && !top) peer_up[np] = z;
          if (l == nrow - 1 && !bottom) peer_dn[np] = z;
        }
      }
      block_sum<2>(w2, wbuf);
      if (lead) {
        x0 += alpha * pole;
        r0 -= alpha * As0;
        const double pr = r0 / ps;
        w2[0] += dnp * pr * pr;
        w2[1] += r0 * (r0 / ps);
      }
      cluster_sum<2>(cl, w2, slots, ctr, rank, csize);
      final_res = sqrt(fmax(0.0, w2[0]));
      iters = it;
      if (final_res <= target || it % kTruePeriod == 0) {
#pragma unroll
        for (int l = 0; l < MR; ++l)
          if (l < nrow && on) put_s(l, xv[l]);
        if (lead && j == 0) pole_s = x0;
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
#pragma unroll
      for (int l = 0; l < MR; ++l) {
        if (l < nrow && on) {
          sv[l] = rv[l] * rt[l].rdg + beta * sv[l];
          ssm[l * np + j] = sv[l];
        }
      }
      if (on) {
        if (!top) halo[j] = halo[np + j] + beta * halo[j];
        if (!bottom) halo[2 * np + j] = halo[3 * np + j] + beta * halo[2 * np + j];
      }
      if (lead && j == 0) pole_s = r0 / ps + beta * pole;
      rho = rho_new;
      __syncthreads();
    }
  }

  if (bad) {
    if (lead && j == 0) *S.status = 2;
    cl.sync();  // no CTA leaves while a peer may still write its memory
    return;
  }
#pragma unroll
  for (int l = 0; l < MR; ++l)
    if (l < nrow && on) S.pot[(size_t)(ra + l + 1) * np + j] = xv[l];
  if (lead)
    for (int q = j; q < np; q += blockDim.x) S.pot[q] = x0;
  if (bottom)
    for (int q = j; q < np; q += blockDim.x) S.pot[(size_t)(S.nt - 1) * np + q] = S.low;
  if (lead && j == 0) {
    *S.stats = gamera_mi_solver_stats{iters, initial, final_res, conv};
    *S.status = conv ? 0 : 1;
  }
  cl.sync();  // no CTA leaves while a peer may still write its memory
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

using PcgKernel = void (*)(const System *, int);

// One launch shape of the solve: kernel, cluster size, threads per CTA and
// dynamic shared memory.
struct Shape {
  PcgKernel kernel = nullptr;
  int csize = 0, threads = 0, rows = 0;
  size_t smem = 0;
};

// Dynamic shared memory of any launch shape (launchable rejects more).
constexpr size_t kShapeSmemCap = 200 * 1024;

// The kernel's shared-memory limit is set to the cap, not to this shape's
// need, so configuring a shape for a small grid never lowers it under a
// shape chosen earlier for a larger one.
cudaError_t configure(const Shape &sh) {
  cudaError_t e = cudaFuncSetAttribute(sh.kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kShapeSmemCap);
  if (e != cudaSuccess) return e;
  if (sh.csize > kPortableCluster)
    e = cudaFuncSetAttribute(sh.kernel, cudaFuncAttributeNonPortableClusterSizeAllowed,
                             1);
  return e;
}

cudaLaunchConfig_t launch_config(const Shape &sh, int count, cudaStream_t stream,
                                 cudaLaunchAttribute *attr) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(sh.csize * count));
  cfg.blockDim = dim3((unsigned)sh.threads);
  cfg.dynamicSmemBytes = sh.smem;
  cfg.stream = stream;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)sh.csize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

bool launchable(const Shape &sh) {
  if (sh.smem > kShapeSmemCap || configure(sh) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = launch_config(sh, 1, nullptr, attr);
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, sh.kernel, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return n >= 1;
}

// Column kernel: MR rows of s plus four halo rows, and the row table.
size_t col_smem(int mr, int np) {
  return ((size_t)mr * np + 4 * (size_t)np) * sizeof(double) + (size_t)mr * sizeof(Row);
}

PcgKernel col_kernel(int mr) {
  switch (mr) {
    case 4: return k_pcg_col<4>;
    case 8: return k_pcg_col<8>;
    case 12: return k_pcg_col<12>;
    case 16: return k_pcg_col<16>;
    default: return nullptr;
  }
}

// Shared memory of a band of `rows` rows: four vectors, four halo rows and
// the row table.
size_t band_smem(int rows, int np) {
  return (4 * (size_t)rows * np + 4 * (size_t)np) * sizeof(double) +
         (size_t)rows * sizeof(Row);
}

constexpr size_t kMaxSmem = kShapeSmemCap;

}  // namespace mi
}  // namespace gcs

using namespace gcs::mi;

struct gcs_mi_plan {
  int count = 0;
  int np = 0, nt = 0;
  Shape shape;
  std::vector<gamera_mi_solver_config> configs;
  Row *d_rows = nullptr;          // count * (nt - 2)
  System *d_sys = nullptr;        // count
  double *d_fac = nullptr;        // count * nt * np
  double *d_pot = nullptr;        // count * nt * np
  gamera_mi_solver_stats *d_stats = nullptr;
  int *d_status = nullptr;
  double *d_coef = nullptr;       // variable Pedersen: count * (5 unknowns + np)
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
  cudaFree(p->d_coef);
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
// Launch shape: the column kernel with the smallest band (most CTAs, at
// most 16) whose rows fit its registers; otherwise the shared-memory kernel
// with about 2048 unknowns per CTA (8 CTAs at most where the device cannot
// co-schedule 16).
int choose_shape(gcs_mi_plan *p, bool variable = false) {
  const int R = p->nt - 2, np = p->np;
  const int threads = (np + 31) / 32 * 32;
  // the variable-conductance mode lives in the shared-memory kernel
  for (int mr : {4, 8, 12, 16}) {
    if (variable) break;
    Shape sh;
    sh.kernel = col_kernel(mr);
    sh.csize = (R + mr - 1) / mr;
    sh.threads = threads;
    sh.rows = mr;
    sh.smem = col_smem(mr, np);
    if (threads > col_threads(mr) || sh.csize > kMaxCluster) continue;
    if (launchable(sh)) {
      p->shape = sh;
      return 0;
    }
  }
  const long long points = (long long)np * R;
  int want = (int)((points + 2047) / 2048);
  if (want < 1) want = 1;
  for (int limit : {kMaxCluster, kPortableCluster}) {
    const int top = limit < R ? limit : R;
    int csize = want < top ? want : top;
    for (; csize <= top; ++csize)
      if (band_smem((R + csize - 1) / csize, np) <= kMaxSmem) break;
    if (csize > top) continue;
    Shape sh;
    sh.kernel = k_pcg;
    sh.csize = csize;
    sh.threads = kThreads;
    sh.rows = (R + csize - 1) / csize;
    sh.smem = band_smem(sh.rows, np);
    if (launchable(sh)) {
      p->shape = sh;
      return 0;
    }
  }
  set_api_error("MI grid too large for the on-chip cluster solve");
  return -1;
}

// The five-point stencil of the conductance-tensor operator with Hall = 0
// (nonorthogonal_mi.c:744-865, same operations): per reduced unknown the
// diagonal, lower, upper, longitude-lower and longitude-upper coefficients
// (`unknowns` entries each), then the np pole edge coefficients; returns the
// pole diagonal.
double build_pedersen_stencil(const gamera_mi_solver_config *c, const double *ped,
                              double *coef) {
  const size_t np = c->longitude_count, nt = c->colatitude_count;
  const size_t n = 1U + np * (nt - 2U);
  const double dth = c->maximum_colatitude / (double)(nt - 1U);
  const double dph = 2.0 * acos(-1.0) / (double)np;
  auto incsq = [](double th) {
    const double co = cos(th);
    return 4.0 * co * co / (1.0 + 3.0 * co * co);
  };
  auto P = [&](size_t i, size_t j) { return ped[i * np + j]; };
  double *pedge = coef + 5 * n;
  double mean = 0.0;
  for (size_t j = 0; j < np; ++j) mean += P(0, j) / (double)np;
  const double half = 0.5 * dth;
  double diag0 = 0.0;
  for (size_t j = 0; j < np; ++j) {
    const double face = 0.5 * (mean + P(1, j));
    pedge[j] = sin(half) * face / (incsq(half) * dth * dth);
    diag0 += pedge[j];
  }
  coef[0] = diag0;
  for (int q = 1; q < 5; ++q) coef[q * n] = 0.0;
  for (size_t i = 1; i + 1 < nt; ++i) {
    const double th = (double)i * dth, sine = sin(th);
    const double lth = th - 0.5 * dth, uth = th + 0.5 * dth;
    for (size_t j = 0; j < np; ++j) {
      const size_t jm = j == 0 ? np - 1 : j - 1, jp = j + 1 == np ? 0 : j + 1;
      const double lower = sin(lth) * 0.5 * (P(i, j) + P(i - 1, j)) / (incsq(lth) * dth * dth);
      const double upper = sin(uth) * 0.5 * (P(i, j) + P(i + 1, j)) / (incsq(uth) * dth * dth);
      const double ll = 0.5 * (P(i, j) + P(i, jm)) / (sine * dph * dph);
      const double lu = 0.5 * (P(i, j) + P(i, jp)) / (sine * dph * dph);
      const size_t ci = 1 + (i - 1) * np + j;
      coef[ci] = lower + upper + ll + lu;
      coef[n + ci] = -lower;
      coef[2 * n + ci] = -upper;
      coef[3 * n + ci] = -ll;
      coef[4 * n + ci] = -lu;
    }
  }
  return diag0;
}

gcs_mi_plan *plan_create(const gamera_mi_solver_config *configs, int count,
                         const double *pedersen = nullptr) {
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
  if (choose_shape(p, pedersen != nullptr) != 0) {
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
    S.gate = nullptr;
    S.coef = nullptr;
    S.pedge = nullptr;
    S.diag0 = 0.0;
    S.unknowns = (long long)(1 + (size_t)p->np * R);
    if (pedersen) {
      // variable Pedersen conductance of system s (nt * np per system)
      const size_t n = 1 + (size_t)p->np * R, per = 5 * n + p->np;
      if (!p->d_coef &&
          !cuda_ok(cudaMalloc(&p->d_coef, count * per * sizeof(double)), "cudaMalloc")) {
        plan_free(p);
        return nullptr;
      }
      std::vector<double> coef(per);
      S.diag0 = build_pedersen_stencil(c, pedersen + s * nodes, coef.data());
      if (!cuda_ok(cudaMemcpy(p->d_coef + s * per, coef.data(), per * sizeof(double),
                              cudaMemcpyHostToDevice), "cudaMemcpy")) {
        plan_free(p);
        return nullptr;
      }
      S.coef = p->d_coef + s * per;
      S.pedge = S.coef + 5 * n;
    }
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
  cudaLaunchConfig_t cfg = launch_config(p->shape, p->count, stream, attr);
  const cudaError_t e = cudaLaunchKernelEx(&cfg, p->shape.kernel,
                                           (const System *)p->d_sys, p->shape.csize);
  p->stream = stream;
  return cuda_ok(e, "MI solve launch") ? 0 : -1;
}

std::mutex g_cache_mutex;
gcs_mi_plan *g_cache = nullptr;  // plan of the last drop-in call

}  // namespace

namespace gcs {

// A plan whose solves run only where *gate != 0 (a coupling update gated by
// its device-side cadence), bound to fixed FAC and potential arrays.  Both
// are set outside any stream capture; the plan's later launches on the same
// arrays need no host synchronisation.
int mi_plan_gate(gcs_mi_plan *p, const int *gate, const double *fac, double *pot) {
  if (!p) return -1;
  for (int q = 0; q < p->count; ++q) p->host_sys[q].gate = gate;
  for (int q = 0; q < p->count; ++q) {
    p->host_sys[q].fac = fac + q * (size_t)p->np * p->nt;
    p->host_sys[q].pot = pot + q * (size_t)p->np * p->nt;
  }
  return cuda_ok(cudaMemcpy(p->d_sys, p->host_sys.data(), p->count * sizeof(System),
                            cudaMemcpyHostToDevice),
                 "cudaMemcpy")
             ? 0
             : -1;
}

// Device status words of a plan's solves (0 converged, 1 not converged,
// 2 non-finite FAC) and its launch.
const int *mi_plan_status(const gcs_mi_plan *p) { return p ? p->d_status : nullptr; }
int mi_plan_launch(gcs_mi_plan *p, cudaStream_t stream) { return plan_launch(p, stream); }

}  // namespace gcs

namespace {

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
  if (cluster_ctas) *cluster_ctas = plan->shape.csize;
  if (threads_per_cta) *threads_per_cta = plan->shape.threads;
  if (shared_bytes) *shared_bytes = plan->shape.smem;
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
int gcs_mi_plan_create_pedersen(const gamera_mi_solver_config *configs,
                                const double *pedersen, int count, gcs_mi_plan **plan) {
  if (!configs || !pedersen || !plan || count < 1) {
    set_api_error("null argument");
    return -1;
  }
  *plan = nullptr;
  for (int s = 0; s < count; ++s)
    if (!valid_config(&configs[s])) {
      set_api_error("invalid MI solver configuration");
      return -1;
    }
  const size_t nodes = configs[0].longitude_count * configs[0].colatitude_count;
  for (size_t q = 0; q < (size_t)count * nodes; ++q)
    if (!std::isfinite(pedersen[q]) || pedersen[q] <= 0.0) {
      set_api_error("Pedersen conductance must be finite and positive");
      return -1;
    }
  *plan = plan_create(configs, count, pedersen);
  return *plan ? 0 : -1;
}

int gcs_mi_solve_pedersen_pcg(const gamera_mi_solver_config *config, const double *fac_a_m2,
                              const double *pedersen, double *potential_v,
                              gamera_mi_solver_stats *stats) {
  if (!valid_config(config) || fac_a_m2 == nullptr || pedersen == nullptr ||
      potential_v == nullptr) {
    set_api_error("invalid MI solver arguments");
    return -1;
  }
  gcs_mi_plan *p = nullptr;
  if (gcs_mi_plan_create_pedersen(config, pedersen, 1, &p) != 0) return -1;
  const size_t bytes = config->longitude_count * config->colatitude_count * sizeof(double);
  cudaStream_t st = nullptr;
  int status = 2;
  gamera_mi_solver_stats s = {};
  const bool ok =
      cuda_ok(cudaMemcpyAsync(p->d_fac, fac_a_m2, bytes, cudaMemcpyHostToDevice, st),
              "cudaMemcpyAsync") &&
      cuda_ok(cudaMemcpyAsync(p->d_pot, potential_v, bytes, cudaMemcpyHostToDevice, st),
              "cudaMemcpyAsync") &&
      plan_launch(p, st) == 0 &&
      cuda_ok(cudaMemcpyAsync(potential_v, p->d_pot, bytes, cudaMemcpyDeviceToHost, st),
              "cudaMemcpyAsync") &&
      cuda_ok(cudaMemcpyAsync(&s, p->d_stats, sizeof(s), cudaMemcpyDeviceToHost, st),
              "cudaMemcpyAsync") &&
      cuda_ok(cudaMemcpyAsync(&status, p->d_status, sizeof(int), cudaMemcpyDeviceToHost,
                              st),
              "cudaMemcpyAsync") &&
      cuda_ok(cudaStreamSynchronize(st), "MI solve");
  plan_free(p);
  if (!ok) return -1;
  if (status == 2) {
    set_api_error("non-finite field-aligned current");
    return -1;
  }
  if (stats) *stats = s;
  return status == 0 ? 0 : -1;
}

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
