// Ionosphere potential with the variable Pedersen + Hall conductance tensor
// (nonorthogonal/src/nonorthogonal/nonorthogonal_mi.c:611-1151): the cached
// five-point stencil, BiCGStab with restarts every 256 iterations, and the
// symmetric Gauss-Seidel (SSOR) preconditioner, solved by one thread-block
// cluster that keeps every vector in L2.
//
// Layout.  The interior unknowns (rows r = 0..R-1 for colatitude rows
// 1..nt-2, longitudes j = 0..np-1) are stored skewed by anti-diagonal: the
// points with r + j = d form one column of Rp doubles (Rp = 32 M >= R rows),
// column F + d, row r at position (r mod M) 32 + r / M of the column.  The
// pole unknown sits at index 0.  Padding rows, off-grid positions of a
// diagonal and the F padding columns hold zeros and stay zero through every
// operation.
//
// SSOR.  The lexicographic forward sweep and the reverse sweep are
// wavefronts along anti-diagonals: point (r, j) depends on (r-1, j),
// (r, j-1) and on the periodic seam (r, 0).  One warp runs a sweep, lane l
// holding rows l M .. l M + M - 1 as M independent chains, so one step
// advances the whole anti-diagonal.  Whole diagonals move between global
// and shared memory by bulk asynchronous copies (tracked by mbarriers,
// every wait bounded), several diagonals per copy.  The preconditioner is
// the reference's (D + L) D^-1 (D + U) with the triangular solves done on
// D^-1-scaled rows, so it equals the reference's to rounding.
//
// Band schedule (the default on grids narrower than 17 longitudes): the
// same sweeps with the rows split into one band per CTA, each band swept by
// its CTA's warp 0 from shared-memory tables and its edge row passed to the
// next CTA through distributed shared memory (band_sweep); identical
// results.
//
// Vector updates, stencil applications and dot products run on all CTAs
// of the cluster (dot products summed in a fixed order, identical on every
// CTA); the sweeps run on one warp of CTA 0 between two cluster barriers.
// The BiCGStab iterates therefore differ from the CPU solver's at rounding
// level, and a converged solve meets the same residual target.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <mutex>
#include <vector>

#include "gamera_cs_b200.h"
#include "gcs_error.h"

namespace cg = cooperative_groups;
using gcs::set_api_error;

namespace {

// The sweep warp holds 32 M interior colatitude rows (rows padded to
// Rp = 32 M): M = 1..8 (up to 256 rows) or 16 (up to 512 rows).  It moves
// diagonals in groups of 12 (a 36-diagonal prefetch ring) where the seam
// allows (at least 25 longitudes) and shared memory fits (up to 6 chains),
// else in groups of 8 (24 diagonals; at least 17 longitudes), of 4 (16
// diagonals; 8 for M = 16), or of 1 for grids of fewer than 9 longitudes:
// every group pays a fixed synchronisation cost in the sweep warp, so
// larger groups are faster.
constexpr int kThreads = 256;
constexpr int kMaxRows = 512;
constexpr int kPad = 16;                    // padding diagonals on each side (>= group - 1)
constexpr unsigned kSpinLimit = 1u << 20;   // polls of a sweep copy's mbarrier
constexpr unsigned kDrainLimit = 1u << 16;  // polls per copy after an abort
constexpr int kMaxCluster = 16;
constexpr int kSlots = 4;
constexpr int kSlotWidth = 4;
constexpr int kRestart = 256;
constexpr int kMaxIterations = 1 << 20;
constexpr int kMaxLongitudes = 8192;        // pole-edge table in shared memory
constexpr size_t kSmemCap = 220 * 1024;     // dynamic shared memory of a launch

// Per-row constants of the full polar grid, computed on the host with the
// reference's formulas (nonorthogonal_mi.c:643-656, :776-865).
struct TRow {
  double s;        // sin(theta)
  double sl, il;   // sin and inclination^2 at theta - dtheta/2
  double su, iu;   // sin and inclination^2 at theta + dtheta/2
  double inc;      // dipole cos(inclination)
};

struct TSys {
  int np, nt, R, Rp, max_iter;
  unsigned core0, core1;  // skewed index range of the grid's diagonals
  double dth, dph, neg_r2, pole_sin, pole_inc2, ps, abs_tol, rel_tol;
  const TRow *rows;             // max(nt, Rp + 2) rows; padding rows have s = 1
  const double *fac, *sp, *sh;  // natural layout (nt x np)
  double *pot;                  // natural layout, initial guess in, solution out
  // skewed vectors
  double *rhs, *x, *res, *shd, *srch, *as, *psv, *mid, *pm, *am, *fw, *pin;
  // skewed stencil: raw coefficients and the D^-1-scaled sweep pairs
  double *dg, *lo, *up, *ll, *lu, *rdg;
  double2 *cf;  // (lo, ll) / dg: forward sweep
  double2 *cb;  // (up, lu) / dg: reverse sweep
  double *pe;   // pole edge coefficients (np)
  double *pole_sum;
  int *fault;   // set when a sweep copy never arrived
  gamera_mi_solver_stats *stats;
  int *status;  // 0 converged, 1 not converged, 2 non-finite FAC, 3 sweep copy lost
  int colored;  // 1: multicolour SSOR by the whole cluster instead of the wavefront
  int band;     // rows per band of the band-pipelined sweeps (0: one sweep warp)
  int nbands;   // bands (CTAs 0 .. nbands - 1 sweep)
};

// Position of row r inside a diagonal of Rp = 32 M rows: the sweep warp's
// lane r / M holds it as chain r % M, at position (r % M) 32 + r / M.
__device__ __forceinline__ int row_pos(int Rp, int r) {
  const int M = Rp >> 5;
  return (r % M) * 32 + r / M;
}
__device__ __forceinline__ int pos_row(int Rp, int q) {
  const int M = Rp >> 5;
  return (q & 31) * M + (q >> 5);
}

// Skewed index of row r, longitude j.
__device__ __forceinline__ size_t sidx(int Rp, int r, int j) {
  return (size_t)(kPad + r + j) * Rp + row_pos(Rp, r);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum of N values over the cluster; every thread of every CTA receives the
// bit-identical result.  Warp butterflies and a butterfly over the warp
// partials give the CTA sum; thread c pushes it into CTA c's slot table
// (a distributed-shared-memory store); after the cluster barrier -- which
// also publishes every earlier global and shared write of the cluster --
// a butterfly over the slots in rank order gives the cluster sum.
template <int NW>
struct Reducer {
  double *wbuf, *slots;
  int ctr, rank, csize;

  template <int N>
  __device__ __forceinline__ void sum(cg::cluster_group &cl, double (&v)[N]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < N; ++q) {
      v[q] = warp_sum(v[q]);
      if (lane == 0) wbuf[warp * kSlotWidth + q] = v[q];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < N; ++q) v[q] = warp_sum(lane < NW ? wbuf[lane * kSlotWidth + q] : 0.0);
    const int slot = ctr & (kSlots - 1);
    ++ctr;
    if ((int)threadIdx.x < csize) {
      double *dst = cl.map_shared_rank(slots, (int)threadIdx.x) +
                    (slot * kMaxCluster + rank) * kSlotWidth;
#pragma unroll
      for (int q = 0; q < N; ++q) dst[q] = v[q];
    }
    cl.sync();
    const double *src = slots + slot * kMaxCluster * kSlotWidth;
#pragma unroll
    for (int q = 0; q < N; ++q) v[q] = warp_sum(lane < csize ? src[lane * kSlotWidth + q] : 0.0);
  }
};

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

// Shared memory of the sweep warp.  Ring: kRG slots of G anti-diagonals
// (G Rp values and G Rp coefficient pairs each) filled by two bulk
// asynchronous copies per group, one mbarrier per slot; group n of the
// warp's running group count uses slot n mod kRG and completes phase
// n / kRG of its barrier.  Stage: two halves of G output diagonals,
// drained to global memory by one bulk copy per group.  edge: each row's
// value at the first longitude of the sweep (captured on the way); seam_f
// and seam_r: the seam coefficients of both directions.
template <int kRG, int G>
struct SweepMem {
  double *val;      // [kRG][G][Rp]
  double2 *cof;     // [kRG][G][Rp]
  double *stage;    // [2][G][Rp]
  double *edge;     // [Rp] by row
  double *seam_f;   // [Rp] by row: lu/dg at longitude np-1
  double *seam_r;   // [Rp] by row: ll/dg at longitude 0
  uint64_t *bar;    // [kRG]
  int Rp;

  // lane 0: fetch diagonals d0 .. d0 + G - 1 of (va, vb) into the slot of group n
  __device__ __forceinline__ void issue(unsigned n, const double *va, const double2 *vb,
                                        size_t d0) const {
    const unsigned slot = n % kRG;
    const unsigned bv = (unsigned)(G * Rp) * 8u, bc = (unsigned)(G * Rp) * 16u;
    const unsigned b = smem_u32(bar + slot);
    // relaxed: the copies carry the data, the arrival orders nothing else
    asm volatile("mbarrier.arrive.expect_tx.relaxed.cta.shared::cta.b64 _, [%0], %1;" ::"r"(b),
                 "r"(bv + bc)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
        "[%3];" ::"r"(smem_u32(val + (size_t)slot * G * Rp)),
        "l"(va + d0 * Rp), "r"(bv), "r"(b)
        : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
        "[%3];" ::"r"(smem_u32(cof + (size_t)slot * G * Rp)),
        "l"(vb + d0 * Rp), "r"(bc), "r"(b)
        : "memory");
  }
  // wait (bounded) until group n's slot is filled
  __device__ __forceinline__ bool wait(unsigned n, unsigned limit = kSpinLimit) const {
    const unsigned b = smem_u32(bar + n % kRG), parity = (n / kRG) & 1u;
    for (unsigned it = 0;; ++it) {
      unsigned ok;
      asm volatile(
          "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
          " selp.u32 %0, 1, 0, p;\n}"
          : "=r"(ok)
          : "r"(b), "r"(parity)
          : "memory");
      if (ok) return true;
      if (it >= limit) return false;
    }
  }
};

template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// The sweep warp gave up waiting for a copy: record it, then wait (again
// bounded) for the groups it still has in flight, n0 .. n1 - 1.
template <int kRG, int G>
__device__ __noinline__ void sweep_abort(const TSys &S, const SweepMem<kRG, G> &sm, unsigned n0,
                                         unsigned n1) {
  if ((threadIdx.x & 31) == 0) {
    atomicExch(S.fault, 1);
    bulk_wait_all();
  }
  for (unsigned n = n0; n < n1; ++n) sm.wait(n, kDrainLimit);
}

// One wavefront sweep by one warp.  Step s handles anti-diagonal
// diag(s) (s for the forward sweep, Rp + np - 2 - s for the reverse).  Lane
// l holds rows l M + m, m < M, as chains:
//   v(r) = a(r) - c.y(r) v_prev(r) - c.x(r) n(r)
// where a is the value stream, c the coefficient pair, v_prev the row's
// previous value (the west / east neighbour) and n the previous step's
// value of the row below / above -- chain m -+ 1 of the same lane, or for
// the lane's first / last chain the neighbouring lane's last / first chain
// by warp shuffle.  Off-grid points and padding rows read zeros and produce
// exact zeros.  Work is grouped G steps at a time: one pair of bulk loads,
// one wait and one bulk store per group, and every load of a step is issued
// before any store.  The seam term of the one point per step on the seam
// longitude is folded into that point's value in the ring, a group ahead,
// from the row's captured edge value (groups of G need the seam
// np - 1 >= 2 G steps after the edge).
//
// Forward (nonorthogonal_mi.c:910-937), on D^-1-scaled rows:
//   fw = in/dg - (lo/dg) fw(r-1, j) - (ll/dg) fw(r, j-1) - (lu/dg) fw(r, 0)|j=np-1
// Reverse (nonorthogonal_mi.c:939-964):
//   out = fw - (up/dg) out(r+1, j) - (lu/dg) out(r, j+1) - (ll/dg) out(r, np-1)|j=0
// with the pole sum sum_j pe_j out(1, j) accumulated from row 0.
template <int M, int kRG, int G, bool kReverse>
__device__ __forceinline__ bool sweep(const TSys &S, const double *__restrict__ in,
                                      double *__restrict__ out, const SweepMem<kRG, G> &sm,
                                      unsigned &gn, const double *pe_s, double boundary,
                                      double &psum) {
  const int lane = threadIdx.x & 31, R = S.R, Rp = S.Rp, np = S.np;
  const int dmax = Rp + np - 2;
  const int ngroups = (Rp + np - 1 + G - 1) / G;  // steps padded to whole groups
  const double2 *coef = kReverse ? S.cb : S.cf;
  const double *seam = kReverse ? sm.seam_r : sm.seam_f;
  // lowest column of group k, and the slot index of step u of a group
  auto group_d0 = [&](int k) {
    return (size_t)(kPad + (kReverse ? dmax - (k * G + G - 1) : k * G));
  };
  auto sub = [&](int u) { return kReverse ? G - 1 - u : u; };
  // seam point of step s: row s - (np - 1) (forward) / dmax - s (reverse);
  // edge point: row s at longitude 0 / row Rp - 1 - s at longitude np - 1
  auto seam_row = [&](int s) { return kReverse ? dmax - s : s - (np - 1); };
  auto edge_row = [&](int s) { return kReverse ? Rp - 1 - s : s; };
  auto pos = [&](int r) { return (r % M) * 32 + r / M; };
  double v[M];
#pragma unroll
  for (int m = 0; m < M; ++m) v[m] = 0.0;
  psum = 0.0;
  // operands (value, coefficient pair) of step u of group k, for this lane's chains
  double ca[M];
  double2 cc[M];
  auto load = [&](int k, int u, double (&a)[M], double2 (&c)[M]) {
    const size_t base = ((size_t)((gn + k) % kRG) * G + sub(u)) * Rp + lane;
    const double *__restrict__ rv = sm.val + base;
    const double2 *__restrict__ rc = sm.cof + base;
#pragma unroll
    for (int m = 0; m < M; ++m) {
      a[m] = rv[32 * m];
      c[m] = rc[32 * m];
    }
  };
  // the value stream was written through the generic proxy (a vector phase,
  // or the forward sweep's drained stores) and is read by bulk copies
  if (lane == 0) bulk_wait_all();
  asm volatile("fence.proxy.async;" ::: "memory");
  __syncwarp();
  if (lane == 0)
    for (int k = 0; k < kRG - 1 && k < ngroups; ++k) sm.issue(gn + k, in, coef, group_d0(k));
  bool ok = true;
  if (lane < G) ok = sm.wait(gn);  // group 0 has no seam point
  for (int k = 0; k < ngroups; ++k) {
    const unsigned n = gn + k;
    if (!__all_sync(0xffffffffu, ok)) {
      sweep_abort(S, sm, n, gn + (unsigned)min(k + kRG - 1, ngroups));
      gn += ngroups;
      return false;
    }
    if (lane == 0) {
      if (k + kRG - 1 < ngroups) sm.issue(n + kRG - 1, in, coef, group_d0(k + kRG - 1));
      bulk_wait_read<1>();  // the stage half of this group is free again
    }
    // lanes u < G: wait for the next group and fold its seam terms
    if (lane < G && k + 1 < ngroups) {
      ok = sm.wait(n + 1);
      const int r = seam_row((k + 1) * G + lane);
      if (ok && r >= 0 && r < R) {
        double *p = sm.val + ((size_t)((n + 1) % kRG) * G + sub(lane)) * Rp + pos(r);
        *p = fma(-seam[r], sm.edge[r], *p);
      }
    }
    __syncwarp();
    if (k == 0) load(0, 0, ca, cc);
    double *gs = sm.stage + (size_t)(k & 1) * G * Rp;
#pragma unroll
    for (int u = 0; u < G; ++u) {
      // operands of the next step, loaded before this step computes and stores
      double na[M];
      double2 nc[M];
      if (u + 1 < G)
        load(k, u + 1, na, nc);
      else if (k + 1 < ngroups)
        load(k + 1, 0, na, nc);
      double nb[M];
      if (kReverse) {
        const double x = __shfl_sync(0xffffffffu, v[0], (lane + 1) & 31);
        nb[M - 1] = lane == 31 ? 0.0 : x;  // no row above the top one
#pragma unroll
        for (int m = 0; m + 1 < M; ++m) nb[m] = v[m + 1];
      } else {
        const double x = __shfl_sync(0xffffffffu, v[M - 1], (lane + 31) & 31);
        nb[0] = lane == 0 ? boundary : x;  // the pole below row 0
#pragma unroll
        for (int m = 1; m < M; ++m) nb[m] = v[m - 1];
      }
#pragma unroll
      for (int m = 0; m < M; ++m) v[m] = fma(-cc[m].x, nb[m], fma(-cc[m].y, v[m], ca[m]));
      if (kReverse) {
        const int d = dmax - (k * G + u);
        psum = fma(pe_s[d < 0 ? 0 : d < np ? d : np - 1], v[0], psum);
      }
      double *__restrict__ st = gs + sub(u) * Rp + lane;
#pragma unroll
      for (int m = 0; m < M; ++m) st[32 * m] = v[m];
#pragma unroll
      for (int m = 0; m < M; ++m) {
        ca[m] = na[m];
        cc[m] = nc[m];
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncwarp();
    if (lane < G) {
      // edge capture for this group's steps
      const int re = edge_row(k * G + lane);
      if (re >= 0 && re < R) sm.edge[re] = gs[sub(lane) * Rp + pos(re)];
    }
    __syncwarp();  // captured edges are visible to the seam folds of later groups
    if (lane == 0) {
      asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(
                       out + group_d0(k) * Rp),
                   "r"(smem_u32(gs)), "r"((unsigned)(G * Rp) * 8u)
                   : "memory");
      asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    }
  }
  gn += ngroups;
  if (lane == 0) {
    bulk_wait_all();
    asm volatile("fence.proxy.async;" ::: "memory");
  }
  __syncwarp();
  return true;
}

// Band-pipelined sweeps.  CTA b of the cluster owns the interior rows
// r0 = b h .. r0 + hb - 1 (hb <= h <= 32 rows, one lane of warp 0 per row).
// Lane l advances its row one longitude per step -- step t handles
// longitude t - l (forward) or np - 1 - t + (hb - 1 - l) (reverse) -- so a
// step covers one anti-diagonal of the band and the row below (forward) /
// above (reverse) is the neighbouring lane's previous-step value, one warp
// shuffle away.  The band's edge row crosses to the next CTA through its
// inbox: the sending lane stores each value into the neighbour's shared
// memory (a distributed-shared-memory store) and the receiving lane polls
// its own copy until the value replaces the empty mark.  The bands thus
// form a pipeline in which each CTA trails the previous one by about hb
// steps, and every point is updated from exactly the operands of the
// single-warp wavefront, in the same order: the two schedules give
// identical results.
//
// Shared memory of a band (per CTA): the forward and reverse coefficient
// pairs and the sweep values at band diagonal d = j + l, slot d h + l (a
// step touches consecutive slots); the forward sweep overwrites its input
// with its output, which the reverse sweep reads back in place.
constexpr unsigned long long kEmpty = 0x7ff4dead0000beefull;  // signalling NaN, never computed
constexpr unsigned kInboxSpinLimit = 1u << 22;                 // polls of one inbox value

struct BandMem {
  double2 *cf, *cb;   // [np + h - 1][h]
  double *val;        // [np + h - 1][h]
  double *inf, *inr;  // inboxes [np]: row below (forward) / above (reverse)
  double *pe;         // [np] pole edges (CTA 0)
  int h;
};

size_t band_smem(int h, int np) {
  return ((size_t)(np + h - 1) * h * 5 + (size_t)np * 3) * sizeof(double);
}

__device__ __forceinline__ unsigned cluster_addr(const void *p, int rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
  return r;
}

__device__ __forceinline__ void inbox_put(unsigned addr, double v) {
  asm volatile("st.relaxed.cluster.shared::cluster.b64 [%0], %1;" ::"r"(addr), "d"(v)
               : "memory");
}

__device__ __forceinline__ double inbox_peek(const double *p) {
  double v;
  asm volatile("ld.relaxed.cluster.shared::cta.b64 %0, [%1];" : "=d"(v) : "r"(smem_u32(p))
               : "memory");
  return v;
}

// Value of an inbox slot, waiting (bounded) for it to arrive; false when
// it never did.
__device__ __forceinline__ bool inbox_take(const double *p, double &v) {
  for (unsigned it = 0; it < kInboxSpinLimit; ++it) {
    v = inbox_peek(p);
    if ((unsigned long long)__double_as_longlong(v) != kEmpty) return true;
  }
  v = 0.0;
  return false;
}

// One sweep of band b (rows r0 .. r0 + hb - 1) by warp 0 of its CTA, the
// recurrences of sweep() on the same D^-1-scaled operands:
//   forward  v = val - (lo/dg) v(r-1, j) - (ll/dg) v(r, j-1) [- (lu/dg) v(r, 0) at j = np-1]
//   reverse  v = fw  - (up/dg) v(r+1, j) - (lu/dg) v(r, j+1) [- (ll/dg) v(r, np-1) at j = 0]
// the forward in place into bm.val, the reverse into out (skewed layout);
// psum accumulates the pole edge sum over row 0 (band 0).  Returns false
// when a value of the neighbouring band never arrived: the fault is
// recorded and the remaining steps use zeros.
template <bool kReverse>
__device__ __noinline__ bool band_sweep(const TSys &S, const BandMem &bm, int b, int r0, int hb,
                                        double boundary, double *__restrict__ out,
                                        double &psum) {
  const int lane = threadIdx.x & 31, np = S.np, h = bm.h, nbands = S.nbands;
  const bool row_on = lane < hb;
  const double2 *__restrict__ cof = kReverse ? bm.cb : bm.cf;
  double *__restrict__ val = bm.val;
  double seam = 0.0;
  if (row_on)
    seam = kReverse ? bm.cf[(size_t)lane * h + lane].y
                    : bm.cb[(size_t)(np - 1 + lane) * h + lane].y;
  // the lane fed by the neighbouring band, and the lane feeding the next one
  const bool link = kReverse ? lane == hb - 1 : lane == 0;
  const bool from_band = kReverse ? b + 1 < nbands : b > 0;
  const bool send =
      (kReverse ? lane == 0 : lane == hb - 1) && (kReverse ? b > 0 : b + 1 < nbands);
  double *inbox = kReverse ? bm.inr : bm.inf;
  const unsigned dst = send ? cluster_addr(inbox, kReverse ? b - 1 : b + 1) : 0u;
  // the row's first point in the skewed output: (kPad + r + j) Rp + row_pos(r)
  double *orow =
      out + (size_t)(kPad + r0 + lane) * S.Rp + (row_on ? row_pos(S.Rp, r0 + lane) : 0);
  const double fixed = kReverse ? 0.0 : boundary;  // pole below row 0; nothing above row R-1
  const bool pole_row = kReverse && b == 0 && lane == 0;
  bool ok = true;
  double v = 0.0, edge = 0.0;
  const int steps = np + hb - 1;
#pragma unroll 2
  for (int t = 0; t < steps; ++t) {
    const int j = kReverse ? np - 1 - t + (hb - 1 - lane) : t - lane;
    const bool on = row_on && j >= 0 && j < np;
    double x =
        kReverse ? __shfl_down_sync(0xffffffffu, v, 1) : __shfl_up_sync(0xffffffffu, v, 1);
    if (link) {
      if (!from_band) {
        x = fixed;
      } else if (on) {
        if (ok) ok = inbox_take(inbox + j, x);
        if (!ok) x = 0.0;
      }
    }
    if (on) {
      const size_t slot = (size_t)(j + lane) * h + lane;
      double a = val[slot];
      const double2 c = cof[slot];
      if (j == (kReverse ? 0 : np - 1)) a = fma(-seam, edge, a);
      v = fma(-c.x, x, fma(-c.y, v, a));
      if (j == (kReverse ? np - 1 : 0)) edge = v;
      if (kReverse)
        orow[(size_t)j * S.Rp] = v;
      else
        val[slot] = v;
      if (pole_row) psum = fma(bm.pe[j], v, psum);
      if (send) inbox_put(dst + (unsigned)j * 8u, v);
    }
  }
  // every value of the inbox has been taken: mark it empty for the next sweep
  if (from_band)
    for (int j = lane; j < np; j += 32) inbox[j] = __longlong_as_double((long long)kEmpty);
  if (!__all_sync(0xffffffffu, ok)) {
    if (lane == 0) atomicExch(S.fault, 1);
    return false;
  }
  return true;
}

// (A p) at a grid point of the skewed layout (nonorthogonal_mi.c:867-900).
__device__ __forceinline__ double apply_at(const TSys &S, const double *p, size_t k, int row,
                                           int j, double pole) {
  const int R = S.R, Rp = S.Rp, np = S.np;
  const size_t q = (size_t)row_pos(Rp, row);
  const double lv = row == 0 ? pole : p[k - q - Rp + row_pos(Rp, row - 1)];
  const double uv = row + 1 < R ? p[k - q + Rp + row_pos(Rp, row + 1)] : 0.0;
  const size_t kw = j == 0 ? k + (size_t)(np - 1) * Rp : k - Rp;
  const size_t ke = j + 1 == np ? k - (size_t)(np - 1) * Rp : k + Rp;
  return S.dg[k] * p[k] + S.lo[k] * lv + S.up[k] * uv + S.ll[k] * p[kw] + S.lu[k] * p[ke];
}

// Colour of grid point (row, j) in the multicolour SSOR: the pole first,
// then (row + j) parity off the seam column and row parity on it (the last
// longitude, whose periodic neighbour j = 0 has the same (row + j) parity
// when np is odd); no two points of one colour are stencil neighbours.
__device__ __forceinline__ int tcolor(int row, int j, int np) {
  return j + 1 < np ? ((row + j) & 1) : 2 + (row & 1);
}

// Partial dot products of one thread.
template <int N>
struct Acc {
  static constexpr int n = N;
  double v[N] = {};
};

// Row and longitude of skewed index k; false off the grid and on padding rows.
__device__ __forceinline__ bool locate(int R, int Rp, int np, unsigned k, int &row, int &j) {
  const unsigned col = k / (unsigned)Rp;
  row = pos_row(Rp, (int)(k - col * (unsigned)Rp));
  j = (int)col - kPad - row;
  return row < R && (unsigned)j < (unsigned)np;
}

// Dynamic shared memory of a launch: the sweep ring (kRG G diagonals of
// Rp values and Rp coefficient pairs), 2 G staged output diagonals, three
// row tables and the pole-edge table.
size_t tensor_smem(int kRG, int G, int Rp, int np) {
  return ((size_t)kRG * G * Rp * 3 + (size_t)(2 * G + 3) * Rp + (size_t)np) * sizeof(double);
}

template <int M, int kRG, int kG>
__global__ void __launch_bounds__(kThreads, 1) k_tensor(TSys S) {
  constexpr int kT = kThreads, kWarps = kT / 32;
  constexpr int kB = 8;  // grid points a thread loads per batch
  extern __shared__ __align__(128) double dyn_smem[];
  __shared__ uint64_t ring_bar[kRG];
  __shared__ double wbuf[kWarps * kSlotWidth];
  __shared__ double slots[kSlots * kMaxCluster * kSlotWidth];
  __shared__ double bcast[2];
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank(), csize = (int)cl.num_blocks();
  Reducer<kWarps> red{wbuf, slots, 0, rank, csize};
  const int np = S.np, nt = S.nt, R = S.R, Rp = S.Rp, t = threadIdx.x, lane = t & 31,
            warp = t >> 5;
  SweepMem<kRG, kG> sm;
  sm.val = dyn_smem;
  sm.cof = reinterpret_cast<double2 *>(dyn_smem + (size_t)kRG * kG * Rp);
  sm.stage = dyn_smem + (size_t)kRG * kG * Rp * 3;
  sm.edge = sm.stage + (size_t)2 * kG * Rp;
  sm.seam_f = sm.edge + Rp;
  sm.seam_r = sm.seam_f + Rp;
  sm.bar = ring_bar;
  sm.Rp = Rp;
  double *pe_s = sm.seam_r + Rp;
  // the band schedule's tables share the dynamic shared memory
  BandMem bm;
  bm.h = S.band;
  {
    const size_t slots = (size_t)(np + S.band - 1) * S.band;
    bm.cf = reinterpret_cast<double2 *>(dyn_smem);
    bm.cb = bm.cf + slots;
    bm.val = reinterpret_cast<double *>(bm.cb + slots);
    bm.inf = bm.val + slots;
    bm.inr = bm.inf + np;
    bm.pe = bm.inr + np;
  }
  if (S.band)
    for (int j = threadIdx.x; j < np; j += kT)
      bm.inf[j] = bm.inr[j] = __longlong_as_double((long long)kEmpty);
  if (rank == 0 && t == 0) {
    for (int q = 0; q < kRG; ++q)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(ring_bar + q))
                   : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *S.fault = 0;
  }
  const unsigned g = (unsigned)(rank * kT + t), G = (unsigned)(csize * kT);
  const bool lead = g == 0;
  const unsigned nq = (unsigned)(R * np);
  const unsigned core0 = S.core0, core1 = S.core1;

  // mean Pedersen conductance of the pole row, every warp 0 alike
  if (warp == 0) {
    double m = 0.0;
    for (int j = lane; j < np; j += 32) m += S.sp[j];
    m = warp_sum(m) / (double)np;
    if (lane == 0) bcast[0] = m;
  }
  __syncthreads();
  const double ppm = bcast[0];
  // pole edges and the cached stencil (nonorthogonal_mi.c:776-865)
  for (unsigned j = g; j < (unsigned)np; j += G) {
    const double fp = 0.5 * (ppm + S.sp[(size_t)np + j]);
    S.pe[j] = S.pole_sin * fp / (S.pole_inc2 * S.dth * S.dth);
  }
  double v3[2] = {0.0, 0.0};  // sum u^2, non-finite FAC count
  for (unsigned q = g; q < nq; q += G) {
    const int row = (int)(q / (unsigned)np), j = (int)(q - (unsigned)row * np), i = row + 1;
    const int jm = j == 0 ? np - 1 : j - 1, jp = j + 1 == np ? 0 : j + 1;
    const TRow &Rw = S.rows[i];
    const size_t full = (size_t)i * np + j;
    const double *P = S.sp, *H = S.sh;
    const double lower = Rw.sl * 0.5 * (P[full] + P[full - np]) / (Rw.il * S.dth * S.dth);
    const double upper = Rw.su * 0.5 * (P[full] + P[full + np]) / (Rw.iu * S.dth * S.dth);
    const double llo = 0.5 * (P[full] + P[(size_t)i * np + jm]) / (Rw.s * S.dph * S.dph);
    const double lup = 0.5 * (P[full] + P[(size_t)i * np + jp]) / (Rw.s * S.dph * S.dph);
    const double d = lower + upper + llo + lup;
    const double f_up = -H[full + np] / S.rows[i + 1].inc;
    const double f_dn = -H[full - np] / S.rows[i - 1].inc;
    const double f_e = -H[(size_t)i * np + jp] / Rw.inc;
    const double f_w = -H[(size_t)i * np + jm] / Rw.inc;
    const double dft = (f_up - f_dn) / (2.0 * S.dth);
    const double dfp = (f_e - f_w) / (2.0 * S.dph);
    const double lo = -lower - dfp / (2.0 * S.dth);
    const double up = -upper + dfp / (2.0 * S.dth);
    const double ll = -llo + dft / (2.0 * S.dph);
    const double lu = -lup - dft / (2.0 * S.dph);
    const size_t k = sidx(Rp, row, j);
    S.dg[k] = d;
    S.lo[k] = lo;
    S.up[k] = up;
    S.ll[k] = ll;
    S.lu[k] = lu;
    S.rdg[k] = 1.0 / d;
    S.cf[k] = make_double2(lo / d, ll / d);
    S.cb[k] = make_double2(up / d, lu / d);
    // right-hand side and initial guess (nonorthogonal_mi.c:999-1029)
    const double f = S.fac[full];
    const double u = S.neg_r2 * f * Rw.inc;
    S.rhs[k] = Rw.s * u;
    v3[0] += u * u;
    v3[1] += isfinite(f) ? 0.0 : 1.0;
    const double gsv = S.pot[full];
    S.x[k] = isfinite(gsv) ? gsv : 0.0;
  }
  if (lead) {
    double m = 0.0;
    for (int j = 0; j < np; ++j) {
      const double gsv = S.pot[j];
      if (isfinite(gsv)) m += gsv / (double)np;
    }
    S.x[0] = m;
    S.rhs[0] = 0.0;
  }
  red.template sum<2>(cl, v3);
  if (v3[1] > 0.0) {
    if (lead) *S.status = 2;
    cl.sync();
    return;
  }
  const double target = fmax(S.abs_tol, S.rel_tol * fmax(sqrt(fmax(0.0, v3[0])), 1.0));
  if (warp == 0) {
    double d0 = 0.0;
    for (int j = lane; j < np; j += 32) d0 += S.pe[j];
    d0 = warp_sum(d0);
    if (lane == 0) bcast[1] = d0;
  }
  if (S.band) {
    // this CTA's band of the sweep coefficients, by band diagonal
    const int h = S.band, r0 = rank * h, hb = rank < S.nbands ? min(h, R - r0) : 0;
    const int slots = (np + h - 1) * h;
    for (int q = t; q < slots; q += kT) {
      const int d = q / h, l = q - d * h, j = d - l;
      const bool on = l < hb && j >= 0 && j < np;
      const size_t k = on ? sidx(Rp, r0 + l, j) : 0;
      bm.cf[q] = on ? S.cf[k] : make_double2(0.0, 0.0);
      bm.cb[q] = on ? S.cb[k] : make_double2(0.0, 0.0);
      bm.val[q] = 0.0;
    }
    if (rank == 0)
      for (int j = t; j < np; j += kT) bm.pe[j] = S.pe[j];
  } else if (rank == 0) {
    for (int j = t; j < np; j += kT) pe_s[j] = S.pe[j];
    for (int r = t; r < Rp; r += kT) {
      sm.seam_f[r] = r < R ? S.cb[sidx(Rp, r, np - 1)].y : 0.0;
      sm.seam_r[r] = r < R ? S.cf[sidx(Rp, r, 0)].y : 0.0;
    }
  }
  __syncthreads();
  const double dg0 = bcast[1], rdg0 = 1.0 / dg0, wp = (double)np / (S.ps * S.ps);
  if (lead) {
    S.dg[0] = dg0;
    S.rdg[0] = rdg0;
  }

  // True residual r = rhs - A x over the grid, with shd = r, srch = as = 0;
  // returns {weighted |r|^2, shd.r}, pole included (nonorthogonal_mi.c:1030-1039).
  auto true_residual = [&](double (&out)[2]) {
    double a[3] = {0.0, 0.0, 0.0};  // weighted norm, plain norm, pole edge sum
    const double x0 = S.x[0];
    for (unsigned k0 = core0 + g; k0 < core1; k0 += kB * G) {
      double r[kB], xr[kB], wr[kB];
      bool on[kB];
#pragma unroll
      for (int b = 0; b < kB; ++b) {
        const unsigned k = k0 + b * G;
        int row = 0, j = 0;
        on[b] = k < core1 && locate(R, Rp, np, k, row, j);
        r[b] = on[b] ? S.rhs[k] - apply_at(S, S.x, k, row, j, x0) : 0.0;
        wr[b] = on[b] ? S.rows[row + 1].s : 1.0;
        xr[b] = on[b] && row == 0 ? S.pe[j] * S.x[k] : 0.0;
      }
#pragma unroll
      for (int b = 0; b < kB; ++b) {
        if (!on[b]) continue;
        const unsigned k = k0 + b * G;
        S.res[k] = r[b];
        S.shd[k] = r[b];
        S.srch[k] = 0.0;
        S.as[k] = 0.0;
        const double wv = r[b] / wr[b];
        a[0] += wv * wv;
        a[1] += r[b] * r[b];
        a[2] += xr[b];
      }
    }
    red.template sum<3>(cl, a);
    const double r0 = S.rhs[0] - (dg0 * x0 - a[2]);
    if (lead) {
      S.res[0] = r0;
      S.shd[0] = r0;
      S.srch[0] = 0.0;
      S.as[0] = 0.0;
    }
    out[0] = a[0] + wp * r0 * r0;
    out[1] = a[1] + r0 * r0;
  };

  // A p on the grid into ap, with the pole row dg0 p0 - (pole edge sum of
  // the SSOR that produced p); accumulates shd.ap (N = 1) or {ap.ap,
  // ap.mid} (N = 2).
  auto apply_phase = [&](const double *p, double *ap, auto &acc) {
    const double p0 = p[0];
    for (unsigned k0 = core0 + g; k0 < core1; k0 += kB * G) {
      double av[kB], o[kB];
      bool on[kB];
#pragma unroll
      for (int b = 0; b < kB; ++b) {
        const unsigned k = k0 + b * G;
        int row = 0, j = 0;
        on[b] = k < core1 && locate(R, Rp, np, k, row, j);
        av[b] = on[b] ? apply_at(S, p, k, row, j, p0) : 0.0;
        o[b] = on[b] ? (acc.n == 1 ? S.shd[k] : S.mid[k]) : 0.0;
      }
#pragma unroll
      for (int b = 0; b < kB; ++b) {
        if (!on[b]) continue;
        ap[k0 + b * G] = av[b];
        if (acc.n == 1) {
          acc.v[0] += o[b] * av[b];
        } else {
          acc.v[0] += av[b] * av[b];
          acc.v[1] += av[b] * o[b];
        }
      }
    }
    if (lead) {
      const double a0 = dg0 * p0 - *S.pole_sum;
      ap[0] = a0;
      if (acc.n == 1) {
        acc.v[0] += S.shd[0] * a0;
      } else {
        acc.v[0] += a0 * a0;
        acc.v[1] += a0 * S.mid[0];
      }
    }
  };

  double nr[2];
  true_residual(nr);
  const double initial = sqrt(fmax(0.0, nr[0]));
  double final_res = initial, rho = nr[1];
  int iters = 0;
  int conv = initial <= target;
  double rho_prev = 1.0, alpha = 1.0, omega = 1.0;
  const int max_iter = S.max_iter < kMaxIterations ? S.max_iter : kMaxIterations;
  const bool sweeper = rank == 0 && warp == 0;
  unsigned gn = 0;  // running group count of the sweep warp's prefetch ring
  // SSOR of in (D^-1-scaled, pole at in[0]) into out, by the sweep warp
  auto ssor = [&](const double *in, double *out) {
    double psum = 0.0;
    if (lane == 0) S.fw[0] = in[0];
    if (sweep<M, kRG, kG, false>(S, in, S.fw, sm, gn, pe_s, in[0], psum) &&
        sweep<M, kRG, kG, true>(S, S.fw, out, sm, gn, pe_s, 0.0, psum) && lane == 0) {
      // pole (nonorthogonal_mi.c:958-963): (dg0 fw0 + sum pe_j out(1, j)) / dg0
      out[0] = (dg0 * S.fw[0] + psum) / dg0;
      *S.pole_sum = psum;
    }
  };
  // The same SSOR by the band pipeline: every CTA stages its band of the
  // input, then warp 0 of each band runs the forward and reverse sweeps.
  auto band_ssor = [&](const double *in, double *out) {
    const int h = S.band, r0 = rank * h, hb = rank < S.nbands ? min(h, R - r0) : 0;
    const double in0 = in[0];
    for (int q = t; q < hb * np; q += kT) {
      const int l = q / np, j = q - l * np;
      bm.val[(size_t)(j + l) * h + l] = in[sidx(Rp, r0 + l, j)];
    }
    __syncthreads();
    if (warp == 0 && hb > 0) {
      double psum = 0.0;
      if (band_sweep<false>(S, bm, rank, r0, hb, in0, out, psum) &&
          band_sweep<true>(S, bm, rank, r0, hb, 0.0, out, psum) && rank == 0 && lane == 0) {
        // pole (nonorthogonal_mi.c:958-963): (dg0 fw0 + sum pe_j out(1, j)) / dg0
        out[0] = (dg0 * in0 + psum) / dg0;
        *S.pole_sum = psum;
      }
    }
  };
  // The reference's triangular SSOR (nonorthogonal_mi.c:910-964) with the
  // unknowns ordered by colour (tcolor) instead of row by row: within a
  // colour every update is independent, so the whole cluster sweeps one
  // colour at a time.  A different ordering of the same splitting: the
  // preconditioner, and so the iteration count, differ from the reference's.
  auto colored_ssor = [&](const double *in, double *out) {
    double *fw = S.fw;
    if (lead) fw[0] = in[0];
    cl.sync();
    const unsigned half = (unsigned)(np / 2);  // colour-0/1 slots per row
    for (int dir = 0; dir < 2; ++dir) {
      const double *src = dir == 0 ? fw : out;
      double *dst = dir == 0 ? fw : out;
      for (int ci = 0; ci < 4; ++ci) {
        const int c = dir == 0 ? ci : 3 - ci;
        // the colour's points, enumerated directly: (row, 2 m + parity) off
        // the seam column for colours 0 and 1, rows of one parity on it for
        // colours 2 and 3
        const unsigned n = c < 2 ? (unsigned)R * half : (unsigned)(R - (c - 2) + 1) / 2;
        for (unsigned t0 = g; t0 < n; t0 += kB * G) {
          size_t kk[kB];
          bool on[kB];
          double v[kB], rd[kB], cf[kB][4], nb[kB][4];
#pragma unroll
          for (int b = 0; b < kB; ++b) {
            const unsigned tt = t0 + b * G;
            int row = 0, j = 0;
            if (c < 2) {
              row = (int)(tt / half);
              j = 2 * (int)(tt - (unsigned)row * half) + ((c + row) & 1);
              on[b] = tt < n && j < np - 1;
            } else {
              row = 2 * (int)tt + (c - 2);
              j = np - 1;
              on[b] = tt < n && row < R;
            }
            kk[b] = 0;
            v[b] = rd[b] = 0.0;
#pragma unroll
            for (int q = 0; q < 4; ++q) cf[b][q] = nb[b][q] = 0.0;
            if (!on[b]) continue;
            const size_t k = sidx(Rp, row, j);
            const size_t q = (size_t)row_pos(Rp, row);
            const int jm = j == 0 ? np - 1 : j - 1, jp = j + 1 == np ? 0 : j + 1;
            kk[b] = k;
            v[b] = dir == 0 ? in[k] : fw[k];
            rd[b] = S.rdg[k];
            // neighbours of an earlier colour (forward) or a later one (reverse)
            const int cn[4] = {row == 0 ? -1 : tcolor(row - 1, j, np),
                               row + 1 < R ? tcolor(row + 1, j, np) : c,
                               tcolor(row, jm, np), tcolor(row, jp, np)};
            const size_t kn[4] = {row == 0 ? 0 : k - q - Rp + row_pos(Rp, row - 1),
                                  row + 1 < R ? k - q + Rp + row_pos(Rp, row + 1) : k,
                                  j == 0 ? k + (size_t)(np - 1) * Rp : k - Rp,
                                  j + 1 == np ? k - (size_t)(np - 1) * Rp : k + Rp};
            const double *co[4] = {S.lo, S.up, S.ll, S.lu};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              if (dir == 0 ? cn[e] < c : cn[e] > c) {
                cf[b][e] = co[e][k];
                nb[b][e] = src[kn[e]];
              }
            }
          }
#pragma unroll
          for (int b = 0; b < kB; ++b) {
            if (!on[b]) continue;
            double x = v[b];
#pragma unroll
            for (int e = 0; e < 4; ++e) x -= cf[b][e] * rd[b] * nb[b][e];
            dst[kk[b]] = x;
          }
        }
        cl.sync();
      }
    }
    // pole (nonorthogonal_mi.c:958-963): (dg0 fw0 + sum pe_j out(1, j)) / dg0
    double ps[1] = {0.0};
    for (unsigned jj = g; jj < (unsigned)np; jj += G) ps[0] += S.pe[jj] * out[sidx(Rp, 0, jj)];
    red.template sum<1>(cl, ps);
    if (lead) {
      out[0] = (dg0 * fw[0] + ps[0]) / dg0;
      *S.pole_sum = ps[0];
    }
  };
  // BiCGStab (nonorthogonal_mi.c:1040-1128)
  for (int it = 1; !conv && it <= max_iter; ++it) {
    if (!isfinite(rho) || fabs(rho) <= DBL_MIN || !isfinite(omega) || fabs(omega) <= DBL_MIN)
      break;
    const double beta = (rho / rho_prev) * (alpha / omega);
    for (unsigned k0 = core0 + g; k0 < core1; k0 += kB * G) {
      double r[kB], sr[kB], a[kB], d[kB];
#pragma unroll
      for (int b = 0; b < kB; ++b) {
        const unsigned k = k0 + b * G;
        const bool on = k < core1;
        r[b] = on ? S.res[k] : 0.0;
        sr[b] = on ? S.srch[k] : 0.0;
        a[b] = on ? S.as[k] : 0.0;
        d[b] = on ? S.rdg[k] : 0.0;
      }
#pragma unroll
      for (int b = 0; b < kB; ++b) {
        const unsigned k = k0 + b * G;
        if (k >= core1) continue;
        const double s = r[b] + beta * (sr[b] - omega * a[b]);
        S.srch[k] = s;
        S.pin[k] = s * d[b];
      }
    }
    if (lead) {
      const double s = S.res[0] + beta * (S.srch[0] - omega * S.as[0]);
      S.srch[0] = s;
      S.pin[0] = s * rdg0;
    }
    cl.sync();
    if (S.colored)
      colored_ssor(S.pin, S.psv);
    else if (S.band)
      band_ssor(S.pin, S.psv);
    else if (sweeper)
      ssor(S.pin, S.psv);
    cl.sync();
    if (*(volatile int *)S.fault) break;
    Acc<1> d2;
    apply_phase(S.psv, S.as, d2);
    red.template sum<1>(cl, d2.v);
    if (!isfinite(d2.v[0]) || fabs(d2.v[0]) <= DBL_MIN) break;
    alpha = rho / d2.v[0];
    double d3[1] = {0.0};
    for (unsigned k0 = core0 + g; k0 < core1; k0 += kB * G) {
      double r[kB], a[kB], d[kB], wr[kB];
#pragma unroll
      for (int b = 0; b < kB; ++b) {
        const unsigned k = k0 + b * G;
        const bool on = k < core1;
        r[b] = on ? S.res[k] : 0.0;
        a[b] = on ? S.as[k] : 0.0;
        d[b] = on ? S.rdg[k] : 0.0;
        // off-grid slots hold zeros; the row weight of any slot is finite
        wr[b] = on ? S.rows[1 + pos_row(Rp, (int)(k % (unsigned)Rp))].s : 1.0;
      }
#pragma unroll
      for (int b = 0; b < kB; ++b) {
        const unsigned k = k0 + b * G;
        if (k >= core1) continue;
        const double m = r[b] - alpha * a[b];
        S.mid[k] = m;
        S.pin[k] = m * d[b];
        const double wv = m / wr[b];
        d3[0] += wv * wv;
      }
    }
    if (lead) {
      const double m0 = S.res[0] - alpha * S.as[0];
      S.mid[0] = m0;
      S.pin[0] = m0 * rdg0;
      d3[0] += wp * m0 * m0;
    }
    red.template sum<1>(cl, d3);
    final_res = sqrt(fmax(0.0, d3[0]));
    if (final_res <= target) {
      for (unsigned k0 = core0 + g; k0 < core1; k0 += kB * G) {
        double x[kB], p[kB];
#pragma unroll
        for (int b = 0; b < kB; ++b) {
          const unsigned k = k0 + b * G;
          const bool on = k < core1;
          x[b] = on ? S.x[k] : 0.0;
          p[b] = on ? S.psv[k] : 0.0;
        }
#pragma unroll
        for (int b = 0; b < kB; ++b) {
          const unsigned k = k0 + b * G;
          if (k < core1) S.x[k] = x[b] + alpha * p[b];
        }
      }
      if (lead) S.x[0] += alpha * S.psv[0];
      cl.sync();
      iters = it;
      conv = 1;
      break;
    }
    if (S.colored)
      colored_ssor(S.pin, S.pm);
    else if (S.band)
      band_ssor(S.pin, S.pm);
    else if (sweeper)
      ssor(S.pin, S.pm);
    cl.sync();
    if (*(volatile int *)S.fault) break;
    Acc<2> d4;
    apply_phase(S.pm, S.am, d4);
    red.template sum<2>(cl, d4.v);
    if (!isfinite(d4.v[0]) || d4.v[0] <= DBL_MIN) break;
    omega = d4.v[1] / d4.v[0];
    if (!isfinite(omega) || fabs(omega) <= DBL_MIN) break;
    double d5[2] = {0.0, 0.0};  // weighted |res|^2, shd.res
    for (unsigned k0 = core0 + g; k0 < core1; k0 += kB * G) {
      double x[kB], p[kB], q[kB], m[kB], a[kB], h[kB], wr[kB];
#pragma unroll
      for (int b = 0; b < kB; ++b) {
        const unsigned k = k0 + b * G;
        const bool on = k < core1;
        x[b] = on ? S.x[k] : 0.0;
        p[b] = on ? S.psv[k] : 0.0;
        q[b] = on ? S.pm[k] : 0.0;
        m[b] = on ? S.mid[k] : 0.0;
        a[b] = on ? S.am[k] : 0.0;
        h[b] = on ? S.shd[k] : 0.0;
        wr[b] = on ? S.rows[1 + pos_row(Rp, (int)(k % (unsigned)Rp))].s : 1.0;
      }
#pragma unroll
      for (int b = 0; b < kB; ++b) {
        const unsigned k = k0 + b * G;
        if (k >= core1) continue;
        S.x[k] = x[b] + (alpha * p[b] + omega * q[b]);
        const double r = m[b] - omega * a[b];
        S.res[k] = r;
        const double wv = r / wr[b];
        d5[0] += wv * wv;
        d5[1] += h[b] * r;
      }
    }
    if (lead) {
      S.x[0] += alpha * S.psv[0] + omega * S.pm[0];
      const double r0 = S.mid[0] - omega * S.am[0];
      S.res[0] = r0;
      d5[0] += wp * r0 * r0;
      d5[1] += S.shd[0] * r0;
    }
    red.template sum<2>(cl, d5);
    final_res = sqrt(fmax(0.0, d5[0]));
    iters = it;
    if (final_res <= target || it % kRestart == 0) {
      true_residual(nr);
      final_res = sqrt(fmax(0.0, nr[0]));
      if (final_res <= target) {
        conv = 1;
        break;
      }
      rho = nr[1];
      rho_prev = 1.0;
      alpha = 1.0;
      omega = 1.0;
      continue;
    }
    rho_prev = rho;
    rho = d5[1];
  }
  cl.sync();
  // expand (nonorthogonal_mi.c:1130-1139); low-latitude potential is 0
  for (unsigned q = g; q < nq; q += G) {
    const int row = (int)(q / (unsigned)np), j = (int)(q - (unsigned)row * np);
    S.pot[(size_t)(row + 1) * np + j] = S.x[sidx(Rp, row, j)];
  }
  const double x0 = S.x[0];
  for (unsigned j = g; j < (unsigned)np; j += G) {
    S.pot[j] = x0;
    S.pot[(size_t)(nt - 1) * np + j] = 0.0;
  }
  if (lead) {
    *S.stats = gamera_mi_solver_stats{iters, initial, final_res, conv};
    *S.status = *(volatile int *)S.fault ? 3 : conv ? 0 : 1;
  }
  cl.sync();  // no CTA leaves while a peer may still write its memory
}

bool cuda_ok(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return true;
  char msg[256];
  snprintf(msg, sizeof(msg), "%s: %s", what, cudaGetErrorString(e));
  set_api_error(msg);
  return false;
}

// nonorthogonal_mi.c:197-207
double cos_inclination(double th, int hemisphere) {
  const double c = cos(th);
  return (double)hemisphere * 2.0 * c / sqrt(1.0 + 3.0 * c * c);
}
double inc2(double a) {
  const double c = cos(a);
  return 4.0 * c * c / (1.0 + 3.0 * c * c);
}

// nonorthogonal_mi.c:611-641 (configuration part)
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

using TensorKernel = void (*)(TSys);

// Kernel instance of M chains per lane (1..8 or 16) and the group size.
struct Launch {
  TensorKernel kernel = nullptr;
  int kRG = 0, G = 0;
};

Launch launch_for(int M, int G) {
  if (G == 12) {
    switch (M) {
      case 1: return {k_tensor<1, 3, 12>, 3, 12};
      case 2: return {k_tensor<2, 3, 12>, 3, 12};
      case 3: return {k_tensor<3, 3, 12>, 3, 12};
      case 4: return {k_tensor<4, 3, 12>, 3, 12};
      case 5: return {k_tensor<5, 3, 12>, 3, 12};
      case 6: return {k_tensor<6, 3, 12>, 3, 12};
      default: return {};
    }
  }
  if (G == 8) {
    switch (M) {
      case 1: return {k_tensor<1, 3, 8>, 3, 8};
      case 2: return {k_tensor<2, 3, 8>, 3, 8};
      case 3: return {k_tensor<3, 3, 8>, 3, 8};
      case 4: return {k_tensor<4, 3, 8>, 3, 8};
      case 5: return {k_tensor<5, 3, 8>, 3, 8};
      case 6: return {k_tensor<6, 3, 8>, 3, 8};
      case 7: return {k_tensor<7, 3, 8>, 3, 8};
      case 8: return {k_tensor<8, 3, 8>, 3, 8};
      default: return {};
    }
  }
  if (G == 4) {
    switch (M) {
      case 1: return {k_tensor<1, 4, 4>, 4, 4};
      case 2: return {k_tensor<2, 4, 4>, 4, 4};
      case 3: return {k_tensor<3, 4, 4>, 4, 4};
      case 4: return {k_tensor<4, 4, 4>, 4, 4};
      case 5: return {k_tensor<5, 4, 4>, 4, 4};
      case 6: return {k_tensor<6, 4, 4>, 4, 4};
      case 7: return {k_tensor<7, 4, 4>, 4, 4};
      case 8: return {k_tensor<8, 4, 4>, 4, 4};
      case 16: return {k_tensor<16, 2, 4>, 2, 4};
      default: return {};
    }
  }
  switch (M) {
    case 1: return {k_tensor<1, 16, 1>, 16, 1};
    case 2: return {k_tensor<2, 16, 1>, 16, 1};
    case 4: return {k_tensor<4, 16, 1>, 16, 1};
    case 8: return {k_tensor<8, 16, 1>, 16, 1};
    case 16: return {k_tensor<16, 8, 1>, 8, 1};
    default: return {};
  }
}

}  // namespace

// Device buffers of one grid size, reused across calls.
struct gcs_mi_tensor_plan {
  gamera_mi_solver_config config{};
  int np = 0, nt = 0, csize = 1;
  TensorKernel kernel = nullptr;
  void *pool = nullptr;
  TSys sys{};
  double *d_fac = nullptr, *d_sp = nullptr, *d_sh = nullptr, *d_pot = nullptr;
  size_t smem = 0;
  int band = 0, nbands = 0;  // band schedule of this grid (0: not available)
};

namespace {

void plan_free(gcs_mi_tensor_plan *p) {
  if (!p) return;
  cudaFree(p->pool);
  delete p;
}

cudaLaunchConfig_t launch_config(int csize, size_t smem, cudaStream_t stream,
                                 cudaLaunchAttribute *attr) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)csize);
  cfg.blockDim = dim3((unsigned)kThreads);
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

// Largest cluster (16, 8, 4, 2, 1 CTAs) the device can co-schedule.  The
// kernel's shared-memory limit is set for the widest grid it serves, so a
// plan for a narrower grid never lowers it under an earlier plan's need.
int pick_cluster(const Launch &L, int Rp, size_t smem) {
  size_t most = tensor_smem(L.kRG, L.G, Rp, kMaxLongitudes);
  if (most > kSmemCap) most = kSmemCap;
  if (cudaFuncSetAttribute(L.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)most) !=
      cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  if (cudaFuncSetAttribute(L.kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
      cudaSuccess)
    cudaGetLastError();
  for (int c = kMaxCluster; c >= 1; c >>= 1) {
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = launch_config(c, smem, nullptr, attr);
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, L.kernel, &cfg) == cudaSuccess && n >= 1) return c;
    cudaGetLastError();
  }
  return 0;
}

// True when one cluster of csize CTAs with smem bytes each can run.
bool cluster_fits(TensorKernel k, int csize, size_t smem) {
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = launch_config(csize, smem, nullptr, attr);
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k, &cfg) == cudaSuccess && n >= 1) return true;
  cudaGetLastError();
  return false;
}

gcs_mi_tensor_plan *plan_create(const gamera_mi_solver_config *c) {
  if (!valid_tensor_config(c) || c->colatitude_count - 2U > (size_t)kMaxRows ||
      c->longitude_count > (size_t)kMaxLongitudes) {
    set_api_error("MI tensor grid outside the supported range (at most 512 interior "
                  "colatitude rows and 8192 longitudes)");
    return nullptr;
  }
  gcs_mi_tensor_plan *p = new gcs_mi_tensor_plan();
  p->config = *c;
  const int np = (int)c->longitude_count, nt = (int)c->colatitude_count, R = nt - 2;
  // sweep chains per lane: M = 1..8 or 16 with groups of 4 diagonals, which
  // need the seam np - 1 >= 8 steps after the edge; narrower grids sweep one
  // diagonal per group with M in {1, 2, 4, 8, 16}
  const bool g4 = np >= 9;
  int M = R <= 256 ? (R + 31) / 32 : 16;
  if (!g4) M = M <= 1 ? 1 : M <= 2 ? 2 : M <= 4 ? 4 : M <= 8 ? 8 : 16;
  const int Rp = 32 * M;  // rows of a diagonal
  const int nrows = nt > Rp + 2 ? nt : Rp + 2;  // row table incl. padding rows
  p->np = np;
  p->nt = nt;
  const size_t nodes = (size_t)np * nt;
  const size_t cols = 2 * (size_t)kPad + Rp + np - 1, len = cols * Rp;
  // 12 vectors, 6 coefficient arrays and 2 coefficient pairs, all skewed
  const size_t doubles = 4 * nodes + (12 + 6 + 4) * len + np + 2;
  const size_t bytes = doubles * sizeof(double) + nrows * sizeof(TRow) +
                       sizeof(gamera_mi_solver_stats) + 64;
  if (!cuda_ok(cudaMalloc(&p->pool, bytes), "cudaMalloc") ||
      !cuda_ok(cudaMemset(p->pool, 0, bytes), "cudaMemset")) {
    plan_free(p);
    return nullptr;
  }
  double *q = (double *)p->pool;
  auto take = [&](size_t k) {
    double *r = q;
    q += k;
    return r;
  };
  TSys &S = p->sys;
  // skewed arrays first: len is a multiple of 32, so every diagonal the bulk
  // copies touch starts on a 256-byte boundary
  S.cf = (double2 *)take(2 * len);
  S.cb = (double2 *)take(2 * len);
  double **vecs[] = {&S.rhs, &S.x, &S.res, &S.shd, &S.srch, &S.as, &S.psv, &S.mid,
                     &S.pm, &S.am, &S.fw, &S.pin, &S.dg, &S.lo, &S.up, &S.ll, &S.lu, &S.rdg};
  for (double **v : vecs) *v = take(len);
  p->d_fac = take(nodes);
  p->d_sp = take(nodes);
  p->d_sh = take(nodes);
  p->d_pot = take(nodes);
  S.pe = take(np);
  S.pole_sum = take(2);
  TRow *rows = (TRow *)q;
  S.stats = (gamera_mi_solver_stats *)(rows + nrows);
  S.status = (int *)(S.stats + 1);
  S.fault = S.status + 1;
  const double dth = c->maximum_colatitude / (double)(nt - 1);
  // padding rows carry a unit row weight and nothing else
  std::vector<TRow> hr(nrows, TRow{1.0, 0.0, 0.0, 0.0, 0.0, 0.0});
  for (int i = 0; i < nt; ++i) {
    const double th = (double)i * dth, lth = th - 0.5 * dth, uth = th + 0.5 * dth;
    hr[i] = TRow{sin(th), sin(lth), inc2(lth), sin(uth), inc2(uth),
                 cos_inclination(th, c->hemisphere)};
  }
  if (!cuda_ok(cudaMemcpy(rows, hr.data(), nrows * sizeof(TRow), cudaMemcpyHostToDevice),
               "cudaMemcpy")) {
    plan_free(p);
    return nullptr;
  }
  S.np = np;
  S.nt = nt;
  S.R = R;
  S.Rp = Rp;
  S.max_iter = c->maximum_iterations;
  S.core0 = (unsigned)(kPad * (size_t)Rp);
  S.core1 = (unsigned)((kPad + (size_t)Rp + np - 1) * Rp);
  S.dth = dth;
  S.dph = 2.0 * acos(-1.0) / (double)np;
  S.neg_r2 = -(c->ionosphere_radius_m * c->ionosphere_radius_m);
  // pole edge of the constant-Pedersen system scales the pole residual
  // (nonorthogonal_mi.c:324-334, :415-431)
  const double th = 0.5 * dth;
  S.pole_sin = sin(th);
  S.pole_inc2 = inc2(th);
  S.ps = (double)np * (sin(th) * c->pedersen_siemens / (inc2(th) * dth * dth));
  S.abs_tol = c->absolute_tolerance;
  S.rel_tol = c->relative_tolerance;
  S.rows = rows;
  S.fac = p->d_fac;
  S.sp = p->d_sp;
  S.sh = p->d_sh;
  S.pot = p->d_pot;
  // (groups of 16 diagonals in a 2-slot ring were tried: 181 x 361 took
  // 470 ms against 192 ms, each group waiting for its whole copy)
  const int G = !g4 ? 1
                : np >= 25 && M <= 6 && tensor_smem(3, 12, Rp, np) <= kSmemCap ? 12
                : np >= 17 && M <= 8 && tensor_smem(3, 8, Rp, np) <= kSmemCap  ? 8
                                                                                 : 4;
  const Launch L = launch_for(M, G);
  p->kernel = L.kernel;
  p->smem = tensor_smem(L.kRG, L.G, Rp, np);
  p->csize = L.kernel ? pick_cluster(L, Rp, p->smem) : 0;
  if (p->csize == 0) {
    set_api_error("no thread-block cluster shape for the MI tensor solve");
    plan_free(p);
    return nullptr;
  }
  // band schedule: one band of at most 32 rows per CTA, its coefficient
  // tables in shared memory beside the ring's room.  The default on grids
  // of fewer than 17 longitudes, where the one-warp sweep cannot move its
  // diagonals in groups of 8 and the band pipeline measured faster (B200:
  // 70 x 12 7.5 -> 5.7 ms, 12 x 8 1.3 -> 0.4 ms, 40 x 5 7.6 -> 2.1 ms); on
  // wider grids the one warp is faster (181 x 361: 163 against 224 ms) and
  // the band schedule is available through gcs_mi_tensor_plan_set_schedule.
  if (p->csize >= 2) {
    const int h = (R + p->csize - 1) / p->csize;
    const size_t need = std::max(p->smem, band_smem(h, np));
    if (h <= 32 && need <= kSmemCap && cluster_fits(p->kernel, p->csize, need)) {
      p->smem = need;
      p->band = h;
      p->nbands = (R + h - 1) / h;
      if (np < 17) {
        S.band = p->band;
        S.nbands = p->nbands;
      }
    }
  }
  return p;
}

std::mutex g_mutex;
gcs_mi_tensor_plan *g_cache = nullptr;

}  // namespace

extern "C" {

int gcs_mi_tensor_plan_create(const gamera_mi_solver_config *config,
                              gcs_mi_tensor_plan **plan) {
  if (!plan) return -1;
  *plan = plan_create(config);
  return *plan ? 0 : -1;
}

int gcs_mi_tensor_plan_set_ordering(gcs_mi_tensor_plan *plan, int colored) {
  if (!plan || (colored != 0 && colored != 1)) return -1;
  plan->sys.colored = colored;
  return 0;
}

int gcs_mi_tensor_plan_set_schedule(gcs_mi_tensor_plan *plan, int banded) {
  if (!plan || (banded != 0 && banded != 1) || (banded && plan->band == 0)) return -1;
  plan->sys.band = banded ? plan->band : 0;
  plan->sys.nbands = banded ? plan->nbands : 0;
  return 0;
}

int gcs_mi_tensor_plan_schedule(const gcs_mi_tensor_plan *plan, int *rows_per_band,
                                int *bands) {
  if (!plan) return -1;
  if (rows_per_band) *rows_per_band = plan->sys.band;
  if (bands) *bands = plan->sys.nbands;
  return plan->sys.band ? 1 : 0;
}

void gcs_mi_tensor_plan_destroy(gcs_mi_tensor_plan *plan) {
  if (plan) cudaDeviceSynchronize();
  plan_free(plan);
}

int gcs_mi_tensor_plan_buffers(gcs_mi_tensor_plan *plan, double **fac, double **pedersen,
                               double **hall, double **potential) {
  if (!plan) return -1;
  if (fac) *fac = plan->d_fac;
  if (pedersen) *pedersen = plan->d_sp;
  if (hall) *hall = plan->d_sh;
  if (potential) *potential = plan->d_pot;
  return 0;
}

// Copies host FAC, conductances and the initial potential into the plan.
int gcs_mi_tensor_plan_upload(gcs_mi_tensor_plan *plan, const double *fac,
                              const double *pedersen, const double *hall,
                              const double *potential) {
  if (!plan || !fac || !pedersen || !hall || !potential) return -1;
  const size_t bytes = (size_t)plan->np * plan->nt * sizeof(double);
  return cuda_ok(cudaMemcpy(plan->d_fac, fac, bytes, cudaMemcpyHostToDevice), "cudaMemcpy") &&
                 cuda_ok(cudaMemcpy(plan->d_sp, pedersen, bytes, cudaMemcpyHostToDevice),
                         "cudaMemcpy") &&
                 cuda_ok(cudaMemcpy(plan->d_sh, hall, bytes, cudaMemcpyHostToDevice),
                         "cudaMemcpy") &&
                 cuda_ok(cudaMemcpy(plan->d_pot, potential, bytes, cudaMemcpyHostToDevice),
                         "cudaMemcpy")
             ? 0
             : -1;
}

// Solve on the plan's buffers (inputs already there), asynchronously.
int gcs_mi_tensor_solve_async(gcs_mi_tensor_plan *plan, void *stream) {
  if (!plan) return -1;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = launch_config(plan->csize, plan->smem, (cudaStream_t)stream, attr);
  return cuda_ok(cudaLaunchKernelEx(&cfg, plan->kernel, plan->sys), "MI tensor solve launch")
             ? 0
             : -1;
}

int gcs_mi_tensor_results(gcs_mi_tensor_plan *plan, gamera_mi_solver_stats *stats,
                          int *status) {
  if (!plan || !cuda_ok(cudaDeviceSynchronize(), "MI tensor solve")) return -1;
  if (stats && !cuda_ok(cudaMemcpy(stats, plan->sys.stats, sizeof(*stats),
                                   cudaMemcpyDeviceToHost), "cudaMemcpy"))
    return -1;
  if (status && !cuda_ok(cudaMemcpy(status, plan->sys.status, sizeof(int),
                                    cudaMemcpyDeviceToHost), "cudaMemcpy"))
    return -1;
  return 0;
}

// Drop-in for nonorthogonal_mi.c:966 (host arrays, synchronous).
int gamera_mi_solve_conductance_tensor(const gamera_mi_solver_config *config,
                                       const double *fac_a_m2, const double *pedersen,
                                       const double *hall, double *potential_v,
                                       gamera_mi_solver_stats *stats) {
  if (!valid_tensor_config(config) || pedersen == nullptr || hall == nullptr ||
      fac_a_m2 == nullptr || potential_v == nullptr) {
    set_api_error("invalid MI tensor solve arguments");
    return -1;
  }
  const size_t nodes = config->longitude_count * config->colatitude_count;
  for (size_t q = 0; q < nodes; ++q)
    if (!std::isfinite(pedersen[q]) || !(pedersen[q] > 0.0) || !std::isfinite(hall[q]) ||
        hall[q] < 0.0) {
      set_api_error("invalid conductance");
      return -1;
    }
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_cache || memcmp(&g_cache->config, config, sizeof(*config)) != 0) {
    gcs_mi_tensor_plan *p = plan_create(config);
    if (!p) return -1;
    plan_free(g_cache);
    g_cache = p;
  }
  gcs_mi_tensor_plan *p = g_cache;
  const size_t bytes = nodes * sizeof(double);
  int status = 2;
  gamera_mi_solver_stats s = {};
  if (!cuda_ok(cudaMemcpy(p->d_fac, fac_a_m2, bytes, cudaMemcpyHostToDevice), "cudaMemcpy") ||
      !cuda_ok(cudaMemcpy(p->d_sp, pedersen, bytes, cudaMemcpyHostToDevice), "cudaMemcpy") ||
      !cuda_ok(cudaMemcpy(p->d_sh, hall, bytes, cudaMemcpyHostToDevice), "cudaMemcpy") ||
      !cuda_ok(cudaMemcpy(p->d_pot, potential_v, bytes, cudaMemcpyHostToDevice),
               "cudaMemcpy") ||
      gcs_mi_tensor_solve_async(p, nullptr) != 0 ||
      gcs_mi_tensor_results(p, &s, &status) != 0 ||
      !cuda_ok(cudaMemcpy(potential_v, p->d_pot, bytes, cudaMemcpyDeviceToHost),
               "cudaMemcpy"))
    return -1;
  if (status == 2) {
    set_api_error("non-finite field-aligned current");
    return -1;
  }
  if (status == 3) {
    set_api_error("MI tensor solve: a sweep copy did not arrive within the wait limit");
    return -1;
  }
  if (stats) *stats = s;
  return status == 0 ? 0 : -1;
}

}  // extern "C"
