// Ionosphere potential with the variable Pedersen + Hall conductance tensor
// (nonorthogonal/src/nonorthogonal/nonorthogonal_mi.c:611-1151): the cached
// five-point stencil, BiCGStab with restarts every 256 iterations, and the
// symmetric Gauss-Seidel (SSOR) preconditioner, on one CTA.
//
// The preconditioner is a lexicographic forward sweep and a reverse sweep.
// Point (i, j) of the forward sweep depends on (i-1, j), (i, j-1) and, on
// the periodic seam, (i, 0): every point of an anti-diagonal i + j = const
// is independent of the others on it.  Thread t owns colatitude row t + 1
// and advances one longitude per step, one row behind the row below it, so
// the rows sweep as a wavefront; each point is computed with the
// reference's operations in the reference's order, so the preconditioner
// output is bitwise the reference's for the same input.  The row's
// coefficients stream into a per-thread shared-memory ring with cp.async
// eight steps ahead; neighbouring rows exchange their last value through
// shared memory and a named barrier over the sweeping warps.  The vector
// updates, stencil applications and dot products run on all threads of the
// CTA (dot products summed in a fixed parallel order, so the BiCGStab
// iterates differ from the CPU solver's at rounding level).
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "gamera_cs_b200.h"
#include "gcs_error.h"

using gcs::set_api_error;

namespace {

constexpr int kT = 512;           // threads of the CTA
constexpr int kWarps = kT / 32;
constexpr int kAhead = 8;         // cp.async lookahead of the sweeps
constexpr int kRestart = 256;
constexpr int kMaxIterations = 1 << 20;

// Per-row constants of the full polar grid, computed on the host with the
// reference's formulas (nonorthogonal_mi.c:643-656, :776-865).
struct TRow {
  double s;        // sin(theta)
  double sl, il;   // sin and inclination^2 at theta - dtheta/2
  double su, iu;   // sin and inclination^2 at theta + dtheta/2
  double inc;      // dipole cos(inclination)
};

struct TSys {
  int np, nt, max_iter, pad;
  double dth, dph, neg_r2, pole_sin, pole_inc2, ps, abs_tol, rel_tol;
  const TRow *rows;
  const double *fac, *sp, *sh;
  double *pot;
  double *rhs, *x, *res, *shd, *srch, *as, *ps_v, *mid, *pm, *am, *fw;
  double *dg, *lo, *up, *ll, *lu, *pe;
  gamera_mi_solver_stats *stats;
  int *status;  // 0 converged, 1 not converged, 2 non-finite FAC
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the CTA; every thread receives the same value.
template <int N>
__device__ __forceinline__ void block_sum(double (&v)[N], double *wbuf) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < N; ++q) {
    v[q] = warp_sum(v[q]);
    if (lane == 0) wbuf[warp * 4 + q] = v[q];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < N; ++q) v[q] = warp_sum(lane < kWarps ? wbuf[lane * 4 + q] : 0.0);
  __syncthreads();
}

__device__ __forceinline__ void sweep_barrier(int n) {
  asm volatile("bar.sync 1, %0;" ::"r"(n) : "memory");
}

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;"); }
__device__ __forceinline__ void cp_wait_ahead() {
  asm volatile("cp.async.wait_group %0;" ::"n"(kAhead - 1) : "memory");
}

__device__ __forceinline__ size_t red(int np, int i, int j) {
  return 1 + (size_t)(i - 1) * np + j;
}

__device__ __forceinline__ double f12(const TSys &S, int i, int j) {
  return -S.sh[(size_t)i * S.np + j] / S.rows[i].inc;
}

// A p (nonorthogonal_mi.c:867-900); the pole row by one thread in order.
__device__ void apply(const TSys &S, const double *p, double *r) {
  const int np = S.np, nt = S.nt;
  const size_t n = 1 + (size_t)np * (nt - 2);
  for (size_t q = 1 + threadIdx.x; q < n; q += kT) {
    const int i = 1 + (int)((q - 1) / np), j = (int)((q - 1) % np);
    const int jm = j == 0 ? np - 1 : j - 1, jp = j + 1 == np ? 0 : j + 1;
    const double lv = i == 1 ? p[0] : p[red(np, i - 1, j)];
    const double uv = i + 2 < nt ? p[red(np, i + 1, j)] : 0.0;
    r[q] = S.dg[q] * p[q] + S.lo[q] * lv + S.up[q] * uv + S.ll[q] * p[red(np, i, jm)] +
           S.lu[q] * p[red(np, i, jp)];
  }
  if (threadIdx.x == 0) {
    double r0 = S.dg[0] * p[0];
    for (int j = 0; j < np; ++j) r0 -= S.pe[j] * p[red(np, 1, j)];
    r[0] = r0;
  }
  __syncthreads();
}

// Symmetric Gauss-Seidel of nonorthogonal_mi.c:910-964 as two wavefronts.
// ring: per-thread kAhead x 4 doubles of shared memory; xch: 2 x kT.
__device__ void ssor(const TSys &S, const double *in, double *out, double *ring,
                     double *xch) {
  const int np = S.np, R = S.nt - 2, t = threadIdx.x;
  const int sweepers = ((R + 31) / 32) * 32;
  double *fw = S.fw;
  if (t == 0) fw[0] = in[0] / S.dg[0];
  __syncthreads();
  if (t < sweepers) {
    const bool row = t < R;
    const int i = t + 1;
    double *my = ring + (size_t)t * kAhead * 4;
    // forward: thread t handles column j = s - t at step s
    auto fetch_f = [&](int j) {
      if (row && j >= 0 && j < np) {
        const size_t c = red(np, i, j);
        double *slot = my + (j % kAhead) * 4;
        cp_async8(slot + 0, in + c);
        cp_async8(slot + 1, S.lo + c);
        cp_async8(slot + 2, S.ll + c);
        cp_async8(slot + 3, j + 1 == np ? S.lu + c : S.dg + c);
      }
      cp_commit();
    };
    for (int u = 0; u < kAhead; ++u) fetch_f(u);
    const double pole = fw[0];
    double left = 0.0, first = 0.0;
    const int steps = R + np - 1;
    for (int s = 0; s < steps; ++s) {
      const int j = s - t;
      cp_wait_ahead();
      double v = 0.0;
      if (row && j >= 0 && j < np) {
        const size_t c = red(np, i, j);
        const double *slot = my + (j % kAhead) * 4;
        const double below = i == 1 ? pole : xch[((s + 1) & 1) * kT + t - 1];
        v = slot[0];
        v -= slot[1] * below;
        if (j > 0) v -= slot[2] * left;
        const double dg = j + 1 == np ? S.dg[c] : slot[3];
        if (j + 1 == np) v -= slot[3] * first;
        v = v / dg;
        fw[c] = v;
        left = v;
        if (j == 0) first = v;
      }
      fetch_f(j + kAhead);
      xch[(s & 1) * kT + t] = v;
      sweep_barrier(sweepers);
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    sweep_barrier(sweepers);
    // reverse: thread t handles column j = np - 1 - (s - (R - 1 - t))
    auto col_b = [&](int s) { return np - 1 - (s - (R - 1 - t)); };
    auto fetch_b = [&](int j) {
      if (row && j >= 0 && j < np) {
        const size_t c = red(np, i, j);
        double *slot = my + (j % kAhead) * 4;
        cp_async8(slot + 0, fw + c);
        cp_async8(slot + 1, S.up + c);
        cp_async8(slot + 2, S.lu + c);
        cp_async8(slot + 3, j == 0 ? S.ll + c : S.dg + c);
      }
      cp_commit();
    };
    for (int u = 0; u < kAhead; ++u) fetch_b(col_b(u));
    double right = 0.0, last = 0.0;
    for (int s = 0; s < steps; ++s) {
      const int j = col_b(s);
      cp_wait_ahead();
      double v = 0.0;
      if (row && j >= 0 && j < np) {
        const size_t c = red(np, i, j);
        const double *slot = my + (j % kAhead) * 4;
        const double dg = j == 0 ? S.dg[c] : slot[3];
        v = dg * slot[0];
        if (i + 2 < S.nt) v -= slot[1] * xch[((s + 1) & 1) * kT + t + 1];
        if (j + 1 < np) v -= slot[2] * right;
        if (j == 0) v -= slot[3] * last;
        v = v / dg;
        out[c] = v;
        right = v;
        if (j + 1 == np) last = v;
      }
      fetch_b(col_b(s + kAhead));
      xch[(s & 1) * kT + t] = v;
      sweep_barrier(sweepers);
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
  }
  __syncthreads();
  if (t == 0) {
    double pv = S.dg[0] * fw[0];
    for (int j = 0; j < np; ++j) pv += S.pe[j] * out[red(np, 1, j)];
    out[0] = pv / S.dg[0];
  }
  __syncthreads();
}

// nonorthogonal_mi.c:415-431 (unweighted rows; pole scaled by ps)
__device__ double norm2_part(const TSys &S, const double *r) {
  const int np = S.np;
  const size_t n = 1 + (size_t)np * (S.nt - 2);
  double a = 0.0;
  for (size_t q = 1 + threadIdx.x; q < n; q += kT) {
    const int i = 1 + (int)((q - 1) / np);
    const double v = r[q] / S.rows[i].s;
    a += v * v;
  }
  if (threadIdx.x == 0) {
    const double pr = r[0] / S.ps;
    a += (double)np * pr * pr;
  }
  return a;
}

__global__ void __launch_bounds__(kT, 1) k_bicgstab(TSys S) {
  extern __shared__ __align__(16) double ring[];
  __shared__ double wbuf[kWarps * 4];
  __shared__ double xch[2 * kT];
  __shared__ double ppm_s;
  const int np = S.np, nt = S.nt, t = threadIdx.x;
  const size_t n = 1 + (size_t)np * (nt - 2);

  // cached stencil (nonorthogonal_mi.c:776-865)
  if (t == 0) {
    double m = 0.0;
    for (int j = 0; j < np; ++j) m += S.sp[j] / (double)np;
    ppm_s = m;
  }
  __syncthreads();
  for (int j = t; j < np; j += kT) {
    const double fp = 0.5 * (ppm_s + S.sp[(size_t)np + j]);
    S.pe[j] = S.pole_sin * fp / (S.pole_inc2 * S.dth * S.dth);
  }
  for (size_t q = 1 + t; q < n; q += kT) {
    const int i = 1 + (int)((q - 1) / np), j = (int)((q - 1) % np);
    const int jm = j == 0 ? np - 1 : j - 1, jp = j + 1 == np ? 0 : j + 1;
    const TRow &R = S.rows[i];
    const size_t full = (size_t)i * np + j;
    const double *P = S.sp;
    const double lower =
        R.sl * 0.5 * (P[full] + P[full - np]) / (R.il * S.dth * S.dth);
    const double upper =
        R.su * 0.5 * (P[full] + P[full + np]) / (R.iu * S.dth * S.dth);
    const double llo = 0.5 * (P[full] + P[(size_t)i * np + jm]) / (R.s * S.dph * S.dph);
    const double lup = 0.5 * (P[full] + P[(size_t)i * np + jp]) / (R.s * S.dph * S.dph);
    S.dg[q] = lower + upper + llo + lup;
    const double dft = (f12(S, i + 1, j) - f12(S, i - 1, j)) / (2.0 * S.dth);
    const double dfp = (f12(S, i, jp) - f12(S, i, jm)) / (2.0 * S.dph);
    S.lo[q] = -lower - dfp / (2.0 * S.dth);
    S.up[q] = -upper + dfp / (2.0 * S.dth);
    S.ll[q] = -llo + dft / (2.0 * S.dph);
    S.lu[q] = -lup - dft / (2.0 * S.dph);
  }
  __syncthreads();
  if (t == 0) {
    double d0 = 0.0;
    for (int j = 0; j < np; ++j) d0 += S.pe[j];
    S.dg[0] = d0;
  }
  // right-hand side and initial guess (nonorthogonal_mi.c:999-1029)
  double v3[3] = {0.0, 0.0, 0.0};  // rhs^2, bad
  for (size_t q = 1 + t; q < n; q += kT) {
    const int i = 1 + (int)((q - 1) / np), j = (int)((q - 1) % np);
    const double f = S.fac[(size_t)i * np + j];
    const double u = S.neg_r2 * f * S.rows[i].inc;
    S.rhs[q] = S.rows[i].s * u;
    v3[0] += u * u;
    v3[1] += isfinite(f) ? 0.0 : 1.0;
    const double g = S.pot[(size_t)i * np + j];
    S.x[q] = isfinite(g) ? g : 0.0;
  }
  if (t == 0) {
    double m = 0.0;
    for (int j = 0; j < np; ++j) {
      const double g = S.pot[j];
      if (isfinite(g)) m += g / (double)np;
    }
    S.x[0] = m;
    S.rhs[0] = 0.0;
  }
  block_sum<3>(v3, wbuf);
  const bool bad = v3[1] > 0.0;
  const double target = fmax(S.abs_tol, S.rel_tol * fmax(sqrt(fmax(0.0, v3[0])), 1.0));
  apply(S, S.x, S.as);
  for (size_t q = t; q < n; q += kT) {
    const double r = S.rhs[q] - S.as[q];
    S.res[q] = r;
    S.shd[q] = r;
    S.srch[q] = 0.0;
    S.as[q] = 0.0;
  }
  __syncthreads();
  double nv[1] = {norm2_part(S, S.res)};
  block_sum<1>(nv, wbuf);
  const double initial = sqrt(fmax(0.0, nv[0]));
  double final_res = initial;
  int iters = 0;
  int conv = initial <= target;
  double rho_prev = 1.0, alpha = 1.0, omega = 1.0;
  const int max_iter = S.max_iter < kMaxIterations ? S.max_iter : kMaxIterations;
  // BiCGStab (nonorthogonal_mi.c:1040-1128)
  for (int it = 1; !bad && !conv && it <= max_iter; ++it) {
    double d1[1] = {0.0};
    for (size_t q = t; q < n; q += kT) d1[0] += S.shd[q] * S.res[q];
    block_sum<1>(d1, wbuf);
    const double rho = d1[0];
    if (!isfinite(rho) || fabs(rho) <= DBL_MIN || !isfinite(omega) || fabs(omega) <= DBL_MIN)
      break;
    const double beta = (rho / rho_prev) * (alpha / omega);
    for (size_t q = t; q < n; q += kT)
      S.srch[q] = S.res[q] + beta * (S.srch[q] - omega * S.as[q]);
    __syncthreads();
    ssor(S, S.srch, S.ps_v, ring, xch);
    apply(S, S.ps_v, S.as);
    double d2[1] = {0.0};
    for (size_t q = t; q < n; q += kT) d2[0] += S.shd[q] * S.as[q];
    block_sum<1>(d2, wbuf);
    if (!isfinite(d2[0]) || fabs(d2[0]) <= DBL_MIN) break;
    alpha = rho / d2[0];
    for (size_t q = t; q < n; q += kT) S.mid[q] = S.res[q] - alpha * S.as[q];
    __syncthreads();
    double d3[1] = {norm2_part(S, S.mid)};
    block_sum<1>(d3, wbuf);
    final_res = sqrt(fmax(0.0, d3[0]));
    if (final_res <= target) {
      for (size_t q = t; q < n; q += kT) S.x[q] += alpha * S.ps_v[q];
      __syncthreads();
      iters = it;
      conv = 1;
      break;
    }
    ssor(S, S.mid, S.pm, ring, xch);
    apply(S, S.pm, S.am);
    double d4[2] = {0.0, 0.0};
    for (size_t q = t; q < n; q += kT) {
      d4[0] += S.am[q] * S.am[q];
      d4[1] += S.am[q] * S.mid[q];
    }
    block_sum<2>(d4, wbuf);
    if (!isfinite(d4[0]) || d4[0] <= DBL_MIN) break;
    omega = d4[1] / d4[0];
    if (!isfinite(omega) || fabs(omega) <= DBL_MIN) break;
    for (size_t q = t; q < n; q += kT) {
      S.x[q] += alpha * S.ps_v[q] + omega * S.pm[q];
      S.res[q] = S.mid[q] - omega * S.am[q];
    }
    __syncthreads();
    double d5[1] = {norm2_part(S, S.res)};
    block_sum<1>(d5, wbuf);
    final_res = sqrt(fmax(0.0, d5[0]));
    iters = it;
    if (final_res <= target || it % kRestart == 0) {
      apply(S, S.x, S.am);
      for (size_t q = t; q < n; q += kT) S.res[q] = S.rhs[q] - S.am[q];
      __syncthreads();
      double d6[1] = {norm2_part(S, S.res)};
      block_sum<1>(d6, wbuf);
      final_res = sqrt(fmax(0.0, d6[0]));
      if (final_res <= target) {
        conv = 1;
        break;
      }
      for (size_t q = t; q < n; q += kT) {
        S.shd[q] = S.res[q];
        S.srch[q] = 0.0;
        S.as[q] = 0.0;
      }
      __syncthreads();
      rho_prev = 1.0;
      alpha = 1.0;
      omega = 1.0;
      continue;
    }
    rho_prev = rho;
  }
  if (bad) {
    if (t == 0) *S.status = 2;
    return;
  }
  // expand (nonorthogonal_mi.c:1130-1139); low-latitude potential is 0
  for (size_t q = 1 + t; q < n; q += kT) {
    const int i = 1 + (int)((q - 1) / np), j = (int)((q - 1) % np);
    S.pot[(size_t)i * np + j] = S.x[q];
  }
  for (int j = t; j < np; j += kT) {
    S.pot[j] = S.x[0];
    S.pot[(size_t)(nt - 1) * np + j] = 0.0;
  }
  if (t == 0) {
    *S.stats = gamera_mi_solver_stats{iters, initial, final_res, conv};
    *S.status = conv ? 0 : 1;
  }
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

}  // namespace

// Device buffers of one grid size, reused across calls.
struct gcs_mi_tensor_plan {
  gamera_mi_solver_config config{};
  int np = 0, nt = 0;
  void *pool = nullptr;
  TSys sys{};
  double *d_fac = nullptr, *d_sp = nullptr, *d_sh = nullptr, *d_pot = nullptr;
  size_t smem = 0;
};

namespace {

void plan_free(gcs_mi_tensor_plan *p) {
  if (!p) return;
  cudaFree(p->pool);
  delete p;
}

gcs_mi_tensor_plan *plan_create(const gamera_mi_solver_config *c) {
  if (!valid_tensor_config(c) || c->colatitude_count - 2U > (size_t)kT ||
      c->longitude_count > (SIZE_MAX - 1U) / (c->colatitude_count - 2U)) {
    set_api_error("invalid or too tall MI tensor grid (at most 512 interior rows)");
    return nullptr;
  }
  gcs_mi_tensor_plan *p = new gcs_mi_tensor_plan();
  p->config = *c;
  const int np = (int)c->longitude_count, nt = (int)c->colatitude_count;
  p->np = np;
  p->nt = nt;
  const size_t nodes = (size_t)np * nt, n = 1 + (size_t)np * (nt - 2);
  const size_t doubles = 4 * nodes + 17 * n + np;
  const size_t bytes = doubles * sizeof(double) + nt * sizeof(TRow) +
                       sizeof(gamera_mi_solver_stats) + 64;
  if (!cuda_ok(cudaMalloc(&p->pool, bytes), "cudaMalloc")) {
    plan_free(p);
    return nullptr;
  }
  double *q = (double *)p->pool;
  auto take = [&](size_t k) {
    double *r = q;
    q += k;
    return r;
  };
  p->d_fac = take(nodes);
  p->d_sp = take(nodes);
  p->d_sh = take(nodes);
  p->d_pot = take(nodes);
  TSys &S = p->sys;
  S.rhs = take(n);
  S.x = take(n);
  S.res = take(n);
  S.shd = take(n);
  S.srch = take(n);
  S.as = take(n);
  S.ps_v = take(n);
  S.mid = take(n);
  S.pm = take(n);
  S.am = take(n);
  S.fw = take(n);
  S.dg = take(n);
  S.lo = take(n);
  S.up = take(n);
  S.ll = take(n);
  S.lu = take(n);
  take(n);  // spare (keeps the row table 8-byte aligned past the vectors)
  S.pe = take(np);
  TRow *rows = (TRow *)q;
  S.stats = (gamera_mi_solver_stats *)(rows + nt);
  S.status = (int *)(S.stats + 1);
  const double dth = c->maximum_colatitude / (double)(nt - 1);
  std::vector<TRow> hr(nt);
  for (int i = 0; i < nt; ++i) {
    const double th = (double)i * dth, lth = th - 0.5 * dth, uth = th + 0.5 * dth;
    hr[i] = TRow{sin(th), sin(lth), inc2(lth), sin(uth), inc2(uth),
                 cos_inclination(th, c->hemisphere)};
  }
  if (!cuda_ok(cudaMemcpy(rows, hr.data(), nt * sizeof(TRow), cudaMemcpyHostToDevice),
               "cudaMemcpy")) {
    plan_free(p);
    return nullptr;
  }
  S.np = np;
  S.nt = nt;
  S.max_iter = c->maximum_iterations;
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
  p->smem = (size_t)kT * kAhead * 4 * sizeof(double);
  if (!cuda_ok(cudaFuncSetAttribute(k_bicgstab, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)p->smem),
               "cudaFuncSetAttribute")) {
    plan_free(p);
    return nullptr;
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
  k_bicgstab<<<1, kT, plan->smem, (cudaStream_t)stream>>>(plan->sys);
  return cuda_ok(cudaGetLastError(), "MI tensor solve launch") ? 0 : -1;
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
  if (stats) *stats = s;
  return status == 0 ? 0 : -1;
}

}  // extern "C"
