// Device Earth radial boundary (no-MI wall) for the six-face step: the
// reference callbacks gamera_cs_earth_fill_radial_ghosts,
// gamera_cs_earth_inner_fluid_flux and gamera_cs_earth_no_mi_emf
// (cubedsphere/cubedsphere_earth_boundary.c) and the solar-wind sampling
// they call (nonorthogonal/src/solar_wind.c), restated as kernels with the
// reference's operation order.  One thread per boundary cell, face or edge;
// all six faces in one launch.  A failure (invalid state, wind sample or
// area) records the host-callback stage, as the reference callback's -1
// fails the step.
#include "gcs_context.h"
#include "gcs_earth.h"
#include "gcs_error.h"
#include "gamera_cs_b200.h"

#include <cfloat>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <utility>
#include <vector>

#include "gcs_kernel_util.cuh"
#include "gcs_physics.cuh"

namespace gcs {
namespace {

struct WindState {
  double rho, p, v[3], b[3];
};

__host__ __device__ inline WindState wind_load(const WindDev &w, int q) {
  const double *a = w.state + 8LL * q;
  WindState s;
  s.rho = a[0];
  s.p = a[1];
  for (int c = 0; c < 3; ++c) {
    s.v[c] = a[2 + c];
    s.b[c] = a[5 + c];
  }
  return s;
}

// solar_wind.c:8-22
__host__ __device__ inline bool wind_finite(const WindState &s) {
  if (!isfinite(s.rho) || !isfinite(s.p) || s.rho <= 0.0 || s.p <= 0.0) return false;
  for (int c = 0; c < 3; ++c)
    if (!isfinite(s.v[c]) || !isfinite(s.b[c])) return false;
  return fabs(s.v[0]) > DBL_MIN;
}

// solar_wind.c:134-160 (binary search of :104-117, interpolation :119-132)
__host__ __device__ bool wind_sample_time(const WindDev &w, double time, WindState *out) {
  if (!isfinite(time)) return false;
  if (w.count == 1 || time <= w.time[0]) {
    *out = wind_load(w, 0);
    return true;
  }
  if (time >= w.time[w.count - 1]) {
    *out = wind_load(w, w.count - 1);
    return true;
  }
  int lo = 0, hi = w.count - 1;
  while (hi - lo > 1) {
    const int mid = lo + (hi - lo) / 2;
    if (w.time[mid] <= time)
      lo = mid;
    else
      hi = mid;
  }
  const WindState a = wind_load(w, lo);
  if (!w.linear) {
    *out = a;
    return true;
  }
  const WindState z = wind_load(w, lo + 1);
  const double fr = (time - w.time[lo]) / (w.time[lo + 1] - w.time[lo]);
  out->rho = a.rho + fr * (z.rho - a.rho);
  out->p = a.p + fr * (z.p - a.p);
  for (int c = 0; c < 3; ++c) {
    out->v[c] = a.v[c] + fr * (z.v[c] - a.v[c]);
    out->b[c] = a.b[c] + fr * (z.b[c] - a.b[c]);
  }
  return wind_finite(*out);
}

// Planar-front ballistic mapping, solar_wind.c:162-200.
__host__ __device__ bool wind_sample_at(const WindDev &w, const double x[3], double t,
                               WindState *out) {
  if (!isfinite(t)) return false;
  const double monitor = t + w.time_offset;
  WindState cur;
  if (!wind_sample_time(w, monitor, &cur)) return false;
  const double csq = w.by * w.by + w.bz * w.bz;
  const double factor = cur.v[0] / (1.0 + csq);
  const double fv[3] = {factor, -factor * w.by, -factor * w.bz};
  double s2 = 0.0, proj = 0.0;
  for (int c = 0; c < 3; ++c) {
    if (!isfinite(x[c])) return false;
    s2 += fv[c] * fv[c];
    proj += (x[c] - w.reference[c]) * fv[c];
  }
  if (!(s2 > DBL_MIN) || !isfinite(s2)) return false;
  const double delay = proj / s2;
  return wind_sample_time(w, monitor - delay, out);
}

// Upstream-to-tail weight, solar_wind.c:202-225, on the state the mapping
// returns for the same point and time.
__host__ __device__ bool wind_weight(const double x[3], const WindState &s, double *weight) {
  double r2 = 0.0, v2 = 0.0, cosine = 0.0;
  for (int c = 0; c < 3; ++c) {
    r2 += x[c] * x[c];
    v2 += s.v[c] * s.v[c];
    cosine -= x[c] * s.v[c];
  }
  if (!(r2 > DBL_MIN) || !(v2 > DBL_MIN)) return false;
  cosine /= sqrt(r2 * v2);
  cosine = fmax(-1.0, fmin(1.0, cosine));
  const double angle = acos(cosine);
  const double half_pi = 0.5 * acos(-1.0);
  if (angle <= half_pi) {
    *weight = 1.0;
  } else if (angle >= 2.0 * half_pi) {
    *weight = 0.0;
  } else {
    const double sc = (angle - half_pi) / half_pi;
    *weight = exp(1.0 - 1.0 / (1.0 - sc * sc));
  }
  return true;
}

// cubedsphere_earth_boundary.c:16-25
__host__ __device__ inline bool sample_wind(const WindDev &w, const double x[3], double t,
                                   WindState *s, double *weight) {
  return wind_sample_at(w, x, t, s) && wind_weight(x, *s, weight);
}

// Times of a launch: the host's values, or the driver-mode values in the
// step parameters (prm non-null).
__device__ inline double radial_time(const StepParams *prm, double time, int old) {
  if (prm == nullptr) return time;
  return old && prm->step > 0 ? prm->time - prm->dt_prev : prm->time;
}

__device__ inline long long plane(const Dims &D, int f, int layers, int l, int j, int k) {
  return (((long long)f * layers + l) * D.N1 + j) * D.N2 + k;
}

// Radial ghost cells of U (old = 0) or U_old (old = 1),
// cubedsphere_earth_boundary.c:27-112: inner ghosts mirror the first active
// layers with the normal velocity reversed (or zero velocity on the strict
// wall); outer ghosts take the last active cell, raise a subsonic outward
// velocity to the sound speed and blend with the sampled wind.
__global__ void k_earth_cells(Dims D, DevState S, EarthDev E, double time, int old,
                              const StepParams *prm, DevStatus *st) {
  if (failed(st)) return;
  time = radial_time(prm, time, old);
  const int jk = blockIdx.x * blockDim.x + threadIdx.x;
  if (jk >= D.E1 * D.E2) return;
  const int l = blockIdx.y, f = blockIdx.z;
  const int j = jk / D.E2, k = jk % D.E2;
  const int outer = D.g + D.nr;
  const bool inner = l < D.g;
  const int i = inner ? l : outer + (l - D.g);
  const int si = inner ? 2 * D.g - 1 - i : outer - 1;
  double *const *U = old ? S.Uo : S.U;
  const long long src = f * D.Nn + D.node(si, j, k);
  const long long dst = f * D.Nn + D.node(i, j, k);
  double u[5];
  for (int m = 0; m < 5; ++m) u[m] = U[m][src];
  Prim p;
  if (cons_to_prim(u, E.gamma, E.rho_floor, E.p_floor, &p)) {
    fail(st, kStageHost, 0, f, i, j, k);
    return;
  }
  const long long q = plane(D, f, 2 * D.g, l, j, k);
  const double x[3] = {E.cell_cen[0][q], E.cell_cen[1][q], E.cell_cen[2][q]};
  const double radius = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  if (!(radius > 0.0)) {
    fail(st, kStageHost, 0, f, i, j, k);
    return;
  }
  double v[3] = {p.vx, p.vy, p.vz};
  if (inner) {
    if (E.mi) {
      const gamera_no_vec3 pt = {{x[0], x[1], x[2]}};
      const gamera_no_vec3 sv = {{v[0], v[1], v[2]}};
      gamera_no_vec3 gv;
      if (mi_ghost_velocity(E.mil, pt, sv, &gv) != 0) {
        fail(st, kStageHost, 0, f, i, j, k);
        return;
      }
      for (int c = 0; c < 3; ++c)
        v[c] = E.strict_wall ? 0.5 * (gv.value[c] + v[c]) : gv.value[c];
    } else if (E.strict_wall) {
      v[0] = v[1] = v[2] = 0.0;
    } else {
      double vn = 0.0;
      for (int c = 0; c < 3; ++c) vn += v[c] * x[c] / radius;
      for (int c = 0; c < 3; ++c) v[c] -= 2.0 * vn * x[c] / radius;
    }
  } else {
    WindState w;
    double wt;
    if (!sample_wind(E.wind, x, time, &w, &wt)) {
      fail(st, kStageHost, 0, f, i, j, k);
      return;
    }
    double vn = 0.0;
    for (int c = 0; c < 3; ++c) vn += v[c] * x[c] / radius;
    const double cs = sqrt(E.gamma * p.p / p.rho);
    if (vn < cs)
      for (int c = 0; c < 3; ++c) v[c] += (cs - vn) * x[c] / radius;
    p.rho = wt * w.rho + (1.0 - wt) * p.rho;
    p.p = wt * w.p + (1.0 - wt) * p.p;
    for (int c = 0; c < 3; ++c) v[c] = wt * w.v[c] + (1.0 - wt) * v[c];
  }
  p.vx = v[0];
  p.vy = v[1];
  p.vz = v[2];
  double out[5];
  if (prim_to_cons(p, E.gamma, E.rho_floor, E.p_floor, out)) {
    fail(st, kStageHost, 0, f, i, j, k);
    return;
  }
  for (int m = 0; m < 5; ++m) U[m][dst] = out[m];
}

// Radial ghost faces of family d, cubedsphere_earth_boundary.c:114-163:
// inner ghosts carry the first active face's flux density; outer ghosts
// blend the wind's residual flux (B_wind . area vector - B0 flux) with the
// last face inside.
__global__ void k_earth_faces(Dims D, DevState S, DevGeom G, EarthDev E, int d,
                              double time, int old, const StepParams *prm, DevStatus *st) {
  if (failed(st)) return;
  time = radial_time(prm, time, old);
  const int e1 = D.E1 + (d == 1), e2 = D.E2 + (d == 2);
  const int jk = blockIdx.x * blockDim.x + threadIdx.x;
  if (jk >= e1 * e2) return;
  const int l = blockIdx.y, f = blockIdx.z;
  const int j = jk / e2, k = jk % e2;
  const int outer = D.g + D.nr;
  double *P = old ? S.Po[d] : S.P[d];
  if (l < D.g) {
    const int i = l;
    const long long c = f * D.Nn + D.node(i, j, k);
    const long long src = f * D.Nn + D.node(D.g, j, k);
    const double sa = G.area[d][src];
    if (!(sa > 0.0)) {
      fail(st, kStageHost, d, f, i, j, k);
      return;
    }
    P[c] = P[src] * G.area[d][c] / sa;
    return;
  }
  const int lo = l - D.g;
  const int i = outer + (d == 0) + lo;
  const long long q = plane(D, f, D.g, lo, j, k);
  const double x[3] = {E.face_cen[d][0][q], E.face_cen[d][1][q], E.face_cen[d][2][q]};
  WindState w;
  double wt;
  if (!sample_wind(E.wind, x, time, &w, &wt)) {
    fail(st, kStageHost, d, f, i, j, k);
    return;
  }
  double wf = -E.face_bg[d][q];
  for (int c = 0; c < 3; ++c) wf += w.b[c] * E.face_av[d][c][q];
  const int si = d == 0 ? outer : outer - 1;
  const long long c = f * D.Nn + D.node(i, j, k);
  P[c] = wt * wf + (1.0 - wt) * P[f * D.Nn + D.node(si, j, k)];
}

// Cell B and old cell B of every cell from the face fluxes and old face
// fluxes (nonorthogonal_step.c:310-358 as called at
// cubedsphere_earth_boundary.c:169-172 after each field's face fill; the
// two fills touch disjoint arrays, so one pass recovers both and reads the
// recovery map once).
__global__ void k_earth_recover(Dims D, DevState S, DevGeom G, DevStatus *st) {
  if (failed(st)) return;
  int f, i, j, k;
  const Box b{0, 0, 0, D.E1, D.E2, D.E0};
  if (!box_coord(b, &f, &i, &j, &k)) return;
  const long long c = f * D.Nn + D.node(i, j, k);
  const long long sdir[3] = {D.stride(0), D.stride(1), 1};
  for (int old = 0; old < 2; ++old) {
    double *const *P = old ? S.Po : S.P;
    double phi[6], bn[3];
    for (int d = 0; d < 3; ++d) {
      phi[2 * d] = P[d][c];
      phi[2 * d + 1] = P[d][c + sdir[d]];
    }
    if (!recover_cell(G, c, phi, bn)) {
      fail(st, kStageHost, 0, f, i, j, k);
      return;
    }
    double *const *B = old ? S.Bo : S.B;
    for (int m = 0; m < 3; ++m) B[m][c] = bn[m];
  }
}

// dB/dr = 0 in the inner ghost cells (cubedsphere_earth_boundary.c:173-182).
__global__ void k_earth_copy_inner(Dims D, DevState S, int old) {
  const int jk = blockIdx.x * blockDim.x + threadIdx.x;
  if (jk >= D.E1 * D.E2) return;
  const int i = blockIdx.y, f = blockIdx.z;
  const int j = jk / D.E2, k = jk % D.E2;
  double *const *B = old ? S.Bo : S.B;
  const long long src = f * D.Nn + D.node(D.g, j, k);
  const long long dst = f * D.Nn + D.node(i, j, k);
  for (int m = 0; m < 3; ++m) B[m][dst] = B[m][src];
}

// No outward mass (and then energy) flux through the inner shell,
// nonorthogonal_step.c:35-72 as called at cubedsphere_earth_boundary.c:259-266.
__global__ void k_earth_trap(Dims D, DevState S) {
  const int jk = blockIdx.x * blockDim.x + threadIdx.x;
  if (jk >= D.n * D.n) return;
  const int f = blockIdx.z;
  const int j = D.g + jk / D.n, k = D.g + jk % D.n;
  const long long c = f * D.Nn + D.node(D.g, j, k);
  if (S.F[0][0][c] > 0.0) {
    S.F[0][0][c] = 0.0;
    if (S.F[0][4][c] > 0.0) S.F[0][4][c] = 0.0;
  }
}

// Outer edges of family d in the last four layers up to the outer shell:
// blend the EMF with the wind's -v x B line integral, the weight falling as
// 1 / (1 + layers inside), cubedsphere_earth_boundary.c:390-425.
__global__ void k_earth_emf_outer(Dims D, DevState S, EarthDev E, int d, double tmid,
                                  const StepParams *prm, DevStatus *st) {
  if (failed(st)) return;
  if (prm) tmid = prm->time + 0.5 * prm->dt;
  const int e1 = D.E1 + (d != 1), e2 = D.E2 + (d != 2);
  const int jk = blockIdx.x * blockDim.x + threadIdx.x;
  if (jk >= e1 * e2) return;
  const int l = 1 + blockIdx.y, f = blockIdx.z;
  const int j = jk / e2, k = jk % e2;
  const int outer = D.g + D.nr;
  const int i = outer - 3 + (l - 1);
  const long long q = plane(D, f, 5, l, j, k);
  if (!E.edge_valid[d][q]) return;
  const double x[3] = {E.edge_mid[d][0][q], E.edge_mid[d][1][q], E.edge_mid[d][2][q]};
  WindState w;
  double wt;
  if (!sample_wind(E.wind, x, tmid, &w, &wt)) {
    fail(st, kStageHost, d, f, i, j, k);
    return;
  }
  if (i < outer) wt /= 1.0 + (double)(outer - i);
  const double el[3] = {-(w.v[1] * w.b[2] - w.v[2] * w.b[1]),
                        -(w.v[2] * w.b[0] - w.v[0] * w.b[2]),
                        -(w.v[0] * w.b[1] - w.v[1] * w.b[0])};
  const double len = E.edge_len[d][q];
  double li = 0.0;
  for (int c = 0; c < 3; ++c) li += el[c] * E.edge_nrm[d][c][q] * len;
  const long long c = f * D.Nn + D.node(i, j, k);
  S.E[d][c] = (1.0 - wt) * S.E[d][c] + wt * li;
}

__device__ inline bool flux_density(const Dims &D, const DevState &S, const DevGeom &G,
                                    int f, int d, int i, int j, int k, double *out) {
  if (i >= D.E0 + (d == 0) || j >= D.E1 + (d == 1) || k >= D.E2 + (d == 2)) return false;
  const long long c = f * D.Nn + D.node(i, j, k);
  const double area = G.area[d][c];
  if (!(area > 0.0)) return false;
  *out = S.Pp[d][c] / area;
  return isfinite(*out);
}

// Wind-front diffusive EMF on the outer shell's j and k edges,
// cubedsphere_earth_boundary.c:298-379.
__global__ void k_earth_emf_diffusive(Dims D, DevState S, DevGeom G, EarthDev E,
                                      double tmid, double dt, const StepParams *prm,
                                      DevStatus *st) {
  if (failed(st)) return;
  if (prm) {
    tmid = prm->time + 0.5 * prm->dt;
    dt = prm->dt;
  }
  const int w1 = D.n + 1;
  const int jk = blockIdx.x * blockDim.x + threadIdx.x;
  if (jk >= w1 * w1) return;
  const int f = blockIdx.z;
  const int j = D.g + jk / w1, k = D.g + jk % w1;
  const int i = D.g + D.nr;
  if (j == 0 || k == 0 || i >= D.E0 + 1 || j >= D.E1 || k >= D.E2 + 1 || j >= D.E1 + 1 ||
      k >= D.E2)
    return;
  const long long qj = plane(D, f, 5, 4, j, k);
  if (!E.edge_valid[1][qj] || !E.edge_valid[2][qj]) return;
  double bikp, bikm, bkip, bkim, bjip, bjim, bijp, bijm;
  if (!flux_density(D, S, G, f, 0, i, j, k, &bikp) ||
      !flux_density(D, S, G, f, 0, i, j, k - 1, &bikm) ||
      !flux_density(D, S, G, f, 2, i, j, k, &bkip) ||
      !flux_density(D, S, G, f, 2, i - 1, j, k, &bkim) ||
      !flux_density(D, S, G, f, 1, i, j, k, &bjip) ||
      !flux_density(D, S, G, f, 1, i - 1, j, k, &bjim) ||
      !flux_density(D, S, G, f, 0, i, j, k, &bijp) ||
      !flux_density(D, S, G, f, 0, i, j - 1, k, &bijm)) {
    fail(st, kStageHost, 1, f, i, j, k);
    return;
  }
  const double cur_j = (bikp - bikm) - (bkip - bkim);
  const double cur_k = (bjip - bjim) - (bijp - bijm);
  const double dl = sqrt(E.edge_len[1][qj] * E.edge_len[2][qj]);
  const double xj[3] = {E.edge_mid[1][0][qj], E.edge_mid[1][1][qj], E.edge_mid[1][2][qj]};
  const double xk[3] = {E.edge_mid[2][0][qj], E.edge_mid[2][1][qj], E.edge_mid[2][2][qj]};
  WindState wj, wk;
  double wtj, wtk;
  if (!(dl > 0.0) || !sample_wind(E.wind, xj, tmid, &wj, &wtj) ||
      !sample_wind(E.wind, xk, tmid, &wk, &wtk)) {
    fail(st, kStageHost, 1, f, i, j, k);
    return;
  }
  const double csq = E.wind.by * E.wind.by + E.wind.bz * E.wind.bz;
  const double front = fmax(fabs(wj.v[0]), fabs(wk.v[0])) / sqrt(1.0 + csq);
  const double speed = fmin(front, E.cfl * dl / dt);
  const long long c = f * D.Nn + D.node(i, j, k);
  S.E[1][c] += wtj * speed * cur_j * dl;
  S.E[2][c] += wtk * speed * cur_k * dl;
}

// E_t = 0 on the inner shell (cubedsphere_earth_boundary.c:428-437), or with
// a ready MI coupling the potential difference along the edge
// (cubedsphere_mi_dipole.c:478-503, applied after the zeroing at :438-441).
__global__ void k_earth_emf_inner(Dims D, DevState S, EarthDev E, int d, DevStatus *st) {
  const int e1 = D.E1 + (d != 1), e2 = D.E2 + (d != 2);
  const int jk = blockIdx.x * blockDim.x + threadIdx.x;
  if (jk >= e1 * e2) return;
  const int f = blockIdx.z;
  const int j = jk / e2, k = jk % e2;
  if (!E.edge_valid[d][plane(D, f, 5, 0, j, k)]) return;
  double emf = 0.0;
  if (E.mi) {
    const long long p = ((long long)f * D.N1 + j) * D.N2 + k;
    const gamera_no_vec3 a = {{E.inner_a[d - 1][0][p], E.inner_a[d - 1][1][p],
                               E.inner_a[d - 1][2][p]}};
    const gamera_no_vec3 b = {{E.inner_b[d - 1][0][p], E.inner_b[d - 1][1][p],
                               E.inner_b[d - 1][2][p]}};
    double pa, pb;
    if (mi_potential(E.mil, a, &pa) != 0 || mi_potential(E.mil, b, &pb) != 0) {
      fail(st, kStageHost, d, f, D.g, j, k);
      return;
    }
    emf = -(pb - pa) / E.mi_potential_norm;
  }
  S.E[d][f * D.Nn + D.node(D.g, j, k)] = emf;
}

inline unsigned blocks(long long n) { return (unsigned)((n + 127) / 128); }

}  // namespace

void launch_earth_radial(const Ctx &X, const EarthStep &es, cudaStream_t s) {
  const Dims &D = X.D;
  const EarthDev &E = *es.dev;
  const StepParams *prm = es.device_times ? X.params : nullptr;
  const dim3 gc(blocks((long long)D.E1 * D.E2), 2 * D.g, kFaces);
  k_earth_cells<<<gc, 128, 0, s>>>(D, X.S, E, es.current_time, 0, prm, X.status);
  k_earth_cells<<<gc, 128, 0, s>>>(D, X.S, E, es.previous_time, 1, prm, X.status);
  const Tile t{128, 1};
  for (int old = 0; old < 2; ++old) {
    const double time = old ? es.previous_time : es.current_time;
    for (int d = 0; d < 3; ++d) {
      const long long pl = (long long)(D.E1 + (d == 1)) * (D.E2 + (d == 2));
      k_earth_faces<<<dim3(blocks(pl), 2 * D.g, kFaces), 128, 0, s>>>(
          D, X.S, X.G, E, d, time, old, prm, X.status);
    }
  }
  k_earth_recover<<<tile_grid(D.E0, D.E1, D.E2, t), tile_block(t), 0, s>>>(D, X.S, X.G,
                                                                            X.status);
  for (int old = 0; old < 2; ++old)
    k_earth_copy_inner<<<dim3(blocks((long long)D.E1 * D.E2), D.g, kFaces), 128, 0, s>>>(
        D, X.S, old);
}

void launch_earth_trap(const Ctx &X, cudaStream_t s) {
  k_earth_trap<<<dim3(blocks((long long)X.D.n * X.D.n), 1, kFaces), 128, 0, s>>>(X.D, X.S);
}

void launch_earth_emf(const Ctx &X, const EarthStep &es, cudaStream_t s) {
  const Dims &D = X.D;
  const EarthDev &E = *es.dev;
  const StepParams *prm = es.device_times ? X.params : nullptr;
  const double tmid = es.step_time + 0.5 * es.step_dt;
  for (int d = 0; d < 3; ++d) {
    const long long pl = (long long)(D.E1 + (d != 1)) * (D.E2 + (d != 2));
    k_earth_emf_outer<<<dim3(blocks(pl), 4, kFaces), 128, 0, s>>>(D, X.S, E, d, tmid, prm,
                                                                   X.status);
  }
  k_earth_emf_diffusive<<<dim3(blocks((long long)(D.n + 1) * (D.n + 1)), 1, kFaces), 128, 0,
                          s>>>(D, X.S, X.G, E, tmid, es.step_dt, prm, X.status);
  for (int d = 1; d < 3; ++d) {
    const long long pl = (long long)(D.E1 + (d != 1)) * (D.E2 + (d != 2));
    k_earth_emf_inner<<<dim3(blocks(pl), 1, kFaces), 128, 0, s>>>(D, X.S, E, d, X.status);
  }
}

}  // namespace gcs

namespace {

int upload_wind(gcs_earth *e, const gamera_solar_wind_series *w) {
  if (!w || w->count < 1 || w->count > (1u << 30) || !w->time || !w->state) {
    gcs::set_api_error("invalid solar-wind series");
    return -1;
  }
  for (int c = 0; c < 3; ++c)
    if (!std::isfinite(w->reference[c])) {
      gcs::set_api_error("invalid solar-wind series");
      return -1;
    }
  const size_t n = w->count;
  void *pool = nullptr;
  if (cudaMalloc(&pool, n * 9 * sizeof(double)) != cudaSuccess) {
    gcs::set_api_error("cannot allocate the solar-wind series");
    return -1;
  }
  std::vector<double> host(n * 9);
  for (size_t q = 0; q < n; ++q) {
    host[q] = w->time[q];
    const gamera_solar_wind_state &s = w->state[q];
    double *a = &host[n + 8 * q];
    a[0] = s.density;
    a[1] = s.pressure;
    for (int c = 0; c < 3; ++c) {
      a[2 + c] = s.velocity[c];
      a[5 + c] = s.magnetic[c];
    }
  }
  if (cudaMemcpy(pool, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice) !=
      cudaSuccess) {
    cudaFree(pool);
    gcs::set_api_error("cannot upload the solar-wind series");
    return -1;
  }
  if (e->wind_pool) cudaFree(e->wind_pool);
  e->wind_pool = pool;
  gcs::WindDev &W = e->dev.wind;
  W.count = (int)n;
  W.linear = w->linear_interpolation;
  W.time = (const double *)pool;
  W.state = (const double *)pool + n;
  for (int c = 0; c < 3; ++c) W.reference[c] = w->reference[c];
  W.time_offset = w->time_offset;
  W.by = w->by_coefficient;
  W.bz = w->bz_coefficient;
  return 0;
}

// Counts of the boundary-layer arrays (layouts of gcs_earth.h).
void earth_counts(const gcs::Dims &D, long long *ncell, long long *nface, long long *nedge,
                  long long *doubles) {
  const long long P = (long long)D.N1 * D.N2;
  *ncell = 6LL * 2 * D.g * P;
  *nface = 6LL * D.g * P;
  *nedge = 6LL * 5 * P;
  *doubles = 3 * *ncell + 3 * 7 * *nface + 3 * 7 * *nedge + 12 * 6LL * P;
}

// Point the boundary's device arrays into its pool: cell centroids, then per
// face family centroid[3], area vector[3], B0 flux, then per edge family
// midpoint[3], direction[3], length, then the edge validity bytes.
gcs::EarthLayers earth_bind(gcs_earth *e, const gcs::Dims &D) {
  long long ncell, nface, nedge, doubles;
  earth_counts(D, &ncell, &nface, &nedge, &doubles);
  double *dp = (double *)e->pool;
  unsigned char *vp = (unsigned char *)e->pool + doubles * sizeof(double);
  gcs::EarthLayers L;
  for (int c = 0; c < 3; ++c) L.cell_cen[c] = dp + c * ncell;
  double *fp = dp + 3 * ncell;
  double *ep = fp + 3 * 7 * nface;
  for (int d = 0; d < 3; ++d) {
    for (int c = 0; c < 3; ++c) {
      L.face_cen[d][c] = fp + (d * 7 + c) * nface;
      L.face_av[d][c] = fp + (d * 7 + 3 + c) * nface;
      L.edge_mid[d][c] = ep + (d * 7 + c) * nedge;
      L.edge_nrm[d][c] = ep + (d * 7 + 3 + c) * nedge;
    }
    L.face_bg[d] = fp + (d * 7 + 6) * nface;
    L.edge_len[d] = ep + (d * 7 + 6) * nedge;
    L.edge_valid[d] = vp + d * nedge;
  }
  double *ip = ep + 3 * 7 * nedge;
  const long long pl = 6LL * D.N1 * D.N2;
  for (int d = 0; d < 2; ++d)
    for (int c = 0; c < 3; ++c) {
      L.inner_a[d][c] = ip + (d * 6 + c) * pl;
      L.inner_b[d][c] = ip + (d * 6 + 3 + c) * pl;
    }
  gcs::EarthDev &E = e->dev;
  for (int d = 0; d < 2; ++d)
    for (int c = 0; c < 3; ++c) {
      E.inner_a[d][c] = L.inner_a[d][c];
      E.inner_b[d][c] = L.inner_b[d][c];
    }
  for (int c = 0; c < 3; ++c) E.cell_cen[c] = L.cell_cen[c];
  for (int d = 0; d < 3; ++d) {
    for (int c = 0; c < 3; ++c) {
      E.face_cen[d][c] = L.face_cen[d][c];
      E.face_av[d][c] = L.face_av[d][c];
      E.edge_mid[d][c] = L.edge_mid[d][c];
      E.edge_nrm[d][c] = L.edge_nrm[d][c];
    }
    E.face_bg[d] = L.face_bg[d];
    E.edge_len[d] = L.edge_len[d];
    E.edge_valid[d] = L.edge_valid[d];
  }
  return L;
}

int earth_create(gcs::Context &C, const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
                 const gamera_cs_earth_boundary *b, gcs_earth **out,
                 bool allow_mi = false) {
  *out = nullptr;
  if (!grid || !b || !b->startup || !b->wind || !b->background ||
      !std::isfinite(b->density_floor) || !(b->density_floor > 0.0) ||
      !std::isfinite(b->pressure_floor) || !(b->pressure_floor > 0.0) ||
      !(b->cfl > 0.0) || !std::isfinite(b->startup->gamma)) {
    gcs::set_api_error("invalid Earth boundary");
    return -1;
  }
  (void)allow_mi;
  const gcs::Dims &D = C.X.D;
  for (int f = 0; f < gcs::kFaces; ++f) {
    const gamera_no_grid &g = grid[f];
    if ((int)g.cell_extent[0] != D.E0 || (int)g.cell_extent[1] != D.E1 ||
        (int)g.cell_extent[2] != D.E2 || !g.cell || !g.vertex ||
        !b->background[f].face_flux[0] || !b->background[f].face_flux[1] ||
        !b->background[f].face_flux[2]) {
      gcs::set_api_error("grid or background does not match the context");
      return -1;
    }
    for (int d = 0; d < 3; ++d)
      if (!g.face[d].value || !g.edge[d].value || !g.edge[d].valid) {
        gcs::set_api_error("grid without face or edge geometry");
        return -1;
      }
  }
  gcs_earth *e = new (std::nothrow) gcs_earth;
  if (!e) return -1;
  e->C = &C;
  const int g = D.g, outer = D.g + D.nr;
  long long ncell, nface, nedge, doubles;
  earth_counts(D, &ncell, &nface, &nedge, &doubles);
  std::vector<double> h(doubles, 0.0);
  std::vector<unsigned char> hv(3 * nedge, 0);
  double *cell = h.data();
  double *face = cell + 3 * ncell;
  double *edge = face + 3 * 7 * nface;
  auto pl = [&](int f, int layers, int l, int j, int k) {
    return (((long long)f * layers + l) * D.N1 + j) * D.N2 + k;
  };
  for (int f = 0; f < 6; ++f) {
    const gamera_no_grid &G = grid[f];
    for (int l = 0; l < 2 * g; ++l) {
      const int i = l < g ? l : outer + (l - g);
      for (int j = 0; j < D.E1; ++j)
        for (int k = 0; k < D.E2; ++k) {
          const gamera_no_vec3 &x = G.cell[((size_t)i * D.E1 + j) * D.E2 + k].centroid;
          for (int c = 0; c < 3; ++c) cell[c * ncell + pl(f, 2 * g, l, j, k)] = x.value[c];
        }
    }
    for (int d = 0; d < 3; ++d) {
      const size_t *fe = G.face[d].extent;
      double *fd = face + d * 7 * nface;
      for (int l = 0; l < g; ++l) {
        const size_t i = outer + (d == 0) + l;
        for (size_t j = 0; j < fe[1]; ++j)
          for (size_t k = 0; k < fe[2]; ++k) {
            const size_t idx = (i * fe[1] + j) * fe[2] + k;
            const gamera_no_face_geometry &fg = G.face[d].value[idx];
            const long long q = pl(f, g, l, (int)j, (int)k);
            for (int c = 0; c < 3; ++c) {
              fd[c * nface + q] = fg.centroid.value[c];
              fd[(3 + c) * nface + q] = fg.area_vector.value[c];
            }
            fd[6 * nface + q] = b->background[f].face_flux[d][idx];
          }
      }
      const size_t *ee = G.edge[d].extent;
      const size_t *ve = G.vertex_extent;
      double *ed = edge + d * 7 * nedge;
      for (int l = 0; l < 5; ++l) {
        const size_t i = l == 0 ? (size_t)g : (size_t)(outer - 3 + (l - 1));
        if (i >= ee[0]) continue;
        for (size_t j = 0; j < ee[1]; ++j)
          for (size_t k = 0; k < ee[2]; ++k) {
            const size_t idx = (i * ee[1] + j) * ee[2] + k;
            const long long q = pl(f, 5, l, (int)j, (int)k);
            hv[d * nedge + q] = G.edge[d].valid[idx];
            const gamera_no_edge_geometry &eg = G.edge[d].value[idx];
            size_t up[3] = {i, j, k};
            ++up[d];
            const gamera_no_vec3 &a = G.vertex[(i * ve[1] + j) * ve[2] + k];
            const gamera_no_vec3 &z = G.vertex[(up[0] * ve[1] + up[1]) * ve[2] + up[2]];
            for (int c = 0; c < 3; ++c) {
              ed[c * nedge + q] = 0.5 * (a.value[c] + z.value[c]);
              ed[(3 + c) * nedge + q] = eg.normal.value[c];
            }
            ed[6 * nedge + q] = eg.length;
            if (l == 0 && d > 0) {
              double *ip = edge + 3 * 7 * nedge;
              const long long plane6 = 6LL * D.N1 * D.N2;
              const long long p = ((long long)f * D.N1 + (long long)j) * D.N2 + (long long)k;
              for (int c = 0; c < 3; ++c) {
                ip[((d - 1) * 6 + c) * plane6 + p] = a.value[c];
                ip[((d - 1) * 6 + 3 + c) * plane6 + p] = z.value[c];
              }
            }
          }
      }
    }
  }
  e->pool_bytes = doubles * sizeof(double) + hv.size();
  if (cudaMalloc(&e->pool, e->pool_bytes) != cudaSuccess ||
      cudaMemcpy(e->pool, h.data(), doubles * sizeof(double), cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemcpy((char *)e->pool + doubles * sizeof(double), hv.data(), hv.size(),
                 cudaMemcpyHostToDevice) != cudaSuccess) {
    gcs_earth_destroy(e);
    gcs::set_api_error("cannot upload the Earth boundary geometry");
    return -1;
  }
  earth_bind(e, D);
  gcs::EarthDev &E = e->dev;
  E.gamma = b->startup->gamma;
  E.rho_floor = b->density_floor;
  E.p_floor = b->pressure_floor;
  E.cfl = b->cfl;
  E.strict_wall = b->strict_inner_gas_wall;
  if (upload_wind(e, b->wind) != 0) {
    gcs_earth_destroy(e);
    return -1;
  }
  e->mi = b->mi;
  if (gcs::earth_sync_mi(e, e->mi) != 0) {
    gcs_earth_destroy(e);
    return -1;
  }
  *out = e;
  return 0;
}

gcs::WindDev host_wind(const gamera_solar_wind_series *w) {
  gcs::WindDev W{};
  W.count = (int)w->count;
  W.linear = w->linear_interpolation;
  W.time = w->time;
  W.state = (const double *)w->state;
  for (int c = 0; c < 3; ++c) W.reference[c] = w->reference[c];
  W.time_offset = w->time_offset;
  W.by = w->by_coefficient;
  W.bz = w->bz_coefficient;
  return W;
}

// cubedsphere_earth_boundary.c:9-14, plus a usable series
bool boundary_ok(const gamera_cs_earth_boundary *b) {
  return b != nullptr && b->startup != nullptr && b->wind != nullptr &&
         b->background != nullptr && std::isfinite(b->density_floor) &&
         b->density_floor > 0.0 && std::isfinite(b->pressure_floor) &&
         b->pressure_floor > 0.0 && b->wind->count >= 1 && b->wind->time != nullptr &&
         b->wind->state != nullptr;
}

// Cache of device boundaries per (context, boundary).
struct EarthEntry {
  gcs_earth *earth;
  const gamera_no_background_field *background;
  std::vector<double> time;
  std::vector<gamera_solar_wind_state> state;
};
std::mutex g_earth_mutex;
std::map<std::pair<const gcs::Context *, const void *>, EarthEntry> g_earth;

bool same_series(const EarthEntry &e, const gamera_solar_wind_series *w) {
  return e.time.size() == w->count &&
         std::memcmp(e.time.data(), w->time, w->count * sizeof(double)) == 0 &&
         std::memcmp(e.state.data(), w->state, w->count * sizeof(gamera_solar_wind_state)) == 0;
}

void remember_series(EarthEntry &e, const gamera_solar_wind_series *w) {
  e.time.assign(w->time, w->time + w->count);
  e.state.assign(w->state, w->state + w->count);
}

}  // namespace

namespace gcs {

gcs_earth *earth_for(Context &C, const gamera_no_grid grid[kFaces],
                     const gamera_cs_earth_boundary *b, bool allow_mi) {
  if (!boundary_ok(b) || !(b->cfl > 0.0)) {
    set_api_error("invalid Earth boundary");
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_earth_mutex);
  const auto key = std::make_pair((const Context *)&C, (const void *)b);
  auto it = g_earth.find(key);
  if (it != g_earth.end() && it->second.background != b->background) {
    gcs_earth_destroy(it->second.earth);
    g_earth.erase(it);
    it = g_earth.end();
  }
  if (it == g_earth.end()) {
    gcs_earth *e = nullptr;
    if (earth_create(C, grid, b, &e, allow_mi) != 0) return nullptr;
    EarthEntry en{e, b->background, {}, {}};
    remember_series(en, b->wind);
    it = g_earth.emplace(key, std::move(en)).first;
  } else if (!same_series(it->second, b->wind)) {
    if (cudaStreamSynchronize(C.stream) != cudaSuccess ||
        upload_wind(it->second.earth, b->wind) != 0)
      return nullptr;
    remember_series(it->second, b->wind);
  }
  // floors, CFL, wall flag and the front mapping may change between calls
  EarthDev &E = it->second.earth->dev;
  const WindDev W = host_wind(b->wind);
  E.wind.linear = W.linear;
  for (int c = 0; c < 3; ++c) E.wind.reference[c] = W.reference[c];
  E.wind.time_offset = W.time_offset;
  E.wind.by = W.by;
  E.wind.bz = W.bz;
  E.gamma = b->startup->gamma;
  E.rho_floor = b->density_floor;
  E.p_floor = b->pressure_floor;
  E.cfl = b->cfl;
  E.strict_wall = b->strict_inner_gas_wall;
  if (earth_sync_mi(it->second.earth, allow_mi ? b->mi : nullptr) != 0) return nullptr;
  return it->second.earth;
}

int earth_sync_mi(gcs_earth *e, const gamera_cs_mi_dipole *mi) {
  EarthDev &E = e->dev;
  MiLookup L;
  double norm;
  if (mi != nullptr && mi_lookup_device(mi, e->C, &L, &norm)) {
    // updated inside the step graph: the wall reads the device potential
    E.mil = L;
    E.mi_potential_norm = norm;
    E.mi = 1;
    return 0;
  }
  if (mi == nullptr || !mi_lookup(mi, &L, &norm)) {
    E.mi = 0;
    return 0;
  }
  const size_t per = (size_t)L.np * (size_t)L.nt;
  if (e->mi_count != 2 * per) {
    if (e->mi_pot) cudaFree(e->mi_pot);
    e->mi_pot = nullptr;
    e->mi_count = 0;
    if (cudaMalloc(&e->mi_pot, 2 * per * sizeof(double)) != cudaSuccess) {
      set_api_error("cannot allocate the MI potential copy");
      return -1;
    }
    e->mi_count = 2 * per;
  }
  // the previous step has finished: every step reads its status back
  if (cudaStreamSynchronize(e->C->stream) != cudaSuccess) return -1;
  for (int h = 0; h < 2; ++h)
    if (cudaMemcpy(e->mi_pot + h * per, L.pot[h], per * sizeof(double),
                   cudaMemcpyHostToDevice) != cudaSuccess)
      return -1;
  L.pot[0] = e->mi_pot;
  L.pot[1] = e->mi_pot + per;
  E.mil = L;
  E.mi_potential_norm = norm;
  E.mi = 1;
  return 0;
}

void earth_forget(const Context &C) {
  std::lock_guard<std::mutex> lock(g_earth_mutex);
  for (auto it = g_earth.begin(); it != g_earth.end();) {
    if (it->first.first == &C) {
      gcs_earth_destroy(it->second.earth);
      it = g_earth.erase(it);
    } else {
      ++it;
    }
  }
}

}  // namespace gcs

namespace {

int fill_radial(const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
                gamera_no_storage storage[GAMERA_CS_FACE_COUNT], const size_t active[3],
                size_t ghost, double t, double tprev, void *context, int receiver) {
  const auto *b = (const gamera_cs_earth_boundary *)context;
  if (!grid || !storage || !active || ghost < 4 || !boundary_ok(b) || !std::isfinite(t) ||
      !std::isfinite(tprev))
    return -1;
  gcs::Context *C = gcs::context_for_grid(grid, active, ghost);
  if (!C) return -1;
  gcs_earth *e = gcs::earth_for(*C, grid, b, true);
  if (!e || C->upload_state(storage) != 0) return -1;
  C->reset_status_async();
  const gcs::EarthStep es{&e->dev, t, tprev, t, 0.0, 0};
  gcs::launch_earth_radial(C->X, es, C->stream);
  gcs::DevStatus s;
  if (cudaGetLastError() != cudaSuccess || C->read_status(&s) != 0 || s.first != 0) {
    C->reset_status_async();
    return -1;
  }
  for (int f = 0; f < gcs::kFaces; ++f) {
    if (receiver >= 0 && f != receiver) continue;
    gamera_no_storage &st = storage[f];
    if (C->transfer_array(f, gcs::kArrU, 0, false, st.conserved) ||
        C->transfer_array(f, gcs::kArrUo, 0, false, st.old_conserved) ||
        C->transfer_array(f, gcs::kArrB, 0, false, (double *)st.cell_magnetic) ||
        C->transfer_array(f, gcs::kArrBo, 0, false, (double *)st.old_cell_magnetic))
      return -1;
    for (int d = 0; d < 3; ++d)
      if (C->transfer_array(f, gcs::kArrP, d, false, st.face_flux[d]) ||
          C->transfer_array(f, gcs::kArrPo, d, false, st.old_face_flux[d]))
        return -1;
  }
  return 0;
}

bool host_flux_density(const gamera_no_grid *grid, const double *flux, int d, size_t i,
                       size_t j, size_t k, double *out) {
  const size_t *fe = grid->face[d].extent;
  if (!flux || i >= fe[0] || j >= fe[1] || k >= fe[2]) return false;
  const size_t idx = (i * fe[1] + j) * fe[2] + k;
  const double area = grid->face[d].value[idx].area;
  if (!(area > 0.0)) return false;
  *out = flux[idx] / area;
  return std::isfinite(*out);
}

void edge_mid(const gamera_no_grid *grid, int d, size_t i, size_t j, size_t k, double x[3]) {
  size_t up[3] = {i, j, k};
  ++up[d];
  const size_t *ve = grid->vertex_extent;
  const gamera_no_vec3 &a = grid->vertex[(i * ve[1] + j) * ve[2] + k];
  const gamera_no_vec3 &z = grid->vertex[(up[0] * ve[1] + up[1]) * ve[2] + up[2]];
  for (int c = 0; c < 3; ++c) x[c] = 0.5 * (a.value[c] + z.value[c]);
}

}  // namespace

extern "C" {

/* cubedsphere_earth_boundary.c:212-231.  Runs the device kernels of the
 * drop-in step on the grid's context (state uploaded, ghosts downloaded);
 * a ready MI coupling sets the inner ghost velocities on the host. */
int gamera_cs_earth_fill_radial_ghosts(const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
                                       gamera_no_storage storage[GAMERA_CS_FACE_COUNT],
                                       const size_t active[3], size_t ghost,
                                       double current_time, double previous_time,
                                       void *context) {
  return fill_radial(grid, storage, active, ghost, current_time, previous_time, context, -1);
}

int gamera_cs_earth_fill_radial_ghosts_face(const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
                                            gamera_no_storage storage[GAMERA_CS_FACE_COUNT],
                                            const size_t active[3], size_t ghost,
                                            double current_time, double previous_time,
                                            void *context, int face) {
  if (face < 0 || face >= GAMERA_CS_FACE_COUNT) return -1;
  return fill_radial(grid, storage, active, ghost, current_time, previous_time, context,
                     face);
}

/* cubedsphere_earth_boundary.c:259-266 with nonorthogonal_step.c:35-72,
 * on one face's host storage. */
int gamera_cs_earth_inner_fluid_flux(gamera_no_storage *storage, const gamera_no_grid *grid,
                                     const size_t lower[3], const size_t upper[3],
                                     void *context) {
  (void)grid;
  (void)context;
  if (!storage || !lower || !upper || !storage->fluid_face_flux[0]) return -1;
  const size_t *fe = storage->face_extent[0];
  if (lower[0] >= fe[0] || lower[1] >= upper[1] || lower[2] >= upper[2] ||
      upper[1] > fe[1] || upper[2] > fe[2])
    return -1;
  for (size_t j = lower[1]; j < upper[1]; ++j)
    for (size_t k = lower[2]; k < upper[2]; ++k) {
      double *fl = &storage->fluid_face_flux[0][((lower[0] * fe[1] + j) * fe[2] + k) * 5];
      if (fl[0] > 0.0) {
        fl[0] = 0.0;
        if (fl[4] > 0.0) fl[4] = 0.0;
      }
    }
  return 0;
}

/* cubedsphere_earth_boundary.c:381-451 on one face's host storage: the
 * same arithmetic as the device EMF kernels. */
int gamera_cs_earth_no_mi_emf(gamera_no_storage *storage, const gamera_no_grid *grid,
                              const size_t lower[3], const size_t upper[3], void *context) {
  const auto *b = (const gamera_cs_earth_boundary *)context;
  if (!storage || !grid || !lower || !upper || !boundary_ok(b) ||
      !std::isfinite(b->step_time) || !(b->step_dt > 0.0))
    return -1;
  const gcs::WindDev W = host_wind(b->wind);
  const double tmid = b->step_time + 0.5 * b->step_dt;
  const size_t outer = upper[0];
  const size_t first = outer > 3 ? outer - 3 : 0;
  for (int d = 0; d < 3; ++d) {
    const size_t *ee = grid->edge[d].extent;
    for (size_t i = first; i <= outer && i < ee[0]; ++i)
      for (size_t j = 0; j < ee[1]; ++j)
        for (size_t k = 0; k < ee[2]; ++k) {
          const size_t idx = (i * ee[1] + j) * ee[2] + k;
          if (!grid->edge[d].valid[idx]) continue;
          double x[3];
          edge_mid(grid, d, i, j, k, x);
          gcs::WindState w;
          double wt;
          if (!gcs::sample_wind(W, x, tmid, &w, &wt)) return -1;
          if (i < outer) wt /= 1.0 + (double)(outer - i);
          const double el[3] = {-(w.v[1] * w.b[2] - w.v[2] * w.b[1]),
                                -(w.v[2] * w.b[0] - w.v[0] * w.b[2]),
                                -(w.v[0] * w.b[1] - w.v[1] * w.b[0])};
          const gamera_no_edge_geometry &g = grid->edge[d].value[idx];
          double li = 0.0;
          for (int c = 0; c < 3; ++c) li += el[c] * g.normal.value[c] * g.length;
          storage->edge_emf[d][idx] = (1.0 - wt) * storage->edge_emf[d][idx] + wt * li;
        }
  }
  {
    const size_t i = upper[0];
    if (i == 0 || !(b->cfl > 0.0)) return -1;
    const size_t *ej = grid->edge[1].extent, *ek = grid->edge[2].extent;
    for (size_t j = lower[1]; j <= upper[1]; ++j)
      for (size_t k = lower[2]; k <= upper[2]; ++k) {
        if (j == 0 || k == 0 || i >= ej[0] || j >= ej[1] || k >= ej[2] || i >= ek[0] ||
            j >= ek[1] || k >= ek[2])
          continue;
        const size_t ij = (i * ej[1] + j) * ej[2] + k, ik = (i * ek[1] + j) * ek[2] + k;
        if (!grid->edge[1].valid[ij] || !grid->edge[2].valid[ik]) continue;
        double bikp, bikm, bkip, bkim, bjip, bjim, bijp, bijm;
        const double *const *pf = storage->predicted_face_flux;
        if (!host_flux_density(grid, pf[0], 0, i, j, k, &bikp) ||
            !host_flux_density(grid, pf[0], 0, i, j, k - 1, &bikm) ||
            !host_flux_density(grid, pf[2], 2, i, j, k, &bkip) ||
            !host_flux_density(grid, pf[2], 2, i - 1, j, k, &bkim) ||
            !host_flux_density(grid, pf[1], 1, i, j, k, &bjip) ||
            !host_flux_density(grid, pf[1], 1, i - 1, j, k, &bjim) ||
            !host_flux_density(grid, pf[0], 0, i, j, k, &bijp) ||
            !host_flux_density(grid, pf[0], 0, i, j - 1, k, &bijm))
          return -1;
        const double cur_j = (bikp - bikm) - (bkip - bkim);
        const double cur_k = (bjip - bjim) - (bijp - bijm);
        const double dl = sqrt(grid->edge[1].value[ij].length * grid->edge[2].value[ik].length);
        double xj[3], xk[3];
        edge_mid(grid, 1, i, j, k, xj);
        edge_mid(grid, 2, i, j, k, xk);
        gcs::WindState wj, wk;
        double wtj, wtk;
        if (!(dl > 0.0) || !gcs::sample_wind(W, xj, tmid, &wj, &wtj) ||
            !gcs::sample_wind(W, xk, tmid, &wk, &wtk))
          return -1;
        const double csq = W.by * W.by + W.bz * W.bz;
        const double front = fmax(fabs(wj.v[0]), fabs(wk.v[0])) / sqrt(1.0 + csq);
        const double speed = fmin(front, b->cfl * dl / b->step_dt);
        storage->edge_emf[1][ij] += wtj * speed * cur_j * dl;
        storage->edge_emf[2][ik] += wtk * speed * cur_k * dl;
      }
  }
  for (int d = 1; d <= 2; ++d) {
    const size_t *ee = grid->edge[d].extent;
    for (size_t j = 0; j < ee[1]; ++j)
      for (size_t k = 0; k < ee[2]; ++k) {
        const size_t idx = (lower[0] * ee[1] + j) * ee[2] + k;
        if (grid->edge[d].valid[idx]) storage->edge_emf[d][idx] = 0.0;
      }
  }
  if (b->mi && gamera_cs_mi_dipole_ready(b->mi) &&
      gamera_cs_mi_dipole_apply_inner_emf(b->mi, storage, grid, lower[0]) != 0)
    return -1;
  return 0;
}

int gcs_earth_create(gcs_context *ctx, const gamera_no_grid grid[GAMERA_CS_FACE_COUNT],
                     const gamera_cs_earth_boundary *b, gcs_earth **out) {
  if (!out) return -1;
  *out = nullptr;
  if (!ctx) return -1;
  return earth_create(ctx->c, grid, b, out);
}

int gcs_earth_create_case(gcs_context *ctx, const gamera_cs_earth_boundary *b,
                          gcs_earth **out) {
  if (!out) return -1;
  *out = nullptr;
  if (!ctx || !b || !b->startup || !b->wind || b->wind->count < 1 || !b->wind->time ||
      !b->wind->state || !std::isfinite(b->density_floor) || !(b->density_floor > 0.0) ||
      !std::isfinite(b->pressure_floor) || !(b->pressure_floor > 0.0) ||
      !(b->cfl > 0.0) || !std::isfinite(b->startup->gamma)) {
    gcs::set_api_error("invalid Earth boundary");
    return -1;
  }
  gcs::Context &C = ctx->c;
  gcs_earth *e = new (std::nothrow) gcs_earth;
  if (!e) return -1;
  e->C = &C;
  long long ncell, nface, nedge, doubles;
  earth_counts(C.X.D, &ncell, &nface, &nedge, &doubles);
  e->pool_bytes = doubles * sizeof(double) + 3 * nedge;
  if (cudaMalloc(&e->pool, e->pool_bytes) != cudaSuccess ||
      cudaMemset(e->pool, 0, e->pool_bytes) != cudaSuccess) {
    gcs_earth_destroy(e);
    gcs::set_api_error("cannot allocate the Earth boundary geometry");
    return -1;
  }
  const gcs::EarthLayers L = earth_bind(e, C.X.D);
  if (C.build_earth_layers(L) != 0) {
    gcs::set_api_error(C.error);
    gcs_earth_destroy(e);
    return -1;
  }
  gcs::EarthDev &E = e->dev;
  E.gamma = b->startup->gamma;
  E.rho_floor = b->density_floor;
  E.p_floor = b->pressure_floor;
  E.cfl = b->cfl;
  E.strict_wall = b->strict_inner_gas_wall;
  if (upload_wind(e, b->wind) != 0) {
    gcs_earth_destroy(e);
    return -1;
  }
  e->mi = b->mi;
  if (gcs::earth_sync_mi(e, e->mi) != 0) {
    gcs_earth_destroy(e);
    return -1;
  }
  *out = e;
  return 0;
}

int gcs_earth_set_wind(gcs_earth *earth, const gamera_solar_wind_series *wind) {
  if (!earth) return -1;
  if (cudaStreamSynchronize(earth->C->stream) != cudaSuccess) return -1;
  return upload_wind(earth, wind);
}

void gcs_earth_destroy(gcs_earth *earth) {
  if (!earth) return;
  if (earth->C) cudaStreamSynchronize(earth->C->stream);
  if (earth->pool) cudaFree(earth->pool);
  if (earth->wind_pool) cudaFree(earth->wind_pool);
  if (earth->mi_pot) cudaFree(earth->mi_pot);
  delete earth;
}

size_t gcs_earth_copy_layers(const gcs_earth *earth, void *host, size_t capacity) {
  if (!earth || !earth->pool) return 0;
  if (host && capacity >= earth->pool_bytes &&
      cudaMemcpy(host, earth->pool, earth->pool_bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
    return 0;
  return earth->pool_bytes;
}

size_t gcs_earth_device_bytes(const gcs_earth *earth) {
  return earth ? earth->pool_bytes + 9 * sizeof(double) * (size_t)earth->dev.wind.count : 0;
}

}  // extern "C"
