// Device-side MHD point operators of the cubed-sphere step.
//
// Every function restates one reference operator with the same operation
// order (so the FP64 path tracks the CPU reference to round-off); the cited
// lines are in the GAMERA-Cube project.  The exceptions are marked where they
// occur: a repeated divisor applied as one reciprocal, sqrt(pi lambda) taken
// as sqrt(pi) sqrt(lambda), each a change in the last bit.  Functions return
// 0 on success and a nonzero value where the reference returns -1.
#pragma once

#include <cfloat>
#include <cmath>

namespace gcs {

// Precision-generic math used by the sweep operators: T = double is the
// plain path (the reference's arithmetic), T = float the FP32-bulk path.
template <typename T> struct Num;
template <> struct Num<double> {
  static constexpr double tiny = DBL_MIN;
  __host__ __device__ static double erfc_(double x) { return ::erfc(x); }
  __host__ __device__ static double exp_(double x) { return ::exp(x); }
  __host__ __device__ static double sqrt_(double x) { return ::sqrt(x); }
  __host__ __device__ static double hypot_(double a, double b) { return ::hypot(a, b); }
};
template <> struct Num<float> {
  static constexpr float tiny = FLT_MIN;
  __host__ __device__ static float erfc_(float x) { return ::erfcf(x); }
  __host__ __device__ static float exp_(float x) { return ::expf(x); }
  __host__ __device__ static float sqrt_(float x) { return ::sqrtf(x); }
  __host__ __device__ static float hypot_(float a, float b) { return ::hypotf(a, b); }
};

template <typename T>
struct PrimT {
  T rho, vx, vy, vz, p;
};
using Prim = PrimT<double>;

template <typename T>
__host__ __device__ inline T dot3(T ax, T ay, T az, T bx, T by, T bz) {
  // nonorthogonal_flux.c:9-15.  The sum starts at +0.0 as in the
  // reference, so a product of -0.0 yields the same +0.0 result.
  T r = T(0.0);
  r += ax * bx;
  r += ay * by;
  r += az * bz;
  return r;
}

// nonorthogonal_reconstruction.c:7-9, 19-26, 53-55
template <typename T>
__host__ __device__ inline T central8(const T s[8]) {
  T r = T(0.0);
  r += T(-3.0 / 840.0) * s[0];
  r += T(29.0 / 840.0) * s[1];
  r += T(-139.0 / 840.0) * s[2];
  r += T(533.0 / 840.0) * s[3];
  r += T(533.0 / 840.0) * s[4];
  r += T(-139.0 / 840.0) * s[5];
  r += T(29.0 / 840.0) * s[6];
  r += T(-3.0 / 840.0) * s[7];
  return r;
}

// nonorthogonal_reconstruction.c:11-13, 57-59
template <typename T>
__host__ __device__ inline T central6(const T s[8]) {
  T r = T(0.0);
  r += T(0.0) * s[0];
  r += T(1.0 / 60.0) * s[1];
  r += T(-8.0 / 60.0) * s[2];
  r += T(37.0 / 60.0) * s[3];
  r += T(37.0 / 60.0) * s[4];
  r += T(-8.0 / 60.0) * s[5];
  r += T(1.0 / 60.0) * s[6];
  r += T(0.0) * s[7];
  return r;
}

// nonorthogonal_reconstruction.c:15-17, 28-34
template <typename T>
__host__ __device__ inline T upwind7_left(const T w[8]) {
  T r = T(0.0);
  r += T(-3.0 / 420.0) * w[0];
  r += T(25.0 / 420.0) * w[1];
  r += T(-101.0 / 420.0) * w[2];
  r += T(319.0 / 420.0) * w[3];
  r += T(214.0 / 420.0) * w[4];
  r += T(-38.0 / 420.0) * w[5];
  r += T(4.0 / 420.0) * w[6];
  return r;
}
template <typename T>
__host__ __device__ inline T upwind7_right(const T w[8]) {
  T r = T(0.0);
  r += T(-3.0 / 420.0) * w[7];
  r += T(25.0 / 420.0) * w[6];
  r += T(-101.0 / 420.0) * w[5];
  r += T(319.0 / 420.0) * w[4];
  r += T(214.0 / 420.0) * w[3];
  r += T(-38.0 / 420.0) * w[2];
  r += T(4.0 / 420.0) * w[1];
  return r;
}

// nonorthogonal_reconstruction.c:36-51 (Fortran SIGN(1,x) == copysign)
template <typename T>
__host__ __device__ inline T pdm_left(T q0, T q1, T q2, T interpolated, T pdmb) {
  const T bounded = fmax(fmin(q1, q2), fmin(interpolated, fmax(q1, q2)));
  const T delta0 = pdmb * (q1 - q0);
  const T delta1 = pdmb * (q2 - q1);
  const T sign0 = copysign(T(1.0), delta0);
  const T sign1 = copysign(T(1.0), delta1);
  const T same = fabs(sign0 + sign1);
  const T slope = bounded - q1;
  return bounded - sign1 * fmax(T(0.0), fabs(slope) - same * fabs(delta0));
}

// nonorthogonal_reconstruction.c:61-93 with the interface volume
// central8(volume) supplied by the caller (it is independent of the
// variable being reconstructed).  The caller guarantees a finite, nonzero
// interface volume (checked once at set-up).
__host__ __device__ inline void up7_pdm(const double vol[8], const double q[8],
                                        double iv, double pdmb, double *left,
                                        double *right) {
  double w[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) w[n] = vol[n] * q[n];
  const double hl = upwind7_left(w) / iv;
  const double hr = upwind7_right(w) / iv;
  *left = pdm_left(q[2], q[3], q[4], hl, pdmb);
  *right = pdm_left(q[5], q[4], q[3], hr, pdmb);
}

// up7_pdm with the division by the interface volume replaced by a multiply
// with its reciprocal (computed once per face for all eight variables):
// the high-order value may differ from the reference's by one rounding.
template <typename T>
__host__ __device__ inline void up7_pdm_rcp(const T vol[8], const T q[8], T riv,
                                            T pdmb, T *left, T *right) {
  T w[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) w[n] = vol[n] * q[n];
  const T hl = upwind7_left(w) * riv;
  const T hr = upwind7_right(w) * riv;
  *left = pdm_left(q[2], q[3], q[4], hl, pdmb);
  *right = pdm_left(q[5], q[4], q[3], hr, pdmb);
}

// nonorthogonal_state.c:60-93
__host__ __device__ inline int cons_to_prim(const double u[5], double gamma,
                                            double rho_floor, double p_floor,
                                            Prim *out) {
  if (!isfinite(u[0]) || u[0] <= DBL_MIN) return 1;
  const double raw = u[0];
  if (!isfinite(u[1]) || !isfinite(u[2]) || !isfinite(u[3])) return 1;
  const double vx = u[1] / raw;
  const double vy = u[2] / raw;
  const double vz = u[3] / raw;
  double v2 = vx * vx;
  v2 += vy * vy;
  v2 += vz * vz;
  if (!isfinite(u[4])) return 1;
  const double kinetic = 0.5 * raw * v2;
  out->vx = vx;
  out->vy = vy;
  out->vz = vz;
  out->rho = fmax(raw, rho_floor);
  out->p = fmax((gamma - 1.0) * (u[4] - kinetic), p_floor);
  return 0;
}

// nonorthogonal_state.c:95-120
__host__ __device__ inline int prim_to_cons(const Prim &pr, double gamma,
                                            double rho_floor, double p_floor,
                                            double u[5]) {
  if (!isfinite(pr.rho) || !isfinite(pr.p)) return 1;
  const double rho = fmax(pr.rho, rho_floor);
  const double p = fmax(pr.p, p_floor);
  if (!isfinite(pr.vx) || !isfinite(pr.vy) || !isfinite(pr.vz)) return 1;
  u[0] = rho;
  u[1] = rho * pr.vx;
  u[2] = rho * pr.vy;
  u[3] = rho * pr.vz;
  double v2 = pr.vx * pr.vx;
  v2 += pr.vy * pr.vy;
  v2 += pr.vz * pr.vz;
  u[4] = p / (gamma - 1.0) + 0.5 * rho * v2;
  return 0;
}

// nonorthogonal_state.c:122-159
__host__ __device__ inline int predict_cell(const double uold[5],
                                            const double ucur[5], double ratio,
                                            double gamma, double rho_floor,
                                            double p_floor, double out[5]) {
  Prim o, c;
  if (cons_to_prim(uold, gamma, rho_floor, p_floor, &o) ||
      cons_to_prim(ucur, gamma, rho_floor, p_floor, &c))
    return 1;
  Prim q;
  q.rho = fmax(c.rho + ratio * (c.rho - o.rho), rho_floor);
  q.p = fmax(c.p + ratio * (c.p - o.p), p_floor);
  q.vx = c.vx + ratio * (c.vx - o.vx);
  q.vy = c.vy + ratio * (c.vy - o.vy);
  q.vz = c.vz + ratio * (c.vz - o.vz);
  return prim_to_cons(q, gamma, rho_floor, p_floor, out);
}

// nonorthogonal_flux.c:25-36
template <typename T>
__host__ __device__ inline bool valid_prim(const PrimT<T> &s) {
  if (!isfinite(s.rho) || !isfinite(s.p) || s.rho <= Num<T>::tiny ||
      s.p <= Num<T>::tiny)
    return false;
  return isfinite(s.vx) && isfinite(s.vy) && isfinite(s.vz);
}

template <typename T>
struct FaceFrame {
  T nx, ny, nz, t1x, t1y, t1z, t2x, t2y, t2z;
};

template <typename T>
struct FluidFlux {
  T f[5];
  T jump[5];
  T vjump[3];
  T vn[2];
};

// nonorthogonal_flux.c:38-105
template <typename T>
__device__ inline int kinetic_fluid_flux(const PrimT<T> st[2], T gamma,
                                         const FaceFrame<T> &fr, FluidFlux<T> *fl) {
  if (!isfinite(gamma) || gamma <= T(1.0) || !valid_prim(st[0]) ||
      !valid_prim(st[1]))
    return 1;
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    fl->f[m] = T(0.0);
    fl->jump[m] = T(0.0);
  }
  fl->vjump[0] = fl->vjump[1] = fl->vjump[2] = T(0.0);
  // p / (gamma - 1) as p * (1 / (gamma - 1)) and sqrt(pi lambda) as
  // sqrt(pi) sqrt(lambda): one division and one square root fewer per
  // side, each a last-bit change
  const T igm1 = T(1.0) / (gamma - T(1.0));
  const T sqrt_pi = T(1.77245385090551602729816748334114518);
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const T sign = side == 0 ? T(-1.0) : T(1.0);
    const T rho = st[side].rho;
    const T p = st[side].p;
    const T vx = st[side].vx, vy = st[side].vy, vz = st[side].vz;
    const T v2 = dot3(vx, vy, vz, vx, vy, vz);
    const T energy = T(0.5) * rho * v2 + p * igm1;
    const T lambda = rho / (T(2.0) * p);
    const T sl = Num<T>::sqrt_(lambda);
    const T vn = dot3(fr.nx, fr.ny, fr.nz, vx, vy, vz);
    const T vt1 = dot3(fr.t1x, fr.t1y, fr.t1z, vx, vy, vz);
    const T vt2 = dot3(fr.t2x, fr.t2y, fr.t2z, vx, vy, vz);
    const T zeroth = T(0.5) * Num<T>::erfc_(sign * sl * vn);
    const T first = vn * zeroth - T(0.5) * sign * Num<T>::exp_(-lambda * vn * vn) /
                                      (sqrt_pi * sl);
    fl->vn[side] = vn;
    fl->f[0] += rho * first;
    fl->f[4] += (energy + T(0.5) * p) * first + T(0.5) * p * zeroth * vn;
    const T mn = rho * vn * first + p * zeroth;
    const T mt1 = rho * vt1 * first;
    const T mt2 = rho * vt2 * first;
    fl->f[1] += fr.nx * mn + fr.t1x * mt1 + fr.t2x * mt2;
    fl->vjump[0] += sign * vx;
    fl->f[2] += fr.ny * mn + fr.t1y * mt1 + fr.t2y * mt2;
    fl->vjump[1] += sign * vy;
    fl->f[3] += fr.nz * mn + fr.t1z * mt1 + fr.t2z * mt2;
    fl->vjump[2] += sign * vz;
    fl->jump[0] += sign * rho;
    fl->jump[1] += sign * rho * vx;
    fl->jump[2] += sign * rho * vy;
    fl->jump[3] += sign * rho * vz;
    fl->jump[4] += sign * energy;
  }
  return 0;
}

template <typename T>
struct MaxwellFlux {
  T m[3];
  T alfven;
  T pmag;
};

// nonorthogonal_flux.c:107-173
template <typename T>
__device__ inline int kinetic_maxwell_flux(const PrimT<T> st[2], const T b[2][3], T bn,
                                           const FaceFrame<T> &fr, bool use_bg,
                                           const T b0[3], T b0n, bool use_boris, T c,
                                           const T vn[2], MaxwellFlux<T> *mx) {
  if (!isfinite(bn) || (use_boris && (!isfinite(c) || c <= Num<T>::tiny))) return 1;
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    if (!valid_prim(st[side])) return 1;
#pragma unroll
    for (int d = 0; d < 3; ++d)
      if (!isfinite(b[side][d]) || (use_bg && !isfinite(b0[d]))) return 1;
  }
  mx->m[0] = mx->m[1] = mx->m[2] = T(0.0);
  mx->alfven = T(0.0);
  mx->pmag = T(0.0);
  const T nrm[3] = {fr.nx, fr.ny, fr.nz};
  const T ic2 = use_boris ? T(1.0) / (c * c) : T(0.0);
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const T sign = side == 0 ? T(-1.0) : T(1.0);
    const T r2 = dot3(b[side][0], b[side][1], b[side][2], b[side][0], b[side][1],
                      b[side][2]);
    const T rp = T(0.5) * r2;
    T tx = b[side][0], ty = b[side][1], tz = b[side][2];
    if (use_bg) {
      tx = b[side][0] + b0[0];
      ty = b[side][1] + b0[1];
      tz = b[side][2] + b0[2];
    }
    const T t2 = dot3(tx, ty, tz, tx, ty, tz);
    // 1 / rho and 1 / c^2 once: two divisions fewer per side
    const T irho = T(1.0) / st[side].rho;
    const T va2 = t2 * irho;
    const T cva2 = use_boris ? va2 / (T(1.0) + va2 * ic2) : va2;
    const T lambda = T(1.0) / (T(2.0) * st[side].p * irho + cva2);
    const T zeroth = T(0.5) * Num<T>::erfc_(sign * Num<T>::sqrt_(lambda) * vn[side]);
    mx->alfven += T(0.5) * Num<T>::sqrt_(cva2);
    mx->pmag += T(0.5) * t2;
    const T bdr =
        use_bg ? dot3(b0[0], b0[1], b0[2], b[side][0], b[side][1], b[side][2]) : T(0.0);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      T stress = rp * nrm[d] - b[side][d] * bn;
      if (use_bg) stress += -b0[d] * bn - b[side][d] * b0n + bdr * nrm[d];
      mx->m[d] += zeroth * stress;
    }
  }
  return 0;
}

// nonorthogonal_flux.c:175-204 (options were validated at entry)
template <typename T>
__device__ inline void apply_hogs(FluidFlux<T> *fl, MaxwellFlux<T> *mx, T ch, T cm,
                                  bool use_boris, T c) {
#pragma unroll
  for (int m = 0; m < 5; ++m) fl->f[m] -= ch * mx->alfven * fl->jump[m];
  if (use_boris) {
    const T ic2 = T(1.0) / (c * c);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const T j = mx->pmag * fl->vjump[d] * ic2;
      mx->m[d] -= cm * mx->alfven * j;
    }
  }
}

// nonorthogonal_flux.c:206-241 (use_boris is true at every call site).  The
// conserved states either side of the face (U[m][lo], U[m][hi]) are read
// only where the diffusion applies.
template <typename T>
__device__ inline int emergency_diffusion(FluidFlux<T> *fl, const PrimT<T> st[2],
                                          const double *const U[5], long long lo_at,
                                          long long hi_at, T c, bool *applied,
                                          T *speed) {
  *applied = false;
  T s2 = T(0.0);
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    if (!valid_prim(st[side])) return 1;
    s2 += dot3(st[side].vx, st[side].vy, st[side].vz, st[side].vx, st[side].vy,
               st[side].vz);
  }
  const T is = Num<T>::sqrt_(T(0.5) * s2);
  *speed = is;
  if (is < T(1.5) * c) return 0;
  T lo[5], hi[5];
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    lo[m] = (T)U[m][lo_at];
    hi[m] = (T)U[m][hi_at];
  }
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    if (!isfinite(lo[m]) || !isfinite(hi[m])) return 1;
    fl->f[m] -= c * (hi[m] - lo[m]);
  }
  *applied = true;
  return 0;
}

// nonorthogonal_operators.c:144-182 (length > DBL_MIN checked at set-up)
template <typename T>
__device__ inline int edge_emf(T vt1, T vt2, T bt1, T bt2, T jump, T rho, T length,
                               T diffusion, bool use_boris, T c, T cfl, T dt, T *emf) {
  if (!isfinite(vt1) || !isfinite(vt2) || !isfinite(bt1) || !isfinite(bt2) ||
      !isfinite(jump) || !isfinite(rho) || rho <= Num<T>::tiny)
    return 1;
  const T flow = Num<T>::hypot_(vt1, vt2);
  T va = Num<T>::hypot_(bt1, bt2) / Num<T>::sqrt_(rho);
  if (use_boris) va = c * va / Num<T>::hypot_(c, va);
  T speed = flow + va;
  speed = fmin(speed, cfl * length / dt);
  const T ideal = -(vt1 * bt2 - vt2 * bt1);
  *emf = (ideal + diffusion * speed * jump) * length;
  return 0;
}

// nonorthogonal_state.c:161-174 (+ vector helpers :9-52)
__device__ inline int apply_boris(double u[5], const double uold[5],
                                  const double bnew[3], const double bold[3],
                                  const double rate[5], const double mrate[3],
                                  double c, double dt, double gamma,
                                  double rho_floor, double p_floor) {
  Prim up;
  if (cons_to_prim(u, gamma, rho_floor, p_floor, &up) || uold[0] <= DBL_MIN)
    return 1;
  const double urho = fmax(up.rho, rho_floor);
  const double up_p = fmax(up.p, p_floor);
  const double orho = uold[0];
  double ov[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) ov[d] = uold[1 + d] / fmax(orho, rho_floor);
  double half[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) half[d] = 0.5 * (bnew[d] + bold[d]);
  const double alpha = dot3(half[0], half[1], half[2], half[0], half[1],
                            half[2]) /
                       (urho * c * c);
  const double drho = dt * rate[0];
  double gas[3], mag[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    gas[d] = dt * rate[1 + d];
    mag[d] = dt * mrate[d];
  }
  double inc[3];
  if (alpha > 1.0e-12) {
    const double frac = 1.0 / (1.0 + alpha);
    // normalized_or_zero (nonorthogonal_state.c:45-52)
    const double norm =
        sqrt(dot3(half[0], half[1], half[2], half[0], half[1], half[2]));
    double unit[3] = {0.0, 0.0, 0.0};
    if (!(norm <= 1.0e-12)) {
      const double inv = 1.0 / norm;
      unit[0] = inv * half[0];
      unit[1] = inv * half[1];
      unit[2] = inv * half[2];
    }
    double tot[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) tot[d] = gas[d] + mag[d];
    // vector_parallel(gas, unit) = unit * dot(gas, unit)
    const double gp = dot3(gas[0], gas[1], gas[2], unit[0], unit[1], unit[2]);
    const double tp = dot3(tot[0], tot[1], tot[2], unit[0], unit[1], unit[2]);
    const double vp = dot3(ov[0], ov[1], ov[2], unit[0], unit[1], unit[2]);
    const double k = alpha * frac * drho;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double par = gp * unit[d];
      const double tperp = tot[d] - tp * unit[d];
      const double vperp = ov[d] - vp * unit[d];
      inc[d] = par + (frac * tperp + k * vperp);
    }
  } else {
#pragma unroll
    for (int d = 0; d < 3; ++d) inc[d] = gas[d] + mag[d];
  }
  Prim res;
  res.rho = urho;
  res.p = up_p;
  res.vx = (orho * ov[0] + inc[0]) / urho;
  res.vy = (orho * ov[1] + inc[1]) / urho;
  res.vz = (orho * ov[2] + inc[2]) / urho;
  return prim_to_cons(res, gamma, rho_floor, p_floor, u);
}

// nonorthogonal_state.c:109-143 (apply_maxwell)
__device__ inline int apply_maxwell(double u[5], const double mrate[3],
                                    double dt, double gamma, double rho_floor,
                                    double p_floor) {
  const double rho = fmax(u[0], rho_floor);
  double m2 = u[1] * u[1];
  m2 += u[2] * u[2];
  m2 += u[3] * u[3];
  const double p = fmax((gamma - 1.0) * (u[4] - 0.5 * m2 / rho), p_floor);
  u[1] += dt * mrate[0];
  u[2] += dt * mrate[1];
  u[3] += dt * mrate[2];
  double n2 = u[1] * u[1];
  n2 += u[2] * u[2];
  n2 += u[3] * u[3];
  u[0] = rho;
  u[4] = 0.5 * n2 / rho + p / (gamma - 1.0);
  return 0;
}

}  // namespace gcs
