// Lookups of a solved ionosphere potential at magnetospheric points
// (cubedsphere/cubedsphere_mi_dipole.c:442-543 with nonorthogonal_mi.c:20-41,
// 168-180): the dipole-mapped bilinear potential lookup, the Earth startup
// background and the E x B drift ghost velocity of the MI-coupled wall.
// Host and device share these functions: the MI coupling's host entry
// points call them on its host copy of the potential, the device Earth
// boundary on a device copy.
#pragma once

#include <cfloat>
#include <cmath>

#include "gamera_cs_types.h"
#include "gcs_device.cuh"

namespace gcs {

struct MiLookup {
  int np, nt;                     // longitudes, colatitudes per hemisphere
  double maximum_colatitude;      // of the polar grid at the ionosphere
  double ionosphere_radius_re;
  double length_norm_m, speed_norm_m_s, magnetic_norm_t;
  const double *pot[2];           // nt x np potential (V) per hemisphere
  gamera_cs_earth_startup startup;
};

GCS_HD inline double mi_vdot(const gamera_no_vec3 &a, const gamera_no_vec3 &b) {
  return a.value[0] * b.value[0] + a.value[1] * b.value[1] + a.value[2] * b.value[2];
}

// nonorthogonal_mi.c:168-180
GCS_HD inline double mi_mapped_colatitude(double th, double r, double ri) {
  if (!isfinite(th) || !isfinite(r) || !isfinite(ri) || r <= 0.0 || ri <= 0.0 || ri > r)
    return (double)NAN;
  double arg = sin(th) * sqrt(ri / r);
  arg = fmax(-1.0, fmin(1.0, arg));
  return asin(arg);
}

// Earth startup background: dipole (nonorthogonal_background.c:422-442)
// times the cut ramp (cubedsphere_earth_startup.c:13-19, :87-97).
GCS_HD inline int mi_startup_background(const gamera_cs_earth_startup &p,
                                        const gamera_no_vec3 &x, gamera_no_vec3 *out) {
  const gamera_no_vec3 &m = p.dipole.moment;
  for (int a = 0; a < 3; ++a)
    if (!isfinite(x.value[a]) || !isfinite(m.value[a])) return -1;
  double r2 = 0.0;
  for (int a = 0; a < 3; ++a) r2 += x.value[a] * x.value[a];
  if (!(r2 > DBL_MIN) || !isfinite(r2)) return -1;
  const double r = sqrt(r2);
  const double ir3 = 1.0 / (r2 * r);
  const double ir5 = ir3 / r2;
  double proj = 0.0;
  for (int a = 0; a < 3; ++a) proj += m.value[a] * x.value[a];
  for (int a = 0; a < 3; ++a)
    out->value[a] = 3.0 * proj * ir5 * x.value[a] - ir3 * m.value[a];
  for (int a = 0; a < 3; ++a)
    if (!isfinite(out->value[a])) return -1;
  const bool valid = isfinite(p.inner_radius) && p.inner_radius > 0.0 &&
                     isfinite(p.density) && p.density > 0.0 && isfinite(p.speed) &&
                     p.speed > 0.0 && isfinite(p.mach) && p.mach > 0.0 &&
                     isfinite(p.gamma) && p.gamma > 1.0 && isfinite(p.ambient_density) &&
                     p.ambient_density > 0.0 && isfinite(p.ambient_pressure) &&
                     p.ambient_pressure > 0.0 && isfinite(p.front_x) &&
                     isfinite(p.front_width) && p.front_width > 0.0 &&
                     isfinite(p.cut_radius) && p.cut_radius > p.inner_radius &&
                     isfinite(p.cut_length) && p.cut_length > 0.0;
  if (!valid) return -1;
  const double rr = sqrt(x.value[0] * x.value[0] + x.value[1] * x.value[1] +
                         x.value[2] * x.value[2]);
  const double sc = (rr - p.cut_radius) / p.cut_length;
  const double w = sc <= 0.0 ? 1.0 : (sc >= 1.0 ? 0.0 : 1.0 - 3.0 * sc * sc + 2.0 * sc * sc * sc);
  for (int a = 0; a < 3; ++a) out->value[a] *= w;
  return 0;
}

// Potential (V) at a point: dipole field-line mapping to the ionosphere and
// bilinear interpolation on the hemisphere's polar grid; 0 beyond the grid.
GCS_HD inline int mi_potential(const MiLookup &L, gamera_no_vec3 point, double *potential_v) {
  const double radius = sqrt(mi_vdot(point, point));
  if (!(radius >= L.ionosphere_radius_re)) return -1;
  const int hemi = point.value[2] >= 0.0 ? 0 : 1;
  const double th = acos(fmin(1.0, fabs(point.value[2]) / radius));
  const double thi = mi_mapped_colatitude(th, radius, L.ionosphere_radius_re);
  if (!isfinite(thi)) return -1;
  if (thi >= L.maximum_colatitude) {
    *potential_v = 0.0;
    return 0;
  }
  const size_t np = (size_t)L.np, nt = (size_t)L.nt;
  const double tq = thi / L.maximum_colatitude * (double)(nt - 1U);
  const size_t t = (size_t)floor(tq);
  const double wt = tq - (double)t;
  double phi = atan2(point.value[1], point.value[0]);
  if (phi < 0.0) phi += 2.0 * acos(-1.0);
  const double pq = phi * (double)np / (2.0 * acos(-1.0));
  const size_t p = (size_t)floor(pq) % np;
  const size_t q = (p + 1U) % np;
  const double wp = pq - floor(pq);
  const double *pot = L.pot[hemi];
  const double lower = (1.0 - wp) * pot[t * np + p] + wp * pot[t * np + q];
  const double upper = (1.0 - wp) * pot[(t + 1U) * np + p] + wp * pot[(t + 1U) * np + q];
  *potential_v = (1.0 - wt) * lower + wt * upper;
  return isfinite(*potential_v) ? 0 : -1;
}

// Ghost velocity of the MI-coupled wall: twice the E x B drift (E from the
// mapped potential by central differences, B the startup background, the
// radial part removed) minus the source velocity.
GCS_HD inline int mi_ghost_velocity(const MiLookup &L, gamera_no_vec3 point,
                                    gamera_no_vec3 source_velocity,
                                    gamera_no_vec3 *ghost_velocity) {
  const double radius = sqrt(mi_vdot(point, point));
  if (!(radius > 0.0)) return -1;
  const double eps = 1e-4 * fmax(1.0, radius);
  gamera_no_vec3 e = {{0.0, 0.0, 0.0}};
  for (int c = 0; c < 3; ++c) {
    gamera_no_vec3 plus = point, minus = point;
    plus.value[c] += eps;
    minus.value[c] -= eps;
    double pp, pm;
    if (mi_potential(L, plus, &pp) != 0 || mi_potential(L, minus, &pm) != 0) return -1;
    e.value[c] = -(pp - pm) / (2.0 * eps * L.length_norm_m * L.speed_norm_m_s *
                               L.magnetic_norm_t);
  }
  gamera_no_vec3 bg;
  if (mi_startup_background(L.startup, point, &bg) != 0) return -1;
  const double b2 = mi_vdot(bg, bg);
  if (!(b2 > 0.0)) return -1;
  gamera_no_vec3 drift = {{(e.value[1] * bg.value[2] - e.value[2] * bg.value[1]) / b2,
                           (e.value[2] * bg.value[0] - e.value[0] * bg.value[2]) / b2,
                           (e.value[0] * bg.value[1] - e.value[1] * bg.value[0]) / b2}};
  const double radial = mi_vdot(drift, point) / (radius * radius);
  for (int c = 0; c < 3; ++c) drift.value[c] -= radial * point.value[c];
  double bsq = 0.0;
  for (int c = 0; c < 3; ++c) bsq += bg.value[c] * bg.value[c];
  if (!(bsq > 0.0) || !isfinite(bsq)) return -1;
  for (int c = 0; c < 3; ++c) {
    ghost_velocity->value[c] = 2.0 * drift.value[c] - source_velocity.value[c];
    if (!isfinite(ghost_velocity->value[c])) return -1;
  }
  return 0;
}

// The lookup parameters and host potential of a ready coupling
// (gcs_mi_dipole.cu); false when it is not ready.
bool mi_lookup(const ::gamera_cs_mi_dipole *s, MiLookup *L, double *potential_norm_v);
// The same for a coupling updated inside context C's step graph, with the
// potential on the device; false otherwise (gcs_mi_dipole.cu).
struct Context;
bool mi_lookup_device(const ::gamera_cs_mi_dipole *s, const Context *C, MiLookup *L,
                      double *potential_norm_v);

}  // namespace gcs
