/*
 * CPU restatement of the GAMERA-Cube cubed-sphere hot path (test oracle).
 * TEST INFRASTRUCTURE ONLY; see gcs_oracle.h.  Every function restates the
 * cited reference function with the same operation order, so that this
 * file reproduces the reference bit for bit on the same host.
 */
#include "gcs_oracle.h"

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "cases_common.h"

typedef gamera_no_vec3 v3;

/* ------------------------------------------------------------ vectors */

static v3 v_zero(void) { v3 r = {{0.0, 0.0, 0.0}}; return r; }
static v3 v_add(v3 a, v3 b) {
  v3 r;
  for (int d = 0; d < 3; ++d) r.value[d] = a.value[d] + b.value[d];
  return r;
}
static v3 v_sub(v3 a, v3 b) {
  v3 r;
  for (int d = 0; d < 3; ++d) r.value[d] = a.value[d] - b.value[d];
  return r;
}
/* geometry.c scales as value * factor; the other files as factor * value */
static v3 v_mul(v3 a, double s) {
  v3 r;
  for (int d = 0; d < 3; ++d) r.value[d] = a.value[d] * s;
  return r;
}
static v3 v_scale(v3 a, double s) {
  v3 r;
  for (int d = 0; d < 3; ++d) r.value[d] = s * a.value[d];
  return r;
}
static double v_dot(v3 a, v3 b) {
  double r = 0.0;
  for (int d = 0; d < 3; ++d) r += a.value[d] * b.value[d];
  return r;
}
static v3 v_cross(v3 a, v3 b) {
  v3 r = {{a.value[1] * b.value[2] - a.value[2] * b.value[1],
           a.value[2] * b.value[0] - a.value[0] * b.value[2],
           a.value[0] * b.value[1] - a.value[1] * b.value[0]}};
  return r;
}
static int v_finite(v3 a) {
  return isfinite(a.value[0]) && isfinite(a.value[1]) && isfinite(a.value[2]);
}

static size_t idx3(const size_t e[3], size_t i, size_t j, size_t k) {
  return (i * e[1] + j) * e[2] + k;
}
static size_t count3(const size_t e[3]) { return e[0] * e[1] * e[2]; }

/* 12-point Gauss-Legendre rule in the reference's node order
 * (nonorthogonal_geometry.c:9-24). */
static const double GN[12] = {
    0.1252334085114689154724,  0.3678314989981801937527,
    0.5873179542866174472967,  0.7699026741943046870369,
    0.9041172563704748566785,  0.9815606342467192506906,
    -0.1252334085114689154724, -0.3678314989981801937527,
    -0.5873179542866174472967, -0.7699026741943046870369,
    -0.9041172563704748566785, -0.9815606342467192506906};
static const double GW[12] = {
    0.2491470458134027850006, 0.2334925365383548087610,
    0.2031674267230659217490, 0.1600783285433462263350,
    0.1069393259953184309603, 0.0471753363865118271946,
    0.2491470458134027850006, 0.2334925365383548087610,
    0.2031674267230659217490, 0.1600783285433462263350,
    0.1069393259953184309603, 0.0471753363865118271946};
static const int LSIGN[8][3] = {{-1, -1, -1}, {+1, -1, -1}, {+1, +1, -1},
                                {-1, +1, -1}, {-1, -1, +1}, {+1, -1, +1},
                                {+1, +1, +1}, {-1, +1, +1}};
static const int FCORNER[3][2][4] = {{{0, 3, 4, 7}, {1, 2, 5, 6}},
                                     {{0, 4, 1, 5}, {3, 7, 2, 6}},
                                     {{0, 1, 3, 2}, {4, 5, 7, 6}}};
static const size_t COFF[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                  {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};

/* ------------------------------------------ geometry (geometry.c) */

static int g_normalize(v3 v, v3 *u) {
  const double n = sqrt(v_dot(v, v));
  if (!isfinite(n) || n <= DBL_MIN) return -1;
  *u = v_mul(v, 1.0 / n);
  return 0;
}

/* nonorthogonal_geometry.c:89-101 */
static v3 g_bilinear(const v3 f[4], double eta, double psi) {
  const v3 de = v_sub(f[1], f[0]);
  const v3 dp = v_sub(f[2], f[0]);
  const v3 dc = v_add(v_sub(f[3], f[2]), v_sub(f[0], f[1]));
  return v_add(f[0], v_add(v_mul(de, eta), v_add(v_mul(dp, psi),
                                                  v_mul(dc, eta * psi))));
}

/* nonorthogonal_geometry.c:103-158 */
static int g_face(const v3 f[4], gamera_no_face_geometry *g) {
  const v3 de = v_sub(f[1], f[0]);
  const v3 dp = v_sub(f[2], f[0]);
  const v3 dc = v_add(v_sub(f[3], f[2]), v_sub(f[0], f[1]));
  g->area = 0.0;
  g->area_vector = v_zero();
  g->centroid = v_zero();
  for (int i = 0; i < 12; ++i) {
    const double eta = 0.5 * (1.0 + GN[i]);
    for (int j = 0; j < 12; ++j) {
      const double psi = 0.5 * (1.0 + GN[j]);
      const double w = 0.25 * GW[i] * GW[j];
      const v3 te = v_add(de, v_mul(dc, psi));
      const v3 tp = v_add(dp, v_mul(dc, eta));
      const v3 oa = v_cross(te, tp);
      const double aw = w * sqrt(v_dot(oa, oa));
      const v3 pt = g_bilinear(f, eta, psi);
      g->area += aw;
      g->area_vector = v_add(g->area_vector, v_mul(oa, w));
      g->centroid = v_add(g->centroid, v_mul(pt, aw));
    }
  }
  if (!isfinite(g->area) || g->area <= DBL_MIN) return -1;
  g->centroid = v_mul(g->centroid, 1.0 / g->area);
  const v3 ce = v_mul(v_add(v_sub(f[3], f[2]), v_sub(f[1], f[0])), 0.5);
  const v3 cp = v_mul(v_add(v_sub(f[3], f[1]), v_sub(f[2], f[0])), 0.5);
  if (g_normalize(v_cross(ce, cp), &g->normal) != 0 ||
      g_normalize(cp, &g->tangent2) != 0 ||
      g_normalize(v_cross(g->tangent2, g->normal), &g->tangent1) != 0)
    return -1;
  return 0;
}

/* nonorthogonal_geometry.c:160-210 */
static int g_volume(const v3 c[8], double *vol, v3 *cen) {
  *vol = 0.0;
  *cen = v_zero();
  for (int i = 0; i < 12; ++i) {
    const double xi = GN[i];
    for (int j = 0; j < 12; ++j) {
      const double eta = GN[j];
      for (int k = 0; k < 12; ++k) {
        const double zeta = GN[k];
        v3 pt = v_zero();
        v3 der[3] = {v_zero(), v_zero(), v_zero()};
        for (int q = 0; q < 8; ++q) {
          const double sx = (double)LSIGN[q][0], sy = (double)LSIGN[q][1],
                       sz = (double)LSIGN[q][2];
          const double fx = 1.0 + sx * xi, fy = 1.0 + sy * eta,
                       fz = 1.0 + sz * zeta;
          const double shape = 0.125 * fx * fy * fz;
          const double ds[3] = {0.125 * sx * fy * fz, 0.125 * fx * sy * fz,
                                0.125 * fx * fy * sz};
          pt = v_add(pt, v_mul(c[q], shape));
          for (int d = 0; d < 3; ++d) der[d] = v_add(der[d], v_mul(c[q], ds[d]));
        }
        const double det = v_dot(der[0], v_cross(der[1], der[2]));
        const double wv = fabs(det) * GW[i] * GW[j] * GW[k];
        *vol += wv;
        *cen = v_add(*cen, v_mul(pt, wv));
      }
    }
  }
  if (!isfinite(*vol) || *vol <= DBL_MIN) return -1;
  *cen = v_mul(*cen, 1.0 / *vol);
  return 0;
}

/* nonorthogonal_geometry.c:212-243 */
static int g_cell(const v3 c[8], gamera_no_cell_geometry *g) {
  if (g_volume(c, &g->volume, &g->centroid) != 0) return -1;
  for (int d = 0; d < 3; ++d) {
    for (int s = 0; s < 2; ++s) {
      v3 f[4];
      for (int q = 0; q < 4; ++q) f[q] = c[FCORNER[d][s][q]];
      if (g_face(f, &g->face[d][s]) != 0) return -1;
    }
    const double ma = fmax(g->face[d][0].area, g->face[d][1].area);
    g->cfl_length[d] = g->volume / ma;
  }
  return 0;
}

/* nonorthogonal_geometry.c:245-262 */
static int g_edge(v3 s, v3 e, v3 avg, gamera_no_edge_geometry *g) {
  const v3 ed = v_sub(e, s);
  g->length = sqrt(v_dot(ed, ed));
  if (!isfinite(g->length) || g->length <= DBL_MIN ||
      g_normalize(ed, &g->normal) != 0 ||
      g_normalize(v_cross(avg, g->normal), &g->tangent1) != 0 ||
      g_normalize(v_cross(g->normal, g->tangent1), &g->tangent2) != 0)
    return -1;
  return 0;
}

/* --------------------------------------------------- grid (grid.c) */

static v3 g_vertex(const gamera_no_grid *g, size_t i, size_t j, size_t k) {
  return g->vertex[idx3(g->vertex_extent, i, j, k)];
}

void gcso_grid_destroy(gamera_no_grid *g) {
  if (!g) return;
  free(g->vertex);
  free(g->cell);
  for (int d = 0; d < 3; ++d) {
    free(g->face[d].value);
    free(g->edge[d].value);
    free(g->edge[d].valid);
  }
  memset(g, 0, sizeof(*g));
}

/* nonorthogonal_grid.c:59-245 */
int gcso_grid_create(const size_t ext[3], const v3 *vertices,
                     gamera_no_grid *g) {
  memset(g, 0, sizeof(*g));
  for (int a = 0; a < 3; ++a) {
    g->cell_extent[a] = ext[a];
    g->vertex_extent[a] = ext[a] + 1;
  }
  for (int d = 0; d < 3; ++d)
    for (int a = 0; a < 3; ++a) {
      g->face[d].extent[a] = ext[a] + (a == d);
      g->edge[d].extent[a] = ext[a] + (a != d);
    }
  const size_t nv = count3(g->vertex_extent), nc = count3(ext);
  g->vertex = malloc(nv * sizeof(v3));
  g->cell = calloc(nc, sizeof(gamera_no_cell_geometry));
  if (!g->vertex || !g->cell) { gcso_grid_destroy(g); return -1; }
  memcpy(g->vertex, vertices, nv * sizeof(v3));
  int failed = 0;
  for (size_t i = 0; i < ext[0]; ++i)
    for (size_t j = 0; j < ext[1]; ++j)
      for (size_t k = 0; k < ext[2]; ++k) {
        v3 c[8];
        for (int q = 0; q < 8; ++q)
          c[q] = g_vertex(g, i + COFF[q][0], j + COFF[q][1], k + COFF[q][2]);
        if (g_cell(c, &g->cell[idx3(ext, i, j, k)]) != 0) failed = 1;
      }
  if (failed) { gcso_grid_destroy(g); return -1; }
  for (int d = 0; d < 3; ++d) {
    const size_t *fe = g->face[d].extent;
    g->face[d].value = calloc(count3(fe), sizeof(gamera_no_face_geometry));
    if (!g->face[d].value) { gcso_grid_destroy(g); return -1; }
    for (size_t i = 0; i < fe[0]; ++i)
      for (size_t j = 0; j < fe[1]; ++j)
        for (size_t k = 0; k < fe[2]; ++k) {
          size_t ci[3] = {i, j, k};
          int side = 0;
          if (ci[d] == ext[d]) { --ci[d]; side = 1; }
          g->face[d].value[idx3(fe, i, j, k)] =
              g->cell[idx3(ext, ci[0], ci[1], ci[2])].face[d][side];
        }
  }
  for (int d = 0; d < 3; ++d) {
    const size_t *ee = g->edge[d].extent;
    g->edge[d].value = calloc(count3(ee), sizeof(gamera_no_edge_geometry));
    g->edge[d].valid = calloc(count3(ee), 1);
    if (!g->edge[d].value || !g->edge[d].valid) { gcso_grid_destroy(g); return -1; }
    for (size_t i = 0; i < ee[0]; ++i)
      for (size_t j = 0; j < ee[1]; ++j)
        for (size_t k = 0; k < ee[2]; ++k) {
          int interior;
          if (d == 0) interior = j > 0 && j < ext[1] && k > 0 && k < ext[2];
          else if (d == 1) interior = i > 0 && i < ext[0] && k > 0 && k < ext[2];
          else interior = i > 0 && i < ext[0] && j > 0 && j < ext[1];
          if (!interior) continue;
          size_t e[3] = {i, j, k};
          ++e[d];
          v3 first, second;
          if (d == 0) {
            first = v_sub(g_vertex(g, i, j, k + 1), g_vertex(g, i, j, k - 1));
            second = v_sub(g_vertex(g, i + 1, j, k + 1),
                           g_vertex(g, i + 1, j, k - 1));
          } else if (d == 1) {
            first = v_sub(g_vertex(g, i + 1, j, k), g_vertex(g, i - 1, j, k));
            second = v_sub(g_vertex(g, i + 1, j + 1, k),
                           g_vertex(g, i - 1, j + 1, k));
          } else {
            first = v_sub(g_vertex(g, i, j + 1, k), g_vertex(g, i, j - 1, k));
            second = v_sub(g_vertex(g, i, j + 1, k + 1),
                           g_vertex(g, i, j - 1, k + 1));
          }
          const v3 avg = v_scale(v_add(first, second), 0.5);
          const size_t x = idx3(ee, i, j, k);
          if (g_edge(g_vertex(g, i, j, k), g_vertex(g, e[0], e[1], e[2]), avg,
                     &g->edge[d].value[x]) != 0) {
            gcso_grid_destroy(g);
            return -1;
          }
          g->edge[d].valid[x] = 1;
        }
  }
  return 0;
}

/* ------------------------------------------- mesh (cubedsphere_mesh.c) */

static const int FRAME[6][3][3] = {
    {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}},   {{-1, 0, 0}, {0, -1, 0}, {0, 0, 1}},
    {{0, 1, 0}, {-1, 0, 0}, {0, 0, 1}},  {{0, -1, 0}, {1, 0, 0}, {0, 0, 1}},
    {{0, 0, 1}, {1, 0, 0}, {0, 1, 0}},   {{0, 0, -1}, {1, 0, 0}, {0, -1, 0}}};

static double m_dot(v3 a, const int b[3]) {
  return a.value[0] * (double)b[0] + a.value[1] * (double)b[1] +
         a.value[2] * (double)b[2];
}

/* cubedsphere_mesh.c:58-75 */
static int m_direction(int face, double a, double b, v3 *out) {
  const double qp = 0.25 * acos(-1.0);
  if (!isfinite(a) || !isfinite(b) || fabs(a) >= 2.0 * qp ||
      fabs(b) >= 2.0 * qp)
    return -1;
  const double u = tan(a), v = tan(b);
  const double il = 1.0 / sqrt(1.0 + u * u + v * v);
  for (int d = 0; d < 3; ++d)
    out->value[d] = il * ((double)FRAME[face][0][d] + u * (double)FRAME[face][1][d] +
                          v * (double)FRAME[face][2][d]);
  return 0;
}

/* cubedsphere_mesh.c:77-103 */
static int m_inverse(v3 dir, int *face, double *a, double *b) {
  if (!v_finite(dir)) return -1;
  int sel = -1;
  double dom = 0.0;
  for (int f = 0; f < 6; ++f) {
    const double p = m_dot(dir, FRAME[f][0]);
    if (p > dom) { dom = p; sel = f; }
  }
  if (sel < 0 || !isfinite(dom)) return -1;
  *face = sel;
  *a = atan2(m_dot(dir, FRAME[sel][1]), dom);
  *b = atan2(m_dot(dir, FRAME[sel][2]), dom);
  return 0;
}

/* cubedsphere_mesh.c:105-162 */
static int m_neighbor(int face, int edge, int *nf, int *ne, int *rev) {
  const double qp = 0.25 * acos(-1.0), eps = 1.0e-7;
  double a = 0.0, b = 0.0;
  if (edge < 2) a = (edge == 0 ? -1.0 : 1.0) * (qp + eps);
  else b = (edge == 2 ? -1.0 : 1.0) * (qp + eps);
  v3 out;
  int t;
  double ta, tb;
  if (m_direction(face, a, b, &out) != 0 || m_inverse(out, &t, &ta, &tb) != 0 ||
      t == face)
    return -1;
  const int de = fabs(ta) > fabs(tb) ? (ta < 0.0 ? 0 : 1) : (tb < 0.0 ? 2 : 3);
  double along[2];
  for (int n = 0; n < 2; ++n) {
    const double pos = n == 0 ? -0.2 : 0.2;
    double sa, sb;
    if (edge < 2) { sa = edge == 0 ? -qp : qp; sb = pos; }
    else { sa = pos; sb = edge == 2 ? -qp : qp; }
    if (m_direction(face, sa, sb, &out) != 0) return -1;
    const double p = m_dot(out, FRAME[t][0]);
    const double xa = atan2(m_dot(out, FRAME[t][1]), p);
    const double xb = atan2(m_dot(out, FRAME[t][2]), p);
    along[n] = de < 2 ? xb : xa;
  }
  *nf = t;
  *ne = de;
  *rev = along[1] < along[0];
  return 0;
}

/* cubedsphere_mesh.c:36-56 */
static int m_key(int face, const size_t act[3], const size_t v[3],
                 int64_t key[4]) {
  for (int a = 0; a < 3; ++a)
    if (v[a] > act[a]) return -1;
  const int64_t n = (int64_t)act[1];
  const int64_t a = 2 * (int64_t)v[1] - n, b = 2 * (int64_t)v[2] - n;
  key[0] = (int64_t)v[0];
  for (int d = 0; d < 3; ++d)
    key[d + 1] = (int64_t)FRAME[face][0][d] * n + (int64_t)FRAME[face][1][d] * a +
                 (int64_t)FRAME[face][2][d] * b;
  return 0;
}

/* cubedsphere_mesh.c:164-254.  stretch <= 0: linear radius (the
 * r_inner + logical * dr path); stretch > 0: legacy exponential radial map
 * nonorthogonal_radial_map.c:152-156 evaluated at logical_i / nr. */
int gcso_generate_vertices(int face, const size_t act[3], size_t ghost,
                           double r_in, double r_out, double stretch, v3 *v) {
  const double qp = 0.25 * acos(-1.0);
  const double da = 2.0 * qp / (double)act[1], db = 2.0 * qp / (double)act[2];
  if (qp + (double)ghost * fmax(da, db) >= 2.0 * qp) return -1;
  if (stretch <= 0.0 && r_in <= (double)ghost * (r_out - r_in) / (double)act[0])
    return -1;
  const size_t ve[3] = {act[0] + 2 * ghost + 1, act[1] + 2 * ghost + 1,
                        act[2] + 2 * ghost + 1};
  const double dr = (r_out - r_in) / (double)act[0];
  for (size_t i = 0; i < ve[0]; ++i) {
    const double li = 0.0 + (double)i - (double)ghost;
    double r = r_in + li * dr;
    if (stretch > 0.0)
      r = r_in + (r_out - r_in) * expm1(stretch * (li / (double)act[0])) /
                     expm1(stretch);
    if (!(r > 0.0) || !isfinite(r)) return -1;
    for (size_t j = 0; j < ve[1]; ++j) {
      const double a = -qp + (0.0 + (double)j - (double)ghost) * da;
      for (size_t k = 0; k < ve[2]; ++k) {
        const double b = -qp + (0.0 + (double)k - (double)ghost) * db;
        v3 dir;
        if (m_direction(face, a, b, &dir) != 0) return -1;
        const size_t x = idx3(ve, i, j, k);
        for (int d = 0; d < 3; ++d) v[x].value[d] = r * dir.value[d];
      }
    }
  }
  return 0;
}

/* cubedsphere_mesh.c:256-303 */
static int m_calibrate(gamera_no_face_geometry *f) {
  const v3 a = f->area_vector;
  const double mag = sqrt(a.value[0] * a.value[0] + a.value[1] * a.value[1] +
                          a.value[2] * a.value[2]);
  if (!isfinite(mag) || mag <= 0.0) return -1;
  v3 n;
  for (int d = 0; d < 3; ++d) n.value[d] = a.value[d] / mag;
  const v3 ot2 = f->tangent2;
  double p = 0.0;
  for (int d = 0; d < 3; ++d) p += ot2.value[d] * n.value[d];
  v3 t2;
  double t2s = 0.0;
  for (int d = 0; d < 3; ++d) {
    t2.value[d] = ot2.value[d] - p * n.value[d];
    t2s += t2.value[d] * t2.value[d];
  }
  if (!isfinite(t2s) || t2s <= 0.0) return -1;
  for (int d = 0; d < 3; ++d) t2.value[d] /= sqrt(t2s);
  const v3 t1 = {{t2.value[1] * n.value[2] - t2.value[2] * n.value[1],
                  t2.value[2] * n.value[0] - t2.value[0] * n.value[2],
                  t2.value[0] * n.value[1] - t2.value[1] * n.value[0]}};
  f->area = mag;
  f->normal = n;
  f->tangent1 = t1;
  f->tangent2 = t2;
  return 0;
}

int gcso_calibrate_face_frames(gamera_no_grid *g) {
  const size_t nc = count3(g->cell_extent);
  for (size_t c = 0; c < nc; ++c)
    for (int d = 0; d < 3; ++d)
      for (int s = 0; s < 2; ++s)
        if (m_calibrate(&g->cell[c].face[d][s]) != 0) return -1;
  for (int d = 0; d < 3; ++d) {
    const size_t nf = count3(g->face[d].extent);
    for (size_t f = 0; f < nf; ++f)
      if (m_calibrate(&g->face[d].value[f]) != 0) return -1;
  }
  return 0;
}

/* --------------------------------------------------- storage (storage.c) */

void gcso_storage_destroy(gamera_no_storage *s) {
  if (!s) return;
  free(s->conserved); free(s->old_conserved); free(s->predicted_conserved);
  free(s->cell_magnetic); free(s->old_cell_magnetic);
  free(s->predicted_cell_magnetic); free(s->hydro_rate); free(s->maxwell_rate);
  for (int d = 0; d < 3; ++d) {
    free(s->face_flux[d]); free(s->old_face_flux[d]);
    free(s->predicted_face_flux[d]); free(s->edge_emf[d]);
    free(s->fluid_face_flux[d]); free(s->maxwell_face_flux[d]);
  }
  memset(s, 0, sizeof(*s));
}

/* nonorthogonal_storage.c:18-88 */
int gcso_storage_create(const size_t ext[3], gamera_no_storage *s) {
  memset(s, 0, sizeof(*s));
  for (int a = 0; a < 3; ++a) s->cell_extent[a] = ext[a];
  const size_t nc = count3(ext);
  s->conserved = calloc(5 * nc, sizeof(double));
  s->old_conserved = calloc(5 * nc, sizeof(double));
  s->predicted_conserved = calloc(5 * nc, sizeof(double));
  s->cell_magnetic = calloc(nc, sizeof(v3));
  s->old_cell_magnetic = calloc(nc, sizeof(v3));
  s->predicted_cell_magnetic = calloc(nc, sizeof(v3));
  s->hydro_rate = calloc(5 * nc, sizeof(double));
  s->maxwell_rate = calloc(nc, sizeof(v3));
  int bad = !s->conserved || !s->old_conserved || !s->predicted_conserved ||
            !s->cell_magnetic || !s->old_cell_magnetic ||
            !s->predicted_cell_magnetic || !s->hydro_rate || !s->maxwell_rate;
  for (int d = 0; d < 3 && !bad; ++d) {
    for (int a = 0; a < 3; ++a) {
      s->face_extent[d][a] = ext[a] + (a == d);
      s->edge_extent[d][a] = ext[a] + (a != d);
    }
    const size_t nf = count3(s->face_extent[d]), ne = count3(s->edge_extent[d]);
    s->face_flux[d] = calloc(nf, sizeof(double));
    s->old_face_flux[d] = calloc(nf, sizeof(double));
    s->predicted_face_flux[d] = calloc(nf, sizeof(double));
    s->fluid_face_flux[d] = calloc(5 * nf, sizeof(double));
    s->maxwell_face_flux[d] = calloc(nf, sizeof(v3));
    s->edge_emf[d] = calloc(ne, sizeof(double));
    bad = !s->face_flux[d] || !s->old_face_flux[d] || !s->predicted_face_flux[d] ||
          !s->fluid_face_flux[d] || !s->maxwell_face_flux[d] || !s->edge_emf[d];
  }
  if (bad) { gcso_storage_destroy(s); return -1; }
  return 0;
}

/* --------------------------------------------- background (background.c) */

/* nonorthogonal_background.c:422-442 */
static int b_dipole(v3 p, v3 m, v3 *field) {
  if (!v_finite(p) || !v_finite(m)) return -1;
  const double r2 = v_dot(p, p);
  if (!(r2 > DBL_MIN) || !isfinite(r2)) return -1;
  const double r = sqrt(r2);
  const double ir3 = 1.0 / (r2 * r);
  const double ir5 = ir3 / r2;
  const double proj = v_dot(m, p);
  *field = v_sub(v_scale(p, 3.0 * proj * ir5), v_scale(m, ir3));
  return v_finite(*field) ? 0 : -1;
}

static v3 b_bilinear(const v3 f[4], double eta, double psi) {
  const v3 de = v_sub(f[1], f[0]);
  const v3 dp = v_sub(f[2], f[0]);
  const v3 dc = v_add(v_sub(f[3], f[2]), v_sub(f[0], f[1]));
  return v_add(f[0], v_add(v_scale(de, eta),
                           v_add(v_scale(dp, psi), v_scale(dc, eta * psi))));
}

/* nonorthogonal_background.c:111-164 */
static int b_face(const v3 f[4], double area_s, v3 m, v3 *avg, double *flux,
                  v3 *stress) {
  const v3 de = v_sub(f[1], f[0]);
  const v3 dp = v_sub(f[2], f[0]);
  const v3 dc = v_add(v_sub(f[3], f[2]), v_sub(f[0], f[1]));
  v3 in = v_zero(), st = v_zero();
  double fl = 0.0;
  if (!(area_s > DBL_MIN) || !isfinite(area_s)) return -1;
  for (int i = 0; i < 12; ++i) {
    const double eta = 0.5 * (1.0 + GN[i]);
    for (int j = 0; j < 12; ++j) {
      const double psi = 0.5 * (1.0 + GN[j]);
      const double w = 0.25 * GW[i] * GW[j];
      const v3 te = v_add(de, v_scale(dc, psi));
      const v3 tp = v_add(dp, v_scale(dc, eta));
      const v3 oa = v_cross(te, tp);
      const double area = sqrt(v_dot(oa, oa));
      const v3 pt = b_bilinear(f, eta, psi);
      v3 fld;
      if (!(area > DBL_MIN) || !isfinite(area) || b_dipole(pt, m, &fld) != 0)
        return -1;
      in = v_add(in, v_scale(fld, w * area));
      const double nf = v_dot(fld, oa);
      fl += w * nf;
      const double pm = 0.5 * v_dot(fld, fld);
      st = v_add(st, v_scale(v_sub(v_scale(oa, pm), v_scale(fld, nf)), w));
    }
  }
  *avg = v_scale(in, 1.0 / area_s);
  *flux = fl;
  *stress = st;
  return v_finite(*avg) && isfinite(*flux) && v_finite(*stress) ? 0 : -1;
}

/* nonorthogonal_background.c:166-215 */
static int b_cell(const v3 c[8], double vol, v3 m, v3 *avg) {
  v3 in = v_zero();
  double iv = 0.0;
  if (!(vol > DBL_MIN) || !isfinite(vol)) return -1;
  for (int i = 0; i < 12; ++i)
    for (int j = 0; j < 12; ++j)
      for (int k = 0; k < 12; ++k) {
        const double xi = GN[i], eta = GN[j], zeta = GN[k];
        v3 pt = v_zero();
        v3 der[3] = {v_zero(), v_zero(), v_zero()};
        for (int q = 0; q < 8; ++q) {
          const double sx = (double)LSIGN[q][0], sy = (double)LSIGN[q][1],
                       sz = (double)LSIGN[q][2];
          const double fx = 1.0 + sx * xi, fy = 1.0 + sy * eta,
                       fz = 1.0 + sz * zeta;
          const double shape = 0.125 * fx * fy * fz;
          const double ds[3] = {0.125 * sx * fy * fz, 0.125 * fx * sy * fz,
                                0.125 * fx * fy * sz};
          pt = v_add(pt, v_scale(c[q], shape));
          for (int d = 0; d < 3; ++d) der[d] = v_add(der[d], v_scale(c[q], ds[d]));
        }
        const double jac = fabs(v_dot(der[0], v_cross(der[1], der[2])));
        const double w = jac * GW[i] * GW[j] * GW[k];
        v3 fld;
        if (!isfinite(w) || b_dipole(pt, m, &fld) != 0) return -1;
        iv += w;
        in = v_add(in, v_scale(fld, w));
      }
  if (!(iv > DBL_MIN) || fabs(iv - vol) > 2.0e-11 * vol) return -1;
  *avg = v_scale(in, 1.0 / vol);
  return v_finite(*avg) ? 0 : -1;
}

/* nonorthogonal_background.c:217-236 */
static int b_edge(v3 s, v3 e, v3 m, v3 *avg) {
  const v3 disp = v_sub(e, s);
  v3 r = v_zero();
  if (!(sqrt(v_dot(disp, disp)) > DBL_MIN)) return -1;
  for (int n = 0; n < 12; ++n) {
    const double t = 0.5 * (1.0 + GN[n]);
    v3 fld;
    if (b_dipole(v_add(s, v_scale(disp, t)), m, &fld) != 0) return -1;
    r = v_add(r, v_scale(fld, 0.5 * GW[n]));
  }
  *avg = r;
  return v_finite(*avg) ? 0 : -1;
}

void gcso_background_destroy(gcso_background *bg) {
  if (!bg) return;
  free(bg->cell_magnetic);
  free(bg->cell_force);
  for (int d = 0; d < 3; ++d) {
    free(bg->face_magnetic[d]);
    free(bg->face_flux[d]);
    free(bg->edge_magnetic[d]);
  }
  memset(bg, 0, sizeof(*bg));
}

/* nonorthogonal_background.c:273-420 with the dipole field */
int gcso_background_create(const gamera_no_grid *g, v3 m, gcso_background *bg) {
  memset(bg, 0, sizeof(*bg));
  const size_t *ce = g->cell_extent;
  const size_t nc = count3(ce);
  v3 *fs[3] = {NULL, NULL, NULL};
  bg->cell_magnetic = calloc(nc, sizeof(v3));
  bg->cell_force = calloc(nc, sizeof(v3));
  int bad = !bg->cell_magnetic || !bg->cell_force;
  for (int d = 0; d < 3 && !bad; ++d) {
    const size_t nf = count3(g->face[d].extent), ne = count3(g->edge[d].extent);
    bg->face_magnetic[d] = calloc(nf, sizeof(v3));
    bg->face_flux[d] = calloc(nf, sizeof(double));
    bg->edge_magnetic[d] = calloc(ne, sizeof(v3));
    fs[d] = calloc(nf, sizeof(v3));
    bad = !bg->face_magnetic[d] || !bg->face_flux[d] || !bg->edge_magnetic[d] ||
          !fs[d];
  }
  for (int d = 0; d < 3 && !bad; ++d) {
    const size_t *fe = g->face[d].extent;
    for (size_t i = 0; i < fe[0]; ++i)
      for (size_t j = 0; j < fe[1]; ++j)
        for (size_t k = 0; k < fe[2]; ++k) {
          size_t cc[3] = {i, j, k};
          int side = 0;
          if (cc[d] == ce[d]) { --cc[d]; side = 1; }
          v3 c[8], f[4];
          for (int q = 0; q < 8; ++q)
            c[q] = g_vertex(g, cc[0] + COFF[q][0], cc[1] + COFF[q][1],
                            cc[2] + COFF[q][2]);
          for (int q = 0; q < 4; ++q) f[q] = c[FCORNER[d][side][q]];
          const size_t x = idx3(fe, i, j, k);
          if (b_face(f, g->face[d].value[x].area, m, &bg->face_magnetic[d][x],
                     &bg->face_flux[d][x], &fs[d][x]) != 0)
            bad = 1;
        }
  }
  for (size_t i = 0; i < ce[0] && !bad; ++i)
    for (size_t j = 0; j < ce[1]; ++j)
      for (size_t k = 0; k < ce[2]; ++k) {
        v3 c[8];
        for (int q = 0; q < 8; ++q)
          c[q] = g_vertex(g, i + COFF[q][0], j + COFF[q][1], k + COFF[q][2]);
        const size_t x = idx3(ce, i, j, k);
        if (b_cell(c, g->cell[x].volume, m, &bg->cell_magnetic[x]) != 0) {
          bad = 1;
          continue;
        }
        v3 um = v_zero();
        for (int d = 0; d < 3; ++d) {
          size_t u[3] = {i, j, k};
          ++u[d];
          const size_t lo = idx3(g->face[d].extent, i, j, k);
          const size_t hi = idx3(g->face[d].extent, u[0], u[1], u[2]);
          um = v_add(um, v_sub(fs[d][hi], fs[d][lo]));
        }
        bg->cell_force[x] = v_scale(um, -1.0 / g->cell[x].volume);
        if (!v_finite(bg->cell_force[x])) bad = 1;
      }
  for (int d = 0; d < 3 && !bad; ++d) {
    const size_t *ee = g->edge[d].extent;
    for (size_t i = 0; i < ee[0]; ++i)
      for (size_t j = 0; j < ee[1]; ++j)
        for (size_t k = 0; k < ee[2]; ++k) {
          size_t e[3] = {i, j, k};
          ++e[d];
          if (b_edge(g_vertex(g, i, j, k), g_vertex(g, e[0], e[1], e[2]), m,
                     &bg->edge_magnetic[d][idx3(ee, i, j, k)]) != 0)
            bad = 1;
        }
  }
  for (int d = 0; d < 3; ++d) {
    free(fs[d]);
    bg->field.face_magnetic[d] = bg->face_magnetic[d];
    bg->field.face_flux[d] = bg->face_flux[d];
    bg->field.edge_magnetic[d] = bg->edge_magnetic[d];
  }
  bg->field.cell_magnetic = bg->cell_magnetic;
  bg->field.cell_force = bg->cell_force;
  if (bad) { gcso_background_destroy(bg); return -1; }
  return 0;
}

/* ------------------------------------------------------- state (state.c) */

typedef struct {
  double density;
  v3 velocity;
  double pressure;
} prim;

static int valid_params(double g, double rf, double pf) {
  return isfinite(g) && g > 1.0 && isfinite(rf) && rf > 0.0 && isfinite(pf) &&
         pf > 0.0;
}

/* nonorthogonal_state.c:60-93 */
static int s_c2p(const double u[5], double g, double rf, double pf, prim *p) {
  if (!valid_params(g, rf, pf) || !isfinite(u[0]) || u[0] <= DBL_MIN) return -1;
  const double raw = u[0];
  double v2 = 0.0;
  for (int d = 0; d < 3; ++d) {
    const double m = u[1 + d];
    if (!isfinite(m)) return -1;
    p->velocity.value[d] = m / raw;
    v2 += p->velocity.value[d] * p->velocity.value[d];
  }
  if (!isfinite(u[4])) return -1;
  const double kin = 0.5 * raw * v2;
  p->density = fmax(raw, rf);
  p->pressure = fmax((g - 1.0) * (u[4] - kin), pf);
  return 0;
}

/* nonorthogonal_state.c:95-120 */
static int s_p2c(const prim *p, double g, double rf, double pf, double u[5]) {
  if (!valid_params(g, rf, pf) || !isfinite(p->density) || !isfinite(p->pressure))
    return -1;
  const double rho = fmax(p->density, rf);
  const double pr = fmax(p->pressure, pf);
  double v2 = 0.0;
  u[0] = rho;
  for (int d = 0; d < 3; ++d) {
    if (!isfinite(p->velocity.value[d])) return -1;
    u[1 + d] = rho * p->velocity.value[d];
    v2 += p->velocity.value[d] * p->velocity.value[d];
  }
  u[4] = pr / (g - 1.0) + 0.5 * rho * v2;
  return 0;
}

/* nonorthogonal_step.c:74-171: post-step pressure control over the cells
 * [lower, upper) of one face (serial; the counts and maxima are
 * order-independent). */
int gcso_apply_pressure_control(gamera_no_storage *s, const gamera_no_grid *g,
                                const size_t lower[3], const size_t upper[3], double dt,
                                double gamma, double rf, double pf, double c,
                                double low_threshold, double low_sound, size_t *low_count,
                                size_t *hot_count, double *max_sound, double *max_pressure) {
  if (!s || !g || !lower || !upper || !s->conserved || !(dt > 0.0) || !(gamma > 1.0) ||
      !(rf > 0.0) || !(pf > 0.0) || !(c > 0.0) || !(low_threshold > 0.0) ||
      !(low_sound >= 0.0))
    return -1;
  size_t low = 0, hot = 0;
  double ms = 0.0, mp = 0.0;
  int failed = 0;
  for (size_t i = lower[0]; i < upper[0]; ++i)
    for (size_t j = lower[1]; j < upper[1]; ++j)
      for (size_t k = lower[2]; k < upper[2]; ++k) {
        const size_t cell = idx3(s->cell_extent, i, j, k);
        double *u = &s->conserved[cell * 5];
        prim p;
        if (s_c2p(u, gamma, rf, pf, &p) != 0) {
          failed = 1;
          continue;
        }
        int changed = 0;
        if (p.density <= low_threshold) {
          p.pressure = fmax(pf, p.density * low_sound * low_sound / gamma);
          ++low;
          changed = 1;
        }
        const double cs = sqrt(gamma * p.pressure / p.density);
        ms = fmax(ms, cs);
        mp = fmax(mp, p.pressure);
        if (cs > 1.5 * c) {
          const v3 x = g->cell[cell].centroid;
          const double r2 = x.value[0] * x.value[0] + x.value[1] * x.value[1] +
                            x.value[2] * x.value[2];
          const double q2 = x.value[0] * x.value[0] + x.value[1] * x.value[1];
          if (!(r2 > 0.0) || !(q2 > DBL_MIN)) {
            failed = 1;
            continue;
          }
          const double L = sqrt(r2) * r2 / q2;
          const double target = p.density * (1.5 * c) * (1.5 * c) / gamma;
          p.pressure -= (dt / (L / cs)) * (p.pressure - target);
          ++hot;
          changed = 1;
        }
        if (changed && s_p2c(&p, gamma, rf, pf, u) != 0) failed = 1;
      }
  if (low_count) *low_count = low;
  if (hot_count) *hot_count = hot;
  if (max_sound) *max_sound = ms;
  if (max_pressure) *max_pressure = mp;
  return failed ? -1 : 0;
}

/* nonorthogonal_state.c:122-159 */
static int s_predict(const double uo[5], const double uc[5], double r, double g,
                     double rf, double pf, double out[5]) {
  if (!isfinite(r)) return -1;
  prim o, c;
  if (s_c2p(uo, g, rf, pf, &o) != 0 || s_c2p(uc, g, rf, pf, &c) != 0) return -1;
  prim q = c;
  q.density = fmax(c.density + r * (c.density - o.density), rf);
  q.pressure = fmax(c.pressure + r * (c.pressure - o.pressure), pf);
  for (int d = 0; d < 3; ++d)
    q.velocity.value[d] = c.velocity.value[d] +
                          r * (c.velocity.value[d] - o.velocity.value[d]);
  return s_p2c(&q, g, rf, pf, out);
}

/* nonorthogonal_state.c:161-174 */
static int s_maxwell(double u[5], v3 rate, double dt, double g, double rf,
                     double pf) {
  if (!isfinite(dt) || !valid_params(g, rf, pf)) return -1;
  const double rho = fmax(u[0], rf);
  double om = 0.0;
  for (int d = 0; d < 3; ++d) om += u[1 + d] * u[1 + d];
  const double pr = fmax((g - 1.0) * (u[4] - 0.5 * om / rho), pf);
  double nm = 0.0;
  for (int d = 0; d < 3; ++d) {
    u[1 + d] += dt * rate.value[d];
    nm += u[1 + d] * u[1 + d];
  }
  u[0] = rho;
  u[4] = 0.5 * nm / rho + pr / (g - 1.0);
  return 0;
}

static v3 s_parallel(v3 v, v3 u) { return v_scale(u, v_dot(v, u)); }
static v3 s_perp(v3 v, v3 u) {
  const v3 p = s_parallel(v, u);
  for (int d = 0; d < 3; ++d) v.value[d] -= p.value[d];
  return v;
}
static v3 s_unit_or_zero(v3 v) {
  const double n = sqrt(v_dot(v, v));
  if (n <= 1.0e-12) return v_zero();
  return v_scale(v, 1.0 / n);
}

/* nonorthogonal_state.c:176-280 */
static int s_boris(double u[5], const double uo[5], v3 bn, v3 bo,
                   const double rate[5], v3 mrate, double c, double dt, double g,
                   double rf, double pf) {
  if (!isfinite(c) || c <= DBL_MIN || !isfinite(dt)) return -1;
  prim up;
  if (s_c2p(u, g, rf, pf, &up) != 0 || uo[0] <= DBL_MIN) return -1;
  const double urho = fmax(up.density, rf);
  const double upr = fmax(up.pressure, pf);
  const double orho = uo[0];
  v3 ov;
  for (int d = 0; d < 3; ++d) ov.value[d] = uo[1 + d] / fmax(orho, rf);
  const v3 half = v_scale(v_add(bn, bo), 0.5);
  const double alpha = v_dot(half, half) / (urho * c * c);
  const double drho = dt * rate[0];
  v3 gas, mag;
  for (int d = 0; d < 3; ++d) {
    gas.value[d] = dt * rate[1 + d];
    mag.value[d] = dt * mrate.value[d];
  }
  v3 inc;
  if (alpha > 1.0e-12) {
    const double frac = 1.0 / (1.0 + alpha);
    const v3 unit = s_unit_or_zero(half);
    const v3 tot = v_add(gas, mag);
    inc = v_add(s_parallel(gas, unit),
                v_add(v_scale(s_perp(tot, unit), frac),
                      v_scale(s_perp(ov, unit), alpha * frac * drho)));
  } else {
    inc = v_add(gas, mag);
  }
  prim r = up;
  r.density = urho;
  r.pressure = upr;
  for (int d = 0; d < 3; ++d)
    r.velocity.value[d] = (orho * ov.value[d] + inc.value[d]) / urho;
  return s_p2c(&r, g, rf, pf, u);
}

/* ------------------------------------- reconstruction (reconstruction.c) */

static const double C8[8] = {-3.0 / 840.0, 29.0 / 840.0, -139.0 / 840.0,
                             533.0 / 840.0, 533.0 / 840.0, -139.0 / 840.0,
                             29.0 / 840.0, -3.0 / 840.0};
static const double C6[8] = {0.0, 1.0 / 60.0, -8.0 / 60.0, 37.0 / 60.0,
                             37.0 / 60.0, -8.0 / 60.0, 1.0 / 60.0, 0.0};
static const double U7[7] = {-3.0 / 420.0, 25.0 / 420.0, -101.0 / 420.0,
                             319.0 / 420.0, 214.0 / 420.0, -38.0 / 420.0,
                             4.0 / 420.0};

static double r_dot8(const double v[8], const double c[8]) {
  double r = 0.0;
  for (int n = 0; n < 8; ++n) r += c[n] * v[n];
  return r;
}
static double r_central8(const double v[8]) { return r_dot8(v, C8); }
static double r_central6(const double v[8]) { return r_dot8(v, C6); }

/* nonorthogonal_reconstruction.c:39-51 */
static double r_pdm(double q0, double q1, double q2, double hi, double b) {
  const double bounded = fmax(fmin(q1, q2), fmin(hi, fmax(q1, q2)));
  const double d0 = b * (q1 - q0), d1 = b * (q2 - q1);
  const double s0 = copysign(1.0, d0), s1 = copysign(1.0, d1);
  const double same = fabs(s0 + s1);
  const double slope = bounded - q1;
  return bounded - s1 * fmax(0.0, fabs(slope) - same * fabs(d0));
}

/* nonorthogonal_reconstruction.c:61-93 */
static int r_up7pdm(const double vol[8], const double q[8], double b,
                    double *left, double *right) {
  if (!isfinite(b) || b < 0.0) return -1;
  double w[8];
  for (int n = 0; n < 8; ++n) w[n] = vol[n] * q[n];
  const double iv = r_central8(vol);
  if (!isfinite(iv) || fabs(iv) <= DBL_MIN) return -1;
  double ls[7], rs[7];
  for (int n = 0; n < 7; ++n) {
    ls[n] = w[n];
    rs[n] = w[7 - n];
  }
  double hl = 0.0, hr = 0.0;
  for (int n = 0; n < 7; ++n) hl += U7[n] * ls[n];
  for (int n = 0; n < 7; ++n) hr += U7[n] * rs[n];
  hl /= iv;
  hr /= iv;
  *left = r_pdm(q[2], q[3], q[4], hl, b);
  *right = r_pdm(q[5], q[4], q[3], hr, b);
  return 0;
}

/* ------------------------------------------------------------ flux.c */

typedef struct {
  double conserved[5], jump[5];
  v3 vjump;
  double vn[2];
} fluid_flux;
typedef struct {
  v3 momentum;
  double alfven, pmag;
} maxwell_flux;

static int valid_prim(prim s) {
  if (!isfinite(s.density) || !isfinite(s.pressure) || s.density <= DBL_MIN ||
      s.pressure <= DBL_MIN)
    return 0;
  return v_finite(s.velocity);
}

/* nonorthogonal_flux.c:38-105 */
static int f_fluid(const prim st[2], double g, const gamera_no_face_geometry *fc,
                   fluid_flux *fl) {
  if (!isfinite(g) || g <= 1.0 || !valid_prim(st[0]) || !valid_prim(st[1]))
    return -1;
  memset(fl, 0, sizeof(*fl));
  const double pi = 3.14159265358979323846264338327950288;
  const double sgn[2] = {-1.0, 1.0};
  for (int s = 0; s < 2; ++s) {
    const double rho = st[s].density, p = st[s].pressure;
    const v3 v = st[s].velocity;
    const double v2 = v_dot(v, v);
    const double en = 0.5 * rho * v2 + p / (g - 1.0);
    const double lam = rho / (2.0 * p);
    const double vn = v_dot(fc->normal, v);
    const double vt1 = v_dot(fc->tangent1, v);
    const double vt2 = v_dot(fc->tangent2, v);
    const double sg = sgn[s];
    const double z = 0.5 * erfc(sg * sqrt(lam) * vn);
    const double f1 = vn * z - 0.5 * sg * exp(-lam * vn * vn) / sqrt(pi * lam);
    fl->vn[s] = vn;
    fl->conserved[0] += rho * f1;
    fl->conserved[4] += (en + 0.5 * p) * f1 + 0.5 * p * z * vn;
    const double mn = rho * vn * f1 + p * z;
    const double m1 = rho * vt1 * f1;
    const double m2 = rho * vt2 * f1;
    for (int d = 0; d < 3; ++d) {
      fl->conserved[1 + d] += fc->normal.value[d] * mn +
                              fc->tangent1.value[d] * m1 +
                              fc->tangent2.value[d] * m2;
      fl->vjump.value[d] += sg * v.value[d];
    }
    fl->jump[0] += sg * rho;
    for (int d = 0; d < 3; ++d) fl->jump[1 + d] += sg * rho * v.value[d];
    fl->jump[4] += sg * en;
  }
  return 0;
}

/* nonorthogonal_flux.c:107-173 */
static int f_maxwell(const prim st[2], const v3 b[2], double bn,
                     const gamera_no_face_geometry *fc, int use_bg, v3 b0,
                     double b0n, int boris, double c, const double vn[2],
                     maxwell_flux *mx) {
  if (!isfinite(bn) || (boris && (!isfinite(c) || c <= DBL_MIN))) return -1;
  for (int s = 0; s < 2; ++s) {
    if (!valid_prim(st[s])) return -1;
    for (int d = 0; d < 3; ++d)
      if (!isfinite(b[s].value[d]) || (use_bg && !isfinite(b0.value[d])))
        return -1;
  }
  mx->momentum = v_zero();
  mx->alfven = 0.0;
  mx->pmag = 0.0;
  const double sgn[2] = {-1.0, 1.0};
  for (int s = 0; s < 2; ++s) {
    const double r2 = v_dot(b[s], b[s]);
    const double rp = 0.5 * r2;
    const v3 t = use_bg ? v_add(b[s], b0) : b[s];
    const double t2 = v_dot(t, t);
    const double va2 = t2 / st[s].density;
    const double cva2 = boris ? va2 / (1.0 + va2 / (c * c)) : va2;
    const double lam = 1.0 / (2.0 * st[s].pressure / st[s].density + cva2);
    const double z = 0.5 * erfc(sgn[s] * sqrt(lam) * vn[s]);
    mx->alfven += 0.5 * sqrt(cva2);
    mx->pmag += 0.5 * t2;
    const double bdr = use_bg ? v_dot(b0, b[s]) : 0.0;
    for (int d = 0; d < 3; ++d) {
      double stress = rp * fc->normal.value[d] - b[s].value[d] * bn;
      if (use_bg)
        stress += -b0.value[d] * bn - b[s].value[d] * b0n +
                  bdr * fc->normal.value[d];
      mx->momentum.value[d] += z * stress;
    }
  }
  return 0;
}

/* nonorthogonal_flux.c:175-204 */
static void f_hogs(fluid_flux *fl, maxwell_flux *mx, double ch, double cm,
                   int boris, double c) {
  for (int m = 0; m < 5; ++m) fl->conserved[m] -= ch * mx->alfven * fl->jump[m];
  if (boris) {
    const double ic2 = 1.0 / (c * c);
    for (int d = 0; d < 3; ++d) {
      const double j = mx->pmag * fl->vjump.value[d] * ic2;
      mx->momentum.value[d] -= cm * mx->alfven * j;
    }
  }
}

/* nonorthogonal_flux.c:206-241 */
static int f_emergency(fluid_flux *fl, const prim st[2], const double *lo,
                       const double *hi, int boris, double c, int *applied) {
  *applied = 0;
  if (!boris) return 0;
  double s2 = 0.0;
  for (int s = 0; s < 2; ++s) {
    if (!valid_prim(st[s])) return -1;
    s2 += v_dot(st[s].velocity, st[s].velocity);
  }
  if (sqrt(0.5 * s2) < 1.5 * c) return 0;
  for (int m = 0; m < 5; ++m) {
    if (!isfinite(lo[m]) || !isfinite(hi[m])) return -1;
    fl->conserved[m] -= c * (hi[m] - lo[m]);
  }
  *applied = 1;
  return 0;
}

/* ------------------------------------------------------- operators.c */

/* Calibrated recovery (cubedsphere/cubedsphere_recovery.c:17-98) over the
 * uncalibrated moment formula (nonorthogonal_operators.c:17-54). */
static int o_moment(const gamera_no_cell_geometry *g, const double fl[3][2],
                    v3 *field) {
  if (!isfinite(g->volume) || g->volume <= DBL_MIN) return -1;
  double div = 0.0;
  *field = v_zero();
  for (int d = 0; d < 3; ++d) {
    const double lo = fl[d][0], hi = fl[d][1];
    div += hi - lo;
    for (int c = 0; c < 3; ++c)
      field->value[c] += hi * g->face[d][1].centroid.value[c] -
                         lo * g->face[d][0].centroid.value[c];
  }
  for (int c = 0; c < 3; ++c)
    field->value[c] = (field->value[c] - div * g->centroid.value[c]) / g->volume;
  return 0;
}

static int o_solve3(const double m[3][3], const double rhs[3], v3 *x) {
  double a[3][4];
  double scale = 0.0;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) {
      a[i][j] = m[i][j];
      scale = fmax(scale, fabs(m[i][j]));
    }
    a[i][3] = rhs[i];
  }
  if (!isfinite(scale) || scale <= DBL_MIN) return -1;
  for (int col = 0; col < 3; ++col) {
    int piv = col;
    for (int r = col + 1; r < 3; ++r)
      if (fabs(a[r][col]) > fabs(a[piv][col])) piv = r;
    if (!isfinite(a[piv][col]) || fabs(a[piv][col]) <= 128.0 * DBL_EPSILON * scale)
      return -1;
    if (piv != col)
      for (int j = col; j < 4; ++j) {
        const double t = a[col][j];
        a[col][j] = a[piv][j];
        a[piv][j] = t;
      }
    const double inv = 1.0 / a[col][col];
    for (int j = col; j < 4; ++j) a[col][j] *= inv;
    for (int r = 0; r < 3; ++r) {
      if (r == col) continue;
      const double f = a[r][col];
      for (int j = col; j < 4; ++j) a[r][j] -= f * a[col][j];
    }
  }
  for (int i = 0; i < 3; ++i) {
    if (!isfinite(a[i][3])) return -1;
    x->value[i] = a[i][3];
  }
  return 0;
}

static int o_recover(const gamera_no_cell_geometry *g, const double fl[3][2],
                     v3 *field) {
  v3 raw;
  if (o_moment(g, fl, &raw) != 0) return -1;
  double resp[3][3];
  for (int b = 0; b < 3; ++b) {
    double bf[3][2];
    for (int d = 0; d < 3; ++d)
      for (int s = 0; s < 2; ++s) bf[d][s] = g->face[d][s].area_vector.value[b];
    v3 col;
    if (o_moment(g, bf, &col) != 0) return -1;
    for (int d = 0; d < 3; ++d) resp[d][b] = col.value[d];
  }
  return o_solve3(resp, raw.value, field);
}

/* nonorthogonal_operators.c:56-79 */
static int o_solve_edge(const double n1[2], const double n2[2], double f1,
                        double f2, double e[2]) {
  const double det = n1[0] * n2[1] - n2[0] * n1[1];
  const double sc = fmax(fmax(fabs(n1[0]), fabs(n1[1])),
                         fmax(fabs(n2[0]), fabs(n2[1])));
  if (!isfinite(det) || sc <= DBL_MIN || fabs(det) <= 64.0 * DBL_EPSILON * sc * sc)
    return -1;
  const double inv = 1.0 / det;
  e[0] = inv * (n2[1] * f1 - n1[1] * f2);
  e[1] = inv * (-n2[0] * f1 + n1[0] * f2);
  return 0;
}

/* nonorthogonal_operators.c:81-113 */
static int o_normal_to_edge(const double area[8], const v3 nrm[8],
                            const gamera_no_edge_geometry *e, double tn[2]) {
  const double ia = r_central6(area);
  if (!isfinite(ia) || fabs(ia) <= DBL_MIN) return -1;
  v3 ne = v_zero();
  for (int c = 0; c < 3; ++c) {
    double w[8];
    for (int n = 0; n < 8; ++n) w[n] = area[n] * nrm[n].value[c];
    ne.value[c] = r_central6(w) / ia;
  }
  const double p1 = v_dot(ne, e->tangent1), p2 = v_dot(ne, e->tangent2);
  const double pn = hypot(p1, p2);
  if (!isfinite(pn) || pn <= DBL_MIN) return -1;
  tn[0] = p1 / pn;
  tn[1] = p2 / pn;
  return 0;
}

/* nonorthogonal_operators.c:144-182 */
static int o_edge_emf(double vt1, double vt2, double bt1, double bt2, double jmp,
                      double rho, const gamera_no_edge_geometry *e, double diff,
                      int boris, double c, double cfl, double dt, double *emf) {
  if (!isfinite(vt1) || !isfinite(vt2) || !isfinite(bt1) || !isfinite(bt2) ||
      !isfinite(jmp) || !isfinite(rho) || rho <= DBL_MIN ||
      !isfinite(e->length) || e->length <= DBL_MIN || !isfinite(diff) ||
      !isfinite(cfl) || cfl < 0.0 || !isfinite(dt) || dt <= DBL_MIN ||
      (boris && (!isfinite(c) || c <= DBL_MIN)))
    return -1;
  const double flow = hypot(vt1, vt2);
  double va = hypot(bt1, bt2) / sqrt(rho);
  if (boris) va = c * va / hypot(c, va);
  double speed = flow + va;
  speed = fmin(speed, cfl * e->length / dt);
  const double ideal = -(vt1 * bt2 - vt2 * bt1);
  *emf = (ideal + diff * speed * jmp) * e->length;
  return 0;
}

#include "gcs_oracle_step.inc"
#include "gcs_oracle_mi.inc"

/* Stand-alone halo fills and seam syncs of the restatement (test
 * infrastructure: checkers of the library's stand-alone entry points). */
int gcso_fill_cell_halos(const gcso_halo_plan *p, gamera_no_storage st[6]) {
  if (!p || !st) return -1;
  h_fill_cells(p, st);
  return 0;
}
int gcso_fill_face_halos(const gcso_halo_plan *p, const gamera_no_grid grid[6],
                         gamera_no_storage st[6]) {
  if (!p || !grid || !st) return -1;
  h_fill_faces(p, grid, st);
  return 0;
}
int gcso_fill_radial_outflow(gamera_no_storage st[6], const size_t act[3], size_t g) {
  if (!st || !act) return -1;
  h_radial(st, act, g);
  return 0;
}
int gcso_sync_faces(gamera_no_storage st[6], const size_t act[3], size_t g,
                    int magnetic) {
  return i_sync(st, act, g, magnetic);
}
int gcso_sync_edges(const gcso_edge_plan *p, gamera_no_storage st[6]) {
  if (!p || !st) return -1;
  i_sync_edges(p, st);
  return 0;
}
