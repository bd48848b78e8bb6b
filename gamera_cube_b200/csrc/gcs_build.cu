// Device case builder: constructs a six-face case (mesh, trilinear cell
// geometry by 12-point Gauss-Legendre quadrature, calibrated face frames,
// edge frames, dipole background B0, initial state) directly in HBM, so a
// production-size run needs no host grid.  The arithmetic restates the
// reference set-up (nonorthogonal_geometry.c, nonorthogonal_grid.c,
// cubedsphere_mesh.c, nonorthogonal_background.c,
// nonorthogonal_initialization.c) in its operation order; device libm
// (tan, atan2, expm1, sqrt) may differ from the host's in the last bit.
#include "gcs_context.h"

#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "gcs_physics.cuh"

namespace gcs {

void convert_cells(const Ctx &X, int f, const gamera_no_cell_geometry *cells,
                   cudaStream_t s);

namespace {

struct V3 {
  double x, y, z;
};
__device__ inline V3 vadd(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ inline V3 vsub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ inline V3 vmul(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ inline V3 vscale(V3 a, double s) { return {s * a.x, s * a.y, s * a.z}; }
__device__ inline double vdot(V3 a, V3 b) {
  double r = 0.0;
  r += a.x * b.x;
  r += a.y * b.y;
  r += a.z * b.z;
  return r;
}
__device__ inline V3 vcross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ inline bool vfinite(V3 a) {
  return isfinite(a.x) && isfinite(a.y) && isfinite(a.z);
}
__device__ inline gamera_no_vec3 tovec(V3 a) {
  gamera_no_vec3 r;
  r.value[0] = a.x;
  r.value[1] = a.y;
  r.value[2] = a.z;
  return r;
}

// 12-point Gauss-Legendre rule in the reference's node order
// (nonorthogonal_geometry.c:9-24).
__constant__ double kGN[12] = {
    0.1252334085114689154724,  0.3678314989981801937527,
    0.5873179542866174472967,  0.7699026741943046870369,
    0.9041172563704748566785,  0.9815606342467192506906,
    -0.1252334085114689154724, -0.3678314989981801937527,
    -0.5873179542866174472967, -0.7699026741943046870369,
    -0.9041172563704748566785, -0.9815606342467192506906};
__constant__ double kGW[12] = {
    0.2491470458134027850006, 0.2334925365383548087610,
    0.2031674267230659217490, 0.1600783285433462263350,
    0.1069393259953184309603, 0.0471753363865118271946,
    0.2491470458134027850006, 0.2334925365383548087610,
    0.2031674267230659217490, 0.1600783285433462263350,
    0.1069393259953184309603, 0.0471753363865118271946};
__constant__ int kLS[8][3] = {{-1, -1, -1}, {+1, -1, -1}, {+1, +1, -1},
                              {-1, +1, -1}, {-1, -1, +1}, {+1, -1, +1},
                              {+1, +1, +1}, {-1, +1, +1}};
__constant__ int kFC[3][2][4] = {{{0, 3, 4, 7}, {1, 2, 5, 6}},
                                 {{0, 4, 1, 5}, {3, 7, 2, 6}},
                                 {{0, 1, 3, 2}, {4, 5, 7, 6}}};
__constant__ int kCO[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                              {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
__constant__ int kFrame[6][3][3] = {
    {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}},  {{-1, 0, 0}, {0, -1, 0}, {0, 0, 1}},
    {{0, 1, 0}, {-1, 0, 0}, {0, 0, 1}}, {{0, -1, 0}, {1, 0, 0}, {0, 0, 1}},
    {{0, 0, 1}, {1, 0, 0}, {0, 1, 0}},  {{0, 0, -1}, {1, 0, 0}, {0, -1, 0}}};

inline unsigned nblk(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

__device__ inline long long tid() {
  return blockIdx.x * (long long)blockDim.x + threadIdx.x;
}

// Vertex (cubedsphere_mesh.c:164-254 + nonorthogonal_radial_map.c:152-156).
__global__ void k_vertices(int face, int nr, int n, int g, double r_in,
                           double r_out, double stretch, V3 *out) {
  const int V0 = nr + 2 * g + 1, V1 = n + 2 * g + 1;
  const long long t = tid();
  if (t >= (long long)V0 * V1 * V1) return;
  const int i = (int)(t / ((long long)V1 * V1));
  const int j = (int)((t / V1) % V1);
  const int k = (int)(t % V1);
  const double qp = 0.25 * acos(-1.0);
  const double da = 2.0 * qp / (double)n;
  const double li = 0.0 + (double)i - (double)g;
  double r = r_in + li * ((r_out - r_in) / (double)nr);
  if (stretch > 0.0)
    r = r_in + (r_out - r_in) * expm1(stretch * (li / (double)nr)) / expm1(stretch);
  const double a = -qp + (0.0 + (double)j - (double)g) * da;
  const double b = -qp + (0.0 + (double)k - (double)g) * da;
  const double u = tan(a), v = tan(b);
  const double il = 1.0 / sqrt(1.0 + u * u + v * v);
  V3 d;
  d.x = il * ((double)kFrame[face][0][0] + u * (double)kFrame[face][1][0] +
              v * (double)kFrame[face][2][0]);
  d.y = il * ((double)kFrame[face][0][1] + u * (double)kFrame[face][1][1] +
              v * (double)kFrame[face][2][1]);
  d.z = il * ((double)kFrame[face][0][2] + u * (double)kFrame[face][1][2] +
              v * (double)kFrame[face][2][2]);
  out[t] = {r * d.x, r * d.y, r * d.z};
}

__device__ inline bool normalize(V3 v, V3 *u) {
  const double nrm = sqrt(vdot(v, v));
  if (!isfinite(nrm) || nrm <= DBL_MIN) return false;
  *u = vmul(v, 1.0 / nrm);
  return true;
}

// nonorthogonal_geometry.c:103-158 followed by the cube calibration of
// cubedsphere_mesh.c:256-282.
__device__ bool face_geometry(const V3 f[4], gamera_no_face_geometry *g) {
  const V3 de = vsub(f[1], f[0]);
  const V3 dp = vsub(f[2], f[0]);
  const V3 dc = vadd(vsub(f[3], f[2]), vsub(f[0], f[1]));
  double area = 0.0;
  V3 av = {0.0, 0.0, 0.0}, cen = {0.0, 0.0, 0.0};
  for (int i = 0; i < 12; ++i) {
    const double eta = 0.5 * (1.0 + kGN[i]);
    for (int j = 0; j < 12; ++j) {
      const double psi = 0.5 * (1.0 + kGN[j]);
      const double w = 0.25 * kGW[i] * kGW[j];
      const V3 te = vadd(de, vmul(dc, psi));
      const V3 tp = vadd(dp, vmul(dc, eta));
      const V3 oa = vcross(te, tp);
      const double aw = w * sqrt(vdot(oa, oa));
      const V3 pt = vadd(f[0], vadd(vmul(de, eta), vadd(vmul(dp, psi),
                                                         vmul(dc, eta * psi))));
      area += aw;
      av = vadd(av, vmul(oa, w));
      cen = vadd(cen, vmul(pt, aw));
    }
  }
  if (!isfinite(area) || area <= DBL_MIN) return false;
  cen = vmul(cen, 1.0 / area);
  const V3 ce = vmul(vadd(vsub(f[3], f[2]), vsub(f[1], f[0])), 0.5);
  const V3 cp = vmul(vadd(vsub(f[3], f[1]), vsub(f[2], f[0])), 0.5);
  V3 nrm, t1, t2;
  if (!normalize(vcross(ce, cp), &nrm) || !normalize(cp, &t2) ||
      !normalize(vcross(t2, nrm), &t1))
    return false;
  // calibration: normal = area vector / |area vector|, t2 re-orthogonalised
  const double mag = sqrt(av.x * av.x + av.y * av.y + av.z * av.z);
  if (!isfinite(mag) || mag <= 0.0) return false;
  const V3 cn = {av.x / mag, av.y / mag, av.z / mag};
  double p = 0.0;
  p += t2.x * cn.x;
  p += t2.y * cn.y;
  p += t2.z * cn.z;
  V3 ct2 = {t2.x - p * cn.x, t2.y - p * cn.y, t2.z - p * cn.z};
  double s2 = 0.0;
  s2 += ct2.x * ct2.x;
  s2 += ct2.y * ct2.y;
  s2 += ct2.z * ct2.z;
  if (!isfinite(s2) || s2 <= 0.0) return false;
  ct2.x /= sqrt(s2);
  ct2.y /= sqrt(s2);
  ct2.z /= sqrt(s2);
  const V3 ct1 = {ct2.y * cn.z - ct2.z * cn.y, ct2.z * cn.x - ct2.x * cn.z,
                  ct2.x * cn.y - ct2.y * cn.x};
  g->area = mag;
  g->area_vector = tovec(av);
  g->centroid = tovec(cen);
  g->normal = tovec(cn);
  g->tangent1 = tovec(ct1);
  g->tangent2 = tovec(ct2);
  return true;
}

// One cell (nonorthogonal_geometry.c:160-243), faces calibrated.
__global__ void k_cells(Dims D, const V3 *vert, gamera_no_cell_geometry *out,
                        int *bad) {
  const long long t = tid();
  const long long nc = (long long)D.E0 * D.E1 * D.E2;
  if (t >= nc) return;
  const int i = (int)(t / ((long long)D.E1 * D.E2));
  const int j = (int)((t / D.E2) % D.E1);
  const int k = (int)(t % D.E2);
  const int V1 = D.E1 + 1, V2 = D.E2 + 1;
  V3 c[8];
  for (int q = 0; q < 8; ++q)
    c[q] = vert[((long long)(i + kCO[q][0]) * V1 + (j + kCO[q][1])) * V2 +
                (k + kCO[q][2])];
  double vol = 0.0;
  V3 cen = {0.0, 0.0, 0.0};
  for (int a = 0; a < 12; ++a) {
    const double xi = kGN[a];
    for (int b = 0; b < 12; ++b) {
      const double eta = kGN[b];
      for (int e = 0; e < 12; ++e) {
        const double zeta = kGN[e];
        V3 pt = {0.0, 0.0, 0.0};
        V3 der[3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
        for (int q = 0; q < 8; ++q) {
          const double sx = (double)kLS[q][0], sy = (double)kLS[q][1],
                       sz = (double)kLS[q][2];
          const double fx = 1.0 + sx * xi, fy = 1.0 + sy * eta,
                       fz = 1.0 + sz * zeta;
          const double shape = 0.125 * fx * fy * fz;
          pt = vadd(pt, vmul(c[q], shape));
          der[0] = vadd(der[0], vmul(c[q], 0.125 * sx * fy * fz));
          der[1] = vadd(der[1], vmul(c[q], 0.125 * fx * sy * fz));
          der[2] = vadd(der[2], vmul(c[q], 0.125 * fx * fy * sz));
        }
        const double det = vdot(der[0], vcross(der[1], der[2]));
        const double wv = fabs(det) * kGW[a] * kGW[b] * kGW[e];
        vol += wv;
        cen = vadd(cen, vmul(pt, wv));
      }
    }
  }
  gamera_no_cell_geometry &g = out[t];
  if (!isfinite(vol) || vol <= DBL_MIN) {
    atomicExch(bad, 1);
    return;
  }
  g.volume = vol;
  g.centroid = tovec(vmul(cen, 1.0 / vol));
  for (int d = 0; d < 3; ++d) {
    for (int s = 0; s < 2; ++s) {
      V3 f[4];
      for (int q = 0; q < 4; ++q) f[q] = c[kFC[d][s][q]];
      if (!face_geometry(f, &g.face[d][s])) atomicExch(bad, 1);
    }
    // cfl length uses the areas before calibration in the reference; the
    // calibrated area replaces the scalar area only after it (see
    // cubedsphere_mesh.c:286-303), so recompute the scalar area here.
  }
}

// Scalar face areas before calibration, for cfl_length
// (nonorthogonal_geometry.c:235-238 runs before the calibration).
__device__ double scalar_area(const V3 f[4]) {
  const V3 de = vsub(f[1], f[0]);
  const V3 dp = vsub(f[2], f[0]);
  const V3 dc = vadd(vsub(f[3], f[2]), vsub(f[0], f[1]));
  double area = 0.0;
  for (int i = 0; i < 12; ++i) {
    const double eta = 0.5 * (1.0 + kGN[i]);
    for (int j = 0; j < 12; ++j) {
      const double psi = 0.5 * (1.0 + kGN[j]);
      const double w = 0.25 * kGW[i] * kGW[j];
      const V3 oa = vcross(vadd(de, vmul(dc, psi)), vadd(dp, vmul(dc, eta)));
      area += w * sqrt(vdot(oa, oa));
    }
  }
  return area;
}

__global__ void k_cfl_length(Dims D, const V3 *vert, gamera_no_cell_geometry *out) {
  const long long t = tid();
  const long long nc = (long long)D.E0 * D.E1 * D.E2;
  if (t >= nc) return;
  const int i = (int)(t / ((long long)D.E1 * D.E2));
  const int j = (int)((t / D.E2) % D.E1);
  const int k = (int)(t % D.E2);
  const int V1 = D.E1 + 1, V2 = D.E2 + 1;
  V3 c[8];
  for (int q = 0; q < 8; ++q)
    c[q] = vert[((long long)(i + kCO[q][0]) * V1 + (j + kCO[q][1])) * V2 +
                (k + kCO[q][2])];
  gamera_no_cell_geometry &g = out[t];
  for (int d = 0; d < 3; ++d) {
    double a[2];
    for (int s = 0; s < 2; ++s) {
      V3 f[4];
      for (int q = 0; q < 4; ++q) f[q] = c[kFC[d][s][q]];
      a[s] = scalar_area(f);
    }
    g.cfl_length[d] = g.volume / fmax(a[0], a[1]);
  }
}

// Face arrays of family d from the calibrated cell faces
// (nonorthogonal_grid.c:97-127); also the face centroids and area vectors
// the halo plan needs.
__global__ void k_faces_from_cells(Dims D, int f, int d,
                                   const gamera_no_cell_geometry *cells,
                                   DevGeom G, gamera_no_vec3 *cen,
                                   gamera_no_vec3 *av) {
  const int e0 = D.E0 + (d == 0), e1 = D.E1 + (d == 1), e2 = D.E2 + (d == 2);
  const long long t = tid();
  if (t >= (long long)e0 * e1 * e2) return;
  int x[3];
  x[0] = (int)(t / ((long long)e1 * e2));
  x[1] = (int)((t / e2) % e1);
  x[2] = (int)(t % e2);
  int ci[3] = {x[0], x[1], x[2]};
  int side = 0;
  if (ci[d] == D.ext(d)) {
    --ci[d];
    side = 1;
  }
  const gamera_no_face_geometry &g =
      cells[((long long)ci[0] * D.E1 + ci[1]) * D.E2 + ci[2]].face[d][side];
  const long long c = f * D.Nn + D.node(x[0], x[1], x[2]);
  G.area[d][c] = g.area;
  for (int q = 0; q < 3; ++q) {
    G.fn[d][q][c] = g.normal.value[q];
    G.ft1[d][q][c] = g.tangent1.value[q];
    G.ft2[d][q][c] = g.tangent2.value[q];
  }
  cen[t] = g.centroid;
  av[t] = g.area_vector;
}

__global__ void k_cell_centroids(Dims D, const gamera_no_cell_geometry *cells,
                                 gamera_no_vec3 *cen) {
  const long long t = tid();
  if (t >= (long long)D.E0 * D.E1 * D.E2) return;
  cen[t] = cells[t].centroid;
}

// Edge frames of family e (nonorthogonal_grid.c:129-210,
// nonorthogonal_geometry.c:245-262).
// Frame of edge (i, j, k) of family e from the vertices: 0 on success, 1
// for an edge on the boundary of the extent (no frame), 2 for a degenerate
// edge.
__device__ int edge_frame(const Dims &D, int e, const V3 *vert, int i, int j, int k,
                          V3 *nrm, V3 *t1, V3 *t2, double *len) {
  int interior;
  if (e == 0) interior = j > 0 && j < D.E1 && k > 0 && k < D.E2;
  else if (e == 1) interior = i > 0 && i < D.E0 && k > 0 && k < D.E2;
  else interior = i > 0 && i < D.E0 && j > 0 && j < D.E1;
  if (!interior) return 1;
  const int V1 = D.E1 + 1, V2 = D.E2 + 1;
  auto vx = [&](int a, int b, int q) {
    return vert[((long long)a * V1 + b) * V2 + q];
  };
  int en[3] = {i, j, k};
  ++en[e];
  V3 first, second;
  if (e == 0) {
    first = vsub(vx(i, j, k + 1), vx(i, j, k - 1));
    second = vsub(vx(i + 1, j, k + 1), vx(i + 1, j, k - 1));
  } else if (e == 1) {
    first = vsub(vx(i + 1, j, k), vx(i - 1, j, k));
    second = vsub(vx(i + 1, j + 1, k), vx(i - 1, j + 1, k));
  } else {
    first = vsub(vx(i, j + 1, k), vx(i, j - 1, k));
    second = vsub(vx(i, j + 1, k + 1), vx(i, j - 1, k + 1));
  }
  const V3 avg = vscale(vadd(first, second), 0.5);
  const V3 ed = vsub(vx(en[0], en[1], en[2]), vx(i, j, k));
  *len = sqrt(vdot(ed, ed));
  if (!isfinite(*len) || *len <= DBL_MIN || !normalize(ed, nrm) ||
      !normalize(vcross(avg, *nrm), t1) || !normalize(vcross(*nrm, *t1), t2))
    return 2;
  return 0;
}

// Edge frames of family e (nonorthogonal_grid.c:129-210,
// nonorthogonal_geometry.c:245-262).
__global__ void k_edges(Dims D, int f, int e, const V3 *vert, DevGeom G,
                        int *bad) {
  const int e0 = D.E0 + (e != 0), e1 = D.E1 + (e != 1), e2 = D.E2 + (e != 2);
  const long long t = tid();
  if (t >= (long long)e0 * e1 * e2) return;
  const int i = (int)(t / ((long long)e1 * e2));
  const int j = (int)((t / e2) % e1);
  const int k = (int)(t % e2);
  const long long c = f * D.Nn + D.node(i, j, k);
  G.edge_ok[e][c] = (unsigned char)kStageEdgeGeometry;
  V3 nrm, t1, t2;
  double len;
  const int r = edge_frame(D, e, vert, i, j, k, &nrm, &t1, &t2, &len);
  if (r == 1) return;
  if (r == 2) {
    atomicExch(bad, 1);
    return;
  }
  G.elen[e][c] = len;
  G.et1[e][0][c] = t1.x;
  G.et1[e][1][c] = t1.y;
  G.et1[e][2][c] = t1.z;
  G.et2[e][0][c] = t2.x;
  G.et2[e][1][c] = t2.y;
  G.et2[e][2][c] = t2.z;
  G.edge_ok[e][c] = 0;
}

// Geometry of the radial boundary layers for the device Earth boundary,
// on the node plane of each face (layouts of gcs_earth.h).
__global__ void k_earth_layer_cells(Dims D, int f, const gamera_no_cell_geometry *cells,
                                    EarthLayers L) {
  const int jk = blockIdx.x * blockDim.x + threadIdx.x;
  if (jk >= D.E1 * D.E2) return;
  const int l = blockIdx.y, j = jk / D.E2, k = jk % D.E2;
  const int i = l < D.g ? l : D.g + D.nr + (l - D.g);
  const gamera_no_vec3 x = cells[((long long)i * D.E1 + j) * D.E2 + k].centroid;
  const long long q = (((long long)f * 2 * D.g + l) * D.N1 + j) * D.N2 + k;
  for (int c = 0; c < 3; ++c) L.cell_cen[c][q] = x.value[c];
}

__global__ void k_earth_layer_faces(Dims D, int f, int d, const gamera_no_vec3 *cen,
                                    const gamera_no_vec3 *av, DevGeom G, DevBg B,
                                    EarthLayers L) {
  const int e1 = D.E1 + (d == 1), e2 = D.E2 + (d == 2);
  const int jk = blockIdx.x * blockDim.x + threadIdx.x;
  if (jk >= e1 * e2) return;
  const int l = blockIdx.y, j = jk / e2, k = jk % e2;
  const int i = D.g + D.nr + (d == 0) + l;
  const long long s = ((long long)i * e1 + j) * e2 + k;
  const long long q = (((long long)f * D.g + l) * D.N1 + j) * D.N2 + k;
  const long long c = f * D.Nn + D.node(i, j, k);
  for (int a = 0; a < 3; ++a) {
    L.face_cen[d][a][q] = cen[s].value[a];
    L.face_av[d][a][q] = av[s].value[a];
  }
  L.face_bg[d][q] = B.fb0n[d][c] * G.area[d][c];
}

__global__ void k_earth_layer_edges(Dims D, int f, int e, const V3 *vert, EarthLayers L) {
  const int e1 = D.E1 + (e != 1), e2 = D.E2 + (e != 2);
  const int jk = blockIdx.x * blockDim.x + threadIdx.x;
  if (jk >= e1 * e2) return;
  const int l = blockIdx.y, j = jk / e2, k = jk % e2;
  const int i = l == 0 ? D.g : D.g + D.nr - 3 + (l - 1);
  const long long q = (((long long)f * 5 + l) * D.N1 + j) * D.N2 + k;
  L.edge_valid[e][q] = 0;
  if (i >= D.E0 + (e != 0)) return;
  const int V1 = D.E1 + 1, V2 = D.E2 + 1;
  int up[3] = {i, j, k};
  ++up[e];
  const V3 a = vert[((long long)i * V1 + j) * V2 + k];
  const V3 z = vert[((long long)up[0] * V1 + up[1]) * V2 + up[2]];
  L.edge_mid[e][0][q] = 0.5 * (a.x + z.x);
  L.edge_mid[e][1][q] = 0.5 * (a.y + z.y);
  L.edge_mid[e][2][q] = 0.5 * (a.z + z.z);
  V3 nrm, t1, t2;
  double len;
  if (l == 0 && e > 0) {
    const long long p = ((long long)f * D.N1 + j) * D.N2 + k;
    L.inner_a[e - 1][0][p] = a.x;
    L.inner_a[e - 1][1][p] = a.y;
    L.inner_a[e - 1][2][p] = a.z;
    L.inner_b[e - 1][0][p] = z.x;
    L.inner_b[e - 1][1][p] = z.y;
    L.inner_b[e - 1][2][p] = z.z;
  }
  if (edge_frame(D, e, vert, i, j, k, &nrm, &t1, &t2, &len) != 0) return;
  L.edge_nrm[e][0][q] = nrm.x;
  L.edge_nrm[e][1][q] = nrm.y;
  L.edge_nrm[e][2][q] = nrm.z;
  L.edge_len[e][q] = len;
  L.edge_valid[e][q] = 1;
}

// Dipole B = 3 (m.r) r / r^5 - m / r^3 (nonorthogonal_background.c:422-442).
__device__ inline V3 dipole(V3 p, V3 m) {
  const double r2 = vdot(p, p);
  const double r = sqrt(r2);
  const double ir3 = 1.0 / (r2 * r);
  const double ir5 = ir3 / r2;
  const double proj = vdot(m, p);
  return vsub(vscale(p, 3.0 * proj * ir5), vscale(m, ir3));
}

// Face B0 average, flux and B0 stress (nonorthogonal_background.c:111-164).
__global__ void k_bg_faces(Dims D, int f, int d, const V3 *vert, V3 m, DevGeom G,
                           DevBg B, V3 *stress, int *bad) {
  const int e0 = D.E0 + (d == 0), e1 = D.E1 + (d == 1), e2 = D.E2 + (d == 2);
  const long long t = tid();
  if (t >= (long long)e0 * e1 * e2) return;
  int x[3];
  x[0] = (int)(t / ((long long)e1 * e2));
  x[1] = (int)((t / e2) % e1);
  x[2] = (int)(t % e2);
  int cc[3] = {x[0], x[1], x[2]};
  int side = 0;
  if (cc[d] == D.ext(d)) {
    --cc[d];
    side = 1;
  }
  const int V1 = D.E1 + 1, V2 = D.E2 + 1;
  V3 c[8], fq[4];
  for (int q = 0; q < 8; ++q)
    c[q] = vert[((long long)(cc[0] + kCO[q][0]) * V1 + (cc[1] + kCO[q][1])) * V2 +
                (cc[2] + kCO[q][2])];
  for (int q = 0; q < 4; ++q) fq[q] = c[kFC[d][side][q]];
  const long long node = f * D.Nn + D.node(x[0], x[1], x[2]);
  const double area_s = G.area[d][node];
  const V3 de = vsub(fq[1], fq[0]);
  const V3 dp = vsub(fq[2], fq[0]);
  const V3 dc = vadd(vsub(fq[3], fq[2]), vsub(fq[0], fq[1]));
  V3 in = {0.0, 0.0, 0.0}, st = {0.0, 0.0, 0.0};
  double fl = 0.0;
  for (int i = 0; i < 12; ++i) {
    const double eta = 0.5 * (1.0 + kGN[i]);
    for (int j = 0; j < 12; ++j) {
      const double psi = 0.5 * (1.0 + kGN[j]);
      const double w = 0.25 * kGW[i] * kGW[j];
      const V3 oa = vcross(vadd(de, vscale(dc, psi)), vadd(dp, vscale(dc, eta)));
      const double area = sqrt(vdot(oa, oa));
      const V3 pt = vadd(fq[0], vadd(vscale(de, eta), vadd(vscale(dp, psi),
                                                            vscale(dc, eta * psi))));
      const V3 fld = dipole(pt, m);
      in = vadd(in, vscale(fld, w * area));
      const double nf = vdot(fld, oa);
      fl += w * nf;
      const double pm = 0.5 * vdot(fld, fld);
      st = vadd(st, vscale(vsub(vscale(oa, pm), vscale(fld, nf)), w));
    }
  }
  const V3 avg = vscale(in, 1.0 / area_s);
  if (!vfinite(avg) || !isfinite(fl) || !vfinite(st)) atomicExch(bad, 1);
  B.fb0[d][0][node] = avg.x;
  B.fb0[d][1][node] = avg.y;
  B.fb0[d][2][node] = avg.z;
  B.fb0n[d][node] = fl / area_s;
  stress[(long long)d * D.Nn + D.node(x[0], x[1], x[2])] = st;
}

// Cell B0 average and pure-B0 force (nonorthogonal_background.c:166-215,
// 365-396).
__global__ void k_bg_cells(Dims D, int f, const V3 *vert, V3 m, DevGeom G,
                           DevBg B, const V3 *stress, int *bad) {
  const long long t = tid();
  if (t >= (long long)D.E0 * D.E1 * D.E2) return;
  const int i = (int)(t / ((long long)D.E1 * D.E2));
  const int j = (int)((t / D.E2) % D.E1);
  const int k = (int)(t % D.E2);
  const int V1 = D.E1 + 1, V2 = D.E2 + 1;
  V3 c[8];
  for (int q = 0; q < 8; ++q)
    c[q] = vert[((long long)(i + kCO[q][0]) * V1 + (j + kCO[q][1])) * V2 +
                (k + kCO[q][2])];
  const long long node = f * D.Nn + D.node(i, j, k);
  const double vol = G.vol[node];
  V3 in = {0.0, 0.0, 0.0};
  double iv = 0.0;
  for (int a = 0; a < 12; ++a)
    for (int b = 0; b < 12; ++b)
      for (int e = 0; e < 12; ++e) {
        const double xi = kGN[a], eta = kGN[b], zeta = kGN[e];
        V3 pt = {0.0, 0.0, 0.0};
        V3 der[3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
        for (int q = 0; q < 8; ++q) {
          const double sx = (double)kLS[q][0], sy = (double)kLS[q][1],
                       sz = (double)kLS[q][2];
          const double fx = 1.0 + sx * xi, fy = 1.0 + sy * eta,
                       fz = 1.0 + sz * zeta;
          pt = vadd(pt, vscale(c[q], 0.125 * fx * fy * fz));
          der[0] = vadd(der[0], vscale(c[q], 0.125 * sx * fy * fz));
          der[1] = vadd(der[1], vscale(c[q], 0.125 * fx * sy * fz));
          der[2] = vadd(der[2], vscale(c[q], 0.125 * fx * fy * sz));
        }
        const double w = fabs(vdot(der[0], vcross(der[1], der[2]))) * kGW[a] *
                         kGW[b] * kGW[e];
        iv += w;
        in = vadd(in, vscale(dipole(pt, m), w));
      }
  if (!(iv > DBL_MIN) || fabs(iv - vol) > 2.0e-11 * vol) atomicExch(bad, 1);
  const V3 avg = vscale(in, 1.0 / vol);
  B.b0[0][node] = avg.x;
  B.b0[1][node] = avg.y;
  B.b0[2][node] = avg.z;
  V3 um = {0.0, 0.0, 0.0};
  for (int d = 0; d < 3; ++d) {
    const long long lo = (long long)d * D.Nn + D.node(i, j, k);
    const long long hi = lo + D.stride(d);
    um = vadd(um, vsub(stress[hi], stress[lo]));
  }
  const V3 force = vscale(um, -1.0 / vol);
  if (!vfinite(force)) atomicExch(bad, 1);
  B.force[0][node] = force.x;
  B.force[1][node] = force.y;
  B.force[2][node] = force.z;
}

// Edge-averaged B0 projected on the edge tangents
// (nonorthogonal_background.c:217-236, nonorthogonal_sweep.c:719-726).
__global__ void k_bg_edges(Dims D, int f, int e, const V3 *vert, V3 m,
                           DevGeom G, DevBg B) {
  const int e0 = D.E0 + (e != 0), e1 = D.E1 + (e != 1), e2 = D.E2 + (e != 2);
  const long long t = tid();
  if (t >= (long long)e0 * e1 * e2) return;
  const int i = (int)(t / ((long long)e1 * e2));
  const int j = (int)((t / e2) % e1);
  const int k = (int)(t % e2);
  const int V1 = D.E1 + 1, V2 = D.E2 + 1;
  int en[3] = {i, j, k};
  ++en[e];
  const V3 s = vert[((long long)i * V1 + j) * V2 + k];
  const V3 disp = vsub(vert[((long long)en[0] * V1 + en[1]) * V2 + en[2]], s);
  V3 r = {0.0, 0.0, 0.0};
  for (int q = 0; q < 12; ++q) {
    const double par = 0.5 * (1.0 + kGN[q]);
    r = vadd(r, vscale(dipole(vadd(s, vscale(disp, par)), m), 0.5 * kGW[q]));
  }
  const long long c = f * D.Nn + D.node(i, j, k);
  B.eb0t1[e][c] = dot3(r.x, r.y, r.z, G.et1[e][0][c], G.et1[e][1][c],
                       G.et1[e][2][c]);
  B.eb0t2[e][c] = dot3(r.x, r.y, r.z, G.et2[e][0][c], G.et2[e][1][c],
                       G.et2[e][2][c]);
}

__device__ inline uint64_t splitmix(uint64_t x) {
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}

// Initial conserved state per cell (the case set of oracle/cases_common.h:
// uniform MHD state, radial shock, solar wind with seeded noise, wind with
// a density pulse).
__global__ void k_init_cells(Dims D, int f, int kind, unsigned long long seed,
                             WindInit w, const gamera_no_cell_geometry *cells,
                             DevState S, int *bad) {
  const long long t = tid();
  if (t >= (long long)D.E0 * D.E1 * D.E2) return;
  const int i = (int)(t / ((long long)D.E1 * D.E2));
  const int j = (int)((t / D.E2) % D.E1);
  const int k = (int)(t % D.E2);
  const gamera_no_vec3 x = cells[t].centroid;
  Prim p;
  double rf = 1e-12, pf = 1e-12;
  if (kind == 0) {
    p = {1.2, 0.23, -0.17, 0.09, 0.74};
  } else if (kind == 1) {
    const double r = sqrt(x.value[0] * x.value[0] + x.value[1] * x.value[1] +
                          x.value[2] * x.value[2]);
    p = r < 2.5 ? Prim{1.0, 0.0, 0.0, 0.0, 1.0} : Prim{0.125, 0.0, 0.0, 0.0, 0.1};
  } else {
    const uint64_t h = splitmix(splitmix((uint64_t)seed) ^ ((uint64_t)f << 56) ^
                                (uint64_t)t);
    const double noise = 2.0 * ((double)(h >> 11) * 0x1.0p-53) - 1.0;
    double rho = w.rho * (1.0 + 0.01 * noise);
    if (w.pulse) rho *= 1.0 + 0.2 * sin(2.0 * acos(-1.0) * x.value[0] / 10.0);
    p = {rho, w.vx, 0.0, 0.0, w.pres};
    rf = 1e-6;
    pf = 1e-8;
  }
  double u[5];
  if (prim_to_cons(p, 5.0 / 3.0, rf, pf, u)) atomicExch(bad, 1);
  const long long c = f * D.Nn + D.node(i, j, k);
  for (int q = 0; q < 5; ++q) {
    S.U[q][c] = u[q];
    S.Uo[q][c] = u[q];
  }
}

// Edge line integrals of A = (B x r) / 2 for a uniform B
// (nonorthogonal_initialization.c:194-249).
__global__ void k_init_lines(Dims D, int e, const V3 *vert, V3 b,
                             double *line) {
  const int e0 = D.E0 + (e != 0), e1 = D.E1 + (e != 1), e2 = D.E2 + (e != 2);
  const long long t = tid();
  if (t >= (long long)e0 * e1 * e2) return;
  const int i = (int)(t / ((long long)e1 * e2));
  const int j = (int)((t / e2) % e1);
  const int k = (int)(t % e2);
  const int V1 = D.E1 + 1, V2 = D.E2 + 1;
  int en[3] = {i, j, k};
  ++en[e];
  const V3 s = vert[((long long)i * V1 + j) * V2 + k];
  const V3 ev = vert[((long long)en[0] * V1 + en[1]) * V2 + en[2]];
  const V3 disp = vsub(ev, s);
  const V3 mid = vscale(vadd(s, ev), 0.5);
  double acc = 0.0;
  for (int n = 0; n < 12; ++n) {
    const V3 p = vadd(mid, vscale(disp, 0.5 * kGN[n]));
    const V3 pot = {0.5 * (b.y * p.z - b.z * p.y), 0.5 * (b.z * p.x - b.x * p.z),
                    0.5 * (b.x * p.y - b.y * p.x)};
    acc += 0.5 * kGW[n] * vdot(pot, disp);
  }
  line[(long long)e * D.Nn + D.node(i, j, k)] = acc;
}

// Face flux = circulation of the edge integrals
// (nonorthogonal_initialization.c:254-313), or the uniform-B flux
// B . area_vector for the uniform and shock cases.
__global__ void k_init_flux(Dims D, int f, int d, const double *line, int uniform,
                            V3 b, const gamera_no_vec3 *av, DevState S) {
  const int e0 = D.E0 + (d == 0), e1 = D.E1 + (d == 1), e2 = D.E2 + (d == 2);
  const long long t = tid();
  if (t >= (long long)e0 * e1 * e2) return;
  const int i = (int)(t / ((long long)e1 * e2));
  const int j = (int)((t / e2) % e1);
  const int k = (int)(t % e2);
  const long long n = D.node(i, j, k);
  double phi;
  if (uniform) {
    phi = 0.0;
    phi += b.x * av[t].value[0];
    phi += b.y * av[t].value[1];
    phi += b.z * av[t].value[2];
  } else {
    const double *L0 = line, *L1 = line + D.Nn, *L2 = line + 2 * D.Nn;
    const long long s0 = D.stride(0), s1 = D.stride(1);
    if (d == 0)
      phi = L1[n] - L1[n + 1] + L2[n + s1] - L2[n];
    else if (d == 1)
      phi = -L0[n] + L0[n + 1] - L2[n + s0] + L2[n];
    else
      phi = L0[n] - L0[n + s1] + L1[n + s0] - L1[n];
  }
  const long long c = f * D.Nn + n;
  S.P[d][c] = phi;
  S.Po[d][c] = phi;
}

__global__ void k_init_b(Dims D, DevState S, DevGeom G, int *bad) {
  const long long t = tid();
  if (t >= kFaces * (long long)D.E0 * D.E1 * D.E2) return;
  const long long per = (long long)D.E0 * D.E1 * D.E2;
  const int f = (int)(t / per);
  const long long r = t % per;
  const int i = (int)(r / ((long long)D.E1 * D.E2));
  const int j = (int)((r / D.E2) % D.E1);
  const int k = (int)(r % D.E2);
  const long long c = f * D.Nn + D.node(i, j, k);
  double phi[6];
  for (int d = 0; d < 3; ++d) {
    phi[2 * d] = S.P[d][c];
    phi[2 * d + 1] = S.P[d][c + D.stride(d)];
  }
  if (!G.cell_ok[c]) {
    atomicExch(bad, 1);
    return;
  }
  for (int q = 0; q < 3; ++q) {
    double s = 0.0;
    for (int col = 0; col < 6; ++col) s += G.rec[q * 6 + col][c] * phi[col];
    S.B[q][c] = s;
    S.Bo[q][c] = s;
  }
}

}  // namespace

#define GCS_BTRY(expr)                                 \
  do {                                                 \
    cudaError_t err_ = (expr);                         \
    if (err_ != cudaSuccess) {                         \
      set_error(cudaGetErrorString(err_), #expr);      \
      return -1;                                       \
    }                                                  \
  } while (0)

WindInit case_wind(int kind) {
  const double bnorm = 100000.0 * sqrt(4.0e-7 * acos(-1.0) * 1.67262192369e-21);
  WindInit w;
  w.rho = 5.0;
  w.vx = kind == 3 ? -4.5 : -4.0;
  w.pres = 5.0e6 * 1.380649e-23 * 1.0e5 / (1.67262192369e-21 * 1.0e10);
  w.bz = -5.0e-9 / bnorm;
  w.pulse = kind == 3;
  return w;
}

WindInit driven_wind(double density_cm3, double velocity_x_kms, double temperature_k,
                     double bz_nt) {
  const double bnorm = 100000.0 * sqrt(4.0e-7 * acos(-1.0) * 1.67262192369e-21);
  WindInit w;
  w.rho = density_cm3;
  w.vx = velocity_x_kms / 100.0;
  w.pres = density_cm3 * 1.0e6 * 1.380649e-23 * temperature_k /
           (1.67262192369e-21 * 1.0e10);
  w.bz = bz_nt * 1.0e-9 / bnorm;
  w.pulse = 0;
  return w;
}

int Context::init_case(int kind, size_t nr, size_t n, unsigned long long seed,
                       const WindInit *driver) {
  if (kind < 0 || kind > 3 || (driver && kind != 2)) {
    set_error("unknown case kind", "init_case");
    return -1;
  }
  const WindInit wi = driver ? *driver : case_wind(kind);
  kind_shock = kind == 1;
  const int wind = kind >= 2;
  const size_t active[3] = {nr, n, n};
  if (allocate(active, 4) != 0) return -1;
  const Dims &D = X.D;
  const long long cells = (long long)D.E0 * D.E1 * D.E2;
  const long long verts = (long long)(D.E0 + 1) * (D.E1 + 1) * (D.E2 + 1);
  // work buffers: vertices, B0 face stress (3 families), edge integrals
  void *work = nullptr;
  const size_t wbytes = verts * sizeof(V3) + 3 * D.Nn * sizeof(V3) +
                        3 * D.Nn * sizeof(double) + sizeof(int);
  GCS_BTRY(cudaMalloc(&work, wbytes));
  V3 *vert = (V3 *)work;
  V3 *stress = vert + verts;
  double *line = (double *)(stress + 3 * D.Nn);
  int *bad = (int *)(line + 3 * D.Nn);
  GCS_BTRY(cudaMemsetAsync(bad, 0, sizeof(int), stream));
  gamera_no_cell_geometry *acells = (gamera_no_cell_geometry *)staging;
  std::vector<gamera_no_vec3> cc[kFaces], fcen[kFaces][3], farea[kFaces][3];
  gamera_no_vec3 *d_cen = nullptr, *d_av = nullptr;
  const size_t fmax = (size_t)(D.E0 + 1) * (D.E1 + 1) * (D.E2 + 1);
  GCS_BTRY(cudaMalloc(&d_cen, fmax * sizeof(gamera_no_vec3)));
  GCS_BTRY(cudaMalloc(&d_av, 3 * fmax * sizeof(gamera_no_vec3)));
  const V3 m = {0.0, 0.0, -6761.730688424097};
  const V3 bimf = {0.0, 0.0, wi.bz};
  const V3 bu = kind == 0 ? V3{0.38, -0.21, 0.16} : V3{0.1, 0.08, -0.03};
  const int bs = 128;
  for (int f = 0; f < kFaces; ++f) {
    const double r_in = kind == 0 ? 2.0 : (kind == 1 ? 2.0 : 2.5);
    const double r_out = kind == 0 ? 2.5 : (kind == 1 ? 3.0 : 30.0);
    k_vertices<<<nblk(verts, bs), bs, 0, stream>>>(f, D.nr, D.n, D.g, r_in, r_out,
                                                   wind ? log(12.0) : 0.0, vert);
    k_cells<<<nblk(cells, 64), 64, 0, stream>>>(D, vert, acells, bad);
    k_cfl_length<<<nblk(cells, bs), bs, 0, stream>>>(D, vert, acells);
    convert_cells(X, f, acells, stream);
    k_cell_centroids<<<nblk(cells, bs), bs, 0, stream>>>(D, acells, d_cen);
    cc[f].resize(cells);
    GCS_BTRY(cudaMemcpyAsync(cc[f].data(), d_cen, cells * sizeof(gamera_no_vec3),
                             cudaMemcpyDeviceToHost, stream));
    {
      // innermost layers (layer-major, so a prefix of each array)
      const int wl = D.g + 4 < D.E0 ? D.g + 4 : D.E0;
      const size_t wc = (size_t)wl * D.E1 * D.E2;
      const size_t wv = (size_t)(wl + 1) * (D.E1 + 1) * (D.E2 + 1);
      win_layers = wl;
      win_vertex[f].resize(wv);
      GCS_BTRY(cudaMemcpyAsync(win_vertex[f].data(), vert, wv * sizeof(gamera_no_vec3),
                               cudaMemcpyDeviceToHost, stream));
      GCS_BTRY(cudaStreamSynchronize(stream));
      win_centroid[f].assign(cc[f].begin(), cc[f].begin() + wc);
    }
    for (int d = 0; d < 3; ++d) {
      const long long fc = (long long)(D.E0 + (d == 0)) * (D.E1 + (d == 1)) *
                           (D.E2 + (d == 2));
      k_faces_from_cells<<<nblk(fc, bs), bs, 0, stream>>>(
          D, f, d, acells, X.G, d_cen, d_av + d * fmax);
      fcen[f][d].resize(fc);
      farea[f][d].resize(fc);
      GCS_BTRY(cudaMemcpyAsync(fcen[f][d].data(), d_cen, fc * sizeof(gamera_no_vec3),
                               cudaMemcpyDeviceToHost, stream));
      GCS_BTRY(cudaMemcpyAsync(farea[f][d].data(), d_av + d * fmax,
                               fc * sizeof(gamera_no_vec3), cudaMemcpyDeviceToHost,
                               stream));
      GCS_BTRY(cudaStreamSynchronize(stream));
      const long long ec = (long long)(D.E0 + (d != 0)) * (D.E1 + (d != 1)) *
                           (D.E2 + (d != 2));
      k_edges<<<nblk(ec, bs), bs, 0, stream>>>(D, f, d, vert, X.G, bad);
    }
    k_init_cells<<<nblk(cells, bs), bs, 0, stream>>>(D, f, kind, seed, wi, acells,
                                                     X.S, bad);
    if (wind) {
      if (!bg_pool && allocate_background() != 0) return -1;
      for (int d = 0; d < 3; ++d) {
        const long long fc = (long long)(D.E0 + (d == 0)) * (D.E1 + (d == 1)) *
                             (D.E2 + (d == 2));
        k_bg_faces<<<nblk(fc, 64), 64, 0, stream>>>(D, f, d, vert, m, X.G, X.BG,
                                                    stress, bad);
      }
      k_bg_cells<<<nblk(cells, 64), 64, 0, stream>>>(D, f, vert, m, X.G, X.BG,
                                                     stress, bad);
      for (int e = 0; e < 3; ++e) {
        const long long ec = (long long)(D.E0 + (e != 0)) * (D.E1 + (e != 1)) *
                             (D.E2 + (e != 2));
        k_bg_edges<<<nblk(ec, bs), bs, 0, stream>>>(D, f, e, vert, m, X.G, X.BG);
        k_init_lines<<<nblk(ec, bs), bs, 0, stream>>>(D, e, vert, bimf, line);
      }
    }
    for (int d = 0; d < 3; ++d) {
      const long long fc = (long long)(D.E0 + (d == 0)) * (D.E1 + (d == 1)) *
                           (D.E2 + (d == 2));
      k_init_flux<<<nblk(fc, bs), bs, 0, stream>>>(D, f, d, line, !wind, bu,
                                                   d_av + d * fmax, X.S);
    }
    GCS_BTRY(cudaGetLastError());
    GCS_BTRY(cudaStreamSynchronize(stream));
  }
  if (derive() != 0) return -1;
  k_init_b<<<nblk(kFaces * cells, bs), bs, 0, stream>>>(D, X.S, X.G, bad);
  int hbad = 0;
  GCS_BTRY(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, stream));
  GCS_BTRY(cudaStreamSynchronize(stream));
  cudaFree(work);
  cudaFree(d_cen);
  cudaFree(d_av);
  if (hbad) {
    set_error("degenerate geometry or invalid initial state", "init_case");
    return -1;
  }
  if (wind) bg_uploaded = 1;
  HaloGeometry geo;
  for (int f = 0; f < kFaces; ++f) {
    geo.cell_centroid[f] = cc[f].data();
    for (int d = 0; d < 3; ++d) {
      geo.face_centroid[f][d] = fcen[f][d].data();
      geo.face_area_vector[f][d] = farea[f][d].data();
    }
  }
  return build_plans(geo);
}

// A wind run on the grid of `o` (same extents, built by init_case): the
// geometry, background, halo/seam/edge plans, FP32 metric copies and the
// per-step scratch arrays are o's; this context owns only the state that
// lives from step to step (U, Uo, B, Bo, Phi, Phi_old), its step
// parameters, status and stream.  Runs sharing a grid must not step
// concurrently (they share the scratch arrays).
int Context::init_member(Context &o, unsigned long long seed, const WindInit &w) {
  if (!o.bg_uploaded || !o.pool || o.owner) {
    set_error("owner is not a device-built wind case", "init_member");
    return -1;
  }
  X = o.X;
  X.params = nullptr;
  X.status = nullptr;
  owner = &o;
  bg_uploaded = 1;
  bulk_b0_threshold = o.bulk_b0_threshold;
  const Dims &D = X.D;
  GCS_BTRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  const long long per = kFaces * D.Nn;
  pool_bytes = (size_t)22 * per * sizeof(double);
  GCS_BTRY(cudaMalloc(&pool, pool_bytes));
  GCS_BTRY(cudaMemsetAsync(pool, 0, pool_bytes, stream));
  double *p = (double *)pool;
  DevState &S = X.S;
  for (int m = 0; m < 5; ++m) {
    S.U[m] = p; p += per;
    S.Uo[m] = p; p += per;
  }
  for (int m = 0; m < 3; ++m) {
    S.B[m] = p; p += per;
    S.Bo[m] = p; p += per;
    S.P[m] = p; p += per;
    S.Po[m] = p; p += per;
  }
  GCS_BTRY(cudaMalloc(&X.params, sizeof(StepParams)));
  GCS_BTRY(cudaMalloc(&X.status, sizeof(DevStatus)));
  GCS_BTRY(cudaMemsetAsync(X.params, 0, sizeof(StepParams), stream));
  reset_status_async();
  // The initial state as init_case builds it for a wind case: vertices and
  // cell centroids of each face rebuilt into scratch (o's staging buffer
  // holds the cell geometry), the IMF edge integrals, Phi and the recovered
  // cell B on the shared recovery maps.
  const long long cells = (long long)D.E0 * D.E1 * D.E2;
  const long long verts = (long long)(D.E0 + 1) * (D.E1 + 1) * (D.E2 + 1);
  void *work = nullptr;
  const size_t wbytes = verts * sizeof(V3) + 3 * D.Nn * sizeof(double) + sizeof(int);
  GCS_BTRY(cudaMalloc(&work, wbytes));
  V3 *vert = (V3 *)work;
  double *line = (double *)(vert + verts);
  int *bad = (int *)(line + 3 * D.Nn);
  GCS_BTRY(cudaMemsetAsync(bad, 0, sizeof(int), stream));
  gamera_no_cell_geometry *acells = (gamera_no_cell_geometry *)o.staging;
  const V3 bimf = {0.0, 0.0, w.bz};
  const int bs = 128;
  for (int f = 0; f < kFaces; ++f) {
    k_vertices<<<nblk(verts, bs), bs, 0, stream>>>(f, D.nr, D.n, D.g, 2.5, 30.0,
                                                   log(12.0), vert);
    k_cells<<<nblk(cells, 64), 64, 0, stream>>>(D, vert, acells, bad);
    k_init_cells<<<nblk(cells, bs), bs, 0, stream>>>(D, f, 2, seed, w, acells, X.S,
                                                     bad);
    for (int e = 0; e < 3; ++e) {
      const long long ec = (long long)(D.E0 + (e != 0)) * (D.E1 + (e != 1)) *
                           (D.E2 + (e != 2));
      k_init_lines<<<nblk(ec, bs), bs, 0, stream>>>(D, e, vert, bimf, line);
    }
    for (int d = 0; d < 3; ++d) {
      const long long fc = (long long)(D.E0 + (d == 0)) * (D.E1 + (d == 1)) *
                           (D.E2 + (d == 2));
      k_init_flux<<<nblk(fc, bs), bs, 0, stream>>>(D, f, d, line, 0, V3{0.0, 0.0, 0.0},
                                                   nullptr, X.S);
    }
    GCS_BTRY(cudaGetLastError());
    GCS_BTRY(cudaStreamSynchronize(stream));
  }
  k_init_b<<<nblk(kFaces * cells, bs), bs, 0, stream>>>(D, X.S, X.G, bad);
  int hbad = 0;
  GCS_BTRY(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, stream));
  GCS_BTRY(cudaStreamSynchronize(stream));
  cudaFree(work);
  if (hbad) {
    set_error("degenerate geometry or invalid initial state", "init_member");
    return -1;
  }
  return 0;
}

__global__ void k_active_centroids(Dims D, const gamera_no_cell_geometry *cells, double *out) {
  const long long count = (long long)D.nr * D.n * D.n;
  const long long t = tid();
  if (t >= count) return;
  const int i = (int)(t / ((long long)D.n * D.n));
  const int j = (int)((t / D.n) % D.n);
  const int k = (int)(t % D.n);
  const gamera_no_vec3 x =
      cells[((long long)(i + D.g) * D.E1 + j + D.g) * D.E2 + k + D.g].centroid;
  for (int a = 0; a < 3; ++a) out[a * count + t] = x.value[a];
}

__global__ void k_active_vertices(Dims D, const V3 *vert, double *out) {
  const long long count = (long long)(D.nr + 1) * (D.n + 1) * (D.n + 1);
  const long long t = tid();
  if (t >= count) return;
  const int i = (int)(t / ((long long)(D.n + 1) * (D.n + 1)));
  const int j = (int)((t / (D.n + 1)) % (D.n + 1));
  const int k = (int)(t % (D.n + 1));
  const V3 x = vert[((long long)(i + D.g) * (D.E1 + 1) + j + D.g) * (D.E2 + 1) + k + D.g];
  out[t] = x.x;
  out[count + t] = x.y;
  out[2 * count + t] = x.z;
}

// Active-cell centroids [3][nr][n][n] and active vertices
// [3][nr+1][n+1][n+1] of one face of a device-built case, rebuilt on the
// device (analysis grid output).
int Context::face_coordinates(int f, std::vector<double> &cen, std::vector<double> &vert_out) {
  if (owner || !staging || grid_cell[0] != nullptr || f < 0 || f >= kFaces) {
    set_error("needs a device-built case", "face_coordinates");
    return -1;
  }
  const Dims &D = X.D;
  const long long cells = (long long)D.E0 * D.E1 * D.E2;
  const long long verts = (long long)(D.E0 + 1) * (D.E1 + 1) * (D.E2 + 1);
  const long long nc = (long long)D.nr * D.n * D.n;
  const long long nv = (long long)(D.nr + 1) * (D.n + 1) * (D.n + 1);
  void *work = nullptr;
  GCS_BTRY(cudaMalloc(&work, verts * sizeof(V3) + 3 * (nc + nv) * sizeof(double) + sizeof(int)));
  V3 *vert = (V3 *)work;
  double *dc = (double *)(vert + verts);
  double *dv = dc + 3 * nc;
  int *bad = (int *)(dv + 3 * nv);
  const int wind = bg_pool != nullptr;
  const double r_in = wind ? 2.5 : 2.0;
  const double r_out = wind ? 30.0 : (kind_shock ? 3.0 : 2.5);
  const int bs = 128;
  k_vertices<<<nblk(verts, bs), bs, 0, stream>>>(f, D.nr, D.n, D.g, r_in, r_out,
                                                 wind ? log(12.0) : 0.0, vert);
  k_cells<<<nblk(cells, 64), 64, 0, stream>>>(D, vert, (gamera_no_cell_geometry *)staging, bad);
  k_active_centroids<<<nblk(nc, bs), bs, 0, stream>>>(D, (gamera_no_cell_geometry *)staging, dc);
  k_active_vertices<<<nblk(nv, bs), bs, 0, stream>>>(D, vert, dv);
  cen.resize(3 * nc);
  vert_out.resize(3 * nv);
  GCS_BTRY(cudaGetLastError());
  GCS_BTRY(cudaMemcpyAsync(cen.data(), dc, 3 * nc * sizeof(double), cudaMemcpyDeviceToHost,
                           stream));
  GCS_BTRY(cudaMemcpyAsync(vert_out.data(), dv, 3 * nv * sizeof(double),
                           cudaMemcpyDeviceToHost, stream));
  GCS_BTRY(cudaStreamSynchronize(stream));
  cudaFree(work);
  return 0;
}

// Boundary-layer geometry of the device Earth boundary for a device-built
// wind case: vertices, cells and faces of each face rebuilt into scratch,
// the radial boundary layers copied into L, outer faces' B0 flux from the
// background (flux / area x area).
int Context::build_earth_layers(const EarthLayers &L) {
  if (owner || !staging || !bg_pool) {
    set_error("needs a device-built wind case", "build_earth_layers");
    return -1;
  }
  const Dims &D = X.D;
  const long long cells = (long long)D.E0 * D.E1 * D.E2;
  const long long verts = (long long)(D.E0 + 1) * (D.E1 + 1) * (D.E2 + 1);
  const size_t fmax = (size_t)verts;
  void *work = nullptr;
  const size_t wbytes = verts * sizeof(V3) + 2 * fmax * sizeof(gamera_no_vec3) + sizeof(int);
  GCS_BTRY(cudaMalloc(&work, wbytes));
  V3 *vert = (V3 *)work;
  gamera_no_vec3 *cen = (gamera_no_vec3 *)(vert + verts);
  gamera_no_vec3 *av = cen + fmax;
  int *bad = (int *)(av + fmax);
  GCS_BTRY(cudaMemsetAsync(bad, 0, sizeof(int), stream));
  gamera_no_cell_geometry *acells = (gamera_no_cell_geometry *)staging;
  const int bs = 128;
  for (int f = 0; f < kFaces; ++f) {
    k_vertices<<<nblk(verts, bs), bs, 0, stream>>>(f, D.nr, D.n, D.g, 2.5, 30.0,
                                                   log(12.0), vert);
    k_cells<<<nblk(cells, 64), 64, 0, stream>>>(D, vert, acells, bad);
    k_earth_layer_cells<<<dim3(nblk((long long)D.E1 * D.E2, bs), 2 * D.g), bs, 0,
                          stream>>>(D, f, acells, L);
    for (int d = 0; d < 3; ++d) {
      const long long fc = (long long)(D.E0 + (d == 0)) * (D.E1 + (d == 1)) *
                           (D.E2 + (d == 2));
      k_faces_from_cells<<<nblk(fc, bs), bs, 0, stream>>>(D, f, d, acells, X.G, cen, av);
      const long long pl = (long long)(D.E1 + (d == 1)) * (D.E2 + (d == 2));
      k_earth_layer_faces<<<dim3(nblk(pl, bs), D.g), bs, 0, stream>>>(D, f, d, cen, av, X.G,
                                                                      X.BG, L);
      const long long pe = (long long)(D.E1 + (d != 1)) * (D.E2 + (d != 2));
      k_earth_layer_edges<<<dim3(nblk(pe, bs), 5), bs, 0, stream>>>(D, f, d, vert, L);
    }
    GCS_BTRY(cudaGetLastError());
    GCS_BTRY(cudaStreamSynchronize(stream));
  }
  int hbad = 0;
  GCS_BTRY(cudaMemcpy(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost));
  cudaFree(work);
  if (hbad) {
    set_error("degenerate boundary-layer geometry", "build_earth_layers");
    return -1;
  }
  return 0;
}

}  // namespace gcs
