// Context set-up: device allocation, conversion of the caller's host grid,
// background and storage (reference array-of-structures layout) into the
// device node layout, and the derived per-cell/face/edge constants that the
// reference recomputes in every call.
#include "gcs_context.h"

#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "gcs_physics.cuh"
#include "gcs_topology.h"

#include <cuda.h>
#include <cudaTypedefs.h>

namespace gcs {

namespace {

__device__ inline long long box_index(int *i, int *j, int *k, int E1, int E2,
                                      int E0) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long jk = (long long)E1 * E2;
  if (t >= jk * E0) return -1;
  *i = (int)(t / jk);
  *j = (int)((t / E2) % E1);
  *k = (int)(t % E2);
  return t;
}

inline unsigned blocks_for(long long n, int bs) {
  return (unsigned)((n + bs - 1) / bs);
}

// Uncalibrated moment recovery of one cell (nonorthogonal_operators.c:
// 17-54), used only to build the calibration response.
__device__ void moment_recovery(const gamera_no_cell_geometry &g,
                                const double flux[3][2], double out[3]) {
  double div = 0.0;
  double fld[3] = {0.0, 0.0, 0.0};
  for (int d = 0; d < 3; ++d) {
    const double lo = flux[d][0], hi = flux[d][1];
    div += hi - lo;
    for (int c = 0; c < 3; ++c)
      fld[c] += hi * g.face[d][1].centroid.value[c] -
                lo * g.face[d][0].centroid.value[c];
  }
  for (int c = 0; c < 3; ++c)
    out[c] = (fld[c] - div * g.centroid.value[c]) / g.volume;
}

// Cells: volume, 1/volume, min cfl length and the calibrated recovery map.
// The calibration (cubedsphere/cubedsphere_recovery.c:17-98) solves
// R b = raw with R the moment-formula response to the three uniform fields;
// raw is linear in the six face fluxes, raw = M phi, so the same pivoted
// elimination applied to the six columns of M yields b = (R^-1 M) phi.
__global__ void k_conv_cells(Dims D, int f, const gamera_no_cell_geometry *cells,
                             DevGeom G) {
  int i, j, k;
  if (box_index(&i, &j, &k, D.E1, D.E2, D.E0) < 0) return;
  const gamera_no_cell_geometry &g =
      cells[((long long)i * D.E1 + j) * D.E2 + k];
  const long long c = f * D.Nn + D.node(i, j, k);
  G.vol[c] = g.volume;
  G.ivol[c] = 1.0 / g.volume;
  double len = g.cfl_length[0];
  for (int d = 1; d < 3; ++d) len = fmin(len, g.cfl_length[d]);
  G.cflmin[c] = len;
  unsigned char ok = isfinite(g.volume) && g.volume > DBL_MIN;
  // response matrix, column = basis field
  double R[3][3];
  for (int basis = 0; basis < 3; ++basis) {
    double bf[3][2], col[3];
    for (int d = 0; d < 3; ++d)
      for (int s = 0; s < 2; ++s) bf[d][s] = g.face[d][s].area_vector.value[basis];
    moment_recovery(g, bf, col);
    for (int d = 0; d < 3; ++d) R[d][basis] = col[d];
  }
  // moment map M (3 x 6): column order i-lo, i-hi, j-lo, j-hi, k-lo, k-hi
  double A[3][9];
  for (int r = 0; r < 3; ++r) {
    for (int q = 0; q < 3; ++q) A[r][q] = R[r][q];
    for (int d = 0; d < 3; ++d) {
      A[r][3 + 2 * d] =
          (g.centroid.value[r] - g.face[d][0].centroid.value[r]) / g.volume;
      A[r][3 + 2 * d + 1] =
          (g.face[d][1].centroid.value[r] - g.centroid.value[r]) / g.volume;
    }
  }
  double scale = 0.0;
  for (int r = 0; r < 3; ++r)
    for (int q = 0; q < 3; ++q) scale = fmax(scale, fabs(A[r][q]));
  if (!isfinite(scale) || scale <= DBL_MIN) ok = 0;
  for (int col = 0; col < 3 && ok; ++col) {
    int piv = col;
    for (int r = col + 1; r < 3; ++r)
      if (fabs(A[r][col]) > fabs(A[piv][col])) piv = r;
    if (!isfinite(A[piv][col]) || fabs(A[piv][col]) <= 128.0 * DBL_EPSILON * scale) {
      ok = 0;
      break;
    }
    if (piv != col)
      for (int q = col; q < 9; ++q) {
        const double t = A[col][q];
        A[col][q] = A[piv][q];
        A[piv][q] = t;
      }
    const double inv = 1.0 / A[col][col];
    for (int q = col; q < 9; ++q) A[col][q] *= inv;
    for (int r = 0; r < 3; ++r) {
      if (r == col) continue;
      const double fct = A[r][col];
      for (int q = col; q < 9; ++q) A[r][q] -= fct * A[col][q];
    }
  }
  for (int r = 0; r < 3; ++r)
    for (int q = 0; q < 6; ++q) {
      const double v = ok ? A[r][3 + q] : 0.0;
      if (!isfinite(v)) ok = 0;
      G.rec[r * 6 + q][c] = v;
    }
  G.cell_ok[c] = ok;
}

__global__ void k_conv_faces(Dims D, int f, int d,
                             const gamera_no_face_geometry *faces, DevGeom G) {
  int i, j, k;
  const int e0 = D.E0 + (d == 0), e1 = D.E1 + (d == 1), e2 = D.E2 + (d == 2);
  if (box_index(&i, &j, &k, e1, e2, e0) < 0) return;
  const gamera_no_face_geometry &g = faces[((long long)i * e1 + j) * e2 + k];
  const long long c = f * D.Nn + D.node(i, j, k);
  G.area[d][c] = g.area;
  for (int q = 0; q < 3; ++q) {
    G.fn[d][q][c] = g.normal.value[q];
    G.ft1[d][q][c] = g.tangent1.value[q];
    G.ft2[d][q][c] = g.tangent2.value[q];
  }
}

__global__ void k_conv_edges(Dims D, int f, int e,
                             const gamera_no_edge_geometry *edges,
                             const unsigned char *valid, DevGeom G) {
  int i, j, k;
  const int e0 = D.E0 + (e != 0), e1 = D.E1 + (e != 1), e2 = D.E2 + (e != 2);
  if (box_index(&i, &j, &k, e1, e2, e0) < 0) return;
  const long long src = ((long long)i * e1 + j) * e2 + k;
  const gamera_no_edge_geometry &g = edges[src];
  const long long c = f * D.Nn + D.node(i, j, k);
  G.elen[e][c] = g.length;
  for (int q = 0; q < 3; ++q) {
    G.et1[e][q][c] = g.tangent1.value[q];
    G.et2[e][q][c] = g.tangent2.value[q];
  }
  G.edge_ok[e][c] = valid[src] ? 0 : (unsigned char)kStageEdgeGeometry;
}

// central8(volume) along the face normal; NaN where the reference
// reconstruction would reject the interface volume.
__global__ void k_derive_iv(Dims D, int d, DevGeom G) {
  int i, j, k;
  const int e0 = D.E0 + (d == 0), e1 = D.E1 + (d == 1), e2 = D.E2 + (d == 2);
  if (box_index(&i, &j, &k, e1, e2, e0) < 0) return;
  const int x[3] = {i, j, k};
  const int f = blockIdx.y;
  const long long c = f * D.Nn + D.node(i, j, k);
  if (x[d] < 4 || x[d] > D.ext(d) - 4) {
    G.iv[d][c] = NAN;
    return;
  }
  double v[8];
  for (int n = 0; n < 8; ++n) v[n] = G.vol[c + (n - 4) * D.stride(d)];
  const double iv = central8(v);
  G.iv[d][c] = (isfinite(iv) && fabs(iv) > DBL_MIN) ? iv : NAN;
}

// nonorthogonal_operators.c:81-113: area-weighted central6 face normal at the
// edge, projected on the edge tangents and normalised.
__device__ bool transverse_normal(const DevGeom &G, int fam, long long c,
                                  long long s, long long ec, int e,
                                  double out[2]) {
  double ar[8];
  for (int n = 0; n < 8; ++n) ar[n] = G.area[fam][c + (n - 4) * s];
  const double ia = central6(ar);
  if (!isfinite(ia) || fabs(ia) <= DBL_MIN) return false;
  double nv[3];
  for (int q = 0; q < 3; ++q) {
    double w[8];
    for (int n = 0; n < 8; ++n) w[n] = ar[n] * G.fn[fam][q][c + (n - 4) * s];
    nv[q] = central6(w) / ia;
  }
  const double p1 = dot3(nv[0], nv[1], nv[2], G.et1[e][0][ec], G.et1[e][1][ec],
                         G.et1[e][2][ec]);
  const double p2 = dot3(nv[0], nv[1], nv[2], G.et2[e][0][ec], G.et2[e][1][ec],
                         G.et2[e][2][ec]);
  const double pn = hypot(p1, p2);
  if (!isfinite(pn) || pn <= DBL_MIN) return false;
  out[0] = p1 / pn;
  out[1] = p2 / pn;
  return true;
}

// Edge constants of the EMF sweep for active edges of family e: the two
// central8 face-area sums, the transverse normals and the inverse 2x2
// determinant (nonorthogonal_sweep.c:309-406, nonorthogonal_operators.c:
// 56-79), with the reference's failure stage of each check.
__global__ void k_derive_edges(Dims D, int e, DevGeom G) {
  int i, j, k;
  const int a = (e + 1) % 3, bb = (e + 2) % 3;
  int cnt[3];
  cnt[e] = D.act(e);
  cnt[a] = D.act(a) + 1;
  cnt[bb] = D.act(bb) + 1;
  if (box_index(&i, &j, &k, cnt[1], cnt[2], cnt[0]) < 0) return;
  const int f = blockIdx.y;
  i += D.g;
  j += D.g;
  k += D.g;
  const long long c = f * D.Nn + D.node(i, j, k);
  if (G.edge_ok[e][c] != 0) return;
  const long long sa = D.stride(a), sb = D.stride(bb);
  unsigned char code = 0;
  // edge velocity: face interface volumes and the edge area
  for (int n = 0; n < 8 && !code; ++n)
    if (isnan(G.iv[a][c + (n - 4) * sb])) code = kStageEdgeVelocity;
  double ar[8];
  for (int n = 0; n < 8; ++n) ar[n] = G.area[a][c + (n - 4) * sb];
  const double ca = central8(ar);
  if (!code && !(isfinite(ca) && fabs(ca) > DBL_MIN)) code = kStageEdgeVelocity;
  double ar2[8];
  for (int n = 0; n < 8; ++n) ar2[n] = G.area[bb][c + (n - 4) * sa];
  const double cb = central8(ar2);
  double n1[2] = {0.0, 0.0}, n2[2] = {0.0, 0.0};
  if (!code && !transverse_normal(G, a, c, sb, c, e, n1)) code = kStageTransverse;
  if (!code && !(isfinite(cb) && fabs(cb) > DBL_MIN)) code = kStageTransverse;
  if (!code && !transverse_normal(G, bb, c, sa, c, e, n2)) code = kStageTransverse;
  double inv = 0.0;
  if (!code) {
    const double det = n1[0] * n2[1] - n2[0] * n1[1];
    const double sc =
        fmax(fmax(fabs(n1[0]), fabs(n1[1])), fmax(fabs(n2[0]), fabs(n2[1])));
    if (!isfinite(det) || sc <= DBL_MIN ||
        fabs(det) <= 64.0 * DBL_EPSILON * sc * sc)
      code = kStageSolveEdge;
    else
      inv = 1.0 / det;
  }
  const double len = G.elen[e][c];
  if (!code && !(isfinite(len) && len > DBL_MIN)) code = kStageEdgeEmf;
  G.ca[e][c] = ca;
  G.cb[e][c] = cb;
  G.en1[e][0][c] = n1[0];
  G.en1[e][1][c] = n1[1];
  G.en2[e][0][c] = n2[0];
  G.en2[e][1][c] = n2[1];
  G.einv[e][c] = inv;
  G.edge_ok[e][c] = code;
}

__global__ void k_conv_bg_cells(Dims D, int f, const gamera_no_vec3 *b0,
                                const gamera_no_vec3 *force, DevBg B) {
  int i, j, k;
  if (box_index(&i, &j, &k, D.E1, D.E2, D.E0) < 0) return;
  const long long s = ((long long)i * D.E1 + j) * D.E2 + k;
  const long long c = f * D.Nn + D.node(i, j, k);
  for (int q = 0; q < 3; ++q) {
    B.b0[q][c] = b0[s].value[q];
    B.force[q][c] = force ? force[s].value[q] : 0.0;
  }
}

__global__ void k_conv_bg_faces(Dims D, int f, int d, const gamera_no_vec3 *b0,
                                const double *flux, DevGeom G, DevBg B) {
  int i, j, k;
  const int e0 = D.E0 + (d == 0), e1 = D.E1 + (d == 1), e2 = D.E2 + (d == 2);
  if (box_index(&i, &j, &k, e1, e2, e0) < 0) return;
  const long long s = ((long long)i * e1 + j) * e2 + k;
  const long long c = f * D.Nn + D.node(i, j, k);
  for (int q = 0; q < 3; ++q) B.fb0[d][q][c] = b0[s].value[q];
  B.fb0n[d][c] = flux[s] / G.area[d][c];
}

__global__ void k_conv_bg_edges(Dims D, int f, int e, const gamera_no_vec3 *b0,
                                DevGeom G, DevBg B) {
  int i, j, k;
  const int e0 = D.E0 + (e != 0), e1 = D.E1 + (e != 1), e2 = D.E2 + (e != 2);
  if (box_index(&i, &j, &k, e1, e2, e0) < 0) return;
  const long long s = ((long long)i * e1 + j) * e2 + k;
  const long long c = f * D.Nn + D.node(i, j, k);
  const gamera_no_vec3 v = b0[s];
  B.eb0t1[e][c] = dot3(v.value[0], v.value[1], v.value[2], G.et1[e][0][c],
                       G.et1[e][1][c], G.et1[e][2][c]);
  B.eb0t2[e][c] = dot3(v.value[0], v.value[1], v.value[2], G.et2[e][0][c],
                       G.et2[e][1][c], G.et2[e][2][c]);
}

// Host array (reference layout, ncomp doubles per element) <-> node arrays.
struct Comp8 {
  double *p[8];
};

__global__ void k_scatter(Dims D, int f, int e0, int e1, int e2, int ncomp,
                          const double *src, Comp8 dst) {
  int i, j, k;
  const long long t = box_index(&i, &j, &k, e1, e2, e0);
  if (t < 0) return;
  const long long c = f * D.Nn + D.node(i, j, k);
  for (int q = 0; q < ncomp; ++q) dst.p[q][c] = src[t * ncomp + q];
}

__global__ void k_gather(Dims D, int f, int e0, int e1, int e2, int ncomp,
                         Comp8 src, double *dst) {
  int i, j, k;
  const long long t = box_index(&i, &j, &k, e1, e2, e0);
  if (t < 0) return;
  const long long c = f * D.Nn + D.node(i, j, k);
  for (int q = 0; q < ncomp; ++q) dst[t * ncomp + q] = src.p[q][c];
}

}  // namespace

// ---------------------------------------------------------------------------

Context::~Context() { release(); }

void Context::release() {
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  graph_exec = nullptr;
  if (pool) cudaFree(pool);
  if (bulk_pool) cudaFree(bulk_pool);
  bulk_pool = nullptr;
  if (bg_pool) cudaFree(bg_pool);
  bg_pool = nullptr;
  if (plans) cudaFree(plans);
  if (staging) cudaFree(staging);
  if (staging_host) cudaFreeHost(staging_host);
  if (X.params) cudaFree(X.params);
  if (X.status) cudaFree(X.status);
  if (pc_dipole) cudaFree(pc_dipole);   // one allocation with pc_stats
  pc_dipole = nullptr;
  pc_stats = nullptr;
  pc_on = 0;
  if (stream) cudaStreamDestroy(stream);
  pool = nullptr;
  plans = nullptr;
  staging = nullptr;
  staging_host = nullptr;
  X.params = nullptr;
  X.status = nullptr;
  stream = nullptr;
}

#define GCS_TRY(expr)                                  \
  do {                                                 \
    cudaError_t err_ = (expr);                         \
    if (err_ != cudaSuccess) {                         \
      set_error(cudaGetErrorString(err_), #expr);      \
      return -1;                                       \
    }                                                  \
  } while (0)

void Context::set_error(const char *what, const char *where) {
  snprintf(error, sizeof(error), "%s (%s)", what, where);
}

int Context::init(const gamera_no_grid grid[kFaces], const size_t active[3],
                  size_t ghost) {
  for (int f = 0; f < kFaces; ++f)
    for (int a = 0; a < 3; ++a)
      if (grid[f].cell_extent[a] != active[a] + 2 * ghost) {
        set_error("grid extent does not match active + 2 ghost", "init");
        return -1;
      }
  if (allocate(active, ghost) != 0) return -1;
  const Dims &D = X.D;
  DevGeom &G = X.G;
  for (int f = 0; f < kFaces; ++f) {
    grid_cell[f] = grid[f].cell;
    for (int d = 0; d < 3; ++d) grid_face[f][d] = grid[f].face[d].value;
  }
  const size_t cells = (size_t)D.E0 * D.E1 * D.E2;
  // ---- geometry conversion, face by face
  for (int f = 0; f < kFaces; ++f) {
    GCS_TRY(cudaMemcpyAsync(staging, grid[f].cell,
                            cells * sizeof(gamera_no_cell_geometry),
                            cudaMemcpyHostToDevice, stream));
    k_conv_cells<<<blocks_for((long long)cells, 128), 128, 0, stream>>>(
        D, f, (const gamera_no_cell_geometry *)staging, G);
    for (int d = 0; d < 3; ++d) {
      const size_t *fe = grid[f].face[d].extent;
      const size_t fc = fe[0] * fe[1] * fe[2];
      GCS_TRY(cudaMemcpyAsync(staging, grid[f].face[d].value,
                              fc * sizeof(gamera_no_face_geometry),
                              cudaMemcpyHostToDevice, stream));
      k_conv_faces<<<blocks_for((long long)fc, 128), 128, 0, stream>>>(
          D, f, d, (const gamera_no_face_geometry *)staging, G);
      const size_t *ee = grid[f].edge[d].extent;
      const size_t ec = ee[0] * ee[1] * ee[2];
      GCS_TRY(cudaMemcpyAsync(staging, grid[f].edge[d].value,
                              ec * sizeof(gamera_no_edge_geometry),
                              cudaMemcpyHostToDevice, stream));
      unsigned char *vbuf = (unsigned char *)staging +
                            ec * sizeof(gamera_no_edge_geometry);
      GCS_TRY(cudaMemcpyAsync(vbuf, grid[f].edge[d].valid, ec,
                              cudaMemcpyHostToDevice, stream));
      k_conv_edges<<<blocks_for((long long)ec, 128), 128, 0, stream>>>(
          D, f, d, (const gamera_no_edge_geometry *)staging, vbuf, G);
    }
    GCS_TRY(cudaStreamSynchronize(stream));
  }
  if (derive() != 0) return -1;
  // ---- ghost-target geometry of the halo plans, gathered from the grid
  std::vector<gamera_no_vec3> cc[kFaces], fcen[kFaces][3], farea[kFaces][3];
  HaloGeometry geo;
  for (int f = 0; f < kFaces; ++f) {
    cc[f].resize(cells);
    for (size_t c = 0; c < cells; ++c) cc[f][c] = grid[f].cell[c].centroid;
    geo.cell_centroid[f] = cc[f].data();
    for (int d = 0; d < 3; ++d) {
      const size_t *fe = grid[f].face[d].extent;
      const size_t fc = fe[0] * fe[1] * fe[2];
      fcen[f][d].resize(fc);
      farea[f][d].resize(fc);
      for (size_t q = 0; q < fc; ++q) {
        fcen[f][d][q] = grid[f].face[d].value[q].centroid;
        farea[f][d][q] = grid[f].face[d].value[q].area_vector;
      }
      geo.face_centroid[f][d] = fcen[f][d].data();
      geo.face_area_vector[f][d] = farea[f][d].data();
    }
  }
  return build_plans(geo);
}

int Context::allocate(const size_t active[3], size_t ghost) {
  if (active[1] != active[2] || active[1] < 9 || ghost != 4 || active[0] < 1 ||
      active[0] > 60000 || active[1] > 60000) {
    set_error("unsupported extents", "init");
    return -1;
  }
  Dims &D = X.D;
  D.nr = (int)active[0];
  D.n = (int)active[1];
  D.g = (int)ghost;
  D.E0 = D.nr + 2 * D.g;
  D.E1 = D.E2 = D.n + 2 * D.g;
  D.N1 = D.E1 + 1;
  // k stride padded to a multiple of 4 nodes: rows then start on 16-byte
  // boundaries in FP64 and FP32 arrays, as the TMA tensor maps of the
  // staged sweeps require (the pad nodes are never read as data)
  D.N2 = (D.E2 + 1 + 3) & ~3;
  D.Nn = (long long)(D.E0 + 1) * D.N1 * D.N2;
  if (D.Nn > 0xffffffffLL) {
    set_error("more than 2^32 nodes per face", "init");
    return -1;
  }
  GCS_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  if (prepare_flux_f64() != 0 || prepare_flux_f32() != 0) {
    set_error("staged flux sweeps cannot be configured on this device", "init");
    return -1;
  }

  // ---- one pool for every node array
  const long long per = kFaces * D.Nn;
  std::vector<double **> arrays;
  DevState &S = X.S;
  DevGeom &G = X.G;
  DevBg &B = X.BG;
  for (int m = 0; m < 5; ++m) {
    arrays.push_back(&S.U[m]);
    arrays.push_back(&S.Uo[m]);
    arrays.push_back(&S.Up[m]);
    arrays.push_back(&S.Pr[m]);
  }
  for (int m = 0; m < 3; ++m) arrays.push_back(&S.BN[m]);
  for (int m = 0; m < 3; ++m) {
    arrays.push_back(&S.B[m]);
    arrays.push_back(&S.Bo[m]);
    arrays.push_back(&S.P[m]);
    arrays.push_back(&S.Po[m]);
    arrays.push_back(&S.Bp[m]);
    arrays.push_back(&S.Pp[m]);
    arrays.push_back(&S.W[m]);
    arrays.push_back(&S.E[m]);
    for (int q = 0; q < 3; ++q) arrays.push_back(&S.FV[m][q]);
    for (int q = 0; q < 5; ++q) arrays.push_back(&S.F[m][q]);
    for (int q = 0; q < 3; ++q) arrays.push_back(&S.M[m][q]);
  }
  arrays.push_back(&G.vol);
  arrays.push_back(&G.ivol);
  arrays.push_back(&G.cflmin);
  for (int q = 0; q < 18; ++q) arrays.push_back(&G.rec[q]);
  for (int d = 0; d < 3; ++d) {
    arrays.push_back(&G.area[d]);
    arrays.push_back(&G.iv[d]);
    arrays.push_back(&G.elen[d]);
    arrays.push_back(&G.einv[d]);
    arrays.push_back(&G.ca[d]);
    arrays.push_back(&G.cb[d]);
    for (int q = 0; q < 3; ++q) {
      arrays.push_back(&G.fn[d][q]);
      arrays.push_back(&G.ft1[d][q]);
      arrays.push_back(&G.ft2[d][q]);
      arrays.push_back(&G.et1[d][q]);
      arrays.push_back(&G.et2[d][q]);
    }
    for (int q = 0; q < 2; ++q) {
      arrays.push_back(&G.en1[d][q]);
      arrays.push_back(&G.en2[d][q]);
    }
  }
  std::memset(&B, 0, sizeof(B));
  const size_t byte_arrays = 4;  // cell_ok + 3 edge_ok
  pool_bytes = arrays.size() * per * sizeof(double) + byte_arrays * per + 256;
  GCS_TRY(cudaMalloc(&pool, pool_bytes));
  GCS_TRY(cudaMemsetAsync(pool, 0, pool_bytes, stream));
  char *p = (char *)pool;
  for (double **a : arrays) {
    *a = (double *)p;
    p += per * sizeof(double);
  }
  G.cell_ok = (unsigned char *)p;
  p += per;
  for (int d = 0; d < 3; ++d) {
    G.edge_ok[d] = (unsigned char *)p;
    p += per;
  }
  GCS_TRY(cudaMalloc(&X.params, sizeof(StepParams)));
  GCS_TRY(cudaMalloc(&X.status, sizeof(DevStatus)));
  GCS_TRY(cudaMemsetAsync(X.params, 0, sizeof(StepParams), stream));
  reset_status_async();

  // ---- staging buffer: the largest host array of one face
  size_t cells = (size_t)D.E0 * D.E1 * D.E2;
  size_t largest = cells * sizeof(gamera_no_cell_geometry);
  for (int d = 0; d < 3; ++d) {
    const size_t fc = (size_t)(D.E0 + (d == 0)) * (D.E1 + (d == 1)) *
                      (D.E2 + (d == 2));
    largest = std::max(largest, fc * sizeof(gamera_no_face_geometry));
    largest = std::max(largest, fc * 5 * sizeof(double));
  }
  staging_bytes = largest;
  GCS_TRY(cudaMalloc(&staging, staging_bytes));
  return 0;
}

// Interface volumes and edge constants from the converted geometry.
int Context::derive() {
  const Dims &D = X.D;
  DevGeom &G = X.G;
  for (int d = 0; d < 3; ++d) {
    const long long fc = (long long)(D.E0 + (d == 0)) * (D.E1 + (d == 1)) *
                         (D.E2 + (d == 2));
    k_derive_iv<<<dim3(blocks_for(fc, 128), kFaces), 128, 0, stream>>>(D, d, G);
  }
  for (int e = 0; e < 3; ++e) {
    const long long ec = (long long)(D.act(e)) * (D.act((e + 1) % 3) + 1) *
                         (D.act((e + 2) % 3) + 1);
    k_derive_edges<<<dim3(blocks_for(ec, 128), kFaces), 128, 0, stream>>>(
        D, e, G);
  }
  GCS_TRY(cudaGetLastError());
  GCS_TRY(cudaStreamSynchronize(stream));
  return 0;
}

// Host plans, then one device allocation for all of them.
int Context::build_plans(const HaloGeometry &geo) {
  const Dims &D = X.D;
  std::vector<HaloCell> hc;
  std::vector<HaloFace> hf;
  std::vector<Seam> seams;
  std::vector<int> offsets;
  std::vector<EdgeMember> members;
  if (build_halo_cells(geo, D, hc) != 0 || build_halo_faces(geo, D, hf) != 0 ||
      build_seams(D, seams) != 0 ||
      build_edge_groups(D, offsets, members) != 0) {
    set_error("plan construction failed", "init");
    return -1;
  }
  const size_t b_hc = hc.size() * sizeof(HaloCell);
  const size_t b_hf = hf.size() * sizeof(HaloFace);
  const size_t b_se = seams.size() * sizeof(Seam);
  const size_t b_of = offsets.size() * sizeof(int);
  const size_t b_me = members.size() * sizeof(EdgeMember);
  auto al = [](size_t x) { return (x + 255) / 256 * 256; };
  plans_bytes = al(b_hc) + al(b_hf) + al(b_se) + al(b_of) + al(b_me);
  GCS_TRY(cudaMalloc(&plans, plans_bytes));
  char *q = (char *)plans;
  X.halo_cells = (HaloCell *)q;
  q += al(b_hc);
  X.halo_faces = (HaloFace *)q;
  q += al(b_hf);
  X.seams = (Seam *)q;
  q += al(b_se);
  X.edge_offsets = (int *)q;
  q += al(b_of);
  X.edge_members = (EdgeMember *)q;
  X.n_halo_cells = (long long)hc.size();
  X.n_halo_faces = (long long)hf.size();
  X.n_edge_groups = (int)offsets.size() - 1;
  GCS_TRY(cudaMemcpyAsync(X.halo_cells, hc.data(), b_hc, cudaMemcpyHostToDevice, stream));
  GCS_TRY(cudaMemcpyAsync(X.halo_faces, hf.data(), b_hf, cudaMemcpyHostToDevice, stream));
  GCS_TRY(cudaMemcpyAsync(X.seams, seams.data(), b_se, cudaMemcpyHostToDevice, stream));
  GCS_TRY(cudaMemcpyAsync(X.edge_offsets, offsets.data(), b_of, cudaMemcpyHostToDevice, stream));
  GCS_TRY(cudaMemcpyAsync(X.edge_members, members.data(), b_me, cudaMemcpyHostToDevice, stream));
  GCS_TRY(cudaStreamSynchronize(stream));
  return 0;
}

// State arrays, seams and edge groups only (no geometry): for the
// reference entry points that take storage without a grid.
int Context::init_topology(const size_t active[3], size_t ghost) {
  if (allocate(active, ghost) != 0) return -1;
  const Dims &D = X.D;
  std::vector<Seam> seams;
  std::vector<int> offsets;
  std::vector<EdgeMember> members;
  if (build_seams(D, seams) != 0 || build_edge_groups(D, offsets, members) != 0) {
    set_error("plan construction failed", "init_topology");
    return -1;
  }
  const size_t b_se = seams.size() * sizeof(Seam);
  const size_t b_of = offsets.size() * sizeof(int);
  const size_t b_me = members.size() * sizeof(EdgeMember);
  auto al = [](size_t x) { return (x + 255) / 256 * 256; };
  plans_bytes = al(b_se) + al(b_of) + al(b_me);
  GCS_TRY(cudaMalloc(&plans, plans_bytes));
  char *q = (char *)plans;
  X.seams = (Seam *)q;
  q += al(b_se);
  X.edge_offsets = (int *)q;
  q += al(b_of);
  X.edge_members = (EdgeMember *)q;
  X.n_halo_cells = 0;
  X.n_halo_faces = 0;
  X.n_edge_groups = (int)offsets.size() - 1;
  GCS_TRY(cudaMemcpyAsync(X.seams, seams.data(), b_se, cudaMemcpyHostToDevice, stream));
  GCS_TRY(cudaMemcpyAsync(X.edge_offsets, offsets.data(), b_of, cudaMemcpyHostToDevice,
                          stream));
  GCS_TRY(cudaMemcpyAsync(X.edge_members, members.data(), b_me, cudaMemcpyHostToDevice,
                          stream));
  GCS_TRY(cudaStreamSynchronize(stream));
  return 0;
}

void convert_cells(const Ctx &X, int f, const gamera_no_cell_geometry *cells,
                   cudaStream_t s) {
  const long long n = (long long)X.D.E0 * X.D.E1 * X.D.E2;
  k_conv_cells<<<blocks_for(n, 128), 128, 0, s>>>(X.D, f, cells, X.G);
}

int Context::allocate_background() {
  const Dims &D = X.D;
  const long long per = kFaces * D.Nn;
  std::vector<double **> arrays;
  DevBg &B = X.BG;
  for (int q = 0; q < 3; ++q) {
    arrays.push_back(&B.b0[q]);
    arrays.push_back(&B.force[q]);
    arrays.push_back(&B.fb0n[q]);
    arrays.push_back(&B.eb0t1[q]);
    arrays.push_back(&B.eb0t2[q]);
    for (int r = 0; r < 3; ++r) arrays.push_back(&B.fb0[q][r]);
  }
  bg_bytes = arrays.size() * per * sizeof(double);
  GCS_TRY(cudaMalloc(&bg_pool, bg_bytes));
  GCS_TRY(cudaMemsetAsync(bg_pool, 0, bg_bytes, stream));
  char *p = (char *)bg_pool;
  for (double **a : arrays) {
    *a = (double *)p;
    p += per * sizeof(double);
  }
  return 0;
}

int Context::upload_background(const gamera_no_background_field bg[kFaces]) {
  if (owner) {
    set_error("the background of a shared grid belongs to its owner", "upload_background");
    return -1;
  }
  const Dims &D = X.D;
  if (!bg_pool && allocate_background() != 0) return -1;
  const size_t cells = (size_t)D.E0 * D.E1 * D.E2;
  for (int f = 0; f < kFaces; ++f) {
    if (bg[f].cell_magnetic == nullptr) {
      set_error("background without cell field", "upload_background");
      return -1;
    }
    double *a = (double *)staging;
    double *b = a + 3 * cells;
    GCS_TRY(cudaMemcpyAsync(a, bg[f].cell_magnetic, cells * 3 * sizeof(double),
                            cudaMemcpyHostToDevice, stream));
    if (bg[f].cell_force)
      GCS_TRY(cudaMemcpyAsync(b, bg[f].cell_force, cells * 3 * sizeof(double),
                              cudaMemcpyHostToDevice, stream));
    k_conv_bg_cells<<<blocks_for((long long)cells, 128), 128, 0, stream>>>(
        D, f, (const gamera_no_vec3 *)a,
        bg[f].cell_force ? (const gamera_no_vec3 *)b : nullptr, X.BG);
    GCS_TRY(cudaStreamSynchronize(stream));
    for (int d = 0; d < 3; ++d) {
      const size_t fc = (size_t)(D.E0 + (d == 0)) * (D.E1 + (d == 1)) *
                        (D.E2 + (d == 2));
      if (bg[f].face_magnetic[d] && bg[f].face_flux[d]) {
        GCS_TRY(cudaMemcpyAsync(a, bg[f].face_magnetic[d], fc * 3 * sizeof(double),
                                cudaMemcpyHostToDevice, stream));
        GCS_TRY(cudaMemcpyAsync(a + 3 * fc, bg[f].face_flux[d], fc * sizeof(double),
                                cudaMemcpyHostToDevice, stream));
        k_conv_bg_faces<<<blocks_for((long long)fc, 128), 128, 0, stream>>>(
            D, f, d, (const gamera_no_vec3 *)a, a + 3 * fc, X.G, X.BG);
      }
      const size_t ec = (size_t)(D.E0 + (d != 0)) * (D.E1 + (d != 1)) *
                        (D.E2 + (d != 2));
      if (bg[f].edge_magnetic[d]) {
        GCS_TRY(cudaStreamSynchronize(stream));
        GCS_TRY(cudaMemcpyAsync(a, bg[f].edge_magnetic[d], ec * 3 * sizeof(double),
                                cudaMemcpyHostToDevice, stream));
        k_conv_bg_edges<<<blocks_for((long long)ec, 128), 128, 0, stream>>>(
            D, f, d, (const gamera_no_vec3 *)a, X.G, X.BG);
      }
      GCS_TRY(cudaStreamSynchronize(stream));
    }
  }
  GCS_TRY(cudaGetLastError());
  for (int f = 0; f < kFaces; ++f) {
    bg_key[f][0] = bg[f].cell_magnetic;
    bg_key[f][1] = bg[f].cell_force;
    for (int d = 0; d < 3; ++d) {
      bg_key[f][2 + d] = bg[f].face_magnetic[d];
      bg_key[f][5 + d] = bg[f].face_flux[d];
      bg_key[f][8 + d] = bg[f].edge_magnetic[d];
    }
  }
  bg_uploaded = 1;
  return 0;
}

bool Context::background_matches(const gamera_no_background_field bg[kFaces]) const {
  if (!bg_uploaded) return false;
  for (int f = 0; f < kFaces; ++f) {
    if (bg_key[f][0] != bg[f].cell_magnetic || bg_key[f][1] != bg[f].cell_force)
      return false;
    for (int d = 0; d < 3; ++d)
      if (bg_key[f][2 + d] != bg[f].face_magnetic[d] ||
          bg_key[f][5 + d] != bg[f].face_flux[d] ||
          bg_key[f][8 + d] != bg[f].edge_magnetic[d])
        return false;
  }
  return true;
}

int Context::transfer_array(int f, int kind, int dir, bool upload, double *host) {
  const Dims &D = X.D;
  int e[3] = {D.E0, D.E1, D.E2};
  Comp8 c{};
  int ncomp = 0;
  switch (kind) {
    case kArrU: ncomp = 5; for (int q = 0; q < 5; ++q) c.p[q] = X.S.U[q]; break;
    case kArrUo: ncomp = 5; for (int q = 0; q < 5; ++q) c.p[q] = X.S.Uo[q]; break;
    case kArrUp: ncomp = 5; for (int q = 0; q < 5; ++q) c.p[q] = X.S.Up[q]; break;
    case kArrB: ncomp = 3; for (int q = 0; q < 3; ++q) c.p[q] = X.S.B[q]; break;
    case kArrBo: ncomp = 3; for (int q = 0; q < 3; ++q) c.p[q] = X.S.Bo[q]; break;
    case kArrBp: ncomp = 3; for (int q = 0; q < 3; ++q) c.p[q] = X.S.Bp[q]; break;
    case kArrP: ncomp = 1; c.p[0] = X.S.P[dir]; e[dir] += 1; break;
    case kArrPo: ncomp = 1; c.p[0] = X.S.Po[dir]; e[dir] += 1; break;
    case kArrPp: ncomp = 1; c.p[0] = X.S.Pp[dir]; e[dir] += 1; break;
    case kArrF: ncomp = 5; for (int q = 0; q < 5; ++q) c.p[q] = X.S.F[dir][q]; e[dir] += 1; break;
    case kArrM: ncomp = 3; for (int q = 0; q < 3; ++q) c.p[q] = X.S.M[dir][q]; e[dir] += 1; break;
    case kArrE: ncomp = 1; c.p[0] = X.S.E[dir];
      for (int a = 0; a < 3; ++a) e[a] += (a != dir);
      break;
    default: set_error("bad array kind", "transfer"); return -1;
  }
  const long long count = (long long)e[0] * e[1] * e[2];
  const size_t bytes = (size_t)count * ncomp * sizeof(double);
  if (!staging && owner) {
    // runs sharing a grid allocate their transfer buffer on first use: the
    // largest state array of one face (5 doubles per node)
    staging_bytes = (size_t)(D.E0 + 1) * (D.E1 + 1) * (D.E2 + 1) * 5 * sizeof(double);
    GCS_TRY(cudaMalloc(&staging, staging_bytes));
  }
  if (bytes > staging_bytes) {
    set_error("staging too small", "transfer");
    return -1;
  }
  if (upload) {
    GCS_TRY(cudaMemcpyAsync(staging, host, bytes, cudaMemcpyHostToDevice, stream));
    k_scatter<<<blocks_for(count, 256), 256, 0, stream>>>(
        D, f, e[0], e[1], e[2], ncomp, (const double *)staging, c);
  } else {
    k_gather<<<blocks_for(count, 256), 256, 0, stream>>>(
        D, f, e[0], e[1], e[2], ncomp, c, (double *)staging);
    GCS_TRY(cudaMemcpyAsync(host, staging, bytes, cudaMemcpyDeviceToHost, stream));
  }
  // The staging buffer is reused by the next transfer.
  GCS_TRY(cudaStreamSynchronize(stream));
  return 0;
}

int Context::upload_state(const gamera_no_storage st[kFaces]) {
  for (int f = 0; f < kFaces; ++f) {
    for (int a = 0; a < 3; ++a)
      if (st[f].cell_extent[a] != (size_t)X.D.ext(a)) {
        set_error("storage extent mismatch", "upload_state");
        return -1;
      }
    if (transfer_array(f, kArrU, 0, true, st[f].conserved) ||
        transfer_array(f, kArrUo, 0, true, st[f].old_conserved) ||
        transfer_array(f, kArrB, 0, true, (double *)st[f].cell_magnetic) ||
        transfer_array(f, kArrBo, 0, true, (double *)st[f].old_cell_magnetic))
      return -1;
    for (int d = 0; d < 3; ++d)
      if (transfer_array(f, kArrP, d, true, st[f].face_flux[d]) ||
          transfer_array(f, kArrPo, d, true, st[f].old_face_flux[d]))
        return -1;
  }
  return 0;
}

int Context::download_state(gamera_no_storage st[kFaces], int scratch) {
  for (int f = 0; f < kFaces; ++f) {
    if (transfer_array(f, kArrU, 0, false, st[f].conserved) ||
        transfer_array(f, kArrUo, 0, false, st[f].old_conserved) ||
        transfer_array(f, kArrB, 0, false, (double *)st[f].cell_magnetic) ||
        transfer_array(f, kArrBo, 0, false, (double *)st[f].old_cell_magnetic))
      return -1;
    for (int d = 0; d < 3; ++d)
      if (transfer_array(f, kArrP, d, false, st[f].face_flux[d]) ||
          transfer_array(f, kArrPo, d, false, st[f].old_face_flux[d]))
        return -1;
    if (scratch) {
      if (transfer_array(f, kArrUp, 0, false, st[f].predicted_conserved) ||
          transfer_array(f, kArrBp, 0, false,
                         (double *)st[f].predicted_cell_magnetic))
        return -1;
      for (int d = 0; d < 3; ++d)
        if (transfer_array(f, kArrPp, d, false, st[f].predicted_face_flux[d]) ||
            transfer_array(f, kArrF, d, false, st[f].fluid_face_flux[d]) ||
            transfer_array(f, kArrM, d, false,
                           (double *)st[f].maxwell_face_flux[d]) ||
            transfer_array(f, kArrE, d, false, st[f].edge_emf[d]))
          return -1;
    }
  }
  return 0;
}

void Context::reset_status_async() {
  DevStatus z;
  std::memset(&z, 0, sizeof(z));
  const double big = DBL_MAX;
  std::memcpy(&z.cfl_min_bits, &big, sizeof(big));
  host_status = z;
  cudaMemcpyAsync(X.status, &host_status, sizeof(DevStatus),
                  cudaMemcpyHostToDevice, stream);
}

int Context::read_status(DevStatus *out) {
  GCS_TRY(cudaMemcpyAsync(out, X.status, sizeof(DevStatus),
                          cudaMemcpyDeviceToHost, stream));
  GCS_TRY(cudaStreamSynchronize(stream));
  return 0;
}

}  // namespace gcs

namespace gcs {

namespace {

// FP32 copy of the layers [lo, N0) of every face of a full FP64 node array
// (the window of the FP32-bulk arrays, Bulk::at).
__global__ void k_to_f32_window(const double *src, float *dst, long long face_nodes,
                                long long Nn, long long shift) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kFaces * face_nodes) return;
  const long long f = t / face_nodes;
  dst[t] = (float)src[f * Nn + shift + (t - f * face_nodes)];
}

__global__ void k_layer_b0(Dims D, DevBg BG, unsigned long long *layer_max) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long cells = (long long)D.E0 * D.E1 * D.E2;
  if (t >= kFaces * cells) return;
  const int f = (int)(t / cells);
  const long long r = t - f * cells;
  const int i = (int)(r / ((long long)D.E1 * D.E2));
  const int j = (int)((r / D.E2) % D.E1), k = (int)(r % D.E2);
  const long long c = f * D.Nn + D.node(i, j, k);
  const double b = sqrt(BG.b0[0][c] * BG.b0[0][c] + BG.b0[1][c] * BG.b0[1][c] +
                        BG.b0[2][c] * BG.b0[2][c]);
  if (isfinite(b)) atomicMax(&layer_max[i], (unsigned long long)__double_as_longlong(b));
}

}  // namespace

// FP32 arrays of the bulk path, one per node per component: 14 sweep
// inputs (Pr 5, Bp 3, BN 3, W 3), 76 metric (vol, iv 3, area 3, face
// frames 27, edge length 3, edge tangents 18, transverse normals 12,
// 1/det 3, central face areas 6) and 18 background (face B0 9, face B0
// normal 3, edge B0 projections 6).  The sweep outputs stay the FP64
// arrays of the state.
int Context::enable_bulk(int on) {
  if (owner) {
    if (on && !owner->X.bulk) {
      set_error("switch the grid owner to FP32-bulk first", "enable_bulk");
      return -1;
    }
    X.B32 = owner->X.B32;
    X.bulk_split = owner->X.bulk_split;
    X.bulk = on ? 1 : 0;
    return 0;
  }
  if (!on) {
    X.bulk = 0;
    return 0;
  }
  const int arrays = 14 + 76 + 18;
  if (!bulk_pool) {
    // the FP32 arrays cover the layers the FP32 sweeps read: from four
    // layers (the Up7 reach) inside the first FP32 layer outwards
    if (set_bulk_split(bulk_b0_threshold) != 0) return -1;
    const Dims &D = X.D;
    const int lo = X.bulk_split > 4 ? X.bulk_split - 4 : 0;
    X.B32.lo = lo;
    X.B32.face_nodes = (long long)(D.E0 + 1 - lo) * D.N1 * D.N2;
    X.B32.shift = (long long)lo * D.N1 * D.N2;
  }
  const long long n = (long long)kFaces * X.B32.face_nodes;
  if (!bulk_pool) {
    bulk_bytes = (size_t)arrays * n * sizeof(float);
    if (cudaMalloc(&bulk_pool, bulk_bytes) != cudaSuccess) {
      bulk_pool = nullptr;
      set_error("cannot allocate the FP32 arrays", "enable_bulk");
      return -1;
    }
    cudaMemsetAsync(bulk_pool, 0, bulk_bytes, stream);
    float *q = (float *)bulk_pool;
    auto take = [&]() {
      float *r = q;
      q += n;
      return r;
    };
    Bulk<float> &B = X.B32;
    for (int m = 0; m < 5; ++m) B.Pr[m] = take();
    for (int d = 0; d < 3; ++d) {
      B.Bp[d] = take();
      B.BN[d] = take();
      B.W[d] = take();
      B.E[d] = X.S.E[d];
      for (int m = 0; m < 3; ++m) B.FV[d][m] = X.S.FV[d][m];
      for (int m = 0; m < 5; ++m) B.F[d][m] = X.S.F[d][m];
      for (int m = 0; m < 3; ++m) B.M[d][m] = X.S.M[d][m];
    }
    const DevGeom &G = X.G;
    const int bs = 256;
    const unsigned nb = (unsigned)((n + bs - 1) / bs);
    auto conv = [&](const double *src) -> const float * {
      float *dst = take();
      if (src)
        k_to_f32_window<<<nb, bs, 0, stream>>>(src, dst, B.face_nodes, X.D.Nn, B.shift);
      return dst;
    };
    B.vol = conv(G.vol);
    for (int d = 0; d < 3; ++d) {
      B.iv[d] = conv(G.iv[d]);
      B.area[d] = conv(G.area[d]);
      B.elen[d] = conv(G.elen[d]);
      B.einv[d] = conv(G.einv[d]);
      B.ca[d] = conv(G.ca[d]);
      B.cb[d] = conv(G.cb[d]);
      for (int m = 0; m < 3; ++m) {
        B.fn[d][m] = conv(G.fn[d][m]);
        B.ft1[d][m] = conv(G.ft1[d][m]);
        B.ft2[d][m] = conv(G.ft2[d][m]);
        B.et1[d][m] = conv(G.et1[d][m]);
        B.et2[d][m] = conv(G.et2[d][m]);
      }
      for (int m = 0; m < 2; ++m) {
        B.en1[d][m] = conv(G.en1[d][m]);
        B.en2[d][m] = conv(G.en2[d][m]);
      }
    }
    for (int d = 0; d < 3; ++d) {
      B.fb0n[d] = take();
      B.eb0t1[d] = take();
      B.eb0t2[d] = take();
      for (int m = 0; m < 3; ++m) B.fb0[d][m] = take();
    }
    bulk_bg_dirty = 1;
  }
  if (bulk_bg_dirty) {
    // the background's FP32 copies follow every background upload
    const DevBg &BG = X.BG;
    Bulk<float> &B = X.B32;
    const int bs = 256;
    const unsigned nb = (unsigned)((n + bs - 1) / bs);
    auto conv = [&](const double *src, const float *dst) {
      if (src)
        k_to_f32_window<<<nb, bs, 0, stream>>>(src, (float *)dst, B.face_nodes, X.D.Nn,
                                               B.shift);
    };
    for (int d = 0; d < 3; ++d) {
      conv(BG.fb0n[d], B.fb0n[d]);
      conv(BG.eb0t1[d], B.eb0t1[d]);
      conv(BG.eb0t2[d], B.eb0t2[d]);
      for (int m = 0; m < 3; ++m) conv(BG.fb0[d][m], B.fb0[d][m]);
    }
    bulk_bg_dirty = 0;
  }
  if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(stream) != cudaSuccess) {
    set_error("FP32 conversion failed", "enable_bulk");
    return -1;
  }
  if (set_bulk_split(bulk_b0_threshold) != 0) return -1;
  X.bulk = 1;
  return 0;
}

// Radial layers whose largest cell |B0| exceeds the threshold, and all
// layers inside them, keep the FP64 sweeps.
int Context::set_bulk_split(double b0_threshold) {
  if (owner) {
    set_error("the FP64 layers of a shared grid are its owner's", "set_bulk_split");
    return -1;
  }
  bulk_b0_threshold = b0_threshold;
  const Dims &D = X.D;
  X.bulk_split = 0;
  if (X.BG.b0[0] == nullptr) return 0;
  unsigned long long *dmax = nullptr;
  std::vector<unsigned long long> hmax(D.E0, 0ULL);
  const long long cells = (long long)kFaces * D.E0 * D.E1 * D.E2;
  if (cudaMalloc(&dmax, D.E0 * sizeof(unsigned long long)) != cudaSuccess) {
    set_error("cannot allocate", "set_bulk_split");
    return -1;
  }
  cudaMemsetAsync(dmax, 0, D.E0 * sizeof(unsigned long long), stream);
  k_layer_b0<<<(unsigned)((cells + 255) / 256), 256, 0, stream>>>(D, X.BG, dmax);
  const bool ok = cudaMemcpyAsync(hmax.data(), dmax, D.E0 * sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost, stream) == cudaSuccess &&
                  cudaStreamSynchronize(stream) == cudaSuccess;
  cudaFree(dmax);
  if (!ok) {
    set_error("layer B0 reduction failed", "set_bulk_split");
    return -1;
  }
  for (int i = D.E0 - 1; i >= 0; --i) {
    double b;
    memcpy(&b, &hmax[i], sizeof(b));
    if (b > b0_threshold) {
      X.bulk_split = i + 1;
      break;
    }
  }
  if (bulk_pool != nullptr && X.bulk_split - 4 < X.B32.lo) {
    // the FP32 window no longer reaches the new first FP32 layer: rebuild
    // the FP32 arrays for the wider window
    cudaStreamSynchronize(stream);
    cudaFree(bulk_pool);
    bulk_pool = nullptr;
    bulk_bytes = 0;
    X.B32 = Bulk<float>{};
    const int was = X.bulk;
    X.bulk = 0;
    if (was) return enable_bulk(1);
  }
  return 0;
}

}  // namespace gcs

namespace gcs {

// Tensor map of one node array of all six faces (layers [lo, N0) of each),
// viewed as the 3-D tensor (k: N2, j: N1, face * (N0 - lo) + i - lo) with k
// contiguous, for the TMA-staged
// sweeps.  The driver's encoder is reached through the runtime's entry-point
// query, so the library links the runtime only.
int encode_cell_map(CUtensorMap *map, const void *base, int elem_bytes, const Dims &D,
                    int lo, int box_x, int box_y, int box_z) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (encode == nullptr) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess || fn == nullptr)
      return -1;
    encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  }
  if (((size_t)base & 15) != 0 || (elem_bytes != 4 && elem_bytes != 8)) return -1;
  const cuuint64_t dims[3] = {(cuuint64_t)D.N2, (cuuint64_t)D.N1,
                              (cuuint64_t)kFaces * (cuuint64_t)(D.E0 + 1 - lo)};
  const cuuint64_t strides[2] = {(cuuint64_t)D.N2 * elem_bytes,
                                 (cuuint64_t)D.N2 * D.N1 * elem_bytes};
  const cuuint32_t box[3] = {(cuuint32_t)box_x, (cuuint32_t)box_y, (cuuint32_t)box_z};
  const cuuint32_t estride[3] = {1, 1, 1};
  const CUresult r = encode(
      map, elem_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
      3, const_cast<void *>(base), dims, strides, box, estride,
      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -1;
}

}  // namespace gcs
