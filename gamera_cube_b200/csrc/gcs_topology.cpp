// Host plan construction for the device halo, seam and edge-EMF kernels.
// See gcs_topology.h for the reference correspondence.
#include "gcs_topology.h"

#include <cmath>
#include <cstdlib>
#include <cstring>

namespace gcs {
namespace topo {

// Right-handed face frames: normal, tangent a, tangent b
// (cubedsphere/cubedsphere_mesh.c:8-14; the frame table defines the cube
// orientation shared with the caller's grid, so it must be the same).
static const int kFrame[kFaces][3][3] = {
    {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}},
    {{-1, 0, 0}, {0, -1, 0}, {0, 0, 1}},
    {{0, 1, 0}, {-1, 0, 0}, {0, 0, 1}},
    {{0, -1, 0}, {1, 0, 0}, {0, 0, 1}},
    {{0, 0, 1}, {1, 0, 0}, {0, 1, 0}},
    {{0, 0, -1}, {1, 0, 0}, {0, -1, 0}}};

static double frame_dot(const double a[3], const int b[3]) {
  return a[0] * (double)b[0] + a[1] * (double)b[1] + a[2] * (double)b[2];
}

// Equiangular gnomonic direction (cubedsphere_mesh.c:58-75).
int direction(int face, double a, double b, double out[3]) {
  const double qp = 0.25 * acos(-1.0);
  if (face < 0 || face >= kFaces || !std::isfinite(a) || !std::isfinite(b) ||
      fabs(a) >= 2.0 * qp || fabs(b) >= 2.0 * qp)
    return -1;
  const double u = tan(a), v = tan(b);
  const double il = 1.0 / sqrt(1.0 + u * u + v * v);
  for (int d = 0; d < 3; ++d)
    out[d] = il * ((double)kFrame[face][0][d] + u * (double)kFrame[face][1][d] +
                   v * (double)kFrame[face][2][d]);
  return 0;
}

// Owning face and face coordinates of a direction (cubedsphere_mesh.c:77-103).
int inverse(const double dir[3], int *face, double *a, double *b) {
  for (int d = 0; d < 3; ++d)
    if (!std::isfinite(dir[d])) return -1;
  int sel = -1;
  double dom = 0.0;
  for (int f = 0; f < kFaces; ++f) {
    const double p = frame_dot(dir, kFrame[f][0]);
    if (p > dom) {
      dom = p;
      sel = f;
    }
  }
  if (sel < 0 || !std::isfinite(dom)) return -1;
  *face = sel;
  *a = atan2(frame_dot(dir, kFrame[sel][1]), dom);
  *b = atan2(frame_dot(dir, kFrame[sel][2]), dom);
  return 0;
}

// Edge adjacency with orientation (cubedsphere_mesh.c:105-162).
int edge_neighbor(int face, int edge, int *nface, int *nedge, int *reversed) {
  const double qp = 0.25 * acos(-1.0);
  const double eps = 1.0e-7;
  double a = 0.0, b = 0.0;
  if (edge == GAMERA_CS_A_LOWER || edge == GAMERA_CS_A_UPPER)
    a = (edge == GAMERA_CS_A_LOWER ? -1.0 : 1.0) * (qp + eps);
  else
    b = (edge == GAMERA_CS_B_LOWER ? -1.0 : 1.0) * (qp + eps);
  double out[3];
  int target;
  double ta, tb;
  if (direction(face, a, b, out) != 0 || inverse(out, &target, &ta, &tb) != 0 ||
      target == face)
    return -1;
  const int dedge = fabs(ta) > fabs(tb)
                        ? (ta < 0.0 ? GAMERA_CS_A_LOWER : GAMERA_CS_A_UPPER)
                        : (tb < 0.0 ? GAMERA_CS_B_LOWER : GAMERA_CS_B_UPPER);
  const double along = 0.2;
  double da[2];
  for (int n = 0; n < 2; ++n) {
    const double pos = n == 0 ? -along : along;
    double sa, sb;
    if (edge == GAMERA_CS_A_LOWER || edge == GAMERA_CS_A_UPPER) {
      sa = edge == GAMERA_CS_A_LOWER ? -qp : qp;
      sb = pos;
    } else {
      sa = pos;
      sb = edge == GAMERA_CS_B_LOWER ? -qp : qp;
    }
    if (direction(face, sa, sb, out) != 0) return -1;
    const double p = frame_dot(out, kFrame[target][0]);
    const double xa = atan2(frame_dot(out, kFrame[target][1]), p);
    const double xb = atan2(frame_dot(out, kFrame[target][2]), p);
    da[n] = dedge < GAMERA_CS_B_LOWER ? xb : xa;
  }
  *nface = target;
  *nedge = dedge;
  *reversed = da[1] < da[0];
  return 0;
}

// Integer identity of a shared vertex (cubedsphere_mesh.c:36-56).
int vertex_key(int face, const size_t active[3], const size_t vertex[3],
               int64_t key[4]) {
  if (face < 0 || face >= kFaces || active[1] == 0 || active[1] != active[2])
    return -1;
  for (int a = 0; a < 3; ++a)
    if (vertex[a] > active[a]) return -1;
  const int64_t n = (int64_t)active[1];
  const int64_t a = 2 * (int64_t)vertex[1] - n;
  const int64_t b = 2 * (int64_t)vertex[2] - n;
  key[0] = (int64_t)vertex[0];
  for (int d = 0; d < 3; ++d)
    key[d + 1] = (int64_t)kFrame[face][0][d] * n +
                 (int64_t)kFrame[face][1][d] * a +
                 (int64_t)kFrame[face][2][d] * b;
  return 0;
}

}  // namespace topo

namespace {

size_t idx3(const size_t e[3], size_t i, size_t j, size_t k) {
  return (i * e[1] + j) * e[2] + k;
}

// cubedsphere_halo.c:25-30
long stencil_start(double x, long n) {
  long s = (long)floor(x) - 3L;
  if (s < 0) s = 0;
  if (s > n - 8L) s = n - 8L;
  return s;
}

// cubedsphere_halo.c:32-57: base tap and the weight of base + 1.
void linear_weight(double x, long start, int *base, double *fraction) {
  const double logical = x - (double)start;
  if (logical < 0.0) {
    *base = 0;
    *fraction = logical;
  } else if (logical >= 7.0) {
    *base = 6;
    *fraction = logical - 6.0;
  } else {
    *base = (int)floor(logical);
    *fraction = logical - (double)*base;
  }
}

}  // namespace

// cubedsphere_halo.c:401-451, 502-514 (cell targets in the reference order).
int build_halo_cells(const HaloGeometry &geo, const Dims &D,
                     std::vector<HaloCell> &out) {
  out.clear();
  const double qp = 0.25 * acos(-1.0);
  const long n = D.n;
  const double da = 2.0 * qp / (double)D.n;
  const double db = 2.0 * qp / (double)D.n;
  for (int f = 0; f < kFaces; ++f) {
    const size_t ext[3] = {(size_t)D.E0, (size_t)D.E1, (size_t)D.E2};
    for (int i = D.g; i < D.g + D.nr; ++i)
      for (int j = 0; j < D.E1; ++j)
        for (int k = 0; k < D.E2; ++k) {
          if (j >= D.g && j < D.g + D.n && k >= D.g && k < D.g + D.n) continue;
          const gamera_no_vec3 pt = geo.cell_centroid[f][idx3(ext, i, j, k)];
          int donor;
          double a, b;
          if (topo::inverse(pt.value, &donor, &a, &b) != 0 || donor == f)
            return -1;
          const double x = (a + qp) / da - 0.5;
          const double y = (b + qp) / db - 0.5;
          const long sx = stencil_start(x, n), sy = stencil_start(y, n);
          int bx, by;
          double fx, fy;
          linear_weight(x, sx, &bx, &fx);
          linear_weight(y, sy, &by, &fy);
          const size_t nx = (size_t)fmax(0.0, fmin((double)(n - 1), nearbyint(x)));
          const size_t ny = (size_t)fmax(0.0, fmin((double)(n - 1), nearbyint(y)));
          HaloCell e;
          e.fx = fx;
          e.fy = fy;
          e.target = (unsigned)D.node(i, j, k);
          e.donor = (unsigned)D.node(i, D.g + (int)sx + bx, D.g + (int)sy + by);
          e.nearest = (unsigned)D.node(i, D.g + (int)nx, D.g + (int)ny);
          e.meta = (unsigned)f | ((unsigned)donor << 4) |
                   (i == D.g ? 256u : 0u) | (i == D.g + D.nr - 1 ? 512u : 0u);
          out.push_back(e);
        }
  }
  return 0;
}

// cubedsphere_halo.c:401-451, 515-535 (magnetic ghost faces).
int build_halo_faces(const HaloGeometry &geo, const Dims &D,
                     std::vector<HaloFace> &out) {
  out.clear();
  const double qp = 0.25 * acos(-1.0);
  const long n = D.n;
  for (int f = 0; f < kFaces; ++f) {
    for (int dir = 0; dir < 3; ++dir) {
      const size_t ext[3] = {(size_t)(D.E0 + (dir == 0)),
                             (size_t)(D.E1 + (dir == 1)),
                             (size_t)(D.E2 + (dir == 2))};
      for (size_t i = 0; i < ext[0]; ++i)
        for (size_t j = 0; j < ext[1]; ++j)
          for (size_t k = 0; k < ext[2]; ++k) {
            const size_t coord[3] = {i, j, k};
            int physical = 1;
            for (int d = 0; d < 3; ++d) {
              const size_t upper = (size_t)(D.g + D.act(d) + (dir == d));
              if (coord[d] < (size_t)D.g || coord[d] >= upper) physical = 0;
            }
            if (physical) continue;
            const size_t xi = idx3(ext, i, j, k);
            const gamera_no_vec3 cen = geo.face_centroid[f][dir][xi];
            const gamera_no_vec3 av = geo.face_area_vector[f][dir][xi];
            int donor;
            double a, b;
            if (topo::inverse(cen.value, &donor, &a, &b) != 0) return -1;
            const double x = (a + qp) * (double)D.n / (2.0 * qp) - 0.5;
            const double y = (b + qp) * (double)D.n / (2.0 * qp) - 0.5;
            const long sx = stencil_start(x, n), sy = stencil_start(y, n);
            int bx, by;
            double fx, fy;
            linear_weight(x, sx, &bx, &fx);
            linear_weight(y, sy, &by, &fy);
            const int si = (int)i < D.g ? D.g
                           : (int)i >= D.g + D.nr ? D.g + D.nr - 1 : (int)i;
            HaloFace e;
            e.fx = fx;
            e.fy = fy;
            e.ax = av.value[0];
            e.ay = av.value[1];
            e.az = av.value[2];
            e.target = (unsigned)D.node((int)i, (int)j, (int)k);
            e.donor = (unsigned)D.node(si, D.g + (int)sx + bx, D.g + (int)sy + by);
            e.meta = (unsigned)f | ((unsigned)dir << 4) | ((unsigned)donor << 8);
            e.pad = 0;
            out.push_back(e);
          }
    }
  }
  return 0;
}

// cubedsphere_interface.c:11-22: the 12 face pairs with face < neighbour.
int build_seams(const Dims &D, std::vector<Seam> &out) {
  out.clear();
  for (int f = 0; f < kFaces; ++f)
    for (int edge = 0; edge < GAMERA_CS_EDGE_COUNT; ++edge) {
      int nf, ne, rev;
      if (topo::edge_neighbor(f, edge, &nf, &ne, &rev) != 0) return -1;
      if (f >= nf) continue;
      Seam s;
      s.face = f;
      s.nface = nf;
      s.src_axis = edge < GAMERA_CS_B_LOWER ? 1 : 2;
      s.dst_axis = ne < GAMERA_CS_B_LOWER ? 1 : 2;
      s.src_b = edge % 2 == 0 ? D.g : D.g + D.act(s.src_axis);
      s.dst_b = ne % 2 == 0 ? D.g : D.g + D.act(s.dst_axis);
      s.orient = edge % 2 == ne % 2 ? -1.0 : 1.0;
      s.reversed = rev;
      out.push_back(s);
    }
  return out.size() == 12 ? 0 : -1;
}

namespace {

// Same element layout and comparator as the reference plan entry
// (cubedsphere_interface.c:95-124) so the C library sort yields the same
// permutation, and therefore the same summation order inside each group.
struct SeamEdge {
  int64_t endpoint[8];
  int face;
  int direction;
  size_t index;
  int sign;
};

int compare_point(const int64_t a[4], const int64_t b[4]) {
  for (int d = 0; d < 4; ++d) {
    if (a[d] < b[d]) return -1;
    if (a[d] > b[d]) return 1;
  }
  return 0;
}

int compare_edge(const void *l, const void *r) {
  const SeamEdge *a = (const SeamEdge *)l;
  const SeamEdge *b = (const SeamEdge *)r;
  for (int d = 0; d < 8; ++d) {
    if (a->endpoint[d] < b->endpoint[d]) return -1;
    if (a->endpoint[d] > b->endpoint[d]) return 1;
  }
  return 0;
}

}  // namespace

// cubedsphere_interface.c:126-209
int build_edge_groups(const Dims &D, std::vector<int> &offsets,
                      std::vector<EdgeMember> &members) {
  const size_t active[3] = {(size_t)D.nr, (size_t)D.n, (size_t)D.n};
  const size_t n = (size_t)D.n, g = (size_t)D.g;
  std::vector<SeamEdge> entries;
  for (int f = 0; f < kFaces; ++f)
    for (int d = 0; d < 3; ++d) {
      const size_t iu = g + active[0] + (d != 0);
      const size_t ju = g + active[1] + (d != 1);
      const size_t ku = g + active[2] + (d != 2);
      for (size_t i = g; i < iu; ++i)
        for (size_t j = g; j < ju; ++j)
          for (size_t k = g; k < ku; ++k) {
            const int on_a = j == g || j == g + n;
            const int on_b = k == g || k == g + n;
            const int shared = d == 0 ? (on_a || on_b) : d == 1 ? on_b : on_a;
            if (!shared) continue;
            size_t sv[3] = {i - g, j - g, k - g};
            size_t ev[3] = {sv[0], sv[1], sv[2]};
            ++ev[d];
            int64_t sk[4], ek[4];
            if (topo::vertex_key(f, active, sv, sk) != 0 ||
                topo::vertex_key(f, active, ev, ek) != 0)
              return -1;
            const int o = compare_point(sk, ek);
            if (o == 0) return -1;
            SeamEdge e;
            std::memset(&e, 0, sizeof(e));
            e.sign = o < 0 ? 1 : -1;
            for (int q = 0; q < 4; ++q) {
              e.endpoint[q] = o < 0 ? sk[q] : ek[q];
              e.endpoint[q + 4] = o < 0 ? ek[q] : sk[q];
            }
            e.face = f;
            e.direction = d;
            e.index = (size_t)D.node((int)i, (int)j, (int)k);
            entries.push_back(e);
          }
    }
  qsort(entries.data(), entries.size(), sizeof(SeamEdge), compare_edge);
  offsets.clear();
  members.clear();
  for (size_t first = 0; first < entries.size();) {
    size_t last = first + 1;
    while (last < entries.size() &&
           compare_edge(&entries[first], &entries[last]) == 0)
      ++last;
    if (last - first < 2 || last - first > 3) return -1;
    offsets.push_back((int)members.size());
    for (size_t t = first; t < last; ++t) {
      EdgeMember m;
      m.node = (unsigned)entries[t].index;
      m.face = (unsigned char)entries[t].face;
      m.dir = (unsigned char)entries[t].direction;
      m.sign = (signed char)entries[t].sign;
      m.pad = 0;
      members.push_back(m);
    }
    first = last;
  }
  offsets.push_back((int)members.size());
  return 0;
}

}  // namespace gcs
