// Host-side cubed-sphere topology used to build the immutable halo, seam and
// edge-group plans.  These run once at set-up on the host with the same
// libm calls and expression order as the reference, so donor indices,
// interpolation fractions and group orders are identical to the reference
// plans (cubedsphere/cubedsphere_mesh.c:8-201, cubedsphere_halo.c:25-57,
// 401-451, cubedsphere_interface.c:95-209).
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "gamera_cs_types.h"
#include "gcs_device.cuh"

namespace gcs {
namespace topo {

int direction(int face, double a, double b, double out[3]);
int inverse(const double dir[3], int *face, double *a, double *b);
int edge_neighbor(int face, int edge, int *nface, int *nedge, int *reversed);
int vertex_key(int face, const size_t active[3], const size_t vertex[3],
               int64_t key[4]);

}  // namespace topo

// Ghost-target geometry the halo plans need, per face: cell centroids over
// the cell extents and, per face family, face centroids and area vectors
// over the face extents (reference index order, k contiguous).
struct HaloGeometry {
  const gamera_no_vec3 *cell_centroid[kFaces];
  const gamera_no_vec3 *face_centroid[kFaces][3];
  const gamera_no_vec3 *face_area_vector[kFaces][3];
};

int build_halo_cells(const HaloGeometry &geo, const Dims &D,
                     std::vector<HaloCell> &out);
int build_halo_faces(const HaloGeometry &geo, const Dims &D,
                     std::vector<HaloFace> &out);
int build_seams(const Dims &D, std::vector<Seam> &out);
int build_edge_groups(const Dims &D, std::vector<int> &offsets,
                      std::vector<EdgeMember> &members);

}  // namespace gcs
