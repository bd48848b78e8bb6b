// Device helpers shared by the step kernels: failure recording, box
// iteration and the calibrated B recovery.
#pragma once

#include <cfloat>

#include "gcs_device.cuh"

namespace gcs {

namespace {

__device__ inline void fail(DevStatus *st, int stage, int dir, int face,
                            int i, int j, int k) {
  atomicCAS(&st->first, 0ULL, pack_failure(stage, dir, face, i, j, k));
  atomicOr(&st->stage_mask, 1u << stage);
}

__device__ inline bool failed(const DevStatus *st) {
  return *(volatile const unsigned long long *)&st->first != 0ULL;
}

// Box iteration over radial layers [i0, i1): a thread block is a tile of
// blockDim.x consecutive points of the flattened (j, k) plane times
// blockDim.y consecutive layers; grid.x over j*k, grid.y over the layer
// groups, grid.z face.
struct Box {
  int i0, j0, k0, nj, nk, i1;
};

__device__ inline bool box_coord(const Box &b, int *f, int *i, int *j,
                                 int *k) {
  const int jk = blockIdx.x * blockDim.x + threadIdx.x;
  const int ii = b.i0 + blockIdx.y * blockDim.y + threadIdx.y;
  if (jk >= b.nj * b.nk || ii >= b.i1) return false;
  *f = blockIdx.z;
  *i = ii;
  *j = b.j0 + jk / b.nk;
  *k = b.k0 + jk % b.nk;
  return true;
}

// Calibrated recovery, cubedsphere/cubedsphere_recovery.c:69-98, applied as
// the precomputed 3x6 map (response inverse times the moment formula of
// nonorthogonal_operators.c:17-54).  Face order: i-lo, i-hi, j-lo, j-hi,
// k-lo, k-hi.
__device__ inline bool recover_cell(const DevGeom &G, long long c,
                                    const double phi[6], double b[3]) {
  if (!G.cell_ok[c]) return false;
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    double s = 0.0;
#pragma unroll
    for (int col = 0; col < 6; ++col) s += G.rec[r * 6 + col][c] * phi[col];
    b[r] = s;
  }
  return isfinite(b[0]) && isfinite(b[1]) && isfinite(b[2]);
}

// cubedsphere_halo.c:103-115
__device__ inline bool halo_valid(const double s[5]) {
  const double rho = s[0];
  if (!isfinite(rho) || rho <= 0.0) return false;
  double m2 = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (!isfinite(s[1 + d])) return false;
    m2 += s[1 + d] * s[1 + d];
  }
  return isfinite(s[4]) && s[4] > 0.5 * m2 / rho;
}

}  // namespace

}  // namespace gcs
