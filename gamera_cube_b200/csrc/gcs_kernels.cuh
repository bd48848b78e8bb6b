// Device context of one six-face cubed-sphere run and the stage launchers.
#pragma once

#include <cuda_runtime.h>

#include "gcs_device.cuh"

namespace gcs {

// Launch tile of a kernel family: blockDim.x consecutive points of the
// flattened (j, k) plane of a radial layer times blockDim.y layers.  The
// kernels compute per point, so the tile changes speed only, never results.
enum TileFamily {
  kTilePredict = 0, kTileFlux, kTileFaceVelocity, kTileEdgeEmf, kTileCt,
  kTileUpdate, kTileRecover, kTileFamilies
};
struct Tile {
  int bx, by;
};
// Largest tile (bx * by) each family's kernels are compiled for.
constexpr int kTileMaxThreads[kTileFamilies] = {256, 128, 256, 128, 256, 128, 256};

struct Ctx {
  Dims D;
  // defaults: the fastest full-step tiles measured at 6 x 96x96x192 (FP64
  // and FP32-bulk agree on these)
  Tile tile[kTileFamilies] = {{128, 1}, {64, 1}, {128, 1}, {64, 1},
                              {128, 1}, {128, 1}, {128, 1}};
  DevState S;
  DevGeom G;
  DevBg BG;
  Seam *seams = nullptr;
  HaloCell *halo_cells = nullptr;
  long long n_halo_cells = 0;
  HaloFace *halo_faces = nullptr;
  long long n_halo_faces = 0;
  int *edge_offsets = nullptr;
  EdgeMember *edge_members = nullptr;
  int n_edge_groups = 0;
  StepParams *params = nullptr;   // device
  DevStatus *status = nullptr;    // device
  int flux_staged = 0;            // 1: TMA-staged flux sweeps (gcs_flux_tma.cuh)
  int bulk = 0;                   // 1: FP32-bulk sweeps (B32)
  int bulk_split = 0;             // radial layers [0, bulk_split) stay FP64
  Bulk<float> B32{};
};

// Grid of a tile over radial layers [0, I) and a J x K plane, six faces.
inline dim3 tile_grid(int I, int J, int K, Tile t) {
  return dim3((unsigned)((J * K + t.bx - 1) / t.bx), (unsigned)((I + t.by - 1) / t.by),
              kFaces);
}
inline dim3 tile_block(Tile t) { return dim3((unsigned)t.bx, (unsigned)t.by, 1); }

// Bulk<double> view of the FP64 arrays.
Bulk<double> bulk64(const Ctx &X);

// FP64 sweeps over the radial range [i0, i1) (gcs_kernels_fp64.cu).
void launch_flux_f64(const Ctx &X, const Opts &O, int i0, int i1, cudaStream_t s);
void launch_face_velocity_f64(const Ctx &X, const Opts &O, int i0, int i1,
                              cudaStream_t s);
void launch_edge_emf_f64(const Ctx &X, const Opts &O, int i0, int i1, cudaStream_t s);

// Kernel attributes and persistent grid sizes of the TMA-staged flux sweeps
// (called at context set-up, before any stream capture).
int prepare_flux_f64();
int prepare_flux_f32();

// FP32-bulk sweeps over the radial range [i0, i1) (gcs_kernels_bulk.cu).
void launch_flux_f32(const Ctx &X, const Opts &O, int i0, int i1, cudaStream_t s);
void launch_face_velocity_f32(const Ctx &X, const Opts &O, int i0, int i1,
                              cudaStream_t s);
void launch_edge_emf_f32(const Ctx &X, const Opts &O, int i0, int i1, cudaStream_t s);

void launch_seam_sync(const Ctx &X, int magnetic, cudaStream_t s);
void launch_halo(const Ctx &X, cudaStream_t s);
void launch_halo_cells_only(const Ctx &X, cudaStream_t s);
void launch_halo_faces_only(const Ctx &X, cudaStream_t s);
void launch_radial_outflow_all(const Ctx &X, cudaStream_t s);
void launch_predict(const Ctx &X, const Opts &O, cudaStream_t s);
void launch_flux(const Ctx &X, const Opts &O, cudaStream_t s);
void launch_emf(const Ctx &X, const Opts &O, cudaStream_t s);
// The two halves of launch_emf: face velocities, then edge EMFs.
void launch_face_velocities(const Ctx &X, const Opts &O, cudaStream_t s);
void launch_edge_emfs(const Ctx &X, const Opts &O, cudaStream_t s);
void launch_edge_sync(const Ctx &X, cudaStream_t s);
void launch_update(const Ctx &X, const Opts &O, cudaStream_t s);
void launch_recover(const Ctx &X, const Opts &O, int with_cfl,
                    cudaStream_t s);
void launch_next_dt(const Ctx &X, double fraction, cudaStream_t s);
void launch_count_step(const Ctx &X, cudaStream_t s);
void launch_step(const Ctx &X, const Opts &O, int driver_mode,
                 cudaStream_t s);
// CFL reduction alone (nonorthogonal_step.c:449-525) into status.
void launch_timestep(const Ctx &X, const Opts &O, cudaStream_t s);

}  // namespace gcs
