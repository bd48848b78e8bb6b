// FP64 instantiation of the flux, face-velocity and edge-EMF sweeps
// (gcs_sweeps.cuh), built with FMA contraction: the sweeps compute the
// reference's expressions with fused multiply-adds (one rounding fewer per
// pair), which stays well inside the plain path's 1e-12 per-step parity and
// shortens the FP64-bound flux sweep by about 5 %.  The halo fills, seam
// and edge syncs, predictor, CT, cell update and B recovery of
// gcs_kernels.cu stay without contraction (bitwise halo and recovery
// results).
#define GCS_SWEEPS_TEMPLATES_ONLY
#include "gcs_sweeps.cuh"

namespace gcs {

void launch_flux_f64(const Ctx &X, const Opts &O, int i0, int i1, cudaStream_t s) {
  Sweeps<double>::flux(X, bulk64(X), O, i0, i1, s);
}
void launch_face_velocity_f64(const Ctx &X, const Opts &O, int i0, int i1, cudaStream_t s) {
  Sweeps<double>::emf(X, bulk64(X), O, i0, i1, s);
}
void launch_edge_emf_f64(const Ctx &X, const Opts &O, int i0, int i1, cudaStream_t s) {
  Sweeps<double>::edge(X, bulk64(X), O, i0, i1, s);
}

int prepare_flux_f64() { return prepare_flux_tma<double>(); }

}  // namespace gcs
