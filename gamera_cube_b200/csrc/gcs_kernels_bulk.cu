// FP32-bulk instantiation of the flux, face-velocity and edge-EMF sweeps
// (gcs_sweeps.cuh), built with FMA contraction.  The predictor, seam and
// edge syncs, CT and cell update are the FP64 kernels of gcs_kernels.cu.
#define GCS_SWEEPS_TEMPLATES_ONLY
#include "gcs_sweeps.cuh"

namespace gcs {

void launch_flux_f32(const Ctx &X, const Opts &O, int i0, int i1, cudaStream_t s) {
  Sweeps<float>::flux(X, X.B32, O, i0, i1, s);
}
void launch_face_velocity_f32(const Ctx &X, const Opts &O, int i0, int i1,
                              cudaStream_t s) {
  Sweeps<float>::emf(X, X.B32, O, i0, i1, s);
}
void launch_edge_emf_f32(const Ctx &X, const Opts &O, int i0, int i1, cudaStream_t s) {
  Sweeps<float>::edge(X, X.B32, O, i0, i1, s);
}

int prepare_flux_f32() { return prepare_flux_tma<float>(); }

}  // namespace gcs
