// Device data layout of the six-face cubed-sphere state.
//
// All six faces of the cube stay resident in HBM.  Every staggered array
// (cells, the three face families, the three edge families) of a face uses
// the same padded node index
//     node(i, j, k) = (i * N1 + j) * N2 + k,   N_a = cell_extent[a] + 1
// (N2 rounded up to a multiple of 4 so rows start on 16-byte boundaries),
// so a cell, its three lower faces and its three lower edges share one
// linear index and neighbours are +-1, +-N2, +-N1*N2 away.  Arrays are
// structure-of-arrays (one double per node per component) and the six faces
// are concatenated: element = face * nodes_per_face + node.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define GCS_HD __host__ __device__
#else
#define GCS_HD
#endif

namespace gcs {

constexpr int kFaces = 6;

struct Dims {
  int nr, n, g;          // active radial cells, active angular cells, ghosts
  int E0, E1, E2;        // cell extents (active + 2 ghosts)
  int N1, N2;            // node strides
  long long Nn;          // nodes per face (N0 * N1 * N2)
  GCS_HD long long node(int i, int j, int k) const {
    return ((long long)i * N1 + j) * N2 + k;
  }
  GCS_HD int ext(int axis) const {
    return axis == 0 ? E0 : (axis == 1 ? E1 : E2);
  }
  GCS_HD int act(int axis) const { return axis == 0 ? nr : n; }
  GCS_HD long long stride(int axis) const {
    return axis == 0 ? (long long)N1 * N2 : (axis == 1 ? (long long)N2 : 1LL);
  }
};

struct DevState {
  double *U[5], *Uo[5];          // conserved, old conserved (cells)
  double *B[3], *Bo[3];          // residual cell B, old (cells)
  double *P[3], *Po[3];          // face magnetic flux per face family
  double *Up[5], *Bp[3], *Pp[3]; // predictor outputs
  double *Pr[5];                 // primitives of Up (sweep options); rho NaN
                                 // where the conversion fails
  double *BN[3];                 // Pp / face area per face family
  double *W[3];                  // (V * m_c) / max(rho, floor) per cell
  double *FV[3][3];              // face velocity per face family, 3 comps
  double *F[3][5];               // area-scaled fluid flux per face family
  double *M[3][3];               // area-scaled Maxwell flux per face family
  double *E[3];                  // line-integrated edge EMF per edge family
};

struct DevGeom {
  double *vol, *ivol, *cflmin;   // volume, 1/volume, min cfl length
  unsigned char *cell_ok;        // recovery matrix valid
  double *rec[18];               // calibrated face-flux -> cell-B, 3 x 6
  double *area[3];               // face area per family
  double *fn[3][3], *ft1[3][3], *ft2[3][3];  // face frame
  double *iv[3];                 // central8(volume) along the face normal
  double *elen[3];               // edge length
  double *et1[3][3], *et2[3][3]; // edge tangents
  double *en1[3][2], *en2[3][2]; // transverse face normals at the edge
  double *einv[3];               // 1 / det of the 2x2 edge system
  double *ca[3], *cb[3];         // central8 face areas for edge stencils
  unsigned char *edge_ok[3];     // edge geometry and 2x2 system valid
};

struct DevBg {
  double *b0[3], *force[3];      // cell B0, pure-B0 stress divergence
  double *fb0[3][3];             // face-averaged B0 per face family
  double *fb0n[3];               // B0 face flux / area per face family
  double *eb0t1[3], *eb0t2[3];   // edge B0 . t1, B0 . t2 per edge family
};

// The arrays the predictor writes for the sweeps and the metric and
// background the sweeps read, in the sweeps' compute type T, plus the sweep
// outputs, which are FP64 in both paths.  Bulk<double> views the FP64
// arrays of DevState/DevGeom/DevBg; Bulk<float> views separate FP32 copies
// (FP32-bulk path) and the same FP64 outputs.
//
// The FP32 arrays cover only the radial layers [lo, N0) of each face (the
// layers the FP32 sweeps read), six faces of face_nodes = (N0 - lo) N1 N2
// nodes each: a node of face f sits at at(f, node) = f face_nodes + node -
// lo N1 N2.  The FP64 view has lo = 0, face_nodes = Nn, so at() is the
// node index of the full arrays.  The sweep outputs (FV, F, M, E) are the
// full FP64 arrays in both views and keep the full index.
template <typename T>
struct Bulk {
  int lo;                    // first radial layer of the arrays of this view
  long long face_nodes;      // nodes per face of this view's arrays
  long long shift;           // lo * N1 * N2
  GCS_HD long long at(int f, long long node) const {
    return (long long)f * face_nodes + node - shift;
  }
  T *Pr[5], *Bp[3], *BN[3], *W[3];
  double *FV[3][3], *F[3][5], *M[3][3], *E[3];
  const T *vol, *iv[3], *area[3];
  const T *fn[3][3], *ft1[3][3], *ft2[3][3];
  const T *elen[3], *et1[3][3], *et2[3][3], *en1[3][2], *en2[3][2], *einv[3];
  const T *ca[3], *cb[3];
  const T *fb0[3][3], *fb0n[3], *eb0t1[3], *eb0t2[3];
};

// Upstream solar-wind state of a wind case in code units: density (proton
// cm^-3, before the seeded +-1% noise), Vx (100 km/s), pressure, IMF Bz and
// the density-pulse flag.
struct WindInit {
  double rho, vx, pres, bz;
  int pulse;
};

// Writable view of the Earth boundary-layer geometry (layouts of
// gcs_earth.h), filled by the device case builder.
struct EarthLayers {
  double *cell_cen[3];
  double *face_cen[3][3], *face_av[3][3], *face_bg[3];
  double *edge_mid[3][3], *edge_nrm[3][3], *edge_len[3];
  unsigned char *edge_valid[3];
  double *inner_a[2][3], *inner_b[2][3];
};

// Scalar parameters of one step.  dt and ratio live in device memory so a
// captured CUDA graph can advance its own time step.
struct StepParams {
  double dt;            // this step
  double ratio;         // predictor ratio 0.5 dt / dt_prev
  double dt_prev;       // previous step
  double cfl_min;       // min CFL step of the state after the last step
  int step;             // number of completed steps
  int pad;
  double time;          // simulation time of the state (driver mode)
};

// Physics options of one call, one group per reference option struct:
// stress sweeps (nonorthogonal_sweep.h:13-25), edge EMF (:40-49), update
// (nonorthogonal_step.h:57-65) and CFL time step (:67-76).
struct Opts {
  double s_gamma, s_rho_floor, s_p_floor, pdm, hogs_h, hogs_m, s_c;
  bool s_mhd, hogs, s_boris, s_bg;
  double e_rho_floor, e_pdm, e_diff, e_c, e_cfl;
  bool e_boris, e_bg;
  double u_gamma, u_rho_floor, u_p_floor, u_c;
  bool u_mhd, u_boris, u_bg;
  double t_gamma, t_rho_floor, t_p_floor, t_cfl, t_c;
  bool t_mhd, t_boris, t_bg;
  double dt_fraction;            // driver mode dt fraction
};

// First failure of a step: stage code, face, direction, node indices.
enum Stage : int {
  kStageNone = 0,
  kStagePredict = 1,
  kStageRecoverPredict = 2,
  kStageReconstruct = 3,
  kStageKineticFluid = 4,
  kStageKineticMaxwell = 5,
  kStageEmergency = 6,
  kStageEdgeGeometry = 7,
  kStageEdgeVelocity = 8,
  kStageTransverse = 9,
  kStageEdgeDensity = 10,
  kStageEdgeEmf = 11,
  kStageUpdate = 12,
  kStageRecoverUpdate = 13,
  kStageRecoverFinal = 14,
  kStageTimestep = 15,
  kStageHost = 16,
  kStageSolveEdge = 17,
  kStageOptions = 18,
  kStagePressureControl = 19,
  kStageTileCopy = 20,   // a staged sweep's tile copy did not arrive in time
  kStageMiCoupling = 21, // an ionosphere coupling update inside the step failed
};

struct DevStatus {
  unsigned long long first;      // packed first failure (0 = none)
  unsigned int stage_mask;       // bit per failed stage
  unsigned int pad;
  unsigned long long emergency_count[kFaces];
  unsigned long long emergency_max_bits[kFaces];  // max speed as bits
  unsigned long long cfl_min_bits;                // min CFL step as bits
};

GCS_HD inline unsigned long long pack_failure(int stage, int dir,
                                                          int face, int i,
                                                          int j, int k) {
  return ((unsigned long long)(stage & 0xff) << 56) |
         ((unsigned long long)(dir & 0xf) << 52) |
         ((unsigned long long)(face & 0xf) << 48) |
         ((unsigned long long)(i & 0xffff) << 32) |
         ((unsigned long long)(j & 0xffff) << 16) |
         (unsigned long long)(k & 0xffff);
}

// Halo plan entries (built on the host from the reference geometry).
// Only the two nonzero weights per axis of the reference's 8x8 bilinear
// stencil are kept (cubedsphere_halo.c:32-57): taps (p0,q0) (p0,q0+1)
// (p0+1,q0) (p0+1,q0+1) in the reference's p-major/q-minor order, with
// weights (1-fx, fx) x (1-fy, fy).
struct HaloCell {
  double fx, fy;
  unsigned int target;    // receiver node
  unsigned int donor;     // donor node of tap (p0, q0)
  unsigned int nearest;   // donor node of the positivity fallback
  unsigned int meta;      // recv | donor << 4 | first layer << 8 | last << 9
};

struct HaloFace {
  double fx, fy;
  double ax, ay, az;      // receiver area vector
  unsigned int target;    // receiver node
  unsigned int donor;     // donor node of tap (p0, q0)
  unsigned int meta;      // recv | dir << 4 | donor << 8
  unsigned int pad;
};

struct Seam {
  int face, nface, src_axis, dst_axis, src_b, dst_b, reversed;
  double orient;
};

struct EdgeMember {
  unsigned int node;
  unsigned char face, dir;
  signed char sign;
  unsigned char pad;
};

}  // namespace gcs
