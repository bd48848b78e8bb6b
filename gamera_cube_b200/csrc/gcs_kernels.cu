// Step kernels of the six-face cubed-sphere MHD hot path (plain FP64).
//
// One launch covers all six cube faces.  The stage order is the reference
// six-face step (cubedsphere/cubedsphere_step.c:48-152):
//   seam Phi sync -> cell halo (+radial outflow) -> face halo -> predictor
//   -> face-flux sweeps -> seam flux sync -> face velocities -> edge EMF
//   -> edge EMF group sync -> CT -> cell update (Reynolds + Boris/Maxwell)
//   -> seam Phi sync -> B recovery (+ CFL reduction in driver mode).
// Each kernel returns early once an earlier stage has recorded a failure,
// so stages after a failing one leave the state untouched, as in the
// reference which returns -1 from the first failing stage.
#include "gcs_kernels.cuh"
#include "gcs_physics.cuh"

#include <cfloat>

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

// Box iteration: grid.x over j*k of the box, grid.y over i, grid.z face.
struct Box {
  int i0, j0, k0, nj, nk;
};

__device__ inline bool box_coord(const Box &b, int *f, int *i, int *j,
                                 int *k) {
  const int jk = blockIdx.x * blockDim.x + threadIdx.x;
  if (jk >= b.nj * b.nk) return false;
  *f = blockIdx.z;
  *i = b.i0 + blockIdx.y;
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

// ---------------------------------------------------------------------------
// Seam synchronisation (cubedsphere_interface.c:7-81).  One thread per seam
// face; each seam face belongs to exactly one (face, edge) pair.
__global__ void k_seam_sync(Dims D, const Seam *seams, DevState S, int magnetic,
                            DevStatus *st) {
  if (failed(st)) return;
  const long long per = (long long)D.nr * D.n;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= 12 * per) return;
  const Seam sm = seams[t / per];
  const int rem = (int)(t % per);
  const int i = D.g + rem / D.n;
  const int along = rem % D.n;
  const int dalong = sm.reversed ? D.n - 1 - along : along;
  int src[3] = {i, D.g + along, D.g + along};
  int tgt[3] = {i, D.g + dalong, D.g + dalong};
  src[sm.src_axis] = sm.src_b;
  tgt[sm.dst_axis] = sm.dst_b;
  const long long s = sm.face * D.Nn + D.node(src[0], src[1], src[2]);
  const long long d = sm.nface * D.Nn + D.node(tgt[0], tgt[1], tgt[2]);
  const double o = sm.orient;
  if (magnetic) {
    double *a = S.P[sm.src_axis], *b = S.P[sm.dst_axis];
    double common = 0.5 * (a[s] + o * b[d]);
    a[s] = common;
    b[d] = o * common;
    a = S.Po[sm.src_axis];
    b = S.Po[sm.dst_axis];
    common = 0.5 * (a[s] + o * b[d]);
    a[s] = common;
    b[d] = o * common;
  } else {
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      double *a = S.F[sm.src_axis][m], *b = S.F[sm.dst_axis][m];
      const double common = 0.5 * (a[s] + o * b[d]);
      a[s] = common;
      b[d] = o * common;
    }
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      double *a = S.M[sm.src_axis][m], *b = S.M[sm.dst_axis][m];
      const double common = 0.5 * (a[s] + o * b[d]);
      a[s] = common;
      b[d] = o * common;
    }
  }
}

// ---------------------------------------------------------------------------
// Tangential cell halo (cubedsphere_halo.c:582-632) fused with the radial
// outflow copy (cubedsphere_halo.c:217-245) of the same (j,k) column: a
// target on the first/last active radial layer also writes the radial
// ghost cells that copy it.
__global__ void k_halo_cells(Dims D, const HaloCell *plan, long long count,
                             int radial, DevState S, DevStatus *st) {
  if (failed(st)) return;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= count) return;
  const HaloCell e = plan[t];
  const int recv = e.meta & 15, donor = (e.meta >> 4) & 15;
  const long long base = donor * D.Nn + e.donor;
  const long long tap[4] = {base, base + 1, base + D.N2, base + D.N2 + 1};
  const double wx0 = 1.0 - e.fx, wx1 = e.fx, wy0 = 1.0 - e.fy, wy1 = e.fy;
  const double w[4] = {wx0 * wy0, wx0 * wy1, wx1 * wy0, wx1 * wy1};
  double cur[5], old[5], cb[3], ob[3];
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    double a = 0.0, b = 0.0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      a += w[q] * S.U[m][tap[q]];
      b += w[q] * S.Uo[m][tap[q]];
    }
    cur[m] = a;
    old[m] = b;
  }
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    double a = 0.0, b = 0.0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      a += w[q] * S.B[m][tap[q]];
      b += w[q] * S.Bo[m][tap[q]];
    }
    cb[m] = a;
    ob[m] = b;
  }
  if (!halo_valid(cur) || !halo_valid(old)) {
    const long long nb = donor * D.Nn + e.nearest;
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      cur[m] = S.U[m][nb];
      old[m] = S.Uo[m][nb];
    }
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      cb[m] = S.B[m][nb];
      ob[m] = S.Bo[m][nb];
    }
  }
  const long long layer = (long long)D.N1 * D.N2;
  const long long tgt = recv * D.Nn + e.target;
  // radial ghost layers that copy this target: [0, g) copies the first
  // active layer, [g + nr, E0) the last one.
  const int below = (radial && (e.meta & 256)) ? D.g : 0;
  const int above = (radial && (e.meta & 512)) ? D.E0 - (D.g + D.nr) : 0;
  for (int r = -below; r <= above; ++r) {
    const long long x = tgt + (long long)r * layer;
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      S.U[m][x] = cur[m];
      S.Uo[m][x] = old[m];
    }
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      S.B[m][x] = cb[m];
      S.Bo[m][x] = ob[m];
    }
  }
}

// Radial outflow ghosts of the active (j,k) columns (cubedsphere_halo.c:
// 217-245); the tangential columns are written by k_halo_cells.
__global__ void k_radial_outflow(Dims D, DevState S, DevStatus *st) {
  if (failed(st)) return;
  const int jk = blockIdx.x * blockDim.x + threadIdx.x;
  if (jk >= D.n * D.n) return;
  const int f = blockIdx.z;
  const int gi = blockIdx.y;  // 0 .. 2g-1
  const int i = gi < D.g ? gi : D.g + D.nr + (gi - D.g);
  const int j = D.g + jk / D.n, k = D.g + jk % D.n;
  const int di = gi < D.g ? D.g : D.g + D.nr - 1;
  const long long x = f * D.Nn + D.node(i, j, k);
  const long long s = f * D.Nn + D.node(di, j, k);
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    S.U[m][x] = S.U[m][s];
    S.Uo[m][x] = S.Uo[m][s];
  }
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    S.B[m][x] = S.B[m][s];
    S.Bo[m][x] = S.Bo[m][s];
  }
}

// Magnetic ghost faces (cubedsphere_halo.c:651-686): interpolated donor B,
// both time levels, projected on the receiver face's area vector.
__global__ void k_halo_faces(Dims D, const HaloFace *plan, long long count,
                             DevState S, DevStatus *st) {
  if (failed(st)) return;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= count) return;
  const HaloFace e = plan[t];
  const int recv = e.meta & 15, dir = (e.meta >> 4) & 15,
            donor = (e.meta >> 8) & 15;
  const long long base = donor * D.Nn + e.donor;
  const long long tap[4] = {base, base + 1, base + D.N2, base + D.N2 + 1};
  const double wx0 = 1.0 - e.fx, wx1 = e.fx, wy0 = 1.0 - e.fy, wy1 = e.fy;
  const double w[4] = {wx0 * wy0, wx0 * wy1, wx1 * wy0, wx1 * wy1};
  double cb[3], ob[3];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    double a = 0.0, b = 0.0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      a += w[q] * S.B[m][tap[q]];
      b += w[q] * S.Bo[m][tap[q]];
    }
    cb[m] = a;
    ob[m] = b;
  }
  double cf = 0.0, of = 0.0;
  cf += cb[0] * e.ax;
  of += ob[0] * e.ax;
  cf += cb[1] * e.ay;
  of += ob[1] * e.ay;
  cf += cb[2] * e.az;
  of += ob[2] * e.az;
  const long long x = recv * D.Nn + e.target;
  S.P[dir][x] = cf;
  S.Po[dir][x] = of;
}

// ---------------------------------------------------------------------------
// Predictor over every cell and face incl. ghosts
// (nonorthogonal_step.c:379-419): U~ = prim^-1(P + r (P - P_old)),
// Phi~ = Phi + r (Phi - Phi_old), B~ = recover(Phi~); plus the per-cell
// momentum weights (V m)/max(rho, floor) of the EMF face velocities
// (nonorthogonal_sweep.c:223-249), which depend on U~ only.  Also stores,
// once per cell and face, two quantities every sweep stencil reads many
// times: the primitive state of U~ under the sweep options
// (nonorthogonal_sweep.c:144-149, rho = NaN marks a failed conversion) and
// the face-normal field Phi~ / area (nonorthogonal_sweep.c:466-467, 391).
__global__ void k_predict(Dims D, DevState S, DevGeom G, Opts O,
                          const StepParams *prm, DevStatus *st) {
  if (failed(st)) return;
  int f, i, j, k;
  const Box b{0, 0, 0, D.N1, D.N2};
  if (!box_coord(b, &f, &i, &j, &k)) return;
  const double r = prm->ratio;
  const long long c = f * D.Nn + D.node(i, j, k);
  const bool cell = i < D.E0 && j < D.E1 && k < D.E2;
  const int coord[3] = {i, j, k};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    bool in = true;
#pragma unroll
    for (int a = 0; a < 3; ++a)
      in = in && coord[a] < D.ext(a) + (a == d ? 1 : 0);
    if (in) {
      const double pp = S.P[d][c] + r * (S.P[d][c] - S.Po[d][c]);
      S.Pp[d][c] = pp;
      S.BN[d][c] = pp / G.area[d][c];
    }
  }
  if (!cell) return;
  double uo[5], uc[5], up[5];
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    uo[m] = S.Uo[m][c];
    uc[m] = S.U[m][c];
  }
  if (predict_cell(uo, uc, r, O.u_gamma, O.u_rho_floor, O.u_p_floor, up)) {
    fail(st, kStagePredict, 0, f, i, j, k);
    return;
  }
#pragma unroll
  for (int m = 0; m < 5; ++m) S.Up[m][c] = up[m];
  Prim pr;
  if (cons_to_prim(up, O.s_gamma, O.s_rho_floor, O.s_p_floor, &pr)) pr.rho = NAN;
  S.Pr[0][c] = pr.rho;
  S.Pr[1][c] = pr.vx;
  S.Pr[2][c] = pr.vy;
  S.Pr[3][c] = pr.vz;
  S.Pr[4][c] = pr.p;
  const double v = G.vol[c];
  const double rho = fmax(up[0], O.e_rho_floor);
#pragma unroll
  for (int m = 0; m < 3; ++m) S.W[m][c] = v * up[1 + m] / rho;
  double phi[6];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const long long u = c + D.stride(d);
    phi[2 * d] = S.P[d][c] + r * (S.P[d][c] - S.Po[d][c]);
    phi[2 * d + 1] = S.P[d][u] + r * (S.P[d][u] - S.Po[d][u]);
  }
  double bp[3];
  if (!recover_cell(G, c, phi, bp)) {
    fail(st, kStageRecoverPredict, 0, f, i, j, k);
    return;
  }
#pragma unroll
  for (int m = 0; m < 3; ++m) S.Bp[m][c] = bp[m];
}

// ---------------------------------------------------------------------------
// Face-flux sweep in direction d (nonorthogonal_sweep.c:408-548).
// Each thread owns one face; the eight-cell stencil of one variable at a
// time is read from the predictor's cell primitives, so only the volumes,
// one stencil and the reconstructed face states are live at once.
template <int d>
__global__ void __launch_bounds__(128, 4) k_flux(Dims D, DevState S, DevGeom G,
                                                 DevBg BG, Opts O,
                                                 DevStatus *st) {
  if (failed(st)) return;
  int f, i, j, k;
  const Box b{D.g, D.g, D.g, D.n + (d == 1), D.n + (d == 2)};
  if (!box_coord(b, &f, &i, &j, &k)) return;
  const long long c = f * D.Nn + D.node(i, j, k);
  const long long sd = D.stride(d);
  const double iv = G.iv[d][c];
  if (isnan(iv)) {
    fail(st, kStageReconstruct, d, f, i, j, k);
    return;
  }
  const double riv = 1.0 / iv;
  double vol[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) vol[n] = G.vol[c + (n - 4) * sd];
  Prim st2[2];
  {
    double q[8], l, r;
    bool ok = true;
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      q[n] = S.Pr[0][c + (n - 4) * sd];
      ok = ok && !isnan(q[n]);
    }
    if (!ok) {
      fail(st, kStageReconstruct, d, f, i, j, k);
      return;
    }
    up7_pdm_rcp(vol, q, riv, O.pdm, &l, &r);
    st2[0].rho = l; st2[1].rho = r;
#pragma unroll
    for (int n = 0; n < 8; ++n) q[n] = S.Pr[1][c + (n - 4) * sd];
    up7_pdm_rcp(vol, q, riv, O.pdm, &l, &r);
    st2[0].vx = l; st2[1].vx = r;
#pragma unroll
    for (int n = 0; n < 8; ++n) q[n] = S.Pr[2][c + (n - 4) * sd];
    up7_pdm_rcp(vol, q, riv, O.pdm, &l, &r);
    st2[0].vy = l; st2[1].vy = r;
#pragma unroll
    for (int n = 0; n < 8; ++n) q[n] = S.Pr[3][c + (n - 4) * sd];
    up7_pdm_rcp(vol, q, riv, O.pdm, &l, &r);
    st2[0].vz = l; st2[1].vz = r;
#pragma unroll
    for (int n = 0; n < 8; ++n) q[n] = S.Pr[4][c + (n - 4) * sd];
    up7_pdm_rcp(vol, q, riv, O.pdm, &l, &r);
    st2[0].p = l; st2[1].p = r;
  }
  double mag[2][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
  if (O.s_mhd) {
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      double q[8];
#pragma unroll
      for (int n = 0; n < 8; ++n) q[n] = S.Bp[m][c + (n - 4) * sd];
      up7_pdm_rcp(vol, q, riv, O.pdm, &mag[0][m], &mag[1][m]);
    }
  }
  FaceFrame fr;
  fr.nx = G.fn[d][0][c]; fr.ny = G.fn[d][1][c]; fr.nz = G.fn[d][2][c];
  fr.t1x = G.ft1[d][0][c]; fr.t1y = G.ft1[d][1][c]; fr.t1z = G.ft1[d][2][c];
  fr.t2x = G.ft2[d][0][c]; fr.t2y = G.ft2[d][1][c]; fr.t2z = G.ft2[d][2][c];
  FluidFlux fl;
  if (kinetic_fluid_flux(st2, O.s_gamma, fr, &fl)) {
    fail(st, kStageKineticFluid, d, f, i, j, k);
    return;
  }
  MaxwellFlux mx;
  mx.m[0] = mx.m[1] = mx.m[2] = 0.0;
  if (O.s_mhd) {
    const double bn = S.BN[d][c];
    double b0[3] = {0.0, 0.0, 0.0};
    double b0n = 0.0;
    if (O.s_bg) {
      b0[0] = BG.fb0[d][0][c];
      b0[1] = BG.fb0[d][1][c];
      b0[2] = BG.fb0[d][2][c];
      b0n = BG.fb0n[d][c];
    }
    if (kinetic_maxwell_flux(st2, mag, bn, fr, O.s_bg, b0, b0n, O.s_boris, O.s_c,
                             fl.vn, &mx)) {
      fail(st, kStageKineticMaxwell, d, f, i, j, k);
      return;
    }
    if (O.hogs) apply_hogs(&fl, &mx, O.hogs_h, O.hogs_m, O.s_boris, O.s_c);
    if (O.hogs && O.s_boris) {
      double lo[5], hi[5];
#pragma unroll
      for (int m = 0; m < 5; ++m) {
        lo[m] = S.Up[m][c - sd];
        hi[m] = S.Up[m][c];
      }
      bool applied;
      double speed;
      if (emergency_diffusion(&fl, st2, lo, hi, O.s_c, &applied, &speed)) {
        fail(st, kStageEmergency, d, f, i, j, k);
        return;
      }
      if (applied) {
        atomicAdd(&st->emergency_count[f], 1ULL);
        atomicMax(&st->emergency_max_bits[f],
                  (unsigned long long)__double_as_longlong(speed));
      }
    }
  }
  const double area = G.area[d][c];
#pragma unroll
  for (int m = 0; m < 5; ++m) S.F[d][m][c] = area * fl.f[m];
#pragma unroll
  for (int m = 0; m < 3; ++m) S.M[d][m][c] = area * mx.m[m];
}

// ---------------------------------------------------------------------------
// Face velocities of face family a (nonorthogonal_sweep.c:223-259):
// central8 of the per-cell weights over central8 of the volumes, for every
// face the edge velocities of edge family (a+2)%3 read.
template <int a>
__global__ void k_face_velocity(Dims D, DevState S, DevGeom G, DevStatus *st) {
  if (failed(st)) return;
  constexpr int e = (a + 2) % 3, bb = (a + 1) % 3;
  int f, x[3];
  int lo[3], cnt[3];
  lo[e] = D.g; cnt[e] = D.act(e);
  lo[a] = D.g; cnt[a] = D.act(a) + 1;
  lo[bb] = 0; cnt[bb] = D.ext(bb);
  const Box b{lo[0], lo[1], lo[2], cnt[1], cnt[2]};
  if (!box_coord(b, &f, &x[0], &x[1], &x[2])) return;
  const long long c = f * D.Nn + D.node(x[0], x[1], x[2]);
  const long long sa = D.stride(a);
  const double riv = 1.0 / G.iv[a][c];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    double w[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) w[n] = S.W[m][c + (n - 4) * sa];
    S.FV[a][m][c] = central8(w) * riv;
  }
}

// ---------------------------------------------------------------------------
// Edge EMF sweep of edge family e (nonorthogonal_sweep.c:624-752).
template <int e>
__global__ void __launch_bounds__(128) k_edge_emf(Dims D, DevState S,
                                                  DevGeom G, DevBg BG, Opts O,
                                                  const StepParams *prm,
                                                  DevStatus *st) {
  if (failed(st)) return;
  constexpr int a = (e + 1) % 3, bb = (e + 2) % 3;
  int f, x[3];
  int cnt[3];
  cnt[e] = D.act(e);
  cnt[a] = D.act(a) + 1;
  cnt[bb] = D.act(bb) + 1;
  const Box b{D.g, D.g, D.g, cnt[1], cnt[2]};
  if (!box_coord(b, &f, &x[0], &x[1], &x[2])) return;
  const long long c = f * D.Nn + D.node(x[0], x[1], x[2]);
  const unsigned char ok = G.edge_ok[e][c];
  if (ok != 0) {
    fail(st, ok, e, f, x[0], x[1], x[2]);
    return;
  }
  const long long sa = D.stride(a), sb = D.stride(bb);
  // edge velocity: faces of family a along bb
  double ar[8], fld[8];
  double v[3];
#pragma unroll
  for (int n = 0; n < 8; ++n) ar[n] = G.area[a][c + (n - 4) * sb];
  const double rca = 1.0 / G.ca[e][c];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    double w[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) w[n] = ar[n] * S.FV[a][m][c + (n - 4) * sb];
    v[m] = central8(w) * rca;
  }
  const double vt1 =
      dot3(v[0], v[1], v[2], G.et1[e][0][c], G.et1[e][1][c], G.et1[e][2][c]);
  const double vt2 =
      dot3(v[0], v[1], v[2], G.et2[e][0][c], G.et2[e][1][c], G.et2[e][2][c]);
  // transverse face fields (nonorthogonal_sweep.c:372-406)
  double fl, fr, sl, sr;
#pragma unroll
  for (int n = 0; n < 8; ++n) fld[n] = S.BN[a][c + (n - 4) * sb];
  up7_pdm_rcp(ar, fld, rca, O.e_pdm, &fl, &fr);
  double ar2[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    ar2[n] = G.area[bb][c + (n - 4) * sa];
    fld[n] = S.BN[bb][c + (n - 4) * sa];
  }
  up7_pdm_rcp(ar2, fld, 1.0 / G.cb[e][c], O.e_pdm, &sl, &sr);
  // 2x2 edge solve (nonorthogonal_operators.c:56-79)
  const double f1 = 0.5 * (fl + fr);
  const double f2 = 0.5 * (sl + sr);
  const double inv = G.einv[e][c];
  const double n10 = G.en1[e][0][c], n11 = G.en1[e][1][c];
  const double n20 = G.en2[e][0][c], n21 = G.en2[e][1][c];
  double ef0 = inv * (n21 * f1 - n11 * f2);
  double ef1 = inv * (-n20 * f1 + n10 * f2);
  if (O.e_bg) {
    ef0 += BG.eb0t1[e][c];
    ef1 += BG.eb0t2[e][c];
  }
  const double jump = (sr - sl) - (fr - fl);
  // edge density (nonorthogonal_sweep.c:351-370)
  double rho = 0.0;
  rho += 0.25 * S.Up[0][c];
  rho += 0.25 * S.Up[0][c - sb];
  rho += 0.25 * S.Up[0][c - sa];
  rho += 0.25 * S.Up[0][c - sa - sb];
  if (!(isfinite(rho) && rho > DBL_MIN)) {
    fail(st, kStageEdgeDensity, e, f, x[0], x[1], x[2]);
    return;
  }
  double emf;
  if (edge_emf(vt1, vt2, ef0, ef1, jump, rho, G.elen[e][c], O.e_diff,
               O.e_boris, O.e_c, O.e_cfl, prm->dt, &emf)) {
    fail(st, kStageEdgeEmf, e, f, x[0], x[1], x[2]);
    return;
  }
  S.E[e][c] = emf;
}

// Signed mean over each group of coincident seam/corner edges
// (cubedsphere_interface.c:217-242); members in the reference's sorted order.
__global__ void k_edge_sync(Dims D, const int *offsets, const EdgeMember *mem,
                            int groups, DevState S, DevStatus *st) {
  if (failed(st)) return;
  const int gi = blockIdx.x * blockDim.x + threadIdx.x;
  if (gi >= groups) return;
  const int b = offsets[gi], e = offsets[gi + 1];
  double common = 0.0;
  for (int t = b; t < e; ++t) {
    const EdgeMember m = mem[t];
    common += (double)m.sign * S.E[m.dir][m.face * D.Nn + m.node];
  }
  common /= (double)(e - b);
  for (int t = b; t < e; ++t) {
    const EdgeMember m = mem[t];
    S.E[m.dir][m.face * D.Nn + m.node] = (double)m.sign * common;
  }
}

// ---------------------------------------------------------------------------
// Save Phi -> Phi_old on every face, then the CT curl on active faces
// (nonorthogonal_step.c:233-298, 361-377).
template <int d>
__global__ void k_ct(Dims D, DevState S, Opts O, const StepParams *prm,
                     DevStatus *st) {
  if (failed(st)) return;
  int f, i, j, k;
  const Box b{0, 0, 0, D.E1 + (d == 1), D.E2 + (d == 2)};
  if (!box_coord(b, &f, &i, &j, &k)) return;
  const long long c = f * D.Nn + D.node(i, j, k);
  const double old = S.P[d][c];
  S.Po[d][c] = old;
  if (!O.u_mhd) return;
  const int x[3] = {i, j, k};
#pragma unroll
  for (int a = 0; a < 3; ++a)
    if (x[a] < D.g || x[a] >= D.g + D.act(a) + (a == d)) return;
  const long long s0 = D.stride(0), s1 = D.stride(1);
  double curl;
  if (d == 0)
    curl = S.E[2][c + s1] - S.E[2][c] - S.E[1][c + 1] + S.E[1][c];
  else if (d == 1)
    curl = S.E[0][c + 1] - S.E[0][c] - S.E[2][c + s0] + S.E[2][c];
  else
    curl = S.E[1][c + s0] - S.E[1][c] - S.E[0][c + s1] + S.E[0][c];
  S.P[d][c] = old - prm->dt * curl;
}

// Cell update (nonorthogonal_step.c:527-610 with the stress rates of
// nonorthogonal_sweep.c:550-622): save U, B as old on every cell, then on
// active cells U += dt * rate, recover B from the CT-updated Phi, and apply
// the Boris (nonorthogonal_state.c:161-280) or Maxwell momentum update.
__global__ void __launch_bounds__(128) k_update(Dims D, DevState S, DevGeom G,
                                                DevBg BG, Opts O,
                                                const StepParams *prm,
                                                DevStatus *st) {
  if (failed(st)) return;
  int f, i, j, k;
  const Box b{0, 0, 0, D.E1, D.E2};
  if (!box_coord(b, &f, &i, &j, &k)) return;
  const long long c = f * D.Nn + D.node(i, j, k);
  double u[5], bo[3];
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    u[m] = S.U[m][c];
    S.Uo[m][c] = u[m];
  }
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    bo[m] = S.B[m][c];
    S.Bo[m][c] = bo[m];
  }
  if (i < D.g || i >= D.g + D.nr || j < D.g || j >= D.g + D.n || k < D.g ||
      k >= D.g + D.n)
    return;
  const double dt = prm->dt;
  const double iv = G.ivol[c];
  double rate[5], mrate[3];
  const long long sdir[3] = {D.stride(0), D.stride(1), 1};
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    double diff = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) diff += S.F[d][m][c] - S.F[d][m][c + sdir[d]];
    rate[m] = diff * iv;
  }
  const double uold[5] = {u[0], u[1], u[2], u[3], u[4]};
#pragma unroll
  for (int m = 0; m < 5; ++m) u[m] += dt * rate[m];
  if (O.u_mhd) {
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      double diff = 0.0;
#pragma unroll
      for (int d = 0; d < 3; ++d)
        diff += S.M[d][m][c] - S.M[d][m][c + sdir[d]];
      mrate[m] = diff * iv;
      if (O.u_bg) mrate[m] += BG.force[m][c];
    }
    double phi[6], bn[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      phi[2 * d] = S.P[d][c];
      phi[2 * d + 1] = S.P[d][c + sdir[d]];
    }
    if (!recover_cell(G, c, phi, bn)) {
      fail(st, kStageRecoverUpdate, 0, f, i, j, k);
      return;
    }
    if (O.u_boris) {
      double nb[3] = {bn[0], bn[1], bn[2]};
      double ob[3] = {bo[0], bo[1], bo[2]};
      if (O.u_bg) {
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          const double b0 = BG.b0[m][c];
          nb[m] = bn[m] + b0;
          ob[m] = bo[m] + b0;
        }
      }
      if (apply_boris(u, uold, nb, ob, rate, mrate, O.u_c, dt, O.u_gamma,
                      O.u_rho_floor, O.u_p_floor)) {
        fail(st, kStageUpdate, 0, f, i, j, k);
        return;
      }
    } else {
      apply_maxwell(u, mrate, dt, O.u_gamma, O.u_rho_floor, O.u_p_floor);
    }
  }
#pragma unroll
  for (int m = 0; m < 5; ++m) S.U[m][c] = u[m];
}

// Final B recovery on every cell (cubedsphere_step.c:142-152), optionally
// fused with the CFL time-step reduction of the next step
// (nonorthogonal_step.c:449-525) over active cells.  mode bit 0: recover
// and store B; bit 1: CFL reduction (with the stored B when bit 0 is clear).
__global__ void __launch_bounds__(256) k_recover(Dims D, DevState S, DevGeom G,
                                                 DevBg BG, Opts O, int mode,
                                                 DevStatus *st) {
  // No early return: every thread reaches the block reduction below.
  const bool skip = failed(st);
  const int with_cfl = mode & 2;
  int f, i, j, k;
  const Box b{0, 0, 0, D.E1, D.E2};
  double cand = DBL_MAX;
  if (!skip && box_coord(b, &f, &i, &j, &k)) {
    const long long c = f * D.Nn + D.node(i, j, k);
    double bn[3];
    bool ok = true;
    if (mode & 1) {
      double phi[6];
      const long long sdir[3] = {D.stride(0), D.stride(1), 1};
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        phi[2 * d] = S.P[d][c];
        phi[2 * d + 1] = S.P[d][c + sdir[d]];
      }
      ok = recover_cell(G, c, phi, bn);
      if (!ok) {
        fail(st, kStageRecoverFinal, 0, f, i, j, k);
      } else {
#pragma unroll
        for (int m = 0; m < 3; ++m) S.B[m][c] = bn[m];
      }
    } else {
#pragma unroll
      for (int m = 0; m < 3; ++m) bn[m] = S.B[m][c];
    }
    if (ok) {
      if (with_cfl && i >= D.g && i < D.g + D.nr && j >= D.g &&
          j < D.g + D.n && k >= D.g && k < D.g + D.n) {
        double u[5];
#pragma unroll
        for (int m = 0; m < 5; ++m) u[m] = S.U[m][c];
        Prim p;
        if (cons_to_prim(u, O.t_gamma, O.t_rho_floor, O.t_p_floor, &p)) {
          fail(st, kStageTimestep, 0, f, i, j, k);
        } else {
          const double cs = sqrt(O.t_gamma * p.p / p.rho);
          double va = 0.0;
          if (O.t_mhd) {
            double bx = bn[0], by = bn[1], bz = bn[2];
            if (O.t_bg) {
              bx = bn[0] + BG.b0[0][c];
              by = bn[1] + BG.b0[1][c];
              bz = bn[2] + BG.b0[2][c];
            }
            double s2 = 0.0;
            s2 += bx * bx;
            s2 += by * by;
            s2 += bz * bz;
            va = sqrt(s2) / sqrt(p.rho);
            if (O.t_boris) va = O.t_c * va / hypot(O.t_c, va);
          }
          double v2 = 0.0;
          v2 += p.vx * p.vx;
          v2 += p.vy * p.vy;
          v2 += p.vz * p.vz;
          const double speed = sqrt(v2) + hypot(cs, va);
          const double cand0 = O.t_cfl * G.cflmin[c] / speed;
          if (!isfinite(cand0) || cand0 <= 0.0)
            fail(st, kStageTimestep, 0, f, i, j, k);
          else
            cand = cand0;
        }
      }
    }
  }
  if (!with_cfl) return;
  // block min (positive doubles order as unsigned 64-bit integers)
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    cand = fmin(cand, __shfl_down_sync(0xffffffffu, cand, o));
  __shared__ double wmin[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) wmin[warp] = cand;
  __syncthreads();
  if (warp == 0) {
    cand = lane < (int)(blockDim.x >> 5) ? wmin[lane] : DBL_MAX;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      cand = fmin(cand, __shfl_down_sync(0xffffffffu, cand, o));
    if (lane == 0 && cand < DBL_MAX)
      atomicMin(&st->cfl_min_bits,
                (unsigned long long)__double_as_longlong(cand));
  }
}

// Driver-mode time step (test_cubedsphere_dipole_background.c:593-670):
// dt = min(fraction * cfl_min, 1.25 dt_prev), ratio = 0.5 dt / dt_prev
// (0 on the first step).  Resets the reduction for the next step.
__global__ void k_next_dt(StepParams *prm, DevStatus *st, double fraction) {
  const double local = __longlong_as_double((long long)st->cfl_min_bits);
  prm->cfl_min = local;
  const double prev = prm->dt;
  double dt = fraction * local;
  if (prm->step > 0) dt = fmin(dt, 1.25 * prev);
  prm->ratio = prm->step > 0 ? 0.5 * dt / prev : 0.0;
  prm->dt_prev = prev;
  prm->dt = dt;
  st->cfl_min_bits = (unsigned long long)__double_as_longlong(DBL_MAX);
}

__global__ void k_count_step(StepParams *prm) { prm->step += 1; }

// ---------------------------------------------------------------------------
// Host-side launchers.

static inline dim3 box_grid(int I, int J, int K, int bs) {
  return dim3((unsigned)((J * K + bs - 1) / bs), (unsigned)I, kFaces);
}

void launch_seam_sync(const Ctx &X, int magnetic, cudaStream_t s) {
  const long long total = 12LL * X.D.nr * X.D.n;
  k_seam_sync<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(
      X.D, X.seams, X.S, magnetic, X.status);
}

void launch_halo_cells_only(const Ctx &X, cudaStream_t s) {
  if (X.n_halo_cells)
    k_halo_cells<<<(unsigned)((X.n_halo_cells + 127) / 128), 128, 0, s>>>(
        X.D, X.halo_cells, X.n_halo_cells, 0, X.S, X.status);
}

void launch_halo_faces_only(const Ctx &X, cudaStream_t s) {
  if (X.n_halo_faces)
    k_halo_faces<<<(unsigned)((X.n_halo_faces + 127) / 128), 128, 0, s>>>(
        X.D, X.halo_faces, X.n_halo_faces, X.S, X.status);
}

void launch_halo(const Ctx &X, cudaStream_t s) {
  if (X.n_halo_cells)
    k_halo_cells<<<(unsigned)((X.n_halo_cells + 127) / 128), 128, 0, s>>>(
        X.D, X.halo_cells, X.n_halo_cells, 1, X.S, X.status);
  k_radial_outflow<<<dim3((X.D.n * X.D.n + 127) / 128, 2 * X.D.g, kFaces),
                     128, 0, s>>>(X.D, X.S, X.status);
  if (X.n_halo_faces)
    k_halo_faces<<<(unsigned)((X.n_halo_faces + 127) / 128), 128, 0, s>>>(
        X.D, X.halo_faces, X.n_halo_faces, X.S, X.status);
}

void launch_predict(const Ctx &X, const Opts &O, cudaStream_t s) {
  k_predict<<<box_grid(X.D.E0 + 1, X.D.N1, X.D.N2, 128), 128, 0, s>>>(
      X.D, X.S, X.G, O, X.params, X.status);
}

void launch_flux(const Ctx &X, const Opts &O, cudaStream_t s) {
  const Dims &D = X.D;
  k_flux<0><<<box_grid(D.nr + 1, D.n, D.n, 128), 128, 0, s>>>(
      D, X.S, X.G, X.BG, O, X.status);
  k_flux<1><<<box_grid(D.nr, D.n + 1, D.n, 128), 128, 0, s>>>(
      D, X.S, X.G, X.BG, O, X.status);
  k_flux<2><<<box_grid(D.nr, D.n, D.n + 1, 128), 128, 0, s>>>(
      D, X.S, X.G, X.BG, O, X.status);
}

void launch_emf(const Ctx &X, const Opts &O, cudaStream_t s) {
  const Dims &D = X.D;
  // face velocities: family a, edge family e=(a+2)%3 active, a faces, bb all
  k_face_velocity<0><<<box_grid(D.nr + 1, D.E1, D.n, 128), 128, 0, s>>>(
      D, X.S, X.G, X.status);  // e=2 (k active), a=0, bb=1 (j all)
  k_face_velocity<1><<<box_grid(D.nr, D.n + 1, D.E2, 128), 128, 0, s>>>(
      D, X.S, X.G, X.status);  // e=0 (i active), a=1, bb=2 (k all)
  k_face_velocity<2><<<box_grid(D.E0, D.n, D.n + 1, 128), 128, 0, s>>>(
      D, X.S, X.G, X.status);  // e=1 (j active), a=2, bb=0 (i all)
  k_edge_emf<0><<<box_grid(D.nr, D.n + 1, D.n + 1, 128), 128, 0, s>>>(
      D, X.S, X.G, X.BG, O, X.params, X.status);
  k_edge_emf<1><<<box_grid(D.nr + 1, D.n, D.n + 1, 128), 128, 0, s>>>(
      D, X.S, X.G, X.BG, O, X.params, X.status);
  k_edge_emf<2><<<box_grid(D.nr + 1, D.n + 1, D.n, 128), 128, 0, s>>>(
      D, X.S, X.G, X.BG, O, X.params, X.status);
}

void launch_edge_sync(const Ctx &X, cudaStream_t s) {
  if (X.n_edge_groups)
    k_edge_sync<<<(X.n_edge_groups + 127) / 128, 128, 0, s>>>(
        X.D, X.edge_offsets, X.edge_members, X.n_edge_groups, X.S, X.status);
}

void launch_update(const Ctx &X, const Opts &O, cudaStream_t s) {
  const Dims &D = X.D;
  k_ct<0><<<box_grid(D.E0 + 1, D.E1, D.E2, 128), 128, 0, s>>>(
      D, X.S, O, X.params, X.status);
  k_ct<1><<<box_grid(D.E0, D.E1 + 1, D.E2, 128), 128, 0, s>>>(
      D, X.S, O, X.params, X.status);
  k_ct<2><<<box_grid(D.E0, D.E1, D.E2 + 1, 128), 128, 0, s>>>(
      D, X.S, O, X.params, X.status);
  k_update<<<box_grid(D.E0, D.E1, D.E2, 128), 128, 0, s>>>(
      D, X.S, X.G, X.BG, O, X.params, X.status);
}

void launch_recover(const Ctx &X, const Opts &O, int with_cfl,
                    cudaStream_t s) {
  const Dims &D = X.D;
  k_recover<<<box_grid(D.E0, D.E1, D.E2, 256), 256, 0, s>>>(
      D, X.S, X.G, X.BG, O, 1 | (with_cfl ? 2 : 0), X.status);
}

void launch_timestep(const Ctx &X, const Opts &O, cudaStream_t s) {
  const Dims &D = X.D;
  k_recover<<<box_grid(D.E0, D.E1, D.E2, 256), 256, 0, s>>>(
      D, X.S, X.G, X.BG, O, 2, X.status);
}

void launch_next_dt(const Ctx &X, double fraction, cudaStream_t s) {
  k_next_dt<<<1, 1, 0, s>>>(X.params, X.status, fraction);
}

void launch_count_step(const Ctx &X, cudaStream_t s) {
  k_count_step<<<1, 1, 0, s>>>(X.params);
}

// Whole step in reference order.
void launch_step(const Ctx &X, const Opts &O, int driver_mode,
                 cudaStream_t s) {
  launch_seam_sync(X, 1, s);
  launch_halo(X, s);
  launch_predict(X, O, s);
  launch_flux(X, O, s);
  launch_seam_sync(X, 0, s);
  if (O.u_mhd) {
    launch_emf(X, O, s);
    launch_edge_sync(X, s);
  }
  launch_update(X, O, s);
  if (O.u_mhd) launch_seam_sync(X, 1, s);
  if (O.u_mhd) launch_recover(X, O, driver_mode, s);
  if (driver_mode) {
    launch_count_step(X, s);
    launch_next_dt(X, O.dt_fraction, s);
  }
}

}  // namespace gcs
