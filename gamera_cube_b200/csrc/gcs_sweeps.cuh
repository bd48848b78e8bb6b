// Predictor, flux and EMF sweeps, CT and cell update, generic in the bulk
// type T of the sweeps.
//
// T = double is the plain FP64 path: every array of the Bulk<double> view
// is the FP64 array of DevState/DevGeom/DevBg and the arithmetic is the
// reference's (gcs_kernels.cu, built without FMA contraction).
// T = float is the FP32-bulk path (gcs_kernels_bulk.cu, built with FMA):
// the predictor still advances the FP64 state and also writes FP32 copies
// of the cell primitives, cell B, face normal fields and EMF weights; the
// flux, face-velocity and edge-EMF sweeps of the radial layers where the
// background field is weak compute in FP32 from FP32 metric and background,
// the layers near the inner boundary (strong dipole) in FP64; every sweep
// stores FP64 fluxes, face velocities and EMFs, which CT and the cell
// update accumulate into the FP64 face flux and conserved state.  Each
// sweep launch covers one radial range [i0, i1).
#pragma once

#ifndef GCS_F32_FLUX_BLOCKS
#define GCS_F32_FLUX_BLOCKS 8
#endif
#ifndef GCS_F32_EDGE_BLOCKS
#define GCS_F32_EDGE_BLOCKS 8
#endif


#include "gcs_kernel_util.cuh"
#include "gcs_kernels.cuh"
#include "gcs_physics.cuh"
#include "gcs_flux_tma.cuh"

namespace gcs {

#ifndef GCS_SWEEPS_TEMPLATES_ONLY
// The non-template kernels below are compiled in gcs_kernels.cu only.

// Predictor over every cell/face (nonorthogonal_step.c:379-419): Phi~, U~,
// B~ in FP64; primitives of U~ with the sweep options (rho NaN where the
// conversion fails), Phi~/area and the EMF weights V m / max(rho, floor)
// for the sweeps, in FP64 and (bulk) FP32.
__global__ void k_predict(Dims D, DevState S, DevGeom G, Bulk<float> B32, int bulk,
                          Opts O, const StepParams *prm, DevStatus *st) {
  if (failed(st)) return;
  int f, i, j, k;
  const Box b{0, 0, 0, D.N1, D.N2, D.E0 + 1};
  if (!box_coord(b, &f, &i, &j, &k)) return;
  const double r = prm->ratio;
  const long long c = f * D.Nn + D.node(i, j, k);
  // FP32 copies exist for the layers [B32.lo, N0) only
  const bool wb = bulk && i >= B32.lo;
  const long long cb = wb ? B32.at(f, D.node(i, j, k)) : 0;
  const bool cell = i < D.E0 && j < D.E1 && k < D.E2;
  const int coord[3] = {i, j, k};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    bool in = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) in = in && coord[a] < D.ext(a) + (a == d ? 1 : 0);
    if (in) {
      const double pp = S.P[d][c] + r * (S.P[d][c] - S.Po[d][c]);
      S.Pp[d][c] = pp;
      const double bn = pp / G.area[d][c];
      S.BN[d][c] = bn;
      if (wb) B32.BN[d][cb] = (float)bn;
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
  const double prv[5] = {pr.rho, pr.vx, pr.vy, pr.vz, pr.p};
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    S.Pr[m][c] = prv[m];
    if (wb) B32.Pr[m][cb] = (float)prv[m];
  }
  const double v = G.vol[c];
  const double rho = fmax(up[0], O.e_rho_floor);
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    const double w = v * up[1 + m] / rho;
    S.W[m][c] = w;
    if (wb) B32.W[m][cb] = (float)w;
  }
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
  for (int m = 0; m < 3; ++m) {
    S.Bp[m][c] = bp[m];
    if (wb) B32.Bp[m][cb] = (float)bp[m];
  }
}
#endif  // GCS_SWEEPS_TEMPLATES_ONLY

// Minimum resident blocks of 128 threads per SM the sweeps are compiled for
// (register caps 128 and 96 in FP64, 64 in FP32), from measured full-step
// sweeps at 6 x 96x96x192.
template <typename T>
struct SweepOccupancy {
  static constexpr int flux = 4;
  static constexpr int edge = 6;
};
template <>
struct SweepOccupancy<float> {
  static constexpr int flux = GCS_F32_FLUX_BLOCKS;
  static constexpr int edge = GCS_F32_EDGE_BLOCKS;
};

// ---------------------------------------------------------------------------
// Face-flux sweep in direction d (nonorthogonal_sweep.c:408-548).
// Each thread owns one face; the eight-cell stencil of one variable at a
// time is read from the predictor's cell primitives, so only the volumes,
// one stencil and the reconstructed face states are live at once.
template <int d, typename T>
__global__ void __launch_bounds__(128, SweepOccupancy<T>::flux) k_flux(Dims D, DevState S, Bulk<T> B,
                                                 Opts O, DevStatus *st, int i0,
                                                 int i1) {
  if (failed(st)) return;
  int f, i, j, k;
  const Box b{i0, D.g, D.g, D.n + (d == 1), D.n + (d == 2), i1};
  if (!box_coord(b, &f, &i, &j, &k)) return;
  const long long c = f * D.Nn + D.node(i, j, k);
  const long long cb = B.at(f, D.node(i, j, k));   // index of the Bulk arrays
  const long long sd = D.stride(d);
  const T iv = B.iv[d][cb];
  if (isnan(iv)) {
    fail(st, kStageReconstruct, d, f, i, j, k);
    return;
  }
  const T riv = T(1.0) / iv;
  const T pdm = (T)O.pdm;
  T vol[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) vol[n] = B.vol[cb + (n - 4) * sd];
  PrimT<T> st2[2];
  {
    T q[8], l, r;
    bool ok = true;
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      q[n] = B.Pr[0][cb + (n - 4) * sd];
      ok = ok && !isnan(q[n]);
    }
    if (!ok) {
      fail(st, kStageReconstruct, d, f, i, j, k);
      return;
    }
    up7_pdm_rcp(vol, q, riv, pdm, &l, &r);
    st2[0].rho = l; st2[1].rho = r;
#pragma unroll
    for (int n = 0; n < 8; ++n) q[n] = B.Pr[1][cb + (n - 4) * sd];
    up7_pdm_rcp(vol, q, riv, pdm, &l, &r);
    st2[0].vx = l; st2[1].vx = r;
#pragma unroll
    for (int n = 0; n < 8; ++n) q[n] = B.Pr[2][cb + (n - 4) * sd];
    up7_pdm_rcp(vol, q, riv, pdm, &l, &r);
    st2[0].vy = l; st2[1].vy = r;
#pragma unroll
    for (int n = 0; n < 8; ++n) q[n] = B.Pr[3][cb + (n - 4) * sd];
    up7_pdm_rcp(vol, q, riv, pdm, &l, &r);
    st2[0].vz = l; st2[1].vz = r;
#pragma unroll
    for (int n = 0; n < 8; ++n) q[n] = B.Pr[4][cb + (n - 4) * sd];
    up7_pdm_rcp(vol, q, riv, pdm, &l, &r);
    st2[0].p = l; st2[1].p = r;
  }
  T mag[2][3] = {{T(0.0), T(0.0), T(0.0)}, {T(0.0), T(0.0), T(0.0)}};
  if (O.s_mhd) {
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      T q[8];
#pragma unroll
      for (int n = 0; n < 8; ++n) q[n] = B.Bp[m][cb + (n - 4) * sd];
      up7_pdm_rcp(vol, q, riv, pdm, &mag[0][m], &mag[1][m]);
    }
  }
  FaceFrame<T> fr;
  fr.nx = B.fn[d][0][cb]; fr.ny = B.fn[d][1][cb]; fr.nz = B.fn[d][2][cb];
  fr.t1x = B.ft1[d][0][cb]; fr.t1y = B.ft1[d][1][cb]; fr.t1z = B.ft1[d][2][cb];
  fr.t2x = B.ft2[d][0][cb]; fr.t2y = B.ft2[d][1][cb]; fr.t2z = B.ft2[d][2][cb];
  FluidFlux<T> fl;
  if (kinetic_fluid_flux(st2, (T)O.s_gamma, fr, &fl)) {
    fail(st, kStageKineticFluid, d, f, i, j, k);
    return;
  }
  MaxwellFlux<T> mx;
  mx.m[0] = mx.m[1] = mx.m[2] = T(0.0);
  if (O.s_mhd) {
    const T bn = B.BN[d][cb];
    T b0[3] = {T(0.0), T(0.0), T(0.0)};
    T b0n = T(0.0);
    if (O.s_bg) {
      b0[0] = B.fb0[d][0][cb];
      b0[1] = B.fb0[d][1][cb];
      b0[2] = B.fb0[d][2][cb];
      b0n = B.fb0n[d][cb];
    }
    if (kinetic_maxwell_flux(st2, mag, bn, fr, O.s_bg, b0, b0n, O.s_boris, (T)O.s_c,
                             fl.vn, &mx)) {
      fail(st, kStageKineticMaxwell, d, f, i, j, k);
      return;
    }
    if (O.hogs)
      apply_hogs(&fl, &mx, (T)O.hogs_h, (T)O.hogs_m, O.s_boris, (T)O.s_c);
    if (O.hogs && O.s_boris) {
      bool applied;
      T speed;
      if (emergency_diffusion(&fl, st2, S.Up, c - sd, c, (T)O.s_c, &applied, &speed)) {
        fail(st, kStageEmergency, d, f, i, j, k);
        return;
      }
      if (applied) {
        atomicAdd(&st->emergency_count[f], 1ULL);
        atomicMax(&st->emergency_max_bits[f],
                  (unsigned long long)__double_as_longlong((double)speed));
      }
    }
  }
  const T area = B.area[d][cb];
#pragma unroll
  for (int m = 0; m < 5; ++m) B.F[d][m][c] = (double)(area * fl.f[m]);
#pragma unroll
  for (int m = 0; m < 3; ++m) B.M[d][m][c] = (double)(area * mx.m[m]);
}

#ifndef GCS_SWEEPS_TEMPLATES_ONLY
// Seam flux synchronisation (cubedsphere_interface.c:40-81): the fluid and
// Maxwell face fluxes of each seam face pair are set to their oriented mean.
__global__ void k_seam_flux(Dims D, const Seam *seams, DevState S, DevStatus *st) {
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

#endif  // GCS_SWEEPS_TEMPLATES_ONLY

// ---------------------------------------------------------------------------
// Face velocities of face family a (nonorthogonal_sweep.c:223-259):
// central8 of the per-cell weights over central8 of the volumes, for every
// face the edge velocities of edge family (a+2)%3 read.
template <int a, typename T>
__global__ void k_face_velocity(Dims D, Bulk<T> B, DevStatus *st, int i0,
                                int i1) {
  if (failed(st)) return;
  constexpr int e = (a + 2) % 3, bb = (a + 1) % 3;
  int f, x[3];
  int lo[3], cnt[3];
  lo[e] = D.g; cnt[e] = D.act(e);
  lo[a] = D.g; cnt[a] = D.act(a) + 1;
  lo[bb] = 0; cnt[bb] = D.ext(bb);
  const Box b{i0, lo[1], lo[2], cnt[1], cnt[2], i1};
  if (!box_coord(b, &f, &x[0], &x[1], &x[2])) return;
  const long long c = f * D.Nn + D.node(x[0], x[1], x[2]);
  const long long cb = B.at(f, D.node(x[0], x[1], x[2]));
  const long long sa = D.stride(a);
  const T riv = T(1.0) / B.iv[a][cb];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    T w[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) w[n] = B.W[m][cb + (n - 4) * sa];
    B.FV[a][m][c] = (double)(central8(w) * riv);
  }
}

// ---------------------------------------------------------------------------
// Edge EMF sweep of edge family e (nonorthogonal_sweep.c:624-752).
template <int e, typename T>
__global__ void __launch_bounds__(128, SweepOccupancy<T>::edge) k_edge_emf(Dims D, DevState S, DevGeom G,
                                                  Bulk<T> B, Opts O,
                                                  const StepParams *prm,
                                                  DevStatus *st, int i0,
                                                  int i1) {
  if (failed(st)) return;
  constexpr int a = (e + 1) % 3, bb = (e + 2) % 3;
  int f, x[3];
  int cnt[3];
  cnt[e] = D.act(e);
  cnt[a] = D.act(a) + 1;
  cnt[bb] = D.act(bb) + 1;
  const Box b{i0, D.g, D.g, cnt[1], cnt[2], i1};
  if (!box_coord(b, &f, &x[0], &x[1], &x[2])) return;
  const long long c = f * D.Nn + D.node(x[0], x[1], x[2]);
  const long long cb = B.at(f, D.node(x[0], x[1], x[2]));
  const unsigned char ok = G.edge_ok[e][c];
  if (ok != 0) {
    fail(st, ok, e, f, x[0], x[1], x[2]);
    return;
  }
  const long long sa = D.stride(a), sb = D.stride(bb);
  const T pdm = (T)O.e_pdm;
  // edge velocity: faces of family a along bb
  T ar[8], fld[8];
  T v[3];
#pragma unroll
  for (int n = 0; n < 8; ++n) ar[n] = B.area[a][cb + (n - 4) * sb];
  const T rca = T(1.0) / B.ca[e][cb];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    T w[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) w[n] = ar[n] * (T)B.FV[a][m][c + (n - 4) * sb];
    v[m] = central8(w) * rca;
  }
  const T vt1 = dot3(v[0], v[1], v[2], B.et1[e][0][cb], B.et1[e][1][cb], B.et1[e][2][cb]);
  const T vt2 = dot3(v[0], v[1], v[2], B.et2[e][0][cb], B.et2[e][1][cb], B.et2[e][2][cb]);
  // transverse face fields (nonorthogonal_sweep.c:372-406)
  T fl, fr, sl, sr;
#pragma unroll
  for (int n = 0; n < 8; ++n) fld[n] = B.BN[a][cb + (n - 4) * sb];
  up7_pdm_rcp(ar, fld, rca, pdm, &fl, &fr);
  T ar2[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    ar2[n] = B.area[bb][cb + (n - 4) * sa];
    fld[n] = B.BN[bb][cb + (n - 4) * sa];
  }
  up7_pdm_rcp(ar2, fld, T(1.0) / B.cb[e][cb], pdm, &sl, &sr);
  // 2x2 edge solve (nonorthogonal_operators.c:56-79)
  const T f1 = T(0.5) * (fl + fr);
  const T f2 = T(0.5) * (sl + sr);
  const T inv = B.einv[e][cb];
  const T n10 = B.en1[e][0][cb], n11 = B.en1[e][1][cb];
  const T n20 = B.en2[e][0][cb], n21 = B.en2[e][1][cb];
  T ef0 = inv * (n21 * f1 - n11 * f2);
  T ef1 = inv * (-n20 * f1 + n10 * f2);
  if (O.e_bg) {
    ef0 += B.eb0t1[e][cb];
    ef1 += B.eb0t2[e][cb];
  }
  const T jump = (sr - sl) - (fr - fl);
  // edge density (nonorthogonal_sweep.c:351-370), from the FP64 state
  double rho = 0.0;
  rho += 0.25 * S.Up[0][c];
  rho += 0.25 * S.Up[0][c - sb];
  rho += 0.25 * S.Up[0][c - sa];
  rho += 0.25 * S.Up[0][c - sa - sb];
  if (!(isfinite(rho) && rho > DBL_MIN)) {
    fail(st, kStageEdgeDensity, e, f, x[0], x[1], x[2]);
    return;
  }
  T emf;
  if (edge_emf(vt1, vt2, ef0, ef1, jump, (T)rho, B.elen[e][cb], (T)O.e_diff, O.e_boris,
               (T)O.e_c, (T)O.e_cfl, (T)prm->dt, &emf)) {
    fail(st, kStageEdgeEmf, e, f, x[0], x[1], x[2]);
    return;
  }
  B.E[e][c] = (double)emf;
}

#ifndef GCS_SWEEPS_TEMPLATES_ONLY
// Signed mean over each group of coincident seam/corner edges
// (cubedsphere_interface.c:217-242); members in the reference's sorted
// order.
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
__global__ void k_ct(Dims D, DevState S, Opts O, const StepParams *prm, DevStatus *st) {
  if (failed(st)) return;
  int f, i, j, k;
  const Box b{0, 0, 0, D.E1 + (d == 1), D.E2 + (d == 2), D.E0 + (d == 0)};
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
  double *const *E = S.E;
  double curl;
  if (d == 0)
    curl = E[2][c + s1] - E[2][c] - E[1][c + 1] + E[1][c];
  else if (d == 1)
    curl = E[0][c + 1] - E[0][c] - E[2][c + s0] + E[2][c];
  else
    curl = E[1][c + s0] - E[1][c] - E[0][c + s1] + E[0][c];
  S.P[d][c] = old - prm->dt * curl;
}

// Cell update (nonorthogonal_step.c:527-610 with the stress rates of
// nonorthogonal_sweep.c:550-622): save U, B as old on every cell, then on
// active cells U += dt * rate, recover B from the CT-updated Phi, and apply
// the Boris (nonorthogonal_state.c:161-280) or Maxwell momentum update.
__global__ void __launch_bounds__(128, 6) k_update(Dims D, DevState S, DevGeom G,
                                                DevBg BG, Opts O,
                                                const StepParams *prm,
                                                DevStatus *st) {
  if (failed(st)) return;
  int f, i, j, k;
  const Box b{0, 0, 0, D.E1, D.E2, D.E0};
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

#endif  // GCS_SWEEPS_TEMPLATES_ONLY

// ---------------------------------------------------------------------------
// Launchers of the sweeps of one precision over the radial range [i0, i1)
// of the range each sweep covers (clamped to it; empty ranges launch
// nothing).

inline bool clamp_range(int lo, int hi, int i0, int i1, int *a, int *n) {
  *a = lo > i0 ? lo : i0;
  const int b = hi < i1 ? hi : i1;
  *n = b - *a;
  return *n > 0;
}

template <typename T>
struct Sweeps {
  static void flux(const Ctx &X, const Bulk<T> &B, const Opts &O, int i0, int i1,
                   cudaStream_t s) {
    const Dims &D = X.D;
    int a, n;
    if (X.flux_staged) {
      if (clamp_range(D.g, D.g + D.nr + 1, i0, i1, &a, &n))
        launch_flux_tma<0, T>(X, B, O, a, a + n, s);
      if (clamp_range(D.g, D.g + D.nr, i0, i1, &a, &n))
        launch_flux_tma<1, T>(X, B, O, a, a + n, s);
      if (clamp_range(D.g, D.g + D.nr, i0, i1, &a, &n))
        launch_flux_tma<2, T>(X, B, O, a, a + n, s);
      return;
    }
    const Tile t = X.tile[kTileFlux];
    if (clamp_range(D.g, D.g + D.nr + 1, i0, i1, &a, &n))
      k_flux<0, T><<<tile_grid(n, D.n, D.n, t), tile_block(t), 0, s>>>(
          D, X.S, B, O, X.status, a, a + n);
    if (clamp_range(D.g, D.g + D.nr, i0, i1, &a, &n))
      k_flux<1, T><<<tile_grid(n, D.n + 1, D.n, t), tile_block(t), 0, s>>>(
          D, X.S, B, O, X.status, a, a + n);
    if (clamp_range(D.g, D.g + D.nr, i0, i1, &a, &n))
      k_flux<2, T><<<tile_grid(n, D.n, D.n + 1, t), tile_block(t), 0, s>>>(
          D, X.S, B, O, X.status, a, a + n);
  }
  static void emf(const Ctx &X, const Bulk<T> &B, const Opts &O, int i0, int i1,
                  cudaStream_t s) {
    const Dims &D = X.D;
    int a, n;
    // face velocities: family a, edge family e=(a+2)%3 active, a faces, bb all
    const Tile t = X.tile[kTileFaceVelocity];
    if (clamp_range(D.g, D.g + D.nr + 1, i0, i1, &a, &n))  // e=2, a=0, bb=1
      k_face_velocity<0, T><<<tile_grid(n, D.E1, D.n, t), tile_block(t), 0, s>>>(
          D, B, X.status, a, a + n);
    if (clamp_range(D.g, D.g + D.nr, i0, i1, &a, &n))  // e=0, a=1, bb=2
      k_face_velocity<1, T><<<tile_grid(n, D.n + 1, D.E2, t), tile_block(t), 0, s>>>(
          D, B, X.status, a, a + n);
    if (clamp_range(0, D.E0, i0, i1, &a, &n))  // e=1, a=2, bb=0 (all i)
      k_face_velocity<2, T><<<tile_grid(n, D.n, D.n + 1, t), tile_block(t), 0, s>>>(
          D, B, X.status, a, a + n);
  }
  static void edge(const Ctx &X, const Bulk<T> &B, const Opts &O, int i0, int i1,
                   cudaStream_t s) {
    const Dims &D = X.D;
    int a, n;
    const Tile t = X.tile[kTileEdgeEmf];
    if (clamp_range(D.g, D.g + D.nr, i0, i1, &a, &n))
      k_edge_emf<0, T><<<tile_grid(n, D.n + 1, D.n + 1, t), tile_block(t), 0, s>>>(
          D, X.S, X.G, B, O, X.params, X.status, a, a + n);
    if (clamp_range(D.g, D.g + D.nr + 1, i0, i1, &a, &n))
      k_edge_emf<1, T><<<tile_grid(n, D.n, D.n + 1, t), tile_block(t), 0, s>>>(
          D, X.S, X.G, B, O, X.params, X.status, a, a + n);
    if (clamp_range(D.g, D.g + D.nr + 1, i0, i1, &a, &n))
      k_edge_emf<2, T><<<tile_grid(n, D.n + 1, D.n, t), tile_block(t), 0, s>>>(
          D, X.S, X.G, B, O, X.params, X.status, a, a + n);
  }
};

}  // namespace gcs
