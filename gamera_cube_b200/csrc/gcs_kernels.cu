// Step kernels of the six-face cubed-sphere MHD hot path (plain FP64; the
// sweeps are templates in gcs_sweeps.cuh, also built in FP32-bulk).
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
#include "gcs_kernel_util.cuh"
#include "gcs_physics.cuh"
#include "gcs_sweeps.cuh"

#include <cfloat>

namespace gcs {


// ---------------------------------------------------------------------------
// Seam Phi synchronisation (cubedsphere_interface.c:7-38).  One thread per
// seam face; each seam face belongs to exactly one (face, edge) pair.  The
// seam flux synchronisation is k_seam_flux (gcs_sweeps.cuh).
__global__ void k_seam_sync(Dims D, const Seam *seams, DevState S, DevStatus *st) {
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
  double *a = S.P[sm.src_axis], *b = S.P[sm.dst_axis];
  double common = 0.5 * (a[s] + o * b[d]);
  a[s] = common;
  b[d] = o * common;
  a = S.Po[sm.src_axis];
  b = S.Po[sm.dst_axis];
  common = 0.5 * (a[s] + o * b[d]);
  a[s] = common;
  b[d] = o * common;
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

// Stand-alone radial outflow fill (cubedsphere_halo.c:217-245) over the full
// tangential extent, ghost columns included.
__global__ void k_radial_outflow_all(Dims D, DevState S) {
  const int jk = blockIdx.x * blockDim.x + threadIdx.x;
  if (jk >= D.E1 * D.E2) return;
  const int f = blockIdx.z;
  const int gi = blockIdx.y;  // 0 .. 2g-1
  const int i = gi < D.g ? gi : D.g + D.nr + (gi - D.g);
  const int j = jk / D.E2, k = jk % D.E2;
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
// Final B recovery on every cell (cubedsphere_step.c:142-152), optionally
// fused with the CFL time-step reduction of the next step
// (nonorthogonal_step.c:449-525) over active cells.  mode bit 0: recover
// and store B; bit 1: CFL reduction (with the stored B when bit 0 is clear).
__global__ void __launch_bounds__(256, 4) k_recover(Dims D, DevState S, DevGeom G,
                                                 DevBg BG, Opts O, int mode,
                                                 DevStatus *st) {
  // No early return: every thread reaches the block reduction below.
  const bool skip = failed(st);
  const int with_cfl = mode & 2;
  int f, i, j, k;
  const Box b{0, 0, 0, D.E1, D.E2, D.E0};
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
  const int lt = threadIdx.y * blockDim.x + threadIdx.x;
  const int lane = lt & 31, warp = lt >> 5;
  if (lane == 0) wmin[warp] = cand;
  __syncthreads();
  if (warp == 0) {
    cand = lane < (int)((blockDim.x * blockDim.y) >> 5) ? wmin[lane] : DBL_MAX;
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

__global__ void k_count_step(StepParams *prm) {
  prm->time += prm->dt;
  prm->step += 1;
}

// ---------------------------------------------------------------------------
// Host-side launchers.

Bulk<double> bulk64(const Ctx &X) {
  Bulk<double> B{};
  B.lo = 0;
  B.face_nodes = X.D.Nn;
  B.shift = 0;
  const DevState &S = X.S;
  const DevGeom &G = X.G;
  const DevBg &BG = X.BG;
  for (int m = 0; m < 5; ++m) B.Pr[m] = S.Pr[m];
  for (int d = 0; d < 3; ++d) {
    B.Bp[d] = S.Bp[d];
    B.BN[d] = S.BN[d];
    B.W[d] = S.W[d];
    B.E[d] = S.E[d];
    B.iv[d] = G.iv[d];
    B.area[d] = G.area[d];
    B.elen[d] = G.elen[d];
    B.einv[d] = G.einv[d];
    B.ca[d] = G.ca[d];
    B.cb[d] = G.cb[d];
    B.fb0n[d] = BG.fb0n[d];
    B.eb0t1[d] = BG.eb0t1[d];
    B.eb0t2[d] = BG.eb0t2[d];
    for (int m = 0; m < 3; ++m) {
      B.FV[d][m] = S.FV[d][m];
      B.M[d][m] = S.M[d][m];
      B.fn[d][m] = G.fn[d][m];
      B.ft1[d][m] = G.ft1[d][m];
      B.ft2[d][m] = G.ft2[d][m];
      B.et1[d][m] = G.et1[d][m];
      B.et2[d][m] = G.et2[d][m];
      B.fb0[d][m] = BG.fb0[d][m];
    }
    for (int m = 0; m < 5; ++m) B.F[d][m] = S.F[d][m];
    for (int m = 0; m < 2; ++m) {
      B.en1[d][m] = G.en1[d][m];
      B.en2[d][m] = G.en2[d][m];
    }
  }
  B.vol = G.vol;
  return B;
}

void launch_seam_sync(const Ctx &X, int magnetic, cudaStream_t s) {
  const long long total = 12LL * X.D.nr * X.D.n;
  if (magnetic)
    k_seam_sync<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(X.D, X.seams, X.S,
                                                                X.status);
  else
    k_seam_flux<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(X.D, X.seams, X.S,
                                                                X.status);
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

void launch_radial_outflow_all(const Ctx &X, cudaStream_t s) {
  k_radial_outflow_all<<<dim3((X.D.E1 * X.D.E2 + 127) / 128, 2 * X.D.g, kFaces), 128, 0,
                         s>>>(X.D, X.S);
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
  const Tile t = X.tile[kTilePredict];
  k_predict<<<tile_grid(X.D.E0 + 1, X.D.N1, X.D.N2, t), tile_block(t), 0, s>>>(
      X.D, X.S, X.G, X.B32, X.bulk, O, X.params, X.status);
}

// Radial layers [0, split) run the FP64 sweeps, [split, E0 + 1) the FP32
// ones (FP32-bulk path); the plain path runs FP64 everywhere.
static int bulk_split(const Ctx &X) { return X.bulk ? X.bulk_split : X.D.E0 + 1; }

void launch_flux(const Ctx &X, const Opts &O, cudaStream_t s) {
  const int sp = bulk_split(X);
  launch_flux_f64(X, O, 0, sp, s);
  if (X.bulk) launch_flux_f32(X, O, sp, X.D.E0 + 1, s);
}

void launch_face_velocities(const Ctx &X, const Opts &O, cudaStream_t s) {
  const int sp = bulk_split(X);
  launch_face_velocity_f64(X, O, 0, sp, s);
  if (X.bulk) launch_face_velocity_f32(X, O, sp, X.D.E0 + 1, s);
}

void launch_edge_emfs(const Ctx &X, const Opts &O, cudaStream_t s) {
  const int sp = bulk_split(X);
  launch_edge_emf_f64(X, O, 0, sp, s);
  if (X.bulk) launch_edge_emf_f32(X, O, sp, X.D.E0 + 1, s);
}

void launch_emf(const Ctx &X, const Opts &O, cudaStream_t s) {
  // every face velocity before any edge EMF reads them
  launch_face_velocities(X, O, s);
  launch_edge_emfs(X, O, s);
}

void launch_edge_sync(const Ctx &X, cudaStream_t s) {
  if (X.n_edge_groups)
    k_edge_sync<<<(X.n_edge_groups + 127) / 128, 128, 0, s>>>(
        X.D, X.edge_offsets, X.edge_members, X.n_edge_groups, X.S, X.status);
}

void launch_update(const Ctx &X, const Opts &O, cudaStream_t s) {
  const Dims &D = X.D;
  const Tile t = X.tile[kTileCt], tu = X.tile[kTileUpdate];
  k_ct<0><<<tile_grid(D.E0 + 1, D.E1, D.E2, t), tile_block(t), 0, s>>>(
      D, X.S, O, X.params, X.status);
  k_ct<1><<<tile_grid(D.E0, D.E1 + 1, D.E2, t), tile_block(t), 0, s>>>(
      D, X.S, O, X.params, X.status);
  k_ct<2><<<tile_grid(D.E0, D.E1, D.E2 + 1, t), tile_block(t), 0, s>>>(
      D, X.S, O, X.params, X.status);
  k_update<<<tile_grid(D.E0, D.E1, D.E2, tu), tile_block(tu), 0, s>>>(
      D, X.S, X.G, X.BG, O, X.params, X.status);
}

void launch_recover(const Ctx &X, const Opts &O, int with_cfl,
                    cudaStream_t s) {
  const Dims &D = X.D;
  const Tile t = X.tile[kTileRecover];
  k_recover<<<tile_grid(D.E0, D.E1, D.E2, t), tile_block(t), 0, s>>>(
      D, X.S, X.G, X.BG, O, 1 | (with_cfl ? 2 : 0), X.status);
}

void launch_timestep(const Ctx &X, const Opts &O, cudaStream_t s) {
  const Dims &D = X.D;
  const Tile t = X.tile[kTileRecover];
  k_recover<<<tile_grid(D.E0, D.E1, D.E2, t), tile_block(t), 0, s>>>(
      D, X.S, X.G, X.BG, O, 2, X.status);
}

__global__ void k_set_failure(DevStatus *st, int stage, int dir) {
  fail(st, stage, dir, 0, 0, 0, 0);
}

void launch_set_failure(const Ctx &X, int stage, int dir, cudaStream_t s) {
  k_set_failure<<<1, 1, 0, s>>>(X.status, stage, dir);
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
