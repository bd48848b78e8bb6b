// Face-flux sweep with the eight-cell Up7 stencil staged in shared memory by
// TMA (nonorthogonal_sweep.c:408-548, the arithmetic of k_flux).
//
// A thread block is persistent: it walks a list of tiles, each tile a
// FX x FY patch of faces of one direction d (FX consecutive faces along the
// contiguous k axis, FY along the sweep axis for d = 0, 1 or along j for
// d = 2).  For every tile one elected thread issues nine tiled bulk tensor
// copies (cp.async.bulk.tensor.3d) of the predicted primitives (5), the
// predicted cell B (3) and the cell volume: the tile's cells plus the four
// Up7 ghost cells on each side along the sweep axis (FY + 8 cells, or
// FX + 8 for d = 2).  The following tiles' copies are in flight while the
// current tile is computed from shared memory, so every cell value is
// read from HBM once per sweep instead of eight times, and no thread waits
// on a global load of the stencil.  (Three stages; see k_flux_tma.)  Per-face arrays (frame, area, interface
// volume, normal field, B0) are read directly (coalesced along k).
//
// The last tile along the sweep axis also computes the extra face FY (FX for
// d = 2) its staged cells cover, so the n + 1 faces of a row need no tile of
// their own.  The tensor maps are encoded on the host at every launch
// (encode_cell_map, gcs_setup.cu) from the arrays of the Bulk view, so a
// context that shares scratch arrays with another gets maps of the arrays it
// reads.  Waits on the stage barriers are bounded: on expiry a warp
// records a kStageTileCopy failure, waits (bounded again) for the other
// stages' copies and returns.
#pragma once

#include <cuda.h>

#include "gcs_kernel_util.cuh"
#include "gcs_kernels.cuh"
#include "gcs_physics.cuh"

namespace gcs {

template <int d, typename T>
struct FluxTile {
  static constexpr int FX = 32;                     // faces along k
  static constexpr int FY = 8;                      // faces along the other tile axis
  static constexpr int THREADS = FX * FY;
  static constexpr int BX = d == 2 ? FX + 8 : FX;   // staged box, cells
  static constexpr int BY = d == 2 ? FY : (d == 1 ? FY + 8 : 1);
  static constexpr int BZ = d == 0 ? FY + 8 : 1;
  static constexpr int CELLS = BX * BY * BZ;
  static constexpr int VARS = 9;                    // 5 primitives, 3 B, volume
  static constexpr unsigned VAR_BYTES = (unsigned)(CELLS * sizeof(T));
  static constexpr unsigned STAGE_BYTES = VARS * VAR_BYTES;
  static constexpr int STAGES = 3;
  // resident blocks per SM the kernel is compiled for: 2 (128 registers) in
  // FP64, 4 (64 registers) in FP32
  static constexpr int MIN_BLOCKS = sizeof(T) == 8 ? 2 : 4;
  // the stage buffers, 128 bytes of alignment slack, the stage barriers,
  // the per-stage counters and a flag
  static constexpr size_t SMEM = STAGES * (size_t)STAGE_BYTES + 128 + 8 * STAGES +
                                 4 * STAGES + 4;
  // smem distance between consecutive stencil cells
  static constexpr int STEP = d == 2 ? 1 : FX;
  static_assert(VAR_BYTES % 128 == 0, "TMA destinations need 128-byte alignment");
};

struct FluxMaps {
  CUtensorMap m[9];
};

// Tile list of one launch: the face box [i0, i1) x [j0, j0 + nj) x
// [k0, k0 + nk) of direction d (ghost-relative starts), cut into tiles.
struct FluxTiles {
  int i0, na, nb;          // first radial layer; faces along the tile axes
  int ta, tb;              // tiles along the sweep (or j) axis and along k
  int rows;                // rows of the third axis (j for d = 0, i for d = 1, 2)
  int row0;                // first row
  int a0;                  // first face along the tile's second axis
  long long count;         // tiles per face times six faces
};

constexpr unsigned kTileSpinLimit = 1u << 22;   // polls of a stage barrier

__device__ __forceinline__ unsigned smem_addr(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ bool bar_wait(unsigned long long *bar, unsigned parity,
                                         unsigned limit) {
  const unsigned b = smem_addr(bar);
  for (unsigned it = 0;; ++it) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(b), "r"(parity)
        : "memory");
    if (ok) return true;
    if (it >= limit) return false;
  }
}

// Tile t of a launch: face f, row, start along the second tile axis (a),
// start along k (b), and the faces the tile covers along each.
struct TileCoord {
  int f, row, a, b, fa, fb;
};

template <int d, typename T>
__device__ __forceinline__ TileCoord tile_coord(const FluxTiles &L, long long t) {
  using S = FluxTile<d, T>;
  TileCoord c;
  const int tb = (int)(t % L.tb);
  long long r = t / L.tb;
  const int ta = (int)(r % L.ta);
  r /= L.ta;
  c.row = L.row0 + (int)(r % L.rows);
  c.f = (int)(r / L.rows);
  if (d == 2) {
    // k is the sweep axis: the last k tile takes up to FX + 1 faces
    c.b = tb * S::FX;
    c.fb = tb == L.tb - 1 ? L.nb - c.b : S::FX;
    c.a = ta * S::FY;
    c.fa = L.na - c.a < S::FY ? L.na - c.a : S::FY;
  } else {
    c.a = ta * S::FY;
    c.fa = ta == L.ta - 1 ? L.na - c.a : S::FY;
    c.b = tb * S::FX;
    c.fb = L.nb - c.b < S::FX ? L.nb - c.b : S::FX;
  }
  return c;
}

// One elected thread: copies of tile t's staged cells into stage buffer sm.
// The cell arrays of the view cover layers [lo, N0) of each face, so the
// tensor's third coordinate is face * (N0 - lo) + i - lo.
template <int d, typename T>
__device__ __forceinline__ void issue_tile(const FluxMaps &maps, const Dims &D,
                                           const FluxTiles &L, long long t, T *sm,
                                           unsigned long long *bar, int lo) {
  using S = FluxTile<d, T>;
  const TileCoord c = tile_coord<d, T>(L, t);
  int x, y, z;
  const int zf = c.f * (D.E0 + 1 - lo) - lo;
  if (d == 0) {
    x = D.g + c.b;
    y = c.row;
    z = zf + L.i0 + c.a - 4;
  } else if (d == 1) {
    x = D.g + c.b;
    y = L.a0 + c.a - 4;
    z = zf + c.row;
  } else {
    x = D.g + c.b - 4;
    y = L.a0 + c.a;
    z = zf + c.row;
  }
  const unsigned b = smem_addr(bar);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b),
               "r"(S::STAGE_BYTES)
               : "memory");
#pragma unroll
  for (int v = 0; v < S::VARS; ++v) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(sm + v * S::CELLS)),
        "l"((unsigned long long)&maps.m[v]), "r"(x), "r"(y), "r"(z), "r"(b)
        : "memory");
  }
}

// The flux of one face from the staged stencil (same operations as k_flux).
template <int d, typename T>
__device__ __forceinline__ void staged_face(const T *sm, int s0, const Dims &D,
                                            const DevState &S, const Bulk<T> &B,
                                            const Opts &O, DevStatus *st, int f, int i,
                                            int j, int k) {
  using Sh = FluxTile<d, T>;
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
  const T *svol = sm + 8 * Sh::CELLS + s0;
  T vol[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) vol[n] = svol[n * Sh::STEP];
  PrimT<T> st2[2];
  {
    T q[8], l, r;
    bool ok = true;
    const T *sp = sm + s0;
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      q[n] = sp[n * Sh::STEP];
      ok = ok && !isnan(q[n]);
    }
    if (!ok) {
      fail(st, kStageReconstruct, d, f, i, j, k);
      return;
    }
    up7_pdm_rcp(vol, q, riv, pdm, &l, &r);
    st2[0].rho = l; st2[1].rho = r;
    sp += Sh::CELLS;
#pragma unroll
    for (int n = 0; n < 8; ++n) q[n] = sp[n * Sh::STEP];
    up7_pdm_rcp(vol, q, riv, pdm, &l, &r);
    st2[0].vx = l; st2[1].vx = r;
    sp += Sh::CELLS;
#pragma unroll
    for (int n = 0; n < 8; ++n) q[n] = sp[n * Sh::STEP];
    up7_pdm_rcp(vol, q, riv, pdm, &l, &r);
    st2[0].vy = l; st2[1].vy = r;
    sp += Sh::CELLS;
#pragma unroll
    for (int n = 0; n < 8; ++n) q[n] = sp[n * Sh::STEP];
    up7_pdm_rcp(vol, q, riv, pdm, &l, &r);
    st2[0].vz = l; st2[1].vz = r;
    sp += Sh::CELLS;
#pragma unroll
    for (int n = 0; n < 8; ++n) q[n] = sp[n * Sh::STEP];
    up7_pdm_rcp(vol, q, riv, pdm, &l, &r);
    st2[0].p = l; st2[1].p = r;
  }
  T mag[2][3] = {{T(0.0), T(0.0), T(0.0)}, {T(0.0), T(0.0), T(0.0)}};
  if (O.s_mhd) {
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const T *sp = sm + (5 + m) * Sh::CELLS + s0;
      T q[8];
#pragma unroll
      for (int n = 0; n < 8; ++n) q[n] = sp[n * Sh::STEP];
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

// Face (x, y) of tile c: x along k, y along the second tile axis.
template <int d, typename T>
__device__ __forceinline__ void tile_face(const T *sm, const TileCoord &c, int x, int y,
                                          const FluxTiles &L, const Dims &D,
                                          const DevState &S, const Bulk<T> &B,
                                          const Opts &O, DevStatus *st) {
  using Sh = FluxTile<d, T>;
  int i, j, k, s0;
  if (d == 0) {
    i = L.i0 + c.a + y;
    j = c.row;
    k = D.g + c.b + x;
    s0 = y * Sh::BX + x;
  } else if (d == 1) {
    i = c.row;
    j = L.a0 + c.a + y;
    k = D.g + c.b + x;
    s0 = y * Sh::BX + x;
  } else {
    i = c.row;
    j = L.a0 + c.a + y;
    k = D.g + c.b + x;
    s0 = y * Sh::BX + x;
  }
  staged_face<d, T>(sm, s0, D, S, B, O, st, c.f, i, j, k);
}

// Warps of a staged flux block.  They share the stage buffers but never wait
// for one another: a warp waits only for the copies of the stage it is about
// to read, and the last warp to finish reading a stage issues its refill
// (the tile kStages iterations ahead).  The extra faces of a last tile along
// the sweep axis go to one warp, a different warp on each iteration.
template <int d, typename T>
__global__ void __launch_bounds__(256, FluxTile<d, T>::MIN_BLOCKS)
    k_flux_tma(const __grid_constant__ FluxMaps maps, Dims D, DevState S, Bulk<T> B,
               Opts O, DevStatus *st, FluxTiles L) {
  using Sh = FluxTile<d, T>;
  constexpr int kWarps = Sh::THREADS / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // stage buffers on a 128-byte boundary (TMA destinations), then the stage
  // barriers, the per-stage count of warps done with the stage, and a flag
  unsigned char *base =
      smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
  unsigned long long *full = (unsigned long long *)(base + Sh::STAGES * Sh::STAGE_BYTES);
  int *done = (int *)(full + Sh::STAGES);
  int &skip = done[Sh::STAGES];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long first = blockIdx.x, stride = gridDim.x;
  // a block leaves before its first copy if an earlier kernel of the step
  // failed (one thread reads the status, so the whole block agrees)
  if (tid == 0) {
    skip = failed(st) ? 1 : 0;
    if (!skip) {
      for (int q = 0; q < Sh::STAGES; ++q) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&full[q])));
        done[q] = 0;
      }
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      for (int q = 0; q < Sh::STAGES; ++q)
        if (first + q * stride < L.count)
          issue_tile<d, T>(maps, D, L, first + q * stride,
                           (T *)(base + q * Sh::STAGE_BYTES), &full[q], B.lo);
    }
  }
  __syncthreads();
  if (skip) return;
  unsigned it = 0;
  for (long long t = first; t < L.count; t += stride, ++it) {
    const int s = (int)(it % Sh::STAGES);
    const unsigned phase = (it / Sh::STAGES) & 1u;
    const bool ok = __all_sync(0xffffffffu, bar_wait(&full[s], phase, kTileSpinLimit));
    if (!ok) {
      // the copies of this stage did not arrive: record it, then wait
      // (bounded) for the copies of the other stages before leaving, so no
      // copy lands in shared memory the block has released
      if (lane == 0) {
        fail(st, kStageTileCopy, d, 0, 0, 0, 0);
        for (int q = 1; q < Sh::STAGES; ++q)
          if (t + q * stride < L.count)
            bar_wait(&full[(s + q) % Sh::STAGES], ((it + q) / Sh::STAGES) & 1u,
                     kTileSpinLimit);
      }
      return;
    }
    const TileCoord c = tile_coord<d, T>(L, t);
    const T *sm = (const T *)(base + s * Sh::STAGE_BYTES);
    // the thread's face, then (one warp per iteration) the extra face of a
    // last tile along the sweep axis; one call site keeps the face code
    // once in the instruction stream
    const int passes = warp == (int)(it % kWarps) ? 2 : 1;
    for (int pass = 0; pass < passes; ++pass) {
      int x, y;
      bool on;
      if (pass == 0) {
        x = tid % Sh::FX;
        y = tid / Sh::FX;
        on = x < c.fb && y < c.fa;
      } else if (d == 2) {
        x = Sh::FX;
        y = lane;
        on = c.fb > Sh::FX && lane < c.fa;
      } else {
        x = lane;
        y = Sh::FY;
        on = c.fa > Sh::FY && lane < c.fb;
      }
      if (on) tile_face<d, T>(sm, c, x, y, L, D, S, B, O, st);
    }
    // this warp is done with the stage; the last warp refills it
    __syncwarp();
    if (lane == 0) {
      __threadfence_block();
      if (atomicAdd(&done[s], 1) == kWarps - 1) {
        done[s] = 0;
        const long long next = t + (long long)Sh::STAGES * stride;
        if (next < L.count) {
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          issue_tile<d, T>(maps, D, L, next, (T *)(base + s * Sh::STAGE_BYTES), &full[s],
                           B.lo);
        }
      }
    }
  }
}

// Host: tensor map of one FP64 or FP32 node array (all six faces, layers
// [lo, N0) of each, viewed as the 3-D tensor k x j x (face, i)) with the
// given box (gcs_setup.cu).
int encode_cell_map(CUtensorMap *map, const void *base, int elem_bytes, const Dims &D,
                    int lo, int box_x, int box_y, int box_z);
// Host: record a failure of the step at a stage (gcs_kernels.cu).
void launch_set_failure(const Ctx &X, int stage, int dir, cudaStream_t s);

// Host: tile list of the flux faces of direction d over radial layers
// [i0, i1) (already clamped to the faces of direction d).
template <int d, typename T>
FluxTiles flux_tiles(const Dims &D, int i0, int i1) {
  using Sh = FluxTile<d, T>;
  FluxTiles L{};
  L.i0 = i0;
  const int n = D.n;
  if (d == 0) {
    L.na = i1 - i0;                       // faces along i (sweep axis)
    L.nb = n;                             // along k
    L.ta = L.na > 1 ? (L.na - 1 + Sh::FY - 1) / Sh::FY : 1;
    L.tb = (n + Sh::FX - 1) / Sh::FX;
    L.rows = n;                           // j
    L.row0 = D.g;
    L.a0 = i0;
  } else if (d == 1) {
    L.na = n + 1;                         // faces along j (sweep axis)
    L.nb = n;
    L.ta = (n + Sh::FY - 1) / Sh::FY;     // last tile takes up to FY + 1 faces
    L.tb = (n + Sh::FX - 1) / Sh::FX;
    L.rows = i1 - i0;                     // i
    L.row0 = i0;
    L.a0 = D.g;
  } else {
    L.na = n;                             // faces along j
    L.nb = n + 1;                         // along k (sweep axis)
    L.ta = (n + Sh::FY - 1) / Sh::FY;
    L.tb = (n + Sh::FX - 1) / Sh::FX;     // last tile takes up to FX + 1 faces
    L.rows = i1 - i0;
    L.row0 = i0;
    L.a0 = D.g;
  }
  L.count = (long long)kFaces * L.rows * L.ta * L.tb;
  return L;
}

// Persistent grid of the staged flux sweep: resident blocks per SM times
// SMs, found once per process (outside any stream capture: the first call
// comes from prepare_flux_tma at context set-up).
template <int d, typename T>
int flux_tma_blocks() {
  using Sh = FluxTile<d, T>;
  static int blocks = 0;
  if (blocks == 0) {
    if (cudaFuncSetAttribute(k_flux_tma<d, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)Sh::SMEM) != cudaSuccess)
      return -1;
    int per_sm = 0, sms = 0, dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_flux_tma<d, T>,
                                                      Sh::THREADS, Sh::SMEM) != cudaSuccess ||
        per_sm <= 0 || sms <= 0)
      return -1;
    blocks = per_sm * sms;
  }
  return blocks;
}

template <typename T>
int prepare_flux_tma() {
  return (flux_tma_blocks<0, T>() > 0 && flux_tma_blocks<1, T>() > 0 &&
          flux_tma_blocks<2, T>() > 0) ? 0 : -1;
}

// Launch of the staged flux sweep of direction d over [i0, i1).
template <int d, typename T>
void launch_flux_tma(const Ctx &X, const Bulk<T> &B, const Opts &O, int i0, int i1,
                     cudaStream_t s) {
  using Sh = FluxTile<d, T>;
  const Dims &D = X.D;
  const FluxTiles L = flux_tiles<d, T>(D, i0, i1);
  if (L.count <= 0) return;
  FluxMaps maps;
  const void *arrays[9] = {B.Pr[0], B.Pr[1], B.Pr[2], B.Pr[3], B.Pr[4],
                           B.Bp[0], B.Bp[1], B.Bp[2], B.vol};
  for (int v = 0; v < 9; ++v)
    if (encode_cell_map(&maps.m[v], arrays[v], (int)sizeof(T), D, B.lo, Sh::BX, Sh::BY,
                        Sh::BZ) != 0) {
      // no sweep without its tensor maps: the step fails at this stage
      launch_set_failure(X, kStageTileCopy, d, s);
      return;
    }
  const int blocks = flux_tma_blocks<d, T>();
  if (blocks <= 0) {
    launch_set_failure(X, kStageTileCopy, d, s);
    return;
  }
  const long long grid = L.count < blocks ? L.count : blocks;
  k_flux_tma<d, T><<<(unsigned)grid, Sh::THREADS, Sh::SMEM, s>>>(maps, D, X.S, B, O,
                                                                  X.status, L);
}

}  // namespace gcs
