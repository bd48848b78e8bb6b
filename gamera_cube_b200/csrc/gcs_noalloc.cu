// Allocation-free CFL time step for callers that cannot allocate device
// memory.
//
// Some callers cannot call cudaMalloc at the point where they need a time
// step: a host code that hands this library device arrays owned by another
// allocator or runtime, a driver that forbids device allocation after its
// start-up, or a coupling loop that must not change the device memory
// footprint while it runs.  gcs_local_timestep_noalloc serves them: the
// caller passes its device inputs and receives the step on the host, and the
// only global memory the reduction uses beyond those inputs is the
// file-scope array below, sized once for the largest supported call.
//
// The array occupies kScratchBytes of every GPU that loads this library
// until the process exits.  With CUDA's default lazy module loading the
// library's device code, and this array with it, is loaded onto a device by
// the first call there of any entry point that touches device code; a
// caller that must fix its footprint at start-up makes one call of this
// entry point then (or runs with CUDA_MODULE_LOADING=EAGER).  Later calls
// change the device memory footprint by nothing.
//
// All calls share the array and it keeps the contents of the last call;
// every slot a call reads is written earlier in the same call, so nothing
// has to be cleared between calls.  Calls that overlap on the GPU (from
// several host threads or streams) race on the array and must be
// serialised by the caller.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdio>

#include "gamera_cs_b200.h"
#include "gcs_physics.cuh"

namespace {

constexpr int kBlock = 256;                // cells per block
constexpr int kMaxBlocks = 65536;          // partial minima
constexpr long long kMaxCells = (long long)kBlock * kMaxBlocks;  // 16,777,216

// Scratch layout: kMaxBlocks partial minima, kMaxBlocks failure flags,
// then the reduced minimum and its failure flag.
struct Scratch {
  double partial[kMaxBlocks];
  int failed[kMaxBlocks];
  double result;
  int result_failed;
};
constexpr size_t kScratchBytes = sizeof(Scratch);

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

thread_local char g_error[256] = "";

// Candidate step of one active cell (nonorthogonal_step.c:479-516).
__device__ inline bool cell_candidate(const gamera_no_cell_geometry *cells,
                                      const double *u, const gamera_no_vec3 *b,
                                      const gamera_no_vec3 *b0, long long c,
                                      const gamera_no_timestep_options o,
                                      double *out) {
  gcs::Prim p;
  if (gcs::cons_to_prim(u + 5 * c, o.gamma, o.density_floor, o.pressure_floor,
                        &p))
    return false;
  const double cs = sqrt(o.gamma * p.p / p.rho);
  double va = 0.0;
  if (o.use_mhd) {
    double bx = b[c].value[0], by = b[c].value[1], bz = b[c].value[2];
    if (o.use_background) {
      bx = bx + b0[c].value[0];
      by = by + b0[c].value[1];
      bz = bz + b0[c].value[2];
    }
    double s2 = 0.0;
    s2 += bx * bx;
    s2 += by * by;
    s2 += bz * bz;
    va = sqrt(s2) / sqrt(p.rho);
    if (o.use_boris) va = o.light_speed * va / hypot(o.light_speed, va);
  }
  double v2 = 0.0;
  v2 += p.vx * p.vx;
  v2 += p.vy * p.vy;
  v2 += p.vz * p.vz;
  const double speed = sqrt(v2) + hypot(cs, va);
  double len = cells[c].cfl_length[0];
  len = fmin(len, cells[c].cfl_length[1]);
  len = fmin(len, cells[c].cfl_length[2]);
  const double cand = o.cfl * len / speed;
  if (!isfinite(cand) || cand <= 0.0) return false;
  *out = cand;
  return true;
}

// Every block writes its partial minimum and failure flag, so the reduction
// below never reads a slot left over from an earlier call.
__global__ void k_partial(Scratch *s, const gamera_no_cell_geometry *cells,
                          const double *u, const gamera_no_vec3 *b,
                          const gamera_no_vec3 *b0, long long e1, long long e2,
                          long long l0, long long l1, long long l2, long long n1,
                          long long n2, long long count,
                          gamera_no_timestep_options o) {
  const long long t = blockIdx.x * (long long)kBlock + threadIdx.x;
  double cand = DBL_MAX;
  int bad = 0;
  if (t < count) {
    const long long i = l0 + t / (n1 * n2);
    const long long j = l1 + (t / n2) % n1;
    const long long k = l2 + t % n2;
    const long long c = (i * e1 + j) * e2 + k;
    if (!cell_candidate(cells, u, b, b0, c, o, &cand)) {
      cand = DBL_MAX;
      bad = 1;
    }
  }
  __shared__ double smin[kBlock / 32];
  __shared__ int sbad[kBlock / 32];
  for (int off = 16; off > 0; off >>= 1) {
    cand = fmin(cand, __shfl_down_sync(0xffffffffu, cand, off));
    bad |= __shfl_down_sync(0xffffffffu, bad, off);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    smin[warp] = cand;
    sbad[warp] = bad;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = smin[0];
    int f = sbad[0];
    for (int w = 1; w < kBlock / 32; ++w) {
      m = fmin(m, smin[w]);
      f |= sbad[w];
    }
    s->partial[blockIdx.x] = m;
    s->failed[blockIdx.x] = f;
  }
}

__global__ void k_final(Scratch *s, int blocks) {
  double m = DBL_MAX;
  int f = 0;
  for (int q = threadIdx.x; q < blocks; q += blockDim.x) {
    m = fmin(m, s->partial[q]);
    f |= s->failed[q];
  }
  __shared__ double smin[1024 / 32];
  __shared__ int sbad[1024 / 32];
  for (int off = 16; off > 0; off >>= 1) {
    m = fmin(m, __shfl_down_sync(0xffffffffu, m, off));
    f |= __shfl_down_sync(0xffffffffu, f, off);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    smin[warp] = m;
    sbad[warp] = f;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x / 32); ++w) {
      smin[0] = fmin(smin[0], smin[w]);
      sbad[0] |= sbad[w];
    }
    s->result = smin[0];
    s->result_failed = sbad[0];
  }
}

// Device address of the scratch array in the current context of the current
// device.  The array's host-side name is only a stand-in and must never be
// passed to a kernel.  The address is looked up on every call rather than
// cached: after cudaDeviceReset, or with another context current on the
// device (a driver-API caller), the module is loaded anew and an address
// kept from before would be stale.
Scratch *scratch_for_current_device() {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
    snprintf(g_error, sizeof(g_error), "no current CUDA device");
    return nullptr;
  }
  void *ptr = nullptr;
  const cudaError_t rc = cudaGetSymbolAddress(&ptr, g_scratch);
  if (rc != cudaSuccess || ptr == nullptr) {
    snprintf(g_error, sizeof(g_error), "cudaGetSymbolAddress failed: %s",
             cudaGetErrorString(rc));
    return nullptr;
  }
  return (Scratch *)ptr;
}

}  // namespace

extern "C" {

int gcs_local_timestep_noalloc(const size_t cell_extent[3],
                               const gamera_no_cell_geometry *cells,
                               const double *conserved,
                               const gamera_no_vec3 *cell_magnetic,
                               const gamera_no_vec3 *background_cell_magnetic,
                               const size_t active_lower[3],
                               const size_t active_upper[3],
                               const gamera_no_timestep_options *options,
                               double *local_dt) {
  if (cell_extent == nullptr || cells == nullptr || conserved == nullptr ||
      active_lower == nullptr || active_upper == nullptr ||
      options == nullptr || local_dt == nullptr) {
    snprintf(g_error, sizeof(g_error), "null argument");
    return -1;
  }
  const gamera_no_timestep_options o = *options;
  if (!std::isfinite(o.gamma) || o.gamma <= 1.0 ||
      !std::isfinite(o.density_floor) || o.density_floor <= 0.0 ||
      !std::isfinite(o.pressure_floor) || o.pressure_floor <= 0.0 ||
      !std::isfinite(o.cfl) || o.cfl <= 0.0 ||
      (o.use_mhd && cell_magnetic == nullptr) ||
      (o.use_background && background_cell_magnetic == nullptr) ||
      (o.use_boris && !(std::isfinite(o.light_speed) && o.light_speed > DBL_MIN))) {
    snprintf(g_error, sizeof(g_error), "invalid time-step options");
    return -1;
  }
  long long n[3];
  for (int a = 0; a < 3; ++a) {
    if (active_lower[a] >= active_upper[a] || active_upper[a] > cell_extent[a]) {
      snprintf(g_error, sizeof(g_error), "invalid active range");
      return -1;
    }
    // each axis is checked on its own first, so the product below cannot
    // overflow
    const size_t na = active_upper[a] - active_lower[a];
    if (na > (size_t)kMaxCells) {
      snprintf(g_error, sizeof(g_error),
               "gcs_local_timestep_noalloc: %zu active cells along axis %d exceed "
               "the maximum of %lld per call",
               na, a, kMaxCells);
      return -1;
    }
    n[a] = (long long)na;
  }
  if (n[0] * n[1] > kMaxCells || n[0] * n[1] * n[2] > kMaxCells) {
    snprintf(g_error, sizeof(g_error),
             "gcs_local_timestep_noalloc: %lld x %lld x %lld active cells exceed "
             "the maximum of %lld per call",
             n[0], n[1], n[2], kMaxCells);
    return -1;
  }
  const long long count = n[0] * n[1] * n[2];
  Scratch *s = scratch_for_current_device();
  if (s == nullptr) return -1;
  const int blocks = (int)((count + kBlock - 1) / kBlock);
  k_partial<<<blocks, kBlock>>>(s, cells, conserved, cell_magnetic,
                                background_cell_magnetic,
                                (long long)cell_extent[1], (long long)cell_extent[2],
                                (long long)active_lower[0],
                                (long long)active_lower[1],
                                (long long)active_lower[2], n[1], n[2], count, o);
  cudaError_t launch = cudaGetLastError();
  if (launch == cudaSuccess) {
    k_final<<<1, 1024>>>(s, blocks);
    launch = cudaGetLastError();
  }
  if (launch != cudaSuccess) {
    // a failed launch leaves the array holding an earlier call's result
    snprintf(g_error, sizeof(g_error), "kernel launch failed: %s",
             cudaGetErrorString(launch));
    return -1;
  }
  double result = 0.0;
  int failed = 1;
  if (cudaMemcpy(&result, &s->result, sizeof(double), cudaMemcpyDeviceToHost) !=
          cudaSuccess ||
      cudaMemcpy(&failed, &s->result_failed, sizeof(int), cudaMemcpyDeviceToHost) !=
          cudaSuccess) {
    snprintf(g_error, sizeof(g_error), "%s", cudaGetErrorString(cudaGetLastError()));
    return -1;
  }
  if (failed) {
    snprintf(g_error, sizeof(g_error), "invalid cell state or time step");
    return -1;
  }
  *local_dt = result;
  return 0;
}

const char *gcs_noalloc_last_error(void) { return g_error; }

size_t gcs_noalloc_scratch_bytes(void) { return kScratchBytes; }

}  // extern "C"
