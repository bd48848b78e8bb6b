// Analysis output of a device-resident run (cubedsphere/cubedsphere_analysis_hdf5.c
// and cubedsphere/docs/OUTPUT_DATA_MODEL.md): per face a float32 frame
// [8][NI][NJ][NK] of rho, p, vx, vy, vz, Bx, By, Bz over the active cells
// (B the total field, residual plus cell B0), computed on the device, and a
// writer of the reference's per-face file set.  HDF5 is not available to
// this library, so each dataset is a raw little-endian file and the
// metadata datasets of the reference (analysis_schema, patch_id, sequence,
// step, coordinate_backend, problem_id, global_cells, logical bounds, times,
// normalization, field_names) go to a JSON file beside it.
#include "gcs_context.h"
#include "gcs_error.h"
#include "gamera_cs_b200.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "gcs_physics.cuh"

namespace gcs {
namespace {

// cubedsphere_analysis_hdf5.c:316-331
__global__ void k_analysis_frame(Dims D, DevState S, DevBg BG, int have_bg, double gamma,
                                 float *out, int *bad) {
  const long long count = (long long)D.nr * D.n * D.n;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= count) return;
  const int f = blockIdx.y;
  const int i = (int)(t / ((long long)D.n * D.n));
  const int j = (int)((t / D.n) % D.n);
  const int k = (int)(t % D.n);
  const long long c = f * D.Nn + D.node(D.g + i, D.g + j, D.g + k);
  double u[5];
  for (int m = 0; m < 5; ++m) u[m] = S.U[m][c];
  Prim p;
  float *o = out + (long long)f * 8 * count + t;
  if (cons_to_prim(u, gamma, 1e-12, 1e-12, &p)) {
    atomicExch(bad, 1);
    for (int q = 0; q < 8; ++q) o[q * count] = 0.0f;
    return;
  }
  double v[8] = {p.rho, p.p, p.vx, p.vy, p.vz, S.B[0][c], S.B[1][c], S.B[2][c]};
  if (have_bg)
    for (int m = 0; m < 3; ++m) v[5 + m] = S.B[m][c] + BG.b0[m][c];
  for (int q = 0; q < 8; ++q) {
    const float x = (float)v[q];
    o[q * count] = x;
    if (!isfinite(v[q]) || !isfinite(x)) atomicExch(bad, 1);
  }
}

}  // namespace
}  // namespace gcs

namespace {

bool write_file(const std::string &path, const void *data, size_t bytes) {
  FILE *fp = fopen(path.c_str(), "wb");
  if (!fp) return false;
  const bool ok = fwrite(data, 1, bytes, fp) == bytes;
  return fclose(fp) == 0 && ok;
}

bool exists(const std::string &path) {
  FILE *fp = fopen(path.c_str(), "rb");
  if (!fp) return false;
  fclose(fp);
  return true;
}

// /normalization of cubedsphere_analysis_hdf5.c:97-101 (x = 1 R_E,
// u = 100 km/s, rho = 1 proton cm^-3).
void normalization(double out[10]) {
  const double mu0 = 4.0e-7 * acos(-1.0);
  const double x = 6371000.0, u = 100000.0, rho = 1.67262192369e-21;
  const double b = u * sqrt(mu0 * rho);
  const double n[10] = {mu0, x, u, x / u, rho, rho * u * u, b, b * x * x * x / mu0, u / x,
                        1.0 / (mu0 * u)};
  for (int q = 0; q < 10; ++q) out[q] = n[q];
}

std::string metadata_json(int face, long sequence, long step, double time_code,
                          double time_seconds, const int cells[3], const char *data_file,
                          const char *what) {
  double norm[10];
  normalization(norm);
  char buf[4096];
  int n = snprintf(buf, sizeof(buf),
                   "{\n  \"analysis_schema\": 1,\n  \"patch_id\": %d,\n  \"sequence\": %ld,\n"
                   "  \"step\": %ld,\n  \"coordinate_backend\": 3,\n  \"problem_id\": 1,\n"
                   "  \"global_cells\": [%d, %d, %d],\n"
                   "  \"logical_lower\": [2.5, -1.0, -1.0],\n"
                   "  \"logical_upper\": [200.0, 1.0, 1.0],\n"
                   "  \"time_code\": %.17g,\n  \"time_seconds\": %.17g,\n"
                   "  \"normalization\": [",
                   face, sequence, step, cells[0], cells[1], cells[2], time_code,
                   time_seconds);
  for (int q = 0; q < 10; ++q)
    n += snprintf(buf + n, sizeof(buf) - n, "%.17g%s", norm[q], q < 9 ? ", " : "");
  n += snprintf(buf + n, sizeof(buf) - n,
                "],\n  \"field_names\": [\"rho\", \"p\", \"vx\", \"vy\", \"vz\", \"Bx\", "
                "\"By\", \"Bz\"],\n  \"%s\": {\"file\": \"%s\", \"dtype\": \"float32\", "
                "\"byte_order\": \"little\", \"shape\": [8, %d, %d, %d]}\n}\n",
                what, data_file, cells[0], cells[1], cells[2]);
  return std::string(buf, n);
}

}  // namespace

extern "C" {

size_t gcs_analysis_frame_floats(const gcs_context *ctx) {
  if (!ctx) return 0;
  const gcs::Dims &D = ctx->c.X.D;
  return (size_t)gcs::kFaces * 8 * (size_t)D.nr * D.n * D.n;
}

int gcs_context_analysis_frame(gcs_context *ctx, double gamma, float *device_out,
                               float *host_out) {
  if (!ctx || !std::isfinite(gamma) || !(gamma > 1.0) || (!device_out && !host_out)) {
    gcs::set_api_error("invalid analysis frame arguments");
    return -1;
  }
  gcs::Context &C = ctx->c;
  const gcs::Dims &D = C.X.D;
  const size_t floats = gcs_analysis_frame_floats(ctx);
  float *out = device_out;
  void *scratch = nullptr;
  const size_t sbytes = (device_out ? 0 : floats * sizeof(float)) + sizeof(int);
  if (cudaMalloc(&scratch, sbytes) != cudaSuccess) {
    gcs::set_api_error("cannot allocate the analysis frame");
    return -1;
  }
  if (!out) out = (float *)scratch;
  int *bad = (int *)((char *)scratch + sbytes - sizeof(int));
  const long long count = (long long)D.nr * D.n * D.n;
  int hbad = 0;
  bool ok = cudaMemsetAsync(bad, 0, sizeof(int), C.stream) == cudaSuccess;
  if (ok) {
    gcs::k_analysis_frame<<<dim3((unsigned)((count + 255) / 256), gcs::kFaces), 256, 0,
                            C.stream>>>(D, C.X.S, C.X.BG, C.bg_uploaded, gamma, out, bad);
    ok = cudaGetLastError() == cudaSuccess &&
         cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, C.stream) ==
             cudaSuccess;
  }
  if (ok && host_out)
    ok = cudaMemcpyAsync(host_out, out, floats * sizeof(float), cudaMemcpyDeviceToHost,
                         C.stream) == cudaSuccess;
  ok = ok && cudaStreamSynchronize(C.stream) == cudaSuccess;
  cudaFree(scratch);
  if (!ok) {
    gcs::set_api_error("analysis frame: CUDA error");
    return -1;
  }
  if (hbad) {
    gcs::set_api_error("analysis frame: invalid state or non-finite field");
    return -1;
  }
  return 0;
}

int gcs_context_write_analysis(gcs_context *ctx, const char *directory, long sequence,
                               long step, double time_code, double time_seconds,
                               double gamma, const gamera_no_grid *grid) {
  if (!ctx || !directory || sequence < 0 || sequence > 2147483647L || step < 0 ||
      !std::isfinite(time_code) || !std::isfinite(time_seconds)) {
    gcs::set_api_error("invalid analysis output arguments");
    return -1;
  }
  gcs::Context &C = ctx->c;
  const gcs::Dims &D = C.X.D;
  const int cells[3] = {D.nr, D.n, D.n};
  const size_t count = (size_t)D.nr * D.n * D.n;
  std::vector<float> frame(gcs_analysis_frame_floats(ctx));
  if (gcs_context_analysis_frame(ctx, gamma, nullptr, frame.data()) != 0) return -1;
  const std::string dir(directory);
  for (int f = 0; f < gcs::kFaces; ++f) {
    char name[64];
    // static grid of the face, written once
    snprintf(name, sizeof(name), "analysis_grid_p%d", f);
    const std::string grid_json = dir + "/" + name + ".json";
    if (!exists(grid_json)) {
      std::vector<double> cen, vert;
      if (grid != nullptr) {
        const gamera_no_grid &G = grid[f];
        cen.assign(3 * count, 0.0);
        const size_t nv = (size_t)(D.nr + 1) * (D.n + 1) * (D.n + 1);
        vert.assign(3 * nv, 0.0);
        for (int i = 0; i < D.nr; ++i)
          for (int j = 0; j < D.n; ++j)
            for (int k = 0; k < D.n; ++k) {
              const size_t q = ((size_t)i * D.n + j) * D.n + k;
              const gamera_no_vec3 &x =
                  G.cell[((size_t)(i + D.g) * D.E1 + j + D.g) * D.E2 + k + D.g].centroid;
              for (int a = 0; a < 3; ++a) cen[a * count + q] = x.value[a];
            }
        const size_t *ve = G.vertex_extent;
        for (int i = 0; i <= D.nr; ++i)
          for (int j = 0; j <= D.n; ++j)
            for (int k = 0; k <= D.n; ++k) {
              const size_t q = ((size_t)i * (D.n + 1) + j) * (D.n + 1) + k;
              const gamera_no_vec3 &x =
                  G.vertex[((size_t)(i + D.g) * ve[1] + j + D.g) * ve[2] + k + D.g];
              for (int a = 0; a < 3; ++a) vert[a * nv + q] = x.value[a];
            }
      } else if (C.face_coordinates(f, cen, vert) != 0) {
        gcs::set_api_error("analysis grid: pass the host grid for this context");
        return -1;
      }
      char cf[96], vf[96];
      snprintf(cf, sizeof(cf), "%s.coordinates.f64", name);
      snprintf(vf, sizeof(vf), "%s.vertices.f64", name);
      char js[1024];
      const int n = snprintf(js, sizeof(js),
                             "{\n  \"patch_id\": %d,\n  \"coordinate_backend\": 3,\n"
                             "  \"units\": \"earth radii\",\n"
                             "  \"coordinates\": {\"file\": \"%s\", \"dtype\": \"float64\", "
                             "\"byte_order\": \"little\", \"shape\": [3, %d, %d, %d]},\n"
                             "  \"vertices\": {\"file\": \"%s\", \"dtype\": \"float64\", "
                             "\"byte_order\": \"little\", \"shape\": [3, %d, %d, %d]}\n}\n",
                             f, cf, D.nr, D.n, D.n, vf, D.nr + 1, D.n + 1, D.n + 1);
      if (!write_file(dir + "/" + cf, cen.data(), cen.size() * sizeof(double)) ||
          !write_file(dir + "/" + vf, vert.data(), vert.size() * sizeof(double)) ||
          !write_file(grid_json, js, (size_t)n)) {
        gcs::set_api_error("analysis grid: cannot write");
        return -1;
      }
    }
    snprintf(name, sizeof(name), "analysis_p%d_%06ld", f, sequence);
    char sf[96];
    snprintf(sf, sizeof(sf), "%s.state.f32", name);
    const std::string meta =
        metadata_json(f, sequence, step, time_code, time_seconds, cells, sf, "state");
    if (!write_file(dir + "/" + sf, frame.data() + (size_t)f * 8 * count,
                    8 * count * sizeof(float)) ||
        !write_file(dir + "/" + name + ".json", meta.data(), meta.size())) {
      gcs::set_api_error("analysis frame: cannot write");
      return -1;
    }
  }
  return 0;
}

}  // extern "C"
