// Learned preconditioner of the conductance-tensor ionosphere solve: a
// four-level convolutional network (encoder of 3x3 convolutions and 2x2
// average pooling, decoder of nearest upsampling, 3x3 convolutions and
// additive skips; 16/32/48/64 channels, about 194,000 parameters) on the
// polar grid, run on BF16 tensor cores with FP32 accumulation by the kernels
// of gcs_learn_kernels.cuh, trained on the GPU by those kernels' forward and
// backward passes with Adam.  It has no counterpart in the reference.
//
// Grid: interior colatitude rows 0..R-1 by longitudes 0..np-1, padded to
// H0 = R rounded up to 8 rows (zeros) and W0 = np rounded up to 32 columns
// (a periodic continuation of the first longitudes), so three poolings
// stay exact.  Input channels: the residual (unit RMS), log(Sigma_P / 5 S),
// Sigma_H / Sigma_P and sin(theta).  Output: one FP32 channel, the
// correction direction.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <random>
#include <vector>

#include "gamera_cs_b200.h"
#include "gcs_error.h"
#include "gcs_learn_kernels.cuh"

using gcs::set_api_error;
using namespace gcs::learn;

namespace {

constexpr int kLevels = 4;
constexpr int kWidth[kLevels] = {16, 32, 48, 64};
constexpr int kInChannels = 4;

bool cuda_ok(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return true;
  char msg[256];
  snprintf(msg, sizeof(msg), "%s: %s", what, cudaGetErrorString(e));
  set_api_error(msg);
  return false;
}

int round_up(int v, int m) { return (v + m - 1) / m * m; }

struct Tensor {
  int c = 0, level = 0;
  bf16 *a = nullptr;   // activation [B][c][H][W]
  float *g = nullptr;  // gradient
};

enum OpKind { kConvOp, kPoolOp, kUpOp };

struct Op {
  OpKind kind;
  int src, dst;
  int conv = -1;  // index into convs
};

struct Conv {
  int cin, cout, relu, skip, level;
  int Kp, Mp;            // forward weight matrix [Mp][Kp]
  int Kpt, Mpt;          // backward-data weight matrix [Mpt][Kpt]
  size_t off;            // offset of [Mp][Kp] in the parameter arrays
  bool final_layer;
};

}  // namespace

struct gcs_mi_net {
  int R = 0, np = 0, H0 = 0, W0 = 0, max_batch = 0;
  std::vector<Tensor> t;
  std::vector<Conv> convs;
  std::vector<Op> ops;
  size_t nparam = 0;           // padded parameter array length
  float *w = nullptr, *gw = nullptr, *m = nullptr, *v = nullptr;
  bf16 *wb = nullptr, *wt = nullptr;
  size_t wt_len = 0, max_act = 0;
  float *out32 = nullptr, *gout = nullptr, *gm = nullptr, *loss = nullptr;
  int adam_t = 0;
  void *pool = nullptr;
  cudaStream_t stream = nullptr;

  int H(int level) const { return H0 >> level; }
  int W(int level) const { return W0 >> level; }
  size_t elems(const Tensor &x, int B) const {
    return (size_t)B * x.c * H(x.level) * W(x.level);
  }
};

namespace {

int add_tensor(gcs_mi_net *n, int c, int level) {
  Tensor x;
  x.c = c;
  x.level = level;
  n->t.push_back(x);
  return (int)n->t.size() - 1;
}

int add_conv(gcs_mi_net *n, int src, int cout, int relu, int skip, bool final_layer = false) {
  Conv c;
  c.cin = n->t[src].c;
  c.cout = cout;
  c.relu = relu;
  c.skip = skip;
  c.level = n->t[src].level;
  c.Kp = round_up(9 * c.cin + 1, 16);
  c.Mp = round_up(cout, 16);
  c.Kpt = round_up(9 * cout + 1, 16);
  c.Mpt = round_up(c.cin, 16);
  c.off = n->nparam;
  c.final_layer = final_layer;
  n->nparam += (size_t)c.Mp * c.Kp;
  n->convs.push_back(c);
  const int dst = add_tensor(n, cout, c.level);
  n->ops.push_back(Op{kConvOp, src, dst, (int)n->convs.size() - 1});
  return dst;
}

int add_pool(gcs_mi_net *n, int src) {
  const int dst = add_tensor(n, n->t[src].c, n->t[src].level + 1);
  n->ops.push_back(Op{kPoolOp, src, dst});
  return dst;
}

int add_up(gcs_mi_net *n, int src) {
  const int dst = add_tensor(n, n->t[src].c, n->t[src].level - 1);
  n->ops.push_back(Op{kUpOp, src, dst});
  return dst;
}

// The network: encoder convolution pairs at four levels, decoder pairs with
// additive skips, a linear output convolution.
void build_graph(gcs_mi_net *n) {
  const int x = add_tensor(n, kInChannels, 0);
  int e[kLevels];
  int h = x;
  for (int l = 0; l < kLevels; ++l) {
    if (l > 0) h = add_pool(n, e[l - 1]);
    h = add_conv(n, h, kWidth[l], 1, -1);
    e[l] = add_conv(n, h, kWidth[l], 1, -1);
  }
  h = e[kLevels - 1];
  for (int l = kLevels - 2; l >= 0; --l) {
    h = add_up(n, h);
    h = add_conv(n, h, kWidth[l], 1, e[l]);
    h = add_conv(n, h, kWidth[l], 1, -1);
  }
  add_conv(n, h, 1, 0, -1, true);
}

unsigned blocks_for(size_t n) {
  size_t b = (n + 255) / 256;
  return (unsigned)(b > 4096 ? 4096 : b);
}

bool launch_conv(const gcs_mi_net *n, const Conv &c, const void *in, bool in_f32,
                 const bf16 *w, int cin, int cout, int Kp, const bf16 *skip, bf16 *out,
                 float *out32, int relu, int accumulate, int B) {
  ConvP p;
  p.in = in;
  p.w = w;
  p.skip = skip;
  p.out = out;
  p.out32 = out32;
  p.B = B;
  p.Cin = cin;
  p.Cout = cout;
  p.H = n->H(c.level);
  p.W = n->W(c.level);
  p.Kp = Kp;
  p.relu = relu;
  p.accumulate = accumulate;
  const dim3 grid((unsigned)((p.W + kPix - 1) / kPix), (unsigned)p.H, (unsigned)B);
  const size_t smem = conv_smem(Kp);
  if (in_f32)
    k_conv<float><<<grid, kConvThreads, smem, n->stream>>>(p);
  else
    k_conv<bf16><<<grid, kConvThreads, smem, n->stream>>>(p);
  return cuda_ok(cudaGetLastError(), "conv launch");
}

bool configure_kernels() {
  const int most = (int)wgrad_smem(round_up(9 * 64 + 1, 16), 64);
  return cuda_ok(cudaFuncSetAttribute(k_conv<bf16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      most),
                 "cudaFuncSetAttribute") &&
         cuda_ok(cudaFuncSetAttribute(k_conv<float>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, most),
                 "cudaFuncSetAttribute") &&
         cuda_ok(cudaFuncSetAttribute(k_conv_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      most),
                 "cudaFuncSetAttribute");
}

bool forward(gcs_mi_net *n, int B) {
  for (const Op &op : n->ops) {
    const Tensor &s = n->t[op.src], &d = n->t[op.dst];
    if (op.kind == kConvOp) {
      const Conv &c = n->convs[op.conv];
      if (!launch_conv(n, c, s.a, false, n->wb + c.off, c.cin, c.cout, c.Kp,
                       c.skip >= 0 ? n->t[c.skip].a : nullptr, c.final_layer ? nullptr : d.a,
                       c.final_layer ? n->out32 : nullptr, c.relu, 0, B))
        return false;
    } else if (op.kind == kPoolOp) {
      const size_t cnt = (size_t)B * d.c * n->H(d.level) * n->W(d.level);
      k_pool<<<blocks_for(cnt), 256, 0, n->stream>>>(s.a, d.a, B * d.c, n->H(d.level),
                                                      n->W(d.level));
    } else {
      const size_t cnt = (size_t)B * s.c * n->H(s.level) * n->W(s.level);
      k_up<<<blocks_for(cnt), 256, 0, n->stream>>>(s.a, d.a, B * s.c, n->H(s.level),
                                                    n->W(s.level));
    }
  }
  return cuda_ok(cudaGetLastError(), "network forward");
}

// Gradients of every parameter for the output gradient in n->gout.
bool backward(gcs_mi_net *n, int B) {
  for (size_t i = 1; i < n->t.size(); ++i)
    if (!cuda_ok(cudaMemsetAsync(n->t[i].g, 0, n->elems(n->t[i], B) * sizeof(float), n->stream),
                 "cudaMemsetAsync"))
      return false;
  if (!cuda_ok(cudaMemsetAsync(n->gw, 0, n->nparam * sizeof(float), n->stream),
               "cudaMemsetAsync"))
    return false;
  for (auto it = n->ops.rbegin(); it != n->ops.rend(); ++it) {
    const Op &op = *it;
    Tensor &s = n->t[op.src], &d = n->t[op.dst];
    if (op.kind == kConvOp) {
      const Conv &c = n->convs[op.conv];
      const size_t cnt = n->elems(d, B);
      const float *g = c.final_layer ? n->gout : d.g;
      k_relu_mask<<<blocks_for(cnt), 256, 0, n->stream>>>(
          g, c.final_layer ? nullptr : d.a, n->gm, c.skip >= 0 ? n->t[c.skip].g : nullptr, cnt,
          c.relu);
      WgradP wp;
      wp.in = s.a;
      wp.g = n->gm;
      wp.gw = n->gw + c.off;
      wp.B = B;
      wp.Cin = c.cin;
      wp.Cout = c.cout;
      wp.H = n->H(c.level);
      wp.W = n->W(c.level);
      wp.Kp = c.Kp;
      wp.Mp = c.Mp;
      const dim3 grid((unsigned)((wp.W + kPix - 1) / kPix), (unsigned)wp.H, (unsigned)B);
      k_conv_wgrad<<<grid, kConvThreads, wgrad_smem(c.Kp, c.Mp), n->stream>>>(wp);
      if (op.src != 0) {
        k_transpose_weights<<<blocks_for((size_t)c.Mpt * c.Kpt), 256, 0, n->stream>>>(
            n->w + c.off, n->wt, c.cin, c.cout, c.Kp, c.Mpt, c.Kpt);
        if (!launch_conv(n, c, n->gm, true, n->wt, c.cout, c.cin, c.Kpt, nullptr, nullptr, s.g,
                         0, 1, B))
          return false;
      }
    } else if (op.kind == kPoolOp) {
      k_pool_back<<<blocks_for(n->elems(d, B)), 256, 0, n->stream>>>(
          d.g, s.g, B * d.c, n->H(d.level), n->W(d.level));
    } else {
      k_up_back<<<blocks_for(n->elems(s, B)), 256, 0, n->stream>>>(
          d.g, s.g, B * s.c, n->H(s.level), n->W(s.level));
    }
  }
  return cuda_ok(cudaGetLastError(), "network backward");
}

// out32 = prediction; loss = sum over valid points (h < R, w < np) of
// (out - target)^2 / (B R np); gout = its gradient.
__global__ void k_loss(const float *out, const float *target, float *gout, float *loss, int B,
                       int H, int W, int R, int np) {
  const size_t n = (size_t)B * H * W;
  const float scale = 1.f / ((float)B * R * np);
  float acc = 0.f;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(i % ((size_t)H * W)), h = r / W, w = r - h * W;
    float gv = 0.f;
    if (h < R && w < np) {
      const float d = out[i] - target[i];
      acc += d * d * scale;
      gv = 2.f * d * scale;
    }
    gout[i] = gv;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc);
}

__global__ void k_to_bf16(const float *in, bf16 *out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16(in[i]);
}

void net_free(gcs_mi_net *n) {
  if (!n) return;
  cudaFree(n->pool);
  delete n;
}

// Packed parameters (host order): for every convolution, output channel
// co: the 9 cin weights [ci][tap] then the bias.
size_t packed_count(const gcs_mi_net *n) {
  size_t c = 0;
  for (const Conv &v : n->convs) c += (size_t)v.cout * (9 * v.cin + 1);
  return c;
}

}  // namespace

extern "C" {

int gcs_mi_net_create(int interior_rows, int longitudes, int max_batch, unsigned seed,
                      gcs_mi_net **out) {
  if (!out || interior_rows < 1 || longitudes < 4 || max_batch < 1 || interior_rows > 4096 ||
      longitudes > 16384 || max_batch > 256) {
    set_api_error("invalid network geometry");
    return -1;
  }
  if (!configure_kernels()) return -1;
  gcs_mi_net *n = new gcs_mi_net();
  n->R = interior_rows;
  n->np = longitudes;
  n->H0 = round_up(interior_rows, 8);
  n->W0 = round_up(longitudes, 32);
  n->max_batch = max_batch;
  build_graph(n);
  // memory: parameters (w, gw, m, v FP32; wb BF16), the backward-data
  // weights, activations (BF16) and gradients (FP32) of every tensor, the
  // FP32 output and its gradient, the ReLU-masked gradient and the loss
  size_t wt = 0, act = 0, maxe = 0;
  for (const Conv &c : n->convs) wt = std::max(wt, (size_t)c.Mpt * c.Kpt);
  for (const Tensor &x : n->t) {
    const size_t e = n->elems(x, max_batch);
    act += e;
    maxe = std::max(maxe, e);
  }
  n->wt_len = wt;
  n->max_act = maxe;
  const size_t out_e = (size_t)max_batch * n->H0 * n->W0;
  const size_t bytes = n->nparam * (4 * sizeof(float) + sizeof(bf16)) + wt * sizeof(bf16) +
                       act * (sizeof(bf16) + sizeof(float)) + 2 * out_e * sizeof(float) +
                       maxe * sizeof(float) + 64 * sizeof(float) + 64 * 256;
  if (!cuda_ok(cudaMalloc(&n->pool, bytes), "cudaMalloc") ||
      !cuda_ok(cudaMemset(n->pool, 0, bytes), "cudaMemset")) {
    net_free(n);
    return -1;
  }
  char *q = static_cast<char *>(n->pool);
  auto take = [&](size_t b) {
    char *r = q;
    q += (b + 255) / 256 * 256;
    return r;
  };
  n->w = (float *)take(n->nparam * sizeof(float));
  n->gw = (float *)take(n->nparam * sizeof(float));
  n->m = (float *)take(n->nparam * sizeof(float));
  n->v = (float *)take(n->nparam * sizeof(float));
  n->wb = (bf16 *)take(n->nparam * sizeof(bf16));
  n->wt = (bf16 *)take(wt * sizeof(bf16));
  for (Tensor &x : n->t) {
    x.a = (bf16 *)take(n->elems(x, max_batch) * sizeof(bf16));
    x.g = (float *)take(n->elems(x, max_batch) * sizeof(float));
  }
  n->out32 = (float *)take(out_e * sizeof(float));
  n->gout = (float *)take(out_e * sizeof(float));
  n->gm = (float *)take(maxe * sizeof(float));
  n->loss = (float *)take(64 * sizeof(float));
  // He initialisation, biases zero
  std::mt19937 rng(seed);
  std::vector<float> hw(n->nparam, 0.f);
  for (const Conv &c : n->convs) {
    std::normal_distribution<float> nd(0.f, std::sqrt(2.f / (9.f * c.cin)) *
                                                 (c.final_layer ? 0.1f : 1.f));
    for (int co = 0; co < c.cout; ++co)
      for (int k = 0; k < 9 * c.cin; ++k) hw[c.off + (size_t)co * c.Kp + k] = nd(rng);
  }
  std::vector<bf16> hb(n->nparam);
  for (size_t i = 0; i < n->nparam; ++i) hb[i] = __float2bfloat16(hw[i]);
  if (!cuda_ok(cudaMemcpy(n->w, hw.data(), n->nparam * sizeof(float), cudaMemcpyHostToDevice),
               "cudaMemcpy") ||
      !cuda_ok(cudaMemcpy(n->wb, hb.data(), n->nparam * sizeof(bf16), cudaMemcpyHostToDevice),
               "cudaMemcpy")) {
    net_free(n);
    return -1;
  }
  *out = n;
  return 0;
}

void gcs_mi_net_destroy(gcs_mi_net *n) {
  if (n) cudaDeviceSynchronize();
  net_free(n);
}

int gcs_mi_net_info(const gcs_mi_net *n, int *H0, int *W0, int *params, int *in_channels) {
  if (!n) return -1;
  if (H0) *H0 = n->H0;
  if (W0) *W0 = n->W0;
  if (params) *params = (int)packed_count(n);
  if (in_channels) *in_channels = kInChannels;
  return 0;
}

// Packed parameters to / from host memory (count = gcs_mi_net_info's params).
int gcs_mi_net_get_params(gcs_mi_net *n, float *host, int count, int gradients) {
  if (!n || !host || count != (int)packed_count(n)) return -1;
  std::vector<float> all(n->nparam);
  if (!cuda_ok(cudaMemcpy(all.data(), gradients ? n->gw : n->w, n->nparam * sizeof(float),
                          cudaMemcpyDeviceToHost),
               "cudaMemcpy"))
    return -1;
  size_t o = 0;
  for (const Conv &c : n->convs)
    for (int co = 0; co < c.cout; ++co)
      for (int k = 0; k <= 9 * c.cin; ++k) host[o++] = all[c.off + (size_t)co * c.Kp + k];
  return 0;
}

int gcs_mi_net_set_params(gcs_mi_net *n, const float *host, int count) {
  if (!n || !host || count != (int)packed_count(n)) return -1;
  std::vector<float> all(n->nparam, 0.f);
  size_t o = 0;
  for (const Conv &c : n->convs)
    for (int co = 0; co < c.cout; ++co)
      for (int k = 0; k <= 9 * c.cin; ++k) all[c.off + (size_t)co * c.Kp + k] = host[o++];
  std::vector<bf16> hb(n->nparam);
  for (size_t i = 0; i < n->nparam; ++i) hb[i] = __float2bfloat16(all[i]);
  n->adam_t = 0;
  return cuda_ok(cudaMemcpy(n->w, all.data(), n->nparam * sizeof(float), cudaMemcpyHostToDevice),
                 "cudaMemcpy") &&
                 cuda_ok(cudaMemcpy(n->wb, hb.data(), n->nparam * sizeof(bf16),
                                    cudaMemcpyHostToDevice),
                         "cudaMemcpy") &&
                 cuda_ok(cudaMemset(n->m, 0, n->nparam * sizeof(float)), "cudaMemset") &&
                 cuda_ok(cudaMemset(n->v, 0, n->nparam * sizeof(float)), "cudaMemset")
             ? 0
             : -1;
}

// Forward pass of B samples: inputs [B][4][H0][W0] FP32 (device), outputs
// [B][H0][W0] FP32 (device); asynchronous on the network's stream (NULL).
int gcs_mi_net_forward(gcs_mi_net *n, const float *inputs, int B, float *outputs) {
  if (!n || !inputs || B < 1 || B > n->max_batch) return -1;
  const size_t ne = n->elems(n->t[0], B);
  k_to_bf16<<<blocks_for(ne), 256, 0, n->stream>>>(inputs, n->t[0].a, ne);
  if (!forward(n, B)) return -1;
  if (outputs &&
      !cuda_ok(cudaMemcpyAsync(outputs, n->out32, (size_t)B * n->H0 * n->W0 * sizeof(float),
                               cudaMemcpyDeviceToDevice, n->stream),
               "cudaMemcpyAsync"))
    return -1;
  return 0;
}

// Loss and parameter gradients for inputs / targets ([B][H0][W0], device),
// then (update != 0) one Adam step with learning rate lr.  The loss is
// returned through *loss (host, synchronous).
int gcs_mi_net_train_step(gcs_mi_net *n, const float *inputs, const float *targets, int B,
                          float lr, int update, float *loss) {
  if (!n || !inputs || !targets || B < 1 || B > n->max_batch) return -1;
  if (gcs_mi_net_forward(n, inputs, B, nullptr) != 0) return -1;
  if (!cuda_ok(cudaMemsetAsync(n->loss, 0, sizeof(float), n->stream), "cudaMemsetAsync"))
    return -1;
  const size_t oe = (size_t)B * n->H0 * n->W0;
  k_loss<<<blocks_for(oe), 256, 0, n->stream>>>(n->out32, targets, n->gout, n->loss, B, n->H0,
                                                n->W0, n->R, n->np);
  if (!backward(n, B)) return -1;
  if (update) {
    ++n->adam_t;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)n->adam_t),
                c2 = 1.f - std::pow(b2, (float)n->adam_t);
    k_adam<<<blocks_for(n->nparam), 256, 0, n->stream>>>(n->w, n->gw, n->m, n->v, n->wb,
                                                         n->nparam, lr, b1, b2, 1e-8f, c1, c2);
  }
  float h = 0.f;
  if (!cuda_ok(cudaMemcpyAsync(&h, n->loss, sizeof(float), cudaMemcpyDeviceToHost, n->stream),
               "cudaMemcpyAsync") ||
      !cuda_ok(cudaStreamSynchronize(n->stream), "network training step"))
    return -1;
  if (loss) *loss = h;
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Flexible GMRES on the conductance-tensor system with the network as the
// (right) preconditioner.
//
// The system is the reference's reduced one (nonorthogonal_mi.c:776-1029):
// unknown 0 the pole, unknown 1 + i np + j interior row i (colatitude row
// i + 1), longitude j.  Every row is divided by its scale -- sin(theta) for
// an interior row, ps / sqrt(np) for the pole (ps the constant-Pedersen
// pole scale of nonorthogonal_mi.c:324-334) -- so the 2-norm of the scaled
// residual is the reference's residual norm (:415-431) and its target
// max(abs_tol, rel_tol max(|u|, 1)) applies unchanged.  All vectors and the
// orthogonalisation (classical Gram-Schmidt, two passes) are FP64 on the
// device; the host reads one Hessenberg column per iteration.  Convergence
// is judged on the true FP64 residual, recomputed at every restart.
namespace {

constexpr int kRestartLen = 40;
constexpr int kDotBlocks = 128;

struct LpSys {
  int np, nt, R, n;
  double dth, dph, neg_r2, pole_sin, pole_inc2, pole_scale;
  const double *fac, *sp, *sh, *pot;  // natural nt x np
  const double *row_s, *row_sl, *row_il, *row_su, *row_iu, *row_inc;  // nt each
  double *dg, *lo, *up, *ll, *lu;     // R x np
  double *pe, *dg0;                   // np, 1
  double *scale;                      // n: row scale of the reduced system
  double *b, *x;                      // n: scaled right-hand side, iterate
  // ring coarse operator T = E^T A' E (E: one value per colatitude ring and
  // the pole), tridiagonal; Thomas factors
  double *tl, *td, *tu, *cp, *cm;     // R + 1 each
};

constexpr int kMaxRingRows = 2048;    // ring rows of the one-block ring solve

// Coefficients (nonorthogonal_mi.c:776-865), scaled right-hand side and the
// initial guess (:999-1029) of the reduced system.
__global__ void k_lp_setup(LpSys S) {
  const int np = S.np, R = S.R;
  const size_t nq = (size_t)R * np;
  __shared__ double ppm_s;
  if (threadIdx.x < 32) {
    double m = 0.0;
    for (int j = threadIdx.x; j < np; j += 32) m += S.sp[j];
    for (int o = 16; o > 0; o >>= 1) m += __shfl_xor_sync(0xffffffffu, m, o);
    if (threadIdx.x == 0) ppm_s = m / (double)np;
  }
  __syncthreads();
  const double ppm = ppm_s;
  const size_t gid = blockIdx.x * (size_t)blockDim.x + threadIdx.x,
               gsz = (size_t)gridDim.x * blockDim.x;
  for (size_t j = gid; j < (size_t)np; j += gsz) {
    const double fp = 0.5 * (ppm + S.sp[(size_t)np + j]);
    S.pe[j] = S.pole_sin * fp / (S.pole_inc2 * S.dth * S.dth);
  }
  for (size_t q = gid; q < nq; q += gsz) {
    const int row = (int)(q / np), j = (int)(q - (size_t)row * np), i = row + 1;
    const int jm = j == 0 ? np - 1 : j - 1, jp = j + 1 == np ? 0 : j + 1;
    const size_t full = (size_t)i * np + j;
    const double *P = S.sp, *H = S.sh;
    const double dth2 = S.dth * S.dth, dph2 = S.dph * S.dph;
    const double lower = S.row_sl[i] * 0.5 * (P[full] + P[full - np]) / (S.row_il[i] * dth2);
    const double upper = S.row_su[i] * 0.5 * (P[full] + P[full + np]) / (S.row_iu[i] * dth2);
    const double llo = 0.5 * (P[full] + P[(size_t)i * np + jm]) / (S.row_s[i] * dph2);
    const double lup = 0.5 * (P[full] + P[(size_t)i * np + jp]) / (S.row_s[i] * dph2);
    const double dft = (-H[full + np] / S.row_inc[i + 1] + H[full - np] / S.row_inc[i - 1]) /
                       (2.0 * S.dth);
    const double dfp = (-H[(size_t)i * np + jp] / S.row_inc[i] +
                        H[(size_t)i * np + jm] / S.row_inc[i]) /
                       (2.0 * S.dph);
    S.dg[q] = lower + upper + llo + lup;
    S.lo[q] = -lower - dfp / (2.0 * S.dth);
    S.up[q] = -upper + dfp / (2.0 * S.dth);
    S.ll[q] = -llo + dft / (2.0 * S.dph);
    S.lu[q] = -lup - dft / (2.0 * S.dph);
    S.scale[1 + q] = S.row_s[i];
    S.b[1 + q] = S.neg_r2 * S.fac[full] * S.row_inc[i];  // = rhs / sin(theta)
    const double g = S.pot[full];
    S.x[1 + q] = isfinite(g) ? g : 0.0;
  }
  if (gid == 0) {
    double m = 0.0;
    for (int j = 0; j < np; ++j) {
      const double g = S.pot[j];
      if (isfinite(g)) m += g / (double)np;
    }
    S.x[0] = m;
    S.b[0] = 0.0;
    S.scale[0] = S.pole_scale;
  }
}

// dg0 = sum_j pe_j (after k_lp_setup).
__global__ void k_lp_dg0(LpSys S) {
  double a = 0.0;
  for (int j = threadIdx.x; j < S.np; j += 32) a += S.pe[j];
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if (threadIdx.x == 0) *S.dg0 = a;
}

// y = S^-1 A p (nonorthogonal_mi.c:867-900), or y = c - S^-1 A p when c.
__global__ void k_lp_apply(LpSys S, const double *p, double *y, const double *c) {
  const int np = S.np, R = S.R;
  const size_t nq = (size_t)R * np;
  const size_t gid = blockIdx.x * (size_t)blockDim.x + threadIdx.x,
               gsz = (size_t)gridDim.x * blockDim.x;
  for (size_t q = gid; q < nq; q += gsz) {
    const int row = (int)(q / np), j = (int)(q - (size_t)row * np);
    const int jm = j == 0 ? np - 1 : j - 1, jp = j + 1 == np ? 0 : j + 1;
    const double lv = row == 0 ? p[0] : p[1 + q - np];
    const double uv = row + 1 < R ? p[1 + q + np] : 0.0;
    const double a = S.dg[q] * p[1 + q] + S.lo[q] * lv + S.up[q] * uv +
                     S.ll[q] * p[1 + (size_t)row * np + jm] +
                     S.lu[q] * p[1 + (size_t)row * np + jp];
    const double v = a / S.scale[1 + q];
    y[1 + q] = c ? c[1 + q] - v : v;
  }
  if (blockIdx.x == 0) {
    __shared__ double part[32];
    double a = 0.0;
    for (int j = threadIdx.x; j < np; j += blockDim.x) a += S.pe[j] * p[1 + j];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x < 32) {
      a = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0;
      for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
      if (threadIdx.x == 0) {
        const double v = (*S.dg0 * p[0] - a) / S.scale[0];
        y[0] = c ? c[0] - v : v;
      }
    }
  }
}

// part[blk][k] = sum over the block's entries of w V_k, k < cnt (w itself
// for k = -1 slot: cnt columns then |w|^2 in column cnt when norm).
__global__ void k_lp_dots(const double *w, const double *V, size_t n, int cnt, int norm,
                          double *part) {
  __shared__ double red[32][kRestartLen + 2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int cols = cnt + (norm ? 1 : 0);
  for (int k = 0; k < cols; ++k) {
    const double *v = k < cnt ? V + (size_t)k * n : w;
    double a = 0.0;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
         q += (size_t)gridDim.x * blockDim.x)
      a += w[q] * v[q];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) red[warp][k] = a;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < cols; k += blockDim.x) {
    double a = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) a += red[q][k];
    part[(size_t)blockIdx.x * (kRestartLen + 2) + k] = a;
  }
}

// out[k] (+)= sum over blocks of part[.][k], k < cols; one warp per column.
__global__ void k_lp_sum(const double *part, int blocks, int cols, double *out, int accumulate) {
  const int k = blockIdx.x;
  if (k >= cols) return;
  double a = 0.0;
  for (int b = threadIdx.x; b < blocks; b += 32) a += part[(size_t)b * (kRestartLen + 2) + k];
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if (threadIdx.x == 0) out[k] = accumulate ? out[k] + a : a;
}

// w -= sum_k h[k] V_k, k < cnt
__global__ void k_lp_orth(double *w, const double *V, size_t n, int cnt, const double *h) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    double a = w[q];
    for (int k = 0; k < cnt; ++k) a -= h[k] * V[(size_t)k * n + q];
    w[q] = a;
  }
}

// out = in / sqrt(nrm2[0]) (nrm2 on the device)
__global__ void k_lp_normalise(const double *in, double *out, size_t n, const double *nrm2) {
  const double s = 1.0 / sqrt(*nrm2);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x)
    out[q] = in[q] * s;
}

// x += sum_k y[k] Z_k
__global__ void k_lp_update(double *x, const double *Z, size_t n, int cnt, const double *y) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    double a = x[q];
    for (int k = 0; k < cnt; ++k) a += y[k] * Z[(size_t)k * n + q];
    x[q] = a;
  }
}

// Network input channel 0 from a unit-norm Krylov vector: unit RMS over
// the interior, periodic continuation in the padding columns, zero rows
// below; channels 1-3 are the fixed features.
__global__ void k_lp_pack(const double *v, float *in, int R, int np, int H0, int W0,
                          const double *nrm2, double count) {
  const double s = sqrt(count / *nrm2);
  const size_t n = (size_t)H0 * W0;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    const int h = (int)(q / W0), w = (int)(q - (size_t)h * W0);
    in[q] = h < R ? (float)(s * v[1 + (size_t)h * np + w % np]) : 0.f;
  }
}

// Z_k from the network output: interior points, the pole the mean of the
// first interior row.  One block.
__global__ void k_lp_unpack(const float *out, double *z, int R, int np, int W0,
                            const double *nrm2, double count) {
  __shared__ double part[32];
  const double s = sqrt(*nrm2 / count);  // the network's output is in units of the input RMS
  double a = 0.0;
  for (int j = threadIdx.x; j < np; j += blockDim.x) a += out[j];
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = a;
  for (size_t q = threadIdx.x; q < (size_t)R * np; q += blockDim.x) {
    const int h = (int)(q / np), w = (int)(q - (size_t)h * np);
    z[1 + q] += s * out[(size_t)h * W0 + w];
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    a = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (threadIdx.x == 0) z[0] += s * a / (double)np;
  }
}

// z = v scale / diag: the Jacobi step of the scaled system.
__global__ void k_lp_jacobi(const LpSys S, const double *v, double *z) {
  const size_t nq = (size_t)S.R * S.np;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q <= nq;
       q += (size_t)gridDim.x * blockDim.x)
    z[q] = q == 0 ? v[0] * S.scale[0] / *S.dg0 : v[q] * S.scale[q] / S.dg[q - 1];
}

// z += omega D'^-1 r (damped Jacobi step of the scaled system)
__global__ void k_lp_jacobi_add(const LpSys S, const double *r, double *z, double omega) {
  const size_t nq = (size_t)S.R * S.np;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q <= nq;
       q += (size_t)gridDim.x * blockDim.x)
    z[q] += omega * (q == 0 ? r[0] * S.scale[0] / *S.dg0 : r[q] * S.scale[q] / S.dg[q - 1]);
}

// Ring coarse operator: row 0 the pole, row i >= 1 interior row i - 1 with
// its coefficients summed over longitude (the Hall terms cancel in the
// sums around a ring).  One block per coarse row.
__global__ void k_lp_ring_setup(LpSys S) {
  const int i = blockIdx.x, np = S.np;
  __shared__ double part[3][32];
  double a = 0.0, l = 0.0, u = 0.0;
  if (i == 0) {
    for (int j = threadIdx.x; j < np; j += blockDim.x) a += S.pe[j];
  } else {
    const int row = i - 1;
    for (int j = threadIdx.x; j < np; j += blockDim.x) {
      const size_t q = (size_t)row * np + j;
      a += S.dg[q] + S.ll[q] + S.lu[q];
      l += S.lo[q];
      u += S.up[q];
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    l += __shfl_xor_sync(0xffffffffu, l, o);
    u += __shfl_xor_sync(0xffffffffu, u, o);
  }
  if ((threadIdx.x & 31) == 0) {
    part[0][threadIdx.x >> 5] = a;
    part[1][threadIdx.x >> 5] = l;
    part[2][threadIdx.x >> 5] = u;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    a = l = u = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a += part[0][w];
      l += part[1][w];
      u += part[2][w];
    }
    if (i == 0) {
      S.td[0] = *S.dg0 / S.scale[0];
      S.tl[0] = 0.0;
      S.tu[0] = -a / S.scale[0];
    } else {
      const double s = S.row_s[i];
      S.td[i] = a / s;
      S.tl[i] = l / s;
      S.tu[i] = i < S.R ? u / s : 0.0;
    }
  }
}

// Thomas factors of the ring operator (one thread).
__global__ void k_lp_ring_factor(LpSys S) {
  double prev = 0.0;
  for (int i = 0; i <= S.R; ++i) {
    const double m = S.td[i] - S.tl[i] * prev;
    S.cm[i] = 1.0 / m;
    prev = S.tu[i] / m;
    S.cp[i] = prev;
  }
}

// z (+)= E T^-1 E^T r: ring sums, the tridiagonal solve, prolongation.
// One block.
__global__ void __launch_bounds__(1024) k_lp_ring_solve(const LpSys S, const double *r,
                                                        double *z, int accumulate) {
  __shared__ double c[kMaxRingRows + 1];
  const int np = S.np, R = S.R, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  for (int i = warp; i <= R; i += nw) {
    double a = 0.0;
    if (i == 0) {
      a = lane == 0 ? r[0] : 0.0;
    } else {
      for (int j = lane; j < np; j += 32) a += r[1 + (size_t)(i - 1) * np + j];
    }
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) c[i] = a;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double prev = 0.0;
    for (int i = 0; i <= R; ++i) {
      prev = (c[i] - S.tl[i] * prev) * S.cm[i];
      c[i] = prev;
    }
    for (int i = R - 1; i >= 0; --i) c[i] -= S.cp[i] * c[i + 1];
  }
  __syncthreads();
  const size_t n = 1 + (size_t)R * np;
  for (size_t q = threadIdx.x; q < n; q += blockDim.x) {
    const double v = q == 0 ? c[0] : c[1 + (q - 1) / np];
    z[q] = accumulate ? z[q] + v : v;
  }
}

// Network feature channels 1-3: log(Sigma_P / 5 S), Sigma_H / Sigma_P,
// sin(theta), on the padded grid.
__global__ void k_lp_features(const LpSys S, float *in, int H0, int W0) {
  const size_t n = (size_t)H0 * W0;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    const int h = (int)(q / W0), w = (int)(q - (size_t)h * W0);
    float f1 = 0.f, f2 = 0.f, f3 = 0.f;
    if (h < S.R) {
      const size_t full = (size_t)(h + 1) * S.np + w % S.np;
      f1 = (float)log(S.sp[full] / 5.0);
      f2 = (float)(S.sh[full] / S.sp[full]);
      f3 = (float)S.row_s[h + 1];
    }
    in[n + q] = f1;
    in[2 * n + q] = f2;
    in[3 * n + q] = f3;
  }
}

// natural potential from the reduced iterate: pole row, interior, 0 at the
// low-latitude boundary (nonorthogonal_mi.c:1130-1139)
__global__ void k_lp_expand(const double *x, double *pot, int R, int np, int nt) {
  const size_t n = (size_t)nt * np;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q / np);
    pot[q] = i == 0 ? x[0] : i == nt - 1 ? 0.0 : x[1 + q - (size_t)np];
  }
}

double cos_incl(double th, int hemisphere) {
  const double c = cos(th);
  return (double)hemisphere * 2.0 * c / sqrt(1.0 + 3.0 * c * c);
}
double incl2(double a) {
  const double c = cos(a);
  return 4.0 * c * c / (1.0 + 3.0 * c * c);
}

}  // namespace

extern "C" int gamera_mi_solve_conductance_tensor(const gamera_mi_solver_config *config,
                                                  const double *fac_a_m2,
                                                  const double *pedersen, const double *hall,
                                                  double *potential_v,
                                                  gamera_mi_solver_stats *stats);

// Device state of one learned-preconditioner solve on one grid.
struct gcs_mi_learned_plan {
  gamera_mi_solver_config config{};
  int np = 0, nt = 0, R = 0;
  size_t n = 0;
  LpSys S{};
  void *pool = nullptr;
  double *V = nullptr, *Z = nullptr, *w = nullptr, *part = nullptr, *h = nullptr,
         *hy = nullptr, *nrm = nullptr, *pot = nullptr, *fac = nullptr, *sp = nullptr,
         *sh = nullptr, *r = nullptr, *t = nullptr, *rn = nullptr;
  float *net_in = nullptr, *net_out = nullptr;
  double *host = nullptr;  // pinned: the last Hessenberg column and norms
};

namespace {

void lp_free(gcs_mi_learned_plan *p) {
  if (!p) return;
  cudaFree(p->pool);
  cudaFreeHost(p->host);
  delete p;
}

gcs_mi_learned_plan *lp_create(const gamera_mi_solver_config *c, const gcs_mi_net *net) {
  if (!c || c->colatitude_count < 3U || c->longitude_count < 4U ||
      c->colatitude_count - 2U > (unsigned)kMaxRingRows ||
      (net && (net->R != (int)c->colatitude_count - 2 || net->np != (int)c->longitude_count))) {
    set_api_error("learned MI solve: network grid and configuration differ");
    return nullptr;
  }
  gcs_mi_learned_plan *p = new gcs_mi_learned_plan();
  p->config = *c;
  p->np = (int)c->longitude_count;
  p->nt = (int)c->colatitude_count;
  p->R = p->nt - 2;
  p->n = 1 + (size_t)p->R * p->np;
  const size_t nodes = (size_t)p->np * p->nt, nq = (size_t)p->R * p->np, n = p->n;
  const int H0 = round_up(p->R, 8), W0 = round_up(p->np, 32);
  const size_t doubles = 5 * nq + p->np + 8 + 5 * n + (2 * (size_t)kRestartLen + 2) * n +
                         5 * ((size_t)p->R + 1 + 32) + 16 +
                         (size_t)kDotBlocks * (kRestartLen + 2) + 2 * (kRestartLen + 2) +
                         4 * nodes + 6 * (size_t)p->nt;
  const size_t floats = 5 * (size_t)H0 * W0;
  if (!cuda_ok(cudaMalloc(&p->pool, doubles * sizeof(double) + floats * sizeof(float) + 4096),
               "cudaMalloc") ||
      !cuda_ok(cudaMallocHost(&p->host, 4 * (kRestartLen + 2) * sizeof(double)),
               "cudaMallocHost")) {
    lp_free(p);
    return nullptr;
  }
  double *q = static_cast<double *>(p->pool);
  auto take = [&](size_t k) {
    double *r = q;
    q += (k + 31) / 32 * 32;
    return r;
  };
  LpSys &S = p->S;
  S.dg = take(nq);
  S.lo = take(nq);
  S.up = take(nq);
  S.ll = take(nq);
  S.lu = take(nq);
  S.pe = take(p->np);
  S.tl = take(p->R + 1);
  S.td = take(p->R + 1);
  S.tu = take(p->R + 1);
  S.cp = take(p->R + 1);
  S.cm = take(p->R + 1);
  p->r = take(n);
  p->t = take(n);
  p->rn = take(8);
  S.dg0 = take(8);
  S.scale = take(n);
  S.b = take(n);
  S.x = take(n);
  p->V = take((size_t)(kRestartLen + 1) * n);
  p->Z = take((size_t)kRestartLen * n);
  p->w = take(n);
  p->part = take((size_t)kDotBlocks * (kRestartLen + 2));
  p->h = take(kRestartLen + 2);
  p->hy = take(kRestartLen + 2);
  p->nrm = take(8);
  p->fac = take(nodes);
  p->sp = take(nodes);
  p->sh = take(nodes);
  p->pot = take(nodes);
  double *rows = take(6 * (size_t)p->nt);
  p->net_in = reinterpret_cast<float *>(q);
  p->net_out = p->net_in + 4 * (size_t)H0 * W0;
  const int nt = p->nt;
  const double dth = c->maximum_colatitude / (double)(nt - 1);
  std::vector<double> hr(6 * (size_t)nt);
  for (int i = 0; i < nt; ++i) {
    const double th = (double)i * dth, lth = th - 0.5 * dth, uth = th + 0.5 * dth;
    hr[i] = sin(th);
    hr[nt + i] = sin(lth);
    hr[2 * nt + i] = incl2(lth);
    hr[3 * nt + i] = sin(uth);
    hr[4 * nt + i] = incl2(uth);
    hr[5 * nt + i] = cos_incl(th, c->hemisphere);
  }
  if (!cuda_ok(cudaMemcpy(rows, hr.data(), hr.size() * sizeof(double), cudaMemcpyHostToDevice),
               "cudaMemcpy")) {
    lp_free(p);
    return nullptr;
  }
  S.row_s = rows;
  S.row_sl = rows + nt;
  S.row_il = rows + 2 * nt;
  S.row_su = rows + 3 * nt;
  S.row_iu = rows + 4 * nt;
  S.row_inc = rows + 5 * nt;
  S.np = p->np;
  S.nt = nt;
  S.R = p->R;
  S.n = (int)n;
  S.dth = dth;
  S.dph = 2.0 * acos(-1.0) / (double)p->np;
  S.neg_r2 = -(c->ionosphere_radius_m * c->ionosphere_radius_m);
  const double th = 0.5 * dth;
  S.pole_sin = sin(th);
  S.pole_inc2 = incl2(th);
  const double ps = (double)p->np * (sin(th) * c->pedersen_siemens / (incl2(th) * dth * dth));
  S.pole_scale = ps / sqrt((double)p->np);
  S.fac = p->fac;
  S.sp = p->sp;
  S.sh = p->sh;
  S.pot = p->pot;
  return p;
}

unsigned lp_blocks(size_t n) {
  const size_t b = (n + 255) / 256;
  return (unsigned)(b > 1184 ? 1184 : b);
}

// h[0..cnt) (+)= (w, V_k); with norm, h[cnt] = |w|^2
void lp_dots(gcs_mi_learned_plan *p, const double *w, int cnt, int norm, double *out,
             int accumulate) {
  k_lp_dots<<<kDotBlocks, 256>>>(w, p->V, p->n, cnt, norm, p->part);
  k_lp_sum<<<cnt + (norm ? 1 : 0), 32>>>(p->part, kDotBlocks, cnt + (norm ? 1 : 0), out,
                                         accumulate);
}

// out = L v, the left preconditioner: Jacobi (method 1) or the two-level
// step (methods 0 and 2): a coarse correction on ring means, E T^-1 E^T
// (one value per colatitude ring and the pole), two damped Jacobi steps and
// the coarse correction again, each on the current residual.  Linear.
// Uses p->r.
void lp_left(gcs_mi_learned_plan *p, int method, const double *v, double *z) {
  LpSys &S = p->S;
  const unsigned nb = lp_blocks(p->n);
  if (method == 1) {
    k_lp_jacobi<<<nb, 256>>>(S, v, z);
    return;
  }
  const int ring_threads = 1024;
  k_lp_ring_solve<<<1, ring_threads>>>(S, v, z, 0);
  k_lp_apply<<<nb, 256>>>(S, z, p->r, v);
  k_lp_jacobi_add<<<nb, 256>>>(S, p->r, z, 0.7);
  k_lp_apply<<<nb, 256>>>(S, z, p->r, v);
  k_lp_jacobi_add<<<nb, 256>>>(S, p->r, z, 0.7);
  k_lp_apply<<<nb, 256>>>(S, z, p->r, v);
  k_lp_ring_solve<<<1, ring_threads>>>(S, p->r, z, 1);
}

// z = N v, the flexible right preconditioner: the network (method 0) on v
// at unit RMS, its output in units of that RMS; the identity otherwise.
bool lp_right(gcs_mi_learned_plan *p, gcs_mi_net *net, int method, const double *v,
              double *z) {
  const size_t n = p->n;
  if (method != 0)
    return cuda_ok(cudaMemcpyAsync(z, v, n * sizeof(double), cudaMemcpyDeviceToDevice),
                   "cudaMemcpyAsync");
  const int H0 = round_up(p->R, 8), W0 = round_up(p->np, 32);
  lp_dots(p, v, 0, 1, p->rn, 0);
  k_lp_pack<<<lp_blocks((size_t)H0 * W0), 256>>>(v, p->net_in, p->R, p->np, H0, W0, p->rn,
                                                 (double)n);
  if (gcs_mi_net_forward(net, p->net_in, 1, nullptr) != 0) return false;
  if (!cuda_ok(cudaMemsetAsync(z, 0, n * sizeof(double)), "cudaMemsetAsync")) return false;
  k_lp_unpack<<<1, 256>>>(net->out32, z, p->R, p->np, W0, p->rn, (double)n);
  return true;
}

// Flexible GMRES(40) on L A x = L b with the right preconditioner N
// (methods: 0 two-level L and the network N, 1 Jacobi L, 2 two-level L and
// N = I).  The left factor is linear, so the Krylov space is that of the
// well-conditioned L A; the inner iteration stops at a reduction of |L r|
// proportional to the true reduction still needed, and every restart
// recomputes the true residual |b - A x| (the reference's norm) and judges
// convergence on it.  Returns 0 converged, 1 not converged, -1 error.
int lp_solve(gcs_mi_learned_plan *p, gcs_mi_net *net, int method, gamera_mi_solver_stats *st) {
  LpSys &S = p->S;
  const size_t n = p->n;
  const unsigned nb = lp_blocks(n);
  const int H0 = round_up(p->R, 8), W0 = round_up(p->np, 32);
  k_lp_setup<<<lp_blocks((size_t)p->R * p->np), 256>>>(S);
  k_lp_dg0<<<1, 32>>>(S);
  if (method != 1) {
    k_lp_ring_setup<<<p->R + 1, 256>>>(S);
    k_lp_ring_factor<<<1, 1>>>(S);
  }
  if (method == 0) k_lp_features<<<lp_blocks((size_t)H0 * W0), 256>>>(S, p->net_in, H0, W0);
  double *hh = p->host;
  // target from |u| = |b| (scaled right-hand side, interior only: b[0] = 0)
  k_lp_dots<<<kDotBlocks, 256>>>(S.b, p->V, n, 0, 1, p->part);
  k_lp_sum<<<1, 32>>>(p->part, kDotBlocks, 1, p->h, 0);
  if (!cuda_ok(cudaMemcpy(hh, p->h, sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy"))
    return -1;
  const gamera_mi_solver_config &c = p->config;
  const double target =
      fmax(c.absolute_tolerance, c.relative_tolerance * fmax(sqrt(fmax(0.0, hh[0])), 1.0));
  const int max_iter = c.maximum_iterations;
  std::vector<double> H((size_t)(kRestartLen + 1) * kRestartLen), cs(kRestartLen),
      sn(kRestartLen), g(kRestartLen + 1), y(kRestartLen);
  int iters = 0;
  double initial = -1.0, res = 0.0;
  for (;;) {
    // true residual r = b - A x, |r|^2; s = L r into V_0, |s|^2
    k_lp_apply<<<nb, 256>>>(S, S.x, p->t, S.b);
    lp_dots(p, p->t, 0, 1, p->h, 0);
    lp_left(p, method, p->t, p->V);
    lp_dots(p, p->V, 0, 1, p->h + 1, 0);
    if (!cuda_ok(cudaMemcpy(hh, p->h, 2 * sizeof(double), cudaMemcpyDeviceToHost),
                 "cudaMemcpy"))
      return -1;
    res = sqrt(fmax(0.0, hh[0]));
    const double beta = sqrt(fmax(0.0, hh[1]));
    if (initial < 0.0) initial = res;
    if (!std::isfinite(res) || !std::isfinite(beta)) return -1;
    if (res <= target || iters >= max_iter || !(beta > 0.0)) break;
    // |L r| reduction matching the true reduction still needed, with margin
    const double inner = 0.3 * beta * target / res;
    k_lp_normalise<<<nb, 256>>>(p->V, p->V, n, p->h + 1);
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int j = 0;
    for (; j < kRestartLen && iters < max_iter; ++j) {
      double *vj = p->V + (size_t)j * n, *zj = p->Z + (size_t)j * n;
      if (!lp_right(p, net, method, vj, zj)) return -1;
      k_lp_apply<<<nb, 256>>>(S, zj, p->t, nullptr);
      lp_left(p, method, p->t, p->w);
      // classical Gram-Schmidt, twice; then |w|^2
      lp_dots(p, p->w, j + 1, 0, p->h, 0);
      k_lp_orth<<<nb, 256>>>(p->w, p->V, n, j + 1, p->h);
      lp_dots(p, p->w, j + 1, 0, p->hy, 0);
      k_lp_orth<<<nb, 256>>>(p->w, p->V, n, j + 1, p->hy);
      lp_dots(p, p->w, 0, 1, p->nrm, 0);  // |w|^2 of the orthogonalised w
      if (!cuda_ok(cudaMemcpy(hh, p->h, (j + 1) * sizeof(double), cudaMemcpyDeviceToHost),
                   "cudaMemcpy") ||
          !cuda_ok(cudaMemcpy(hh + kRestartLen + 2, p->hy, (j + 1) * sizeof(double),
                              cudaMemcpyDeviceToHost),
                   "cudaMemcpy") ||
          !cuda_ok(cudaMemcpy(hh + 2 * (kRestartLen + 2), p->nrm, sizeof(double),
                              cudaMemcpyDeviceToHost),
                   "cudaMemcpy"))
        return -1;
      ++iters;
      double *col = &H[(size_t)j * (kRestartLen + 1)];
      for (int k = 0; k <= j; ++k) col[k] = hh[k] + hh[kRestartLen + 2 + k];
      const double hn = sqrt(fmax(0.0, hh[2 * (kRestartLen + 2)]));
      col[j + 1] = hn;
      for (int k = 0; k < j; ++k) {
        const double a = cs[k] * col[k] + sn[k] * col[k + 1];
        col[k + 1] = -sn[k] * col[k] + cs[k] * col[k + 1];
        col[k] = a;
      }
      const double r = hypot(col[j], col[j + 1]);
      cs[j] = r > 0.0 ? col[j] / r : 1.0;
      sn[j] = r > 0.0 ? col[j + 1] / r : 0.0;
      col[j] = r;
      col[j + 1] = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      if (!(hn > 0.0) || fabs(g[j + 1]) <= inner) {
        ++j;
        break;
      }
      k_lp_normalise<<<nb, 256>>>(p->w, p->V + (size_t)(j + 1) * n, n, p->nrm);
    }
    // y = H^-1 g (upper triangular), x += Z y
    for (int k = j - 1; k >= 0; --k) {
      double a = g[k];
      for (int l = k + 1; l < j; ++l) a -= H[(size_t)l * (kRestartLen + 1) + k] * y[l];
      y[k] = a / H[(size_t)k * (kRestartLen + 1) + k];
    }
    if (!cuda_ok(cudaMemcpy(p->hy, y.data(), j * sizeof(double), cudaMemcpyHostToDevice),
                 "cudaMemcpy"))
      return -1;
    k_lp_update<<<nb, 256>>>(S.x, p->Z, n, j, p->hy);
  }
  if (!cuda_ok(cudaGetLastError(), "learned MI solve")) return -1;
  if (st) *st = gamera_mi_solver_stats{iters, initial, res, res <= target ? 1 : 0};
  return res <= target ? 0 : 1;
}

std::mutex g_lp_mutex;
gcs_mi_learned_plan *g_lp_cache = nullptr;

}  // namespace

extern "C" {

// Conductance-tensor solve (host arrays, synchronous) by lp_solve's method
// (0 needs the network).  When
// the iteration limit is reached without convergence the reference
// algorithm (gamera_mi_solve_conductance_tensor) continues from the
// iterate; *fallback reports it.  Same arguments, validation and result
// convention as gamera_mi_solve_conductance_tensor.
int gcs_mi_solve_conductance_tensor_learned(gcs_mi_net *net, int method,
                                            const gamera_mi_solver_config *config,
                                            const double *fac_a_m2, const double *pedersen,
                                            const double *hall, double *potential_v,
                                            gamera_mi_solver_stats *stats, int *fallback) {
  if (fallback) *fallback = 0;
  if (method < 0 || method > 2 || (method == 0 && !net)) {
    set_api_error("learned MI solve: method 0 needs a network, methods are 0, 1, 2");
    return -1;
  }
  if (!config || !fac_a_m2 || !pedersen || !hall || !potential_v || config->maximum_iterations <= 0 ||
      !(config->relative_tolerance > 0.0) || config->colatitude_count < 3U ||
      config->longitude_count < 4U) {
    set_api_error("invalid learned MI solve arguments");
    return -1;
  }
  const size_t nodes = (size_t)config->longitude_count * config->colatitude_count;
  for (size_t q = 0; q < nodes; ++q) {
    if (!std::isfinite(pedersen[q]) || !(pedersen[q] > 0.0) || !std::isfinite(hall[q]) ||
        hall[q] < 0.0) {
      set_api_error("invalid conductance");
      return -1;
    }
    if (!std::isfinite(fac_a_m2[q])) {
      set_api_error("non-finite field-aligned current");
      return -1;
    }
  }
  std::lock_guard<std::mutex> lock(g_lp_mutex);
  if (!g_lp_cache || memcmp(&g_lp_cache->config, config, sizeof(*config)) != 0 ||
      (net && (net->R != g_lp_cache->R || net->np != g_lp_cache->np))) {
    gcs_mi_learned_plan *p = lp_create(config, net);
    if (!p) return -1;
    lp_free(g_lp_cache);
    g_lp_cache = p;
  }
  gcs_mi_learned_plan *p = g_lp_cache;
  const size_t bytes = nodes * sizeof(double);
  if (!cuda_ok(cudaMemcpy(p->fac, fac_a_m2, bytes, cudaMemcpyHostToDevice), "cudaMemcpy") ||
      !cuda_ok(cudaMemcpy(p->sp, pedersen, bytes, cudaMemcpyHostToDevice), "cudaMemcpy") ||
      !cuda_ok(cudaMemcpy(p->sh, hall, bytes, cudaMemcpyHostToDevice), "cudaMemcpy") ||
      !cuda_ok(cudaMemcpy(p->pot, potential_v, bytes, cudaMemcpyHostToDevice), "cudaMemcpy"))
    return -1;
  gamera_mi_solver_stats s{};
  const int rc = lp_solve(p, method == 0 ? net : nullptr, method, &s);
  if (rc < 0) return -1;
  k_lp_expand<<<lp_blocks(nodes), 256>>>(p->S.x, p->pot, p->R, p->np, p->nt);
  if (!cuda_ok(cudaMemcpy(potential_v, p->pot, bytes, cudaMemcpyDeviceToHost), "cudaMemcpy"))
    return -1;
  if (rc == 1) {
    // the reference algorithm continues from the iterate
    if (fallback) *fallback = 1;
    gamera_mi_solver_stats f{};
    const int frc = gamera_mi_solve_conductance_tensor(config, fac_a_m2, pedersen, hall,
                                                        potential_v, &f);
    if (stats) *stats = gamera_mi_solver_stats{s.iterations + f.iterations, s.initial_residual,
                                               f.final_residual, f.converged};
    return frc;
  }
  if (stats) *stats = s;
  return 0;
}

}  // extern "C"

extern "C" {

// One application, on host vectors of the reduced system (1 + R np
// doubles), of the scaled operator (what = 1: y = S^-1 A v) or of the
// preconditioner of `method` (what = 0: y = M v), for the configuration and
// conductances given -- the pieces of the learned solve, for checking them
// against a CPU restatement.
int gcs_mi_learned_apply(gcs_mi_net *net, int method, int what,
                         const gamera_mi_solver_config *config, const double *pedersen,
                         const double *hall, const double *v, double *y) {
  if (!config || !pedersen || !hall || !v || !y || method < 0 || method > 2 || what < 0 ||
      what > 2 || (method == 0 && !net && what == 2)) {
    set_api_error("invalid learned MI apply arguments");
    return -1;
  }
  std::lock_guard<std::mutex> lock(g_lp_mutex);
  gcs_mi_learned_plan *p = lp_create(config, net);
  if (!p) return -1;
  const size_t nodes = (size_t)config->longitude_count * config->colatitude_count;
  std::vector<double> zeros(nodes, 0.0);
  int rc = -1;
  const size_t nb = p->n * sizeof(double);
  if (cuda_ok(cudaMemcpy(p->sp, pedersen, nodes * sizeof(double), cudaMemcpyHostToDevice),
              "cudaMemcpy") &&
      cuda_ok(cudaMemcpy(p->sh, hall, nodes * sizeof(double), cudaMemcpyHostToDevice),
              "cudaMemcpy") &&
      cuda_ok(cudaMemcpy(p->fac, zeros.data(), nodes * sizeof(double), cudaMemcpyHostToDevice),
              "cudaMemcpy") &&
      cuda_ok(cudaMemcpy(p->pot, zeros.data(), nodes * sizeof(double), cudaMemcpyHostToDevice),
              "cudaMemcpy")) {
    LpSys &S = p->S;
    const int H0 = round_up(p->R, 8), W0 = round_up(p->np, 32);
    k_lp_setup<<<lp_blocks((size_t)p->R * p->np), 256>>>(S);
    k_lp_dg0<<<1, 32>>>(S);
    k_lp_ring_setup<<<p->R + 1, 256>>>(S);
    k_lp_ring_factor<<<1, 1>>>(S);
    if (method == 0 && what == 0)
      k_lp_features<<<lp_blocks((size_t)H0 * W0), 256>>>(S, p->net_in, H0, W0);
    double *dv = p->V, *dy = p->Z;
    if (cuda_ok(cudaMemcpy(dv, v, nb, cudaMemcpyHostToDevice), "cudaMemcpy")) {
      bool ok = true;
      if (what == 1)
        k_lp_apply<<<lp_blocks(p->n), 256>>>(S, dv, dy, nullptr);
      else if (what == 2)
        ok = lp_right(p, method == 0 ? net : nullptr, method, dv, dy);
      else
        lp_left(p, method, dv, dy);
      if (ok && cuda_ok(cudaMemcpy(y, dy, nb, cudaMemcpyDeviceToHost), "cudaMemcpy")) rc = 0;
    }
  }
  lp_free(p);
  return rc;
}

}  // extern "C"
