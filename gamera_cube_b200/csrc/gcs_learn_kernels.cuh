// Kernels of the learned ionosphere preconditioner: a 3x3 convolution on
// BF16 tensor cores with FP32 accumulation (forward, and backward data via
// flipped, transposed weights), its weight gradient, 2x2 average pooling,
// nearest 2x upsampling, the ReLU mask and the Adam update.
//
// Tensors are [batch][channel][H][W], periodic in W (longitude) and
// zero-padded in H (colatitude).  Activations are BF16; gradients FP32.  A
// convolution's weights are [Mp][Kp] (Mp = output channels rounded up to
// 16, Kp = 9 Cin + 1 rounded up to 16): column 9 ci + t is tap t = 3 (dh+1)
// + (dw+1) of input channel ci, column 9 Cin the bias (its im2col row is
// all ones), the rest zero.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <mma.h>

namespace gcs {
namespace learn {

using bf16 = __nv_bfloat16;
namespace wm = nvcuda::wmma;

constexpr int kConvThreads = 256;   // 8 warps
constexpr int kPix = 64;            // pixels (one row segment) per block
constexpr int kLd = kPix + 8;       // shared-memory row stride of the im2col tile

__device__ __forceinline__ float to_f(float v) { return v; }
__device__ __forceinline__ float to_f(bf16 v) { return __bfloat162float(v); }

struct ConvP {
  const void *in;     // [B][Cin][H][W], bf16 or float
  const bf16 *w;      // [Mp][Kp]
  const bf16 *skip;   // optional [B][Cout][H][W] added before the activation
  bf16 *out;          // optional [B][Cout][H][W]
  float *out32;       // optional [B][Cout][H][W] (FP32, written or accumulated)
  int B, Cin, Cout, H, W, Kp, relu, accumulate;
};

// Shared-memory bytes of k_conv / k_conv_wgrad for a Kp and Mp.
inline size_t conv_smem(int Kp) {
  return (size_t)Kp * kLd * sizeof(bf16) + 8 * 256 * sizeof(float);
}
inline size_t wgrad_smem(int Kp, int Mp) {
  return (size_t)(Kp + Mp) * kLd * sizeof(bf16) + 8 * 256 * sizeof(float);
}

// im2col of one 64-pixel row segment: col[k][n] for k < Kp.
template <typename Tin>
__device__ __forceinline__ void fill_im2col(bf16 *col, const Tin *in, int Cin, int H, int W,
                                            int Kp, int h, int w0) {
  const int K9 = Cin * 9;
  for (int idx = threadIdx.x; idx < Kp * kPix; idx += blockDim.x) {
    const int k = idx / kPix, n = idx - k * kPix;
    float v = 0.f;
    if (k < K9) {
      const int ci = k / 9, t = k - ci * 9;
      const int hh = h + t / 3 - 1;
      if (hh >= 0 && hh < H) {
        const int ww = (w0 + n + t % 3 - 1 + W) % W;
        v = to_f(in[((size_t)ci * H + hh) * W + ww]);
      }
    } else if (k == K9) {
      v = 1.f;
    }
    col[k * kLd + n] = __float2bfloat16(v);
  }
}

// out[b][co][h][w0..w0+63] = act(sum_k W[co][k] col[k][n] + skip); grid
// (ceil(W / 64), H, B).
template <typename Tin>
__global__ void __launch_bounds__(kConvThreads) k_conv(ConvP p) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  bf16 *col = reinterpret_cast<bf16 *>(smem_raw);
  float *stage = reinterpret_cast<float *>(col + (size_t)p.Kp * kLd);
  const int b = blockIdx.z, h = blockIdx.y, w0 = blockIdx.x * kPix;
  const Tin *in = static_cast<const Tin *>(p.in) + (size_t)b * p.Cin * p.H * p.W;
  fill_im2col(col, in, p.Cin, p.H, p.W, p.Kp, h, w0);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int Mt = (p.Cout + 15) >> 4, tiles = Mt * (kPix / 16);
  float *st = stage + warp * 256;
  for (int tile = warp; tile < tiles; tile += kConvThreads / 32) {
    const int mt = tile / (kPix / 16), nt = tile % (kPix / 16);
    wm::fragment<wm::accumulator, 16, 16, 16, float> acc;
    wm::fill_fragment(acc, 0.f);
    for (int kk = 0; kk < p.Kp; kk += 16) {
      wm::fragment<wm::matrix_a, 16, 16, 16, bf16, wm::row_major> a;
      wm::fragment<wm::matrix_b, 16, 16, 16, bf16, wm::row_major> bm;
      wm::load_matrix_sync(a, p.w + (size_t)mt * 16 * p.Kp + kk, p.Kp);
      wm::load_matrix_sync(bm, col + (size_t)kk * kLd + nt * 16, kLd);
      wm::mma_sync(acc, a, bm, acc);
    }
    wm::store_matrix_sync(st, acc, 16, wm::mem_row_major);
    __syncwarp();
    for (int e = lane; e < 256; e += 32) {
      const int i = e >> 4, j = e & 15, co = mt * 16 + i, w = w0 + nt * 16 + j;
      if (co < p.Cout && w < p.W) {
        const size_t o = (((size_t)b * p.Cout + co) * p.H + h) * p.W + w;
        float v = st[e];
        if (p.skip) v += __bfloat162float(p.skip[o]);
        if (p.relu) v = fmaxf(v, 0.f);
        if (p.out) p.out[o] = __float2bfloat16(v);
        if (p.out32) p.out32[o] = p.accumulate ? p.out32[o] + v : v;
      }
    }
    __syncwarp();
  }
}

struct WgradP {
  const bf16 *in;     // layer input [B][Cin][H][W]
  const float *g;     // gradient at the layer output (after the ReLU mask) [B][Cout][H][W]
  float *gw;          // [Mp][Kp], accumulated
  int B, Cin, Cout, H, W, Kp, Mp;
};

// gw[co][k] += sum over the block's 64 pixels of g[co][pix] col[k][pix];
// grid (ceil(W / 64), H, B).
__global__ void __launch_bounds__(kConvThreads) k_conv_wgrad(WgradP p) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  bf16 *col = reinterpret_cast<bf16 *>(smem_raw);
  bf16 *ga = col + (size_t)p.Kp * kLd;
  float *stage = reinterpret_cast<float *>(ga + (size_t)p.Mp * kLd);
  const int b = blockIdx.z, h = blockIdx.y, w0 = blockIdx.x * kPix;
  fill_im2col(col, p.in + (size_t)b * p.Cin * p.H * p.W, p.Cin, p.H, p.W, p.Kp, h, w0);
  for (int idx = threadIdx.x; idx < p.Mp * kPix; idx += blockDim.x) {
    const int co = idx / kPix, n = idx - co * kPix;
    float v = 0.f;
    if (co < p.Cout && w0 + n < p.W)
      v = p.g[(((size_t)b * p.Cout + co) * p.H + h) * p.W + w0 + n];
    ga[co * kLd + n] = __float2bfloat16(v);
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int Mt = p.Mp >> 4, Kt = p.Kp >> 4, tiles = Mt * Kt;
  float *st = stage + warp * 256;
  for (int tile = warp; tile < tiles; tile += kConvThreads / 32) {
    const int mt = tile / Kt, kt = tile % Kt;
    wm::fragment<wm::accumulator, 16, 16, 16, float> acc;
    wm::fill_fragment(acc, 0.f);
#pragma unroll
    for (int pk = 0; pk < kPix; pk += 16) {
      wm::fragment<wm::matrix_a, 16, 16, 16, bf16, wm::row_major> a;
      wm::fragment<wm::matrix_b, 16, 16, 16, bf16, wm::col_major> bm;
      wm::load_matrix_sync(a, ga + (size_t)mt * 16 * kLd + pk, kLd);
      wm::load_matrix_sync(bm, col + (size_t)kt * 16 * kLd + pk, kLd);
      wm::mma_sync(acc, a, bm, acc);
    }
    wm::store_matrix_sync(st, acc, 16, wm::mem_row_major);
    __syncwarp();
    for (int e = lane; e < 256; e += 32) {
      const int i = e >> 4, j = e & 15, co = mt * 16 + i;
      if (co < p.Cout) atomicAdd(&p.gw[(size_t)co * p.Kp + kt * 16 + j], st[e]);
    }
    __syncwarp();
  }
}

// Backward-data weights: wt[ci][9 co + t] = w[co][9 ci + 8 - t] (flipped
// taps, transposed channels), bias column and padding zero.
__global__ void k_transpose_weights(const float *w, bf16 *wt, int Cin, int Cout, int Kp,
                                    int Mpt, int Kpt) {
  const int n = Mpt * Kpt;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
    const int ci = idx / Kpt, k = idx - ci * Kpt;
    float v = 0.f;
    if (ci < Cin && k < Cout * 9) {
      const int co = k / 9, t = k - co * 9;
      v = w[(size_t)co * Kp + ci * 9 + 8 - t];
    }
    wt[idx] = __float2bfloat16(v);
  }
}

// out = avg 2x2 (in); in [B][C][2H][2W], out [B][C][H][W].
__global__ void k_pool(const bf16 *in, bf16 *out, int BC, int H, int W) {
  const size_t n = (size_t)BC * H * W;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t bc = i / ((size_t)H * W);
    const int r = (int)(i - bc * H * W), h = r / W, w = r - h * W;
    const bf16 *src = in + bc * 4 * H * W + (size_t)(2 * h) * (2 * W) + 2 * w;
    const float s = __bfloat162float(src[0]) + __bfloat162float(src[1]) +
                    __bfloat162float(src[2 * W]) + __bfloat162float(src[2 * W + 1]);
    out[i] = __float2bfloat16(0.25f * s);
  }
}
// gin[2h+i][2w+j] += g[h][w] / 4
__global__ void k_pool_back(const float *g, float *gin, int BC, int H, int W) {
  const size_t n = (size_t)BC * H * W;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t bc = i / ((size_t)H * W);
    const int r = (int)(i - bc * H * W), h = r / W, w = r - h * W;
    float *dst = gin + bc * 4 * H * W + (size_t)(2 * h) * (2 * W) + 2 * w;
    const float q = 0.25f * g[i];
    dst[0] += q;
    dst[1] += q;
    dst[2 * W] += q;
    dst[2 * W + 1] += q;
  }
}
// out[2h+i][2w+j] = in[h][w]; in [B][C][H][W]
__global__ void k_up(const bf16 *in, bf16 *out, int BC, int H, int W) {
  const size_t n = (size_t)BC * H * W;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t bc = i / ((size_t)H * W);
    const int r = (int)(i - bc * H * W), h = r / W, w = r - h * W;
    bf16 *dst = out + bc * 4 * H * W + (size_t)(2 * h) * (2 * W) + 2 * w;
    dst[0] = dst[1] = dst[2 * W] = dst[2 * W + 1] = in[i];
  }
}
// gin[h][w] += sum of g over the 2x2 block
__global__ void k_up_back(const float *g, float *gin, int BC, int H, int W) {
  const size_t n = (size_t)BC * H * W;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t bc = i / ((size_t)H * W);
    const int r = (int)(i - bc * H * W), h = r / W, w = r - h * W;
    const float *src = g + bc * 4 * H * W + (size_t)(2 * h) * (2 * W) + 2 * w;
    gin[i] += src[0] + src[1] + src[2 * W] + src[2 * W + 1];
  }
}
// gm = g (act > 0) for ReLU layers; also adds gm into gskip when given.
__global__ void k_relu_mask(const float *g, const bf16 *act, float *gm, float *gskip, size_t n,
                            int relu) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const float v = relu && !(__bfloat162float(act[i]) > 0.f) ? 0.f : g[i];
    gm[i] = v;
    if (gskip) gskip[i] += v;
  }
}
// Adam (decoupled from the BF16 copy): w, m, v FP32; wb = bf16(w).
__global__ void k_adam(float *w, const float *g, float *m, float *v, bf16 *wb, size_t n,
                       float lr, float b1, float b2, float eps, float c1, float c2) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    wb[i] = __float2bfloat16(wi);
  }
}

}  // namespace learn
}  // namespace gcs
