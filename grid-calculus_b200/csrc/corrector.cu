// Learned coarse-step corrector for 2-D Cahn-Hilliard: a 6-layer periodic
// 3x3 CNN (32 channels, GELU), BF16 weights and activations, FP32
// accumulation on the tensor cores (mma.sync m16n8k16 bf16), trained and run
// by the kernels in this file.
//
// Network: x0 = [c, 0, ..., 0] (32 channels, NHWC), for l = 1..6:
//   z_l = conv3x3_periodic(x_{l-1}, W_l) + b_l,  x_l = gelu(z_l) (l < 6);
// the correction is delta = s_out * (z_6[ch 0] - mean(z_6[ch 0])) per sample
// (zero mean, so the coarse step c + delta conserves mass).  Every layer is
// computed as a 32 -> 32 convolution (the first layer's input channels
// 1..31 are zero and the last layer's outputs 1..31 are unused), so one
// implicit-GEMM kernel serves all layers: M = pixels, N = 32 output
// channels, K = 9 taps x 32 input channels.
//
// Parameters (FP32 master, packed): per layer W[9][32 ci][32 co] then b[32];
// tap t covers offset (dy, dx) = (t / 3 - 1, t % 3 - 1).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace gcb {
namespace {

constexpr int kLayers = 6;
constexpr int kC = 32;                       // channels
constexpr int kTaps = 9;
constexpr int kLayerParams = kTaps * kC * kC + kC;
constexpr int kParams = kLayers * kLayerParams;
constexpr int kPixStride = 40;               // bf16 per pixel in shared memory (80 B: conflict-free)
constexpr int kTR = 8, kTC = 16;             // conv tile: 8 rows x 16 columns of pixels
constexpr int kConvThreads = 128;            // 4 warps, 2 rows (2 m16 tiles) each
constexpr int kHaloR = kTR + 2, kHaloC = kTC + 2;

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

// ---- forward / backward-data convolution ----------------------------------
// out[p][n] = sum_t sum_k in[p + off_t][k] * Bw[t][n][k]  (+ epilogue)
// Epilogue kinds:
//   EPI_FWD    z = acc + bias; store z (bf16) and gelu(z) (bf16)
//   EPI_LAST   z0 = acc + bias (channel 0 only); store z0 (fp32)
//   EPI_BWD    dz_prev = acc * gelu'(z_prev); store (bf16)
enum Epi { EPI_FWD = 0, EPI_LAST = 1, EPI_BWD = 2 };

template <int EPI, int NT>
__global__ void __launch_bounds__(kConvThreads) conv3x3_kernel(
    const __nv_bfloat16* __restrict__ in, const __nv_bfloat16* __restrict__ bw, const float* __restrict__ bias,
    __nv_bfloat16* __restrict__ out_z, __nv_bfloat16* __restrict__ out_y, float* __restrict__ out_f,
    const __nv_bfloat16* __restrict__ z_prev, int H, int W, int tiles_x, int tiles_per_img) {
  __shared__ __align__(16) __nv_bfloat16 s_in[kHaloR * kHaloC * kPixStride];
  __shared__ __align__(16) __nv_bfloat16 s_w[kTaps * kC * kPixStride];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tig = lane & 3;
  const int img = blockIdx.x / tiles_per_img;
  const int tile = blockIdx.x - img * tiles_per_img;
  const int y0 = (tile / tiles_x) * kTR, x0 = (tile % tiles_x) * kTC;
  const size_t img_off = static_cast<size_t>(img) * H * W;

  // Weights: [t][n][k] dense 32 -> padded rows of 40.
  for (int v = tid; v < kTaps * kC * (kC / 8); v += kConvThreads) {
    const int row = v >> 2, q = v & 3;  // row = t * 32 + n
    *reinterpret_cast<uint4*>(&s_w[row * kPixStride + q * 8]) = reinterpret_cast<const uint4*>(bw)[v];
  }
  // Input tile with a one-pixel periodic halo.
  for (int v = tid; v < kHaloR * kHaloC * (kC / 8); v += kConvThreads) {
    const int pix = v >> 2, q = v & 3;
    const int r = pix / kHaloC, c = pix - r * kHaloC;
    const int gy = wrap(y0 - 1 + r, H), gx = wrap(x0 - 1 + c, W);
    const size_t gp = img_off + static_cast<size_t>(gy) * W + gx;
    *reinterpret_cast<uint4*>(&s_in[pix * kPixStride + q * 8]) =
        reinterpret_cast<const uint4*>(in + gp * kC)[q];
  }
  __syncthreads();

  float acc[2][NT][4];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[mt][nt][e] = 0.f;

#pragma unroll
  for (int t = 0; t < kTaps; ++t) {
    const int dy = t / 3 - 1, dx = t % 3 - 1;
#pragma unroll
    for (int kh = 0; kh < 2; ++kh) {
      uint32_t b[NT][2];
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        const __nv_bfloat16* wp = &s_w[(t * kC + nt * 8 + g) * kPixStride + kh * 16 + tig * 2];
        b[nt][0] = *reinterpret_cast<const uint32_t*>(wp);
        b[nt][1] = *reinterpret_cast<const uint32_t*>(wp + 8);
      }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        const int r = warp * 2 + mt + 1 + dy;
        const __nv_bfloat16* p0 = &s_in[(r * kHaloC + g + 1 + dx) * kPixStride + kh * 16 + tig * 2];
        const __nv_bfloat16* p1 = p0 + 8 * kPixStride;
        uint32_t a[4];
        a[0] = *reinterpret_cast<const uint32_t*>(p0);
        a[1] = *reinterpret_cast<const uint32_t*>(p1);
        a[2] = *reinterpret_cast<const uint32_t*>(p0 + 8);
        a[3] = *reinterpret_cast<const uint32_t*>(p1 + 8);
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) mma_bf16(acc[mt][nt], a, b[nt]);
      }
    }
  }

  // Epilogue: C fragment rows are pixels g and g + 8, columns 2 tig, 2 tig + 1.
#pragma unroll
  for (int mt = 0; mt < 2; ++mt) {
    const int oy = y0 + warp * 2 + mt;
    if (oy >= H) continue;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int ox = x0 + g + half * 8;
      if (ox >= W) continue;
      const size_t gp = img_off + static_cast<size_t>(oy) * W + ox;
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        const int n = nt * 8 + tig * 2;
        float v0 = acc[mt][nt][half * 2], v1 = acc[mt][nt][half * 2 + 1];
        if constexpr (EPI == EPI_FWD) {
          v0 += bias[n];
          v1 += bias[n + 1];
          *reinterpret_cast<uint32_t*>(out_z + gp * kC + n) = pack_bf16(v0, v1);
          *reinterpret_cast<uint32_t*>(out_y + gp * kC + n) = pack_bf16(gelu(v0), gelu(v1));
        } else if constexpr (EPI == EPI_LAST) {
          if (n == 0) out_f[gp] = v0 + bias[0];
        } else {
          const __nv_bfloat162 zp = *reinterpret_cast<const __nv_bfloat162*>(z_prev + gp * kC + n);
          const float2 zf = __bfloat1622float2(zp);
          *reinterpret_cast<uint32_t*>(out_z + gp * kC + n) = pack_bf16(v0 * gelu_grad(zf.x), v1 * gelu_grad(zf.y));
        }
      }
    }
  }
}

// ---- weight gradient ------------------------------------------------------
// dW[t][ci][co] = sum_p x[p + off_t][ci] dz[p][co];  db[co] = sum_p dz[p][co].
// Persistent CTAs accumulate over many tiles in registers and write one
// partial per CTA; a second kernel sums the partials in CTA order.
constexpr int kWgThreads = 128;  // 4 warps: warp w owns ci block (w >> 1), co blocks 2 (w & 1) .. +1

__global__ void __launch_bounds__(kWgThreads) conv3x3_wgrad_kernel(
    const __nv_bfloat16* __restrict__ x, const __nv_bfloat16* __restrict__ dz, int H, int W, int tiles_x,
    int tiles_per_img, int n_tiles, float* __restrict__ partial) {
  // Channel-major staging: xt[ci][10][18 + 2], dzt[co][8][16 + 8].
  constexpr int XS = kHaloC + 2, DS = kTC + 8;
  __shared__ __align__(16) __nv_bfloat16 xt[kC * kHaloR * XS];
  __shared__ __align__(16) __nv_bfloat16 dzt[kC * kTR * DS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tig = lane & 3;
  const int mb = warp >> 1;            // ci block of 16
  const int nb0 = (warp & 1) * 2;      // two co blocks of 8
  float acc[kTaps][2][4];
#pragma unroll
  for (int t = 0; t < kTaps; ++t)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[t][j][e] = 0.f;
  float dbias = 0.f;  // thread tid < 32: channel tid

  for (int tl = blockIdx.x; tl < n_tiles; tl += gridDim.x) {
    const int img = tl / tiles_per_img;
    const int tile = tl - img * tiles_per_img;
    const int y0 = (tile / tiles_x) * kTR, x0 = (tile % tiles_x) * kTC;
    const size_t img_off = static_cast<size_t>(img) * H * W;
    __syncthreads();
    for (int pix = tid; pix < kHaloR * kHaloC; pix += kWgThreads) {
      const int r = pix / kHaloC, c = pix - r * kHaloC;
      const size_t gp = img_off + static_cast<size_t>(wrap(y0 - 1 + r, H)) * W + wrap(x0 - 1 + c, W);
      const __nv_bfloat16* src = x + gp * kC;
#pragma unroll
      for (int ci = 0; ci < kC; ++ci) xt[(ci * kHaloR + r) * XS + c] = src[ci];
    }
    for (int pix = tid; pix < kTR * kTC; pix += kWgThreads) {
      const int r = pix / kTC, c = pix - r * kTC;
      const int oy = y0 + r, ox = x0 + c;
      const bool in = oy < H && ox < W;
      const size_t gp = img_off + static_cast<size_t>(in ? oy : 0) * W + (in ? ox : 0);
      const __nv_bfloat16* src = dz + gp * kC;
#pragma unroll
      for (int co = 0; co < kC; ++co) dzt[(co * kTR + r) * DS + c] = in ? src[co] : __float2bfloat16(0.f);
    }
    __syncthreads();
    if (tid < kC) {
      float s = 0.f;
      for (int r = 0; r < kTR; ++r)
        for (int c = 0; c < kTC; ++c) s += __bfloat162float(dzt[(tid * kTR + r) * DS + c]);
      dbias += s;
    }
#pragma unroll
    for (int t = 0; t < kTaps; ++t) {
      const int dy = t / 3 - 1, dx = t % 3 - 1;
#pragma unroll
      for (int kb = 0; kb < kTR; ++kb) {  // 16 pixels = one tile row per k step
        // A[m = ci][k = pixel], row-major; two 16-bit loads per pair (pixel offset may be odd).
        uint32_t a[4];
        const int xr = kb + 1 + dy;
        auto xa = [&](int ci, int px) { return xt[(ci * kHaloR + xr) * XS + px + 1 + dx]; };
        const int ci0 = mb * 16 + g, ci1 = ci0 + 8, k0 = tig * 2, k1 = k0 + 8;
        a[0] = pack_bf16(__bfloat162float(xa(ci0, k0)), __bfloat162float(xa(ci0, k0 + 1)));
        a[1] = pack_bf16(__bfloat162float(xa(ci1, k0)), __bfloat162float(xa(ci1, k0 + 1)));
        a[2] = pack_bf16(__bfloat162float(xa(ci0, k1)), __bfloat162float(xa(ci0, k1 + 1)));
        a[3] = pack_bf16(__bfloat162float(xa(ci1, k1)), __bfloat162float(xa(ci1, k1 + 1)));
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int co = (nb0 + j) * 8 + g;
          uint32_t b[2];
          b[0] = *reinterpret_cast<const uint32_t*>(&dzt[(co * kTR + kb) * DS + tig * 2]);
          b[1] = *reinterpret_cast<const uint32_t*>(&dzt[(co * kTR + kb) * DS + tig * 2 + 8]);
          mma_bf16(acc[t][j], a, b);
        }
      }
    }
  }
  // Partial layout: [cta][t][ci][co] then [cta][9216 + co] for the bias.
  float* dst = partial + static_cast<size_t>(blockIdx.x) * kLayerParams;
#pragma unroll
  for (int t = 0; t < kTaps; ++t)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int ci0 = mb * 16 + g, co = (nb0 + j) * 8 + tig * 2;
      dst[(t * kC + ci0) * kC + co] = acc[t][j][0];
      dst[(t * kC + ci0) * kC + co + 1] = acc[t][j][1];
      dst[(t * kC + ci0 + 8) * kC + co] = acc[t][j][2];
      dst[(t * kC + ci0 + 8) * kC + co + 1] = acc[t][j][3];
    }
  if (tid < kC) dst[kTaps * kC * kC + tid] = dbias;
}

// Sums partials in CTA order into grad (one thread per parameter).
__global__ void sum_partials(const float* __restrict__ partial, int n_parts, float* __restrict__ grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kLayerParams) return;
  float s = 0.f;
  for (int k = 0; k < n_parts; ++k) s += partial[static_cast<size_t>(k) * kLayerParams + i];
  grad[i] = s;
}

// ---- input, output, loss --------------------------------------------------
// Channel 0 = c, channel 1 = feature_scale * f (the right-hand side when
// features are on, else 0), channels 2..31 = 0.
template <class T>
__global__ void pack_input(const T* __restrict__ c, const T* __restrict__ f, float feature_scale, size_t n,
                           __nv_bfloat16* __restrict__ x0) {
  for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<size_t>(gridDim.x) * blockDim.x) {
    uint4* dst = reinterpret_cast<uint4*>(x0 + p * kC);
    uint4 z = make_uint4(0, 0, 0, 0);
    const float fv = f ? feature_scale * static_cast<float>(f[p]) : 0.f;
    z.x = pack_bf16(static_cast<float>(c[p]), fv);
    dst[0] = z;
    dst[1] = make_uint4(0, 0, 0, 0);
    dst[2] = make_uint4(0, 0, 0, 0);
    dst[3] = make_uint4(0, 0, 0, 0);
  }
}

// Per-sample mean of f over H*W pixels (one CTA per sample, fixed order).
__global__ void sample_mean(const float* __restrict__ f, int hw, float* __restrict__ mean) {
  __shared__ double sh[256];
  const float* s = f + static_cast<size_t>(blockIdx.x) * hw;
  double acc = 0.0;
  for (int i = threadIdx.x; i < hw; i += 256) acc += s[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w >= 1; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) mean[blockIdx.x] = static_cast<float>(sh[0] / hw);
}

// delta = s_out (z - mean_z)
__global__ void project_delta(const float* __restrict__ z, const float* __restrict__ mean, int hw, size_t n,
                              float s_out, float* __restrict__ delta) {
  for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<size_t>(gridDim.x) * blockDim.x)
    delta[p] = s_out * (z[p] - mean[p / hw]);
}

// (target - c)^2, for the per-sample step size of the normalised loss.
__global__ void step_sq(const float* __restrict__ c, const float* __restrict__ target, size_t n,
                        float* __restrict__ out) {
  for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const float d = target[p] - c[p];
    out[p] = d * d;
  }
}

// r = c + delta - target, stored; per-CTA partial sums of r^2 / den[sample]
// (den = 1 for the plain loss; fixed grid).
__global__ void residual_kernel(const float* __restrict__ c, const float* __restrict__ delta,
                                const float* __restrict__ target, size_t n, int hw,
                                const float* __restrict__ den, float* __restrict__ r,
                                double* __restrict__ part) {
  __shared__ double sh[256];
  double acc = 0.0;
  for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const float v = c[p] + delta[p] - target[p];
    r[p] = v;
    const double w = den ? 1.0 / static_cast<double>(den[p / hw]) : 1.0;
    acc += static_cast<double>(v) * v * w;
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w >= 1; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// dz6 (channel 0) = s_out * 2/N (r - mean_sample(r)) / den[sample];
// other channels 0.
__global__ void last_layer_grad(const float* __restrict__ r, const float* __restrict__ rmean, int hw, size_t n,
                                float scale, const float* __restrict__ den, __nv_bfloat16* __restrict__ dz) {
  for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<size_t>(gridDim.x) * blockDim.x) {
    uint4* dst = reinterpret_cast<uint4*>(dz + p * kC);
    const float w = den ? 1.0f / den[p / hw] : 1.0f;
    __nv_bfloat16 v = __float2bfloat16(scale * w * (r[p] - rmean[p / hw]));
    uint4 z = make_uint4(static_cast<uint32_t>(*reinterpret_cast<uint16_t*>(&v)), 0, 0, 0);
    dst[0] = z;
    dst[1] = make_uint4(0, 0, 0, 0);
    dst[2] = make_uint4(0, 0, 0, 0);
    dst[3] = make_uint4(0, 0, 0, 0);
  }
}

// FP32 master -> bf16 [l][t][n = co][k = ci] (forward) and
// [l][t][n = ci][k = co] with the tap flipped (backward data).
__global__ void layout_weights(const float* __restrict__ params, __nv_bfloat16* __restrict__ fwd,
                               __nv_bfloat16* __restrict__ bwd) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kLayers * kTaps * kC * kC) return;
  const int l = i / (kTaps * kC * kC);
  const int rem = i - l * kTaps * kC * kC;
  const int t = rem / (kC * kC), ci = (rem / kC) % kC, co = rem % kC;
  const float w = params[l * kLayerParams + rem];  // W[t][ci][co]
  const size_t lb = static_cast<size_t>(l) * kTaps * kC * kC;
  fwd[lb + (t * kC + co) * kC + ci] = __float2bfloat16(w);
  bwd[lb + ((kTaps - 1 - t) * kC + ci) * kC + co] = __float2bfloat16(w);
}

__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// cand = psi + delta
__global__ void apply_delta(const double* __restrict__ psi, const float* __restrict__ delta, size_t n,
                            double* __restrict__ cand) {
  for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<size_t>(gridDim.x) * blockDim.x)
    cand[p] = psi[p] + static_cast<double>(delta[p]);
}

// Trapezoid residual of a coarse step: sums of ((c1 - c0)/dt - (f0 + f1)/2)^2
// and ((f0 + f1)/2)^2, per CTA (fixed grid).
__global__ void trapezoid_residual(const double* __restrict__ c0, const double* __restrict__ c1,
                                   const double* __restrict__ f0, const double* __restrict__ f1, size_t n,
                                   double inv_dt, double* __restrict__ part) {
  __shared__ double sr[256], sf[256];
  double ar = 0.0, af = 0.0;
  for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const double fm = 0.5 * (f0[p] + f1[p]);
    const double r = (c1[p] - c0[p]) * inv_dt - fm;
    ar += r * r;
    af += fm * fm;
  }
  sr[threadIdx.x] = ar;
  sf[threadIdx.x] = af;
  __syncthreads();
  for (int w = 128; w >= 1; w >>= 1) {
    if (threadIdx.x < w) {
      sr[threadIdx.x] += sr[threadIdx.x + w];
      sf[threadIdx.x] += sf[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = sr[0];
    part[2 * blockIdx.x + 1] = sf[0];
  }
}

}  // namespace
}  // namespace gcb

using namespace gcb;

struct gc_corrector {
  gc_context* ctx = nullptr;
  int H = 0, W = 0, max_batch = 0;
  float s_out = 0.05f;
  float* params = nullptr;  // FP32 master
  float* grad = nullptr;
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  int adam_t = 0;
  __nv_bfloat16* w_fwd = nullptr;
  __nv_bfloat16* w_bwd = nullptr;
  __nv_bfloat16* x[kLayers] = {};   // layer inputs (x[0] = packed c)
  __nv_bfloat16* z[kLayers] = {};   // pre-activations of layers 1..5 (z[0..4])
  __nv_bfloat16* dz_a = nullptr;    // backward ping-pong
  __nv_bfloat16* dz_b = nullptr;
  float* zlast = nullptr;           // z_6 channel 0
  float* delta = nullptr;
  float* resid = nullptr;
  float* mean = nullptr;            // per-sample means
  float* mean2 = nullptr;
  float* cbuf = nullptr;            // fp32 copies of inputs / targets
  float* tbuf = nullptr;
  double* part = nullptr;
  float* wpart = nullptr;           // per-CTA weight-gradient partials
  int wparts = 0;
  double* adv = nullptr;            // advance scratch: cand, f0, f1 (H x W each)
  // Right-hand-side input feature: channel 1 = feature_dt * f(c), f the
  // Cahn-Hilliard RHS with chp (off until gc_corrector_set_physics).
  bool feature = false;
  gc_ch_params chp{1.0, 1.0, 2};
  double feature_dt = 0.0;
  double* fbuf = nullptr;           // f(c), max_batch x H x W (double-sized)
  float* den = nullptr;             // per-sample step size (normalised loss)
  bool normalized = false;
  bool weights_dirty = true;
};

namespace gcb {
namespace {

constexpr int kRedBlocks = 256;

gc_status corr_layout(gc_corrector* c) {
  if (!c->weights_dirty) return GC_OK;
  const int n = kLayers * kTaps * kC * kC;
  layout_weights<<<div_up(n, 256), 256, 0, c->ctx->stream>>>(c->params, c->w_fwd, c->w_bwd);
  GC_CHECK_LAUNCH("layout_weights");
  c->weights_dirty = false;
  return GC_OK;
}

template <class T>
gc_status corr_forward(gc_corrector* c, int batch, const T* in) {
  gc_status s = corr_layout(c);
  if (s != GC_OK) return s;
  const int H = c->H, W = c->W;
  const size_t n = static_cast<size_t>(batch) * H * W;
  cudaStream_t st = c->ctx->stream;
  const T* feat = nullptr;
  if (c->feature) {
    const gc_grid g{W, H, 1, 1.0, 1.0, 1.0};
    T* fb = reinterpret_cast<T*>(c->fbuf);
    for (int b = 0; b < batch; ++b) {
      gc_status fs = gc_ch_rhs(c->ctx, &g, sizeof(T) == 8 ? GC_F64 : GC_F32, &c->chp, in + static_cast<size_t>(b) * H * W,
                               fb + static_cast<size_t>(b) * H * W);
      if (fs != GC_OK) return fs;
    }
    feat = fb;
  }
  pack_input<T><<<c->ctx->num_sms * 8, 256, 0, st>>>(in, feat, static_cast<float>(c->feature_dt), n, c->x[0]);
  GC_CHECK_LAUNCH("pack_input");
  const int tiles_x = div_up(W, kTC), tiles_y = div_up(H, kTR);
  const int tpi = tiles_x * tiles_y;
  for (int l = 0; l < kLayers; ++l) {
    const __nv_bfloat16* wl = c->w_fwd + static_cast<size_t>(l) * kTaps * kC * kC;
    const float* bl = c->params + static_cast<size_t>(l) * kLayerParams + kTaps * kC * kC;
    if (l + 1 < kLayers) {
      conv3x3_kernel<EPI_FWD, 4><<<batch * tpi, kConvThreads, 0, st>>>(c->x[l], wl, bl, c->z[l], c->x[l + 1],
                                                                      nullptr, nullptr, H, W, tiles_x, tpi);
    } else {
      conv3x3_kernel<EPI_LAST, 1><<<batch * tpi, kConvThreads, 0, st>>>(c->x[l], wl, bl, nullptr, nullptr,
                                                                       c->zlast, nullptr, H, W, tiles_x, tpi);
    }
    GC_CHECK_LAUNCH("conv3x3_kernel (forward)");
  }
  sample_mean<<<batch, 256, 0, st>>>(c->zlast, H * W, c->mean);
  project_delta<<<c->ctx->num_sms * 8, 256, 0, st>>>(c->zlast, c->mean, H * W, n, c->s_out, c->delta);
  GC_CHECK_LAUNCH("project_delta");
  return GC_OK;
}

// Forward + loss + backward into c->grad (no update). loss = mean((c + delta - target)^2).
gc_status corr_backward(gc_corrector* c, int batch, const float* cin, const float* target, double* loss) {
  gc_status s = corr_forward<float>(c, batch, cin);
  if (s != GC_OK) return s;
  const int H = c->H, W = c->W, hw = H * W;
  const size_t n = static_cast<size_t>(batch) * hw;
  cudaStream_t st = c->ctx->stream;
  const float* den = nullptr;
  if (c->normalized) {
    step_sq<<<c->ctx->num_sms * 8, 256, 0, st>>>(cin, target, n, c->resid);
    sample_mean<<<batch, 256, 0, st>>>(c->resid, hw, c->den);
    den = c->den;
  }
  residual_kernel<<<kRedBlocks, 256, 0, st>>>(cin, c->delta, target, n, hw, den, c->resid, c->part);
  GC_CHECK_LAUNCH("residual_kernel");
  sample_mean<<<batch, 256, 0, st>>>(c->resid, hw, c->mean2);
  const float scale = c->s_out * 2.0f / static_cast<float>(n);
  __nv_bfloat16* dz = c->dz_a;
  __nv_bfloat16* dzn = c->dz_b;
  last_layer_grad<<<c->ctx->num_sms * 8, 256, 0, st>>>(c->resid, c->mean2, hw, n, scale, den, dz);
  GC_CHECK_LAUNCH("last_layer_grad");
  const int tiles_x = div_up(W, kTC), tiles_y = div_up(H, kTR);
  const int tpi = tiles_x * tiles_y;
  const int n_tiles = batch * tpi;
  const int wg_grid = std::min(n_tiles, c->wparts);
  for (int l = kLayers - 1; l >= 0; --l) {
    // weight gradient of layer l+1 (index l): input x[l], output gradient dz
    conv3x3_wgrad_kernel<<<wg_grid, kWgThreads, 0, st>>>(c->x[l], dz, H, W, tiles_x, tpi, n_tiles, c->wpart);
    GC_CHECK_LAUNCH("conv3x3_wgrad_kernel");
    sum_partials<<<div_up(kLayerParams, 256), 256, 0, st>>>(c->wpart, wg_grid, c->grad + static_cast<size_t>(l) * kLayerParams);
    GC_CHECK_LAUNCH("sum_partials");
    if (l > 0) {
      const __nv_bfloat16* wl = c->w_bwd + static_cast<size_t>(l) * kTaps * kC * kC;
      conv3x3_kernel<EPI_BWD, 4><<<n_tiles, kConvThreads, 0, st>>>(dz, wl, nullptr, dzn, nullptr, nullptr,
                                                                   c->z[l - 1], H, W, tiles_x, tpi);
      GC_CHECK_LAUNCH("conv3x3_kernel (backward)");
      std::swap(dz, dzn);
    }
  }
  if (loss) {
    std::vector<double> h(kRedBlocks);
    GC_CUDA(cudaMemcpyAsync(h.data(), c->part, sizeof(double) * kRedBlocks, cudaMemcpyDeviceToHost, st));
    GC_CUDA(cudaStreamSynchronize(st));
    double sum = 0.0;
    for (double v : h) sum += v;
    *loss = sum / static_cast<double>(n);
  }
  return GC_OK;
}

}  // namespace
}  // namespace gcb

extern "C" {

GC_API gc_status gc_corrector_create(gc_context* ctx, int32_t height, int32_t width, int32_t max_batch,
                                     gc_corrector** out) {
  Call call(ctx);
  if (call.st != GC_OK) return call.st;
  if (!out || height < 3 || width < 3 || max_batch < 1)
    return fail(GC_ERR_INVALID_ARG, "gc_corrector_create: need height, width >= 3 and max_batch >= 1");
  *out = nullptr;
  gc_corrector* c = new gc_corrector();
  c->ctx = ctx;
  c->H = height;
  c->W = width;
  c->max_batch = max_batch;
  const size_t n = static_cast<size_t>(max_batch) * height * width;
  cudaError_t e = cudaSuccess;
  auto alloc = [&](void** p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, bytes);
  };
  alloc(reinterpret_cast<void**>(&c->params), sizeof(float) * kParams);
  alloc(reinterpret_cast<void**>(&c->grad), sizeof(float) * kParams);
  alloc(reinterpret_cast<void**>(&c->adam_m), sizeof(float) * kParams);
  alloc(reinterpret_cast<void**>(&c->adam_v), sizeof(float) * kParams);
  alloc(reinterpret_cast<void**>(&c->w_fwd), sizeof(__nv_bfloat16) * kLayers * kTaps * kC * kC);
  alloc(reinterpret_cast<void**>(&c->w_bwd), sizeof(__nv_bfloat16) * kLayers * kTaps * kC * kC);
  for (int l = 0; l < kLayers; ++l) alloc(reinterpret_cast<void**>(&c->x[l]), sizeof(__nv_bfloat16) * n * kC);
  for (int l = 0; l + 1 < kLayers; ++l) alloc(reinterpret_cast<void**>(&c->z[l]), sizeof(__nv_bfloat16) * n * kC);
  alloc(reinterpret_cast<void**>(&c->dz_a), sizeof(__nv_bfloat16) * n * kC);
  alloc(reinterpret_cast<void**>(&c->dz_b), sizeof(__nv_bfloat16) * n * kC);
  alloc(reinterpret_cast<void**>(&c->zlast), sizeof(float) * n);
  alloc(reinterpret_cast<void**>(&c->delta), sizeof(float) * n);
  alloc(reinterpret_cast<void**>(&c->resid), sizeof(float) * n);
  alloc(reinterpret_cast<void**>(&c->mean), sizeof(float) * max_batch);
  alloc(reinterpret_cast<void**>(&c->mean2), sizeof(float) * max_batch);
  alloc(reinterpret_cast<void**>(&c->cbuf), sizeof(float) * n);
  alloc(reinterpret_cast<void**>(&c->fbuf), sizeof(double) * n);
  alloc(reinterpret_cast<void**>(&c->den), sizeof(float) * max_batch);
  alloc(reinterpret_cast<void**>(&c->tbuf), sizeof(float) * n);
  alloc(reinterpret_cast<void**>(&c->part), sizeof(double) * 2 * kRedBlocks);
  c->wparts = ctx->num_sms * 4;
  alloc(reinterpret_cast<void**>(&c->wpart), sizeof(float) * kLayerParams * c->wparts);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->params, 0, sizeof(float) * kParams, ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->adam_m, 0, sizeof(float) * kParams, ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->adam_v, 0, sizeof(float) * kParams, ctx->stream);
  if (e != cudaSuccess) {
    gc_corrector_destroy(c);
    return cuda_fail(e, "gc_corrector_create");
  }
  *out = c;
  return GC_OK;
}

GC_API gc_status gc_corrector_destroy(gc_corrector* c) {
  if (!c) return GC_OK;
  cudaSetDevice(c->ctx->device);
  cudaStreamSynchronize(c->ctx->stream);
  void* ptrs[] = {c->params, c->grad, c->adam_m, c->adam_v, c->w_fwd, c->w_bwd, c->dz_a, c->dz_b, c->zlast,
                  c->delta, c->resid, c->mean, c->mean2, c->cbuf, c->tbuf, c->part, c->wpart, c->adv,
                  c->fbuf, c->den};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (auto* p : c->x)
    if (p) cudaFree(p);
  for (auto* p : c->z)
    if (p) cudaFree(p);
  delete c;
  return GC_OK;
}

GC_API int32_t gc_corrector_num_params(void) { return kParams; }

GC_API gc_status gc_corrector_set_physics(gc_corrector* c, const gc_ch_params* p, double feature_dt) {
  if (!c) return fail(GC_ERR_INVALID_ARG, "gc_corrector_set_physics: null corrector");
  if (!p) {
    c->feature = false;
    return GC_OK;
  }
  if (p->order != 2 && p->order != 4 && p->order != 6)
    return fail(GC_ERR_UNSUPPORTED, "gc_corrector_set_physics: order must be 2, 4 or 6");
  c->feature = true;
  c->chp = *p;
  c->feature_dt = feature_dt;
  return GC_OK;
}

GC_API gc_status gc_corrector_set_loss(gc_corrector* c, int32_t normalized) {
  if (!c) return fail(GC_ERR_INVALID_ARG, "gc_corrector_set_loss: null corrector");
  c->normalized = normalized != 0;
  return GC_OK;
}

GC_API gc_status gc_corrector_set_params(gc_corrector* c, const float* host, int32_t n, float s_out) {
  if (!c || !host || n != kParams) return fail(GC_ERR_INVALID_ARG, "gc_corrector_set_params: need all parameters");
  Call call(c->ctx);
  if (call.st != GC_OK) return call.st;
  GC_CUDA(cudaMemcpyAsync(c->params, host, sizeof(float) * kParams, cudaMemcpyHostToDevice, c->ctx->stream));
  GC_CUDA(cudaMemsetAsync(c->adam_m, 0, sizeof(float) * kParams, c->ctx->stream));
  GC_CUDA(cudaMemsetAsync(c->adam_v, 0, sizeof(float) * kParams, c->ctx->stream));
  GC_CUDA(cudaStreamSynchronize(c->ctx->stream));
  c->adam_t = 0;
  c->s_out = s_out;
  c->weights_dirty = true;
  return GC_OK;
}

GC_API gc_status gc_corrector_get_params(gc_corrector* c, float* host, int32_t n) {
  if (!c || !host || n != kParams) return fail(GC_ERR_INVALID_ARG, "gc_corrector_get_params: need all parameters");
  Call call(c->ctx);
  if (call.st != GC_OK) return call.st;
  GC_CUDA(cudaMemcpyAsync(host, c->params, sizeof(float) * kParams, cudaMemcpyDeviceToHost, c->ctx->stream));
  GC_CUDA(cudaStreamSynchronize(c->ctx->stream));
  return GC_OK;
}

// delta_out = zero-mean correction for each of `batch` fields c (fp32 or fp64, batch x H x W).
GC_API gc_status gc_corrector_forward(gc_corrector* c, int32_t batch, gc_dtype dt, const void* cin,
                                      float* delta_out) {
  if (!c || !cin || !delta_out) return fail(GC_ERR_INVALID_ARG, "gc_corrector_forward: null pointer");
  Call call(c->ctx);
  if (call.st != GC_OK) return call.st;
  if (batch < 1 || batch > c->max_batch) return fail(GC_ERR_INVALID_ARG, "gc_corrector_forward: batch out of range");
  gc_status s = dt == GC_F64 ? corr_forward<double>(c, batch, static_cast<const double*>(cin))
                             : corr_forward<float>(c, batch, static_cast<const float*>(cin));
  if (s != GC_OK) return s;
  GC_CUDA(cudaMemcpyAsync(delta_out, c->delta, sizeof(float) * batch * c->H * c->W, cudaMemcpyDeviceToDevice,
                          c->ctx->stream));
  return GC_OK;
}

// Gradient of the loss mean((c + delta(c) - target)^2) into grad_host
// (kParams floats), without updating the parameters.
GC_API gc_status gc_corrector_gradient(gc_corrector* c, int32_t batch, const float* cin, const float* target,
                                       float* grad_host, double* loss) {
  if (!c || !cin || !target) return fail(GC_ERR_INVALID_ARG, "gc_corrector_gradient: null pointer");
  Call call(c->ctx);
  if (call.st != GC_OK) return call.st;
  if (batch < 1 || batch > c->max_batch) return fail(GC_ERR_INVALID_ARG, "gc_corrector_gradient: batch out of range");
  gc_status s = corr_backward(c, batch, cin, target, loss);
  if (s != GC_OK) return s;
  if (grad_host) {
    GC_CUDA(cudaMemcpyAsync(grad_host, c->grad, sizeof(float) * kParams, cudaMemcpyDeviceToHost, c->ctx->stream));
    GC_CUDA(cudaStreamSynchronize(c->ctx->stream));
  }
  return GC_OK;
}

// One Adam step on the loss above (fp32 inputs and targets on the device).
GC_API gc_status gc_corrector_train_step(gc_corrector* c, int32_t batch, const float* cin, const float* target,
                                         float lr, double* loss) {
  if (!c || !cin || !target) return fail(GC_ERR_INVALID_ARG, "gc_corrector_train_step: null pointer");
  Call call(c->ctx);
  if (call.st != GC_OK) return call.st;
  if (batch < 1 || batch > c->max_batch) return fail(GC_ERR_INVALID_ARG, "gc_corrector_train_step: batch out of range");
  gc_status s = corr_backward(c, batch, cin, target, loss);
  if (s != GC_OK) return s;
  ++c->adam_t;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, static_cast<float>(c->adam_t));
  const float c2 = 1.f - std::pow(b2, static_cast<float>(c->adam_t));
  adam_kernel<<<div_up(kParams, 256), 256, 0, c->ctx->stream>>>(c->params, c->grad, c->adam_m, c->adam_v, kParams,
                                                                lr, b1, b2, 1e-8f, c1, c2);
  GC_CHECK_LAUNCH("adam_kernel");
  c->weights_dirty = true;
  return GC_OK;
}

// Advances one 2-D double field by n_coarse coarse steps of
// dt_fine * fine_per_coarse.  Each coarse step proposes c + delta(c) and
// accepts it when the free energy does not rise by more than energy_tol and
// the trapezoid residual |(c1 - c0)/Dt - (f(c0) + f(c1))/2| / |(f(c0) + f(c1))/2|
// is at most residual_tol; otherwise the step is taken by fine_per_coarse
// plain RK4 steps.
GC_API gc_status gc_corrector_advance(gc_corrector* c, const gc_grid* g, const gc_ch_params* cp, double* psi,
                                      int32_t n_coarse, const gc_corrector_policy* pol,
                                      gc_corrector_stats* stats) {
  if (!c || !g || !cp || !psi || !pol) return fail(GC_ERR_INVALID_ARG, "gc_corrector_advance: null pointer");
  Call call(c->ctx);
  if (call.st != GC_OK) return call.st;
  if (g->nz != 1 || g->ny != c->H || g->nx != c->W)
    return fail(GC_ERR_GRID_MISMATCH, "gc_corrector_advance: grid must be 2-D and match the corrector's size");
  if (n_coarse < 0 || pol->fine_per_coarse < 1 || !(pol->dt_fine > 0.0))
    return fail(GC_ERR_INVALID_ARG, "gc_corrector_advance: bad policy or step count");
  gc_context* ctx = c->ctx;
  const size_t n = static_cast<size_t>(c->H) * c->W;
  if (!c->adv) GC_CUDA(cudaMalloc(&c->adv, sizeof(double) * 3 * n));
  double* cand = c->adv;
  double* f0 = c->adv + n;
  double* f1 = c->adv + 2 * n;
  const double dt_coarse = pol->dt_fine * pol->fine_per_coarse;
  gc_integrand fe{GC_INTEGRAND_CH_FREE_ENERGY, cp->kappa};
  double F0 = 0.0;
  gc_status s = gc_evaluate(ctx, g, GC_F64, psi, &fe, GC_SUM_PAIRWISE, &F0);
  if (s != GC_OK) return s;
  bool f0_valid = false;
  gc_corrector_stats st{};
  std::vector<double> part(2 * kRedBlocks);
  for (int k = 0; k < n_coarse; ++k) {
    if ((s = corr_forward<double>(c, 1, psi)) != GC_OK) return s;
    apply_delta<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(psi, c->delta, n, cand);
    GC_CHECK_LAUNCH("apply_delta");
    double F1 = 0.0;
    if ((s = gc_evaluate(ctx, g, GC_F64, cand, &fe, GC_SUM_PAIRWISE, &F1)) != GC_OK) return s;
    bool accept = F1 <= F0 + pol->energy_tol;
    double res = 0.0;
    if (accept) {
      if (!f0_valid && (s = gc_ch_rhs(ctx, g, GC_F64, cp, psi, f0)) != GC_OK) return s;
      if ((s = gc_ch_rhs(ctx, g, GC_F64, cp, cand, f1)) != GC_OK) return s;
      trapezoid_residual<<<kRedBlocks, 256, 0, ctx->stream>>>(psi, cand, f0, f1, n, 1.0 / dt_coarse,
                                                              reinterpret_cast<double*>(c->part));
      GC_CHECK_LAUNCH("trapezoid_residual");
      GC_CUDA(cudaMemcpyAsync(part.data(), c->part, sizeof(double) * 2 * kRedBlocks, cudaMemcpyDeviceToHost,
                              ctx->stream));
      GC_CUDA(cudaStreamSynchronize(ctx->stream));
      double sr = 0.0, sf = 0.0;
      for (int b = 0; b < kRedBlocks; ++b) {
        sr += part[2 * b];
        sf += part[2 * b + 1];
      }
      res = sf > 0.0 ? std::sqrt(sr / sf) : 0.0;
      accept = res <= pol->residual_tol;
    }
    st.last_residual = res;
    if (accept) {
      GC_CUDA(cudaMemcpyAsync(psi, cand, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));
      std::swap(f0, f1);  // f(psi) of the new state is known
      f0_valid = true;
      F0 = F1;
      ++st.accepted;
    } else {
      if ((s = gc_ch_integrate(ctx, g, GC_F64, cp, psi, pol->dt_fine, pol->fine_per_coarse, GC_RK4)) != GC_OK)
        return s;
      if ((s = gc_evaluate(ctx, g, GC_F64, psi, &fe, GC_SUM_PAIRWISE, &F0)) != GC_OK) return s;
      f0_valid = false;
      ++st.fallbacks;
    }
  }
  if (stats) {
    stats->accepted += st.accepted;
    stats->fallbacks += st.fallbacks;
    stats->last_residual = st.last_residual;
  }
  return GC_OK;
}

}  // extern "C"
