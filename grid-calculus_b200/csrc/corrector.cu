// Learned coarse-step corrector for 2-D Cahn-Hilliard: a 6-layer periodic
// 3x3 CNN (32 channels, GELU in tanh form), BF16 weights and activations, FP32
// accumulation on the tensor cores -- tcgen05 MMAs with tensor-memory
// accumulators for the forward and backward-data convolutions, mma.sync
// for the weight gradient -- trained and run by the kernels in this file.
//
// Network: x0 = [c, u, e, 0, ..., 0] (32 channels, NHWC), for l = 1..6:
//   z_l = conv3x3_periodic(x_{l-1}, W_l) + b_l,  x_l = gelu(z_l) (l < 6);
// the correction is delta = s_out * rho * (z_6[ch 0] - mean(z_6[ch 0]))
// per sample (zero mean, so the coarse step conserves mass).
// Without a base step: u = e = 0, rho = 1 and the coarse step is c + delta.
// With a base step B (one RKC2 step of the coarse dt Dt, gc_ch_rkc) the
// coarse step is B(c) + delta, and the network sees the base step's
// increment and its error indicator, each scaled to unit RMS per sample:
//   u = (B(c) - c) / rms(B(c) - c),
//   e = est / rms(est),  est = (B(c) - c) / Dt - (f(c) + f(B(c))) / 2
// (the trapezoid residual of the base step, f the Cahn-Hilliard RHS), with
// rho = Dt rms(est): the correction is learned in units of the base step's
// own error indicator, so small late-time errors are corrected as precisely
// as large early ones.  Every layer is computed as a 32 -> 32 convolution
// (the first layer's input channels 3..31 are zero and the last layer's
// outputs 1..31 are unused), so one implicit-GEMM kernel serves all layers:
// M = pixels, N = 32 output channels, K = 9 taps x 32 input channels.
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
#include "tma.cuh"

namespace gcb {
namespace {

constexpr int kLayers = 6;
constexpr int kC = 32;                       // channels
constexpr int kTaps = 9;
constexpr int kLayerParams = kTaps * kC * kC + kC;
constexpr int kParams = kLayers * kLayerParams;
// Weight-gradient tiles: 8 rows x 16 columns of pixels.
constexpr int kTR = 8, kTC = 16;
constexpr int kHaloR = kTR + 2, kHaloC = kTC + 2;

__device__ __forceinline__ uint32_t pack_bf16_rn(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

// GELU in its tanh form (Hendrycks & Gimpel 2016):
//   gelu(z) = z/2 (1 + tanh(u)),  u = sqrt(2/pi) (z + 0.044715 z^3),
//   gelu'(z) = (1 + tanh(u))/2 + z/2 (1 - tanh(u)^2) sqrt(2/pi) (1 + 3 0.044715 z^2),
// with the hardware tanh: tanh.approx.f32 for one value, tanh.approx.bf16x2
// for the pairs the convolution epilogues produce (one transcendental-unit
// instruction per two values: that unit bounds the epilogue; the bf16
// result is as precise as the bf16 activations it feeds).
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float2 tanh_hw2(float a, float b) {
  const uint32_t in = pack_bf16_rn(a, b);
  uint32_t out;
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(out) : "r"(in));
  return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&out));
}
constexpr float kGeluA = 0.7978845608028654f;   // sqrt(2/pi)
constexpr float kGeluB = 0.044715f;
__device__ __forceinline__ float2 gelu2(float z0, float z1) {
  const float2 t = tanh_hw2(kGeluA * fmaf(kGeluB * z0 * z0, z0, z0), kGeluA * fmaf(kGeluB * z1 * z1, z1, z1));
  return make_float2(0.5f * z0 * (1.0f + t.x), 0.5f * z1 * (1.0f + t.y));
}
__device__ __forceinline__ float2 gelu_grad2(float z0, float z1) {
  const float a0 = z0 * z0, a1 = z1 * z1;
  const float2 t = tanh_hw2(kGeluA * fmaf(kGeluB * a0, z0, z0), kGeluA * fmaf(kGeluB * a1, z1, z1));
  return make_float2(0.5f * (1.0f + t.x) + 0.5f * z0 * (1.0f - t.x * t.x) * kGeluA * fmaf(3.0f * kGeluB, a0, 1.0f),
                     0.5f * (1.0f + t.y) + 0.5f * z1 * (1.0f - t.y * t.y) * kGeluA * fmaf(3.0f * kGeluB, a1, 1.0f));
}
__device__ __forceinline__ float gelu(float z) {
  const float t = tanh_hw(kGeluA * fmaf(kGeluB * z * z, z, z));
  return 0.5f * z * (1.0f + t);
}
__device__ __forceinline__ float gelu_grad(float z) {
  const float z2 = z * z;
  const float t = tanh_hw(kGeluA * fmaf(kGeluB * z2, z, z));
  return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * kGeluA * fmaf(3.0f * kGeluB, z2, 1.0f);
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

__device__ __forceinline__ void cp_async16(void* s, const void* g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Epilogue kinds of the convolution:
//   EPI_FWD    z = acc + bias; store gelu(z) (bf16) and, for training, z (bf16)
//   EPI_LAST   z0 = acc + bias (channel 0 only); store z0 (fp32)
//   EPI_BWD    dz_prev = acc * gelu'(z_prev); store (bf16)
enum Epi { EPI_FWD = 0, EPI_LAST = 1, EPI_BWD = 2 };

// ---- tcgen05 (UMMA) forward / backward-data convolution ---------------------
// The same implicit GEMM on the 5th-generation tensor cores.  A tile is two
// image rows of 128 consecutive pixels; each row is one UMMA M = 128 with
// N = 32 output channels and K = 9 taps x 32 input channels in 18 MMAs of
// K = 16, accumulated in tensor memory.  Operands live in shared memory in
// the K-major no-swizzle layout (8-row x 16-byte core matrices): the staged
// input rows y-1 .. y+2 (130 pixels each with the periodic halo) are kept
// as four planes of 8 channels, pixel-contiguous at 16 bytes, so the A
// operand of output row j and tap (dy, dx) is the same plane started
// (j + 1 + dy) rows and (1 + dx) pixels in -- a shift of the descriptor's
// start address.  Weights are [tap][8-channel chunk][n][8].
// Software pipeline per CTA: one thread issues tile i's 36 MMAs and commits
// them to an mbarrier; meanwhile all warps wait for tile i-1's
// accumulators, stage tile i+1 by cp.async into the buffer tile i-1 used,
// and run tile i-1's epilogue (each warp reads its 32 TMEM lanes = pixels,
// 32 columns = channels; 16-byte stores).  Tiles and accumulators are
// double-buffered.  Every mbarrier wait is bounded; on expiry the CTA
// records GC_ERR_TIMEOUT, stops, and frees its tensor memory.
constexpr int kUM = 128;                       // pixels per tile row = UMMA M
constexpr int kUR = 2;                         // output rows per tile
constexpr int kUCols = kUM + 2;                // staged pixels per row
constexpr int kUPix = (kUR + 2) * kUCols;      // staged pixels
constexpr int kUChunk = kUPix * 16;            // bytes of one 8-channel plane
constexpr int kUIn = 4 * kUChunk;              // one staged tile
constexpr int kUW = kTaps * 4 * kC * 16;       // weights
constexpr int kUSmem = kUW + 2 * kUIn + 64;    // + two mbarriers and the TMEM address
constexpr int kUThreads = 256;                 // 8 warps: warp w reads TMEM lanes 32 (w % 4), channels 16 (w / 4) ..
constexpr uint32_t kUTmemCols = 2 * kUR * 32;  // two tiles x kUR accumulators of 32 columns
constexpr long long kUWaitCycles = 4000000000LL;  // about 2 s at 2 GHz
// Instruction descriptor: D f32, A and B bf16, both K-major, N = 32, M = 128.
constexpr uint32_t kUIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

// Shared-memory matrix descriptor, no swizzle: start address, leading byte
// offset (between the two 8-element K chunks), stride byte offset (between
// 8-row groups), version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      ::"r"(d_tmem), "l"(a), "l"(b), "r"(kUIdesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Epilogue of channels c0 .. c0 + 15 of one output pixel from their
// accumulator values.
template <int EPI, bool STORE_Z>
__device__ __forceinline__ void conv_epilogue(const uint32_t (&r)[16], int c0, size_t gp,
                                              const float* __restrict__ bias, __nv_bfloat16* __restrict__ out_z,
                                              __nv_bfloat16* __restrict__ out_y, float* __restrict__ out_f,
                                              const __nv_bfloat16* __restrict__ z_prev) {
  if constexpr (EPI == EPI_LAST) {
    if (c0 == 0) out_f[gp] = __uint_as_float(r[0]) + bias[0];
  } else if constexpr (EPI == EPI_FWD) {
    uint32_t o[8], zb[8];
#pragma unroll
    for (int n = 0; n < 16; n += 2) {
      const float v0 = __uint_as_float(r[n]) + __ldg(bias + c0 + n);
      const float v1 = __uint_as_float(r[n + 1]) + __ldg(bias + c0 + n + 1);
      zb[n / 2] = pack_bf16(v0, v1);
      const float2 gy = gelu2(v0, v1);
      o[n / 2] = pack_bf16(gy.x, gy.y);
    }
    if constexpr (STORE_Z) {
      uint4* dz = reinterpret_cast<uint4*>(out_z + gp * kC + c0);
      dz[0] = make_uint4(zb[0], zb[1], zb[2], zb[3]);
      dz[1] = make_uint4(zb[4], zb[5], zb[6], zb[7]);
    }
    uint4* dy = reinterpret_cast<uint4*>(out_y + gp * kC + c0);
    dy[0] = make_uint4(o[0], o[1], o[2], o[3]);
    dy[1] = make_uint4(o[4], o[5], o[6], o[7]);
  } else {
    uint32_t o[8];
    const uint4* zp = reinterpret_cast<const uint4*>(z_prev + gp * kC + c0);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const uint4 zz = __ldg(zp + q);
      const uint32_t zw[4] = {zz.x, zz.y, zz.z, zz.w};
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const float2 zf = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&zw[h]));
        const int n = 8 * q + 2 * h;
        const float2 gd = gelu_grad2(zf.x, zf.y);
        o[4 * q + h] = pack_bf16(__uint_as_float(r[n]) * gd.x, __uint_as_float(r[n + 1]) * gd.y);
      }
    }
    uint4* dz = reinterpret_cast<uint4*>(out_z + gp * kC + c0);
    dz[0] = make_uint4(o[0], o[1], o[2], o[3]);
    dz[1] = make_uint4(o[4], o[5], o[6], o[7]);
  }
}

template <int EPI, bool STORE_Z>
__global__ void __launch_bounds__(kUThreads) conv3x3_umma_kernel(
    const __nv_bfloat16* __restrict__ in, const __nv_bfloat16* __restrict__ bw, const float* __restrict__ bias,
    __nv_bfloat16* __restrict__ out_z, __nv_bfloat16* __restrict__ out_y, float* __restrict__ out_f,
    const __nv_bfloat16* __restrict__ z_prev, int H, int W, int tiles_x, int tiles_per_img, int n_tiles,
    int* status) {
  extern __shared__ __align__(128) unsigned char usm[];
  unsigned char* s_w = usm;
  unsigned char* s_in = usm + kUW;  // [2][4 chunks][kUPix][16 B]
  uint64_t* bar = reinterpret_cast<uint64_t*>(usm + kUW + 2 * kUIn);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // Weights: global [t][n][k] -> [t][k / 8][n][8].
  for (int v = tid; v < kTaps * kC * 4; v += kUThreads) {
    const int t = v >> 7, n = (v >> 2) & 31, q = v & 3;
    cp_async16(s_w + t * 2048 + q * 512 + n * 16, bw + (t * kC + n) * kC + q * 8);
  }
  auto origin = [&](int tl, int& img, int& y0, int& x0) {
    img = tl / tiles_per_img;
    const int tile = tl - img * tiles_per_img;
    const int ty = tile / tiles_x;
    y0 = ty * kUR;
    x0 = (tile - ty * tiles_x) * kUM;
  };
  auto issue = [&](int tl, int buf) {
    int img, y0, x0;
    origin(tl, img, y0, x0);
    const size_t img_off = static_cast<size_t>(img) * H * W;
    unsigned char* dst = s_in + buf * kUIn;
    for (int v = tid; v < kUPix * 4; v += kUThreads) {
      const int pix = v >> 2, q = v & 3;
      const int r = pix / kUCols, c = pix - r * kUCols;
      const size_t gp = img_off + static_cast<size_t>(wrap(y0 - 1 + r, H)) * W + wrap(x0 - 1 + c, W);
      cp_async16(dst + q * kUChunk + pix * 16, in + gp * kC + q * 8);
    }
  };
  // Warp w: TMEM lanes (pixels) 32 (w % 4) .. + 31, channels 16 (w / 4) .. + 15.
  const int quad = warp & 3, c0 = (warp >> 2) * 16;
  auto epilogue = [&](int tl, int buf) {
    int img, y0, x0;
    origin(tl, img, y0, x0);
    const int ox = x0 + quad * 32 + lane;
#pragma unroll
    for (int j = 0; j < kUR; ++j) {
      uint32_t r[16];
      tmem_ld16(*tmem_slot + (static_cast<uint32_t>(quad * 32) << 16) + buf * (kUR * 32) + j * 32 + c0, r);
      const int oy = y0 + j;
      if (ox < W && oy < H)
        conv_epilogue<EPI, STORE_Z>(r, c0, static_cast<size_t>(img) * H * W + static_cast<size_t>(oy) * W + ox,
                                    bias, out_z, out_y, out_f, z_prev);
    }
  };
  // Bounded wait for the accumulators of the tile issued at iteration k.
  auto wait_mma = [&](int k) -> bool {
    const long long t0 = clock64();
    while (!mbar_try_wait(&bar[k & 1], (k >> 1) & 1))
      if (clock64() - t0 > kUWaitCycles) {
        if (status) atomicExch(status, static_cast<int>(GC_ERR_TIMEOUT));
        return false;
      }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    return true;
  };

  issue(blockIdx.x, 0);  // the grid never exceeds n_tiles
  cp_commit();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kUTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  bool failed = false;
  int it = 0, prev = -1;
  for (int tl = blockIdx.x; tl < n_tiles; tl += gridDim.x, ++it) {
    const int buf = it & 1;
    cp_wait<0>();              // this tile's copies
    fence_proxy_async_smem();  // cp.async writes -> visible to the tensor core's reads
    if (__syncthreads_or(failed)) break;
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = smem_u32(s_in + buf * kUIn), b0 = smem_u32(s_w);
#pragma unroll
      for (int j = 0; j < kUR; ++j) {
        const uint32_t d = tmem + buf * (kUR * 32) + j * 32;
#pragma unroll
        for (int t = 0; t < kTaps; ++t) {
          const int dy = t / 3 - 1, dx = t % 3 - 1;
          const uint32_t pix0 = static_cast<uint32_t>((j + 1 + dy) * kUCols + 1 + dx);
#pragma unroll
          for (int kh = 0; kh < 2; ++kh) {
            const uint64_t ad = umma_desc(a0 + 2 * kh * kUChunk + pix0 * 16, kUChunk, 128);
            const uint64_t bd = umma_desc(b0 + t * 2048 + 2 * kh * 512, 512, 128);
            umma_bf16(d, ad, bd, (t | kh) != 0);
          }
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   ::"r"(smem_u32(&bar[buf])) : "memory");
    }
    // The previous tile's MMAs: once done, its staging buffer takes the next
    // tile and its accumulators are written out while this tile's MMAs run.
    if (prev >= 0 && !wait_mma(it - 1)) {
      failed = true;
      continue;  // the loop's barrier makes every thread stop
    }
    if (tl + static_cast<int>(gridDim.x) < n_tiles) issue(tl + gridDim.x, buf ^ 1);
    cp_commit();
    if (prev >= 0) epilogue(prev, buf ^ 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    prev = tl;
  }
  if (!failed && prev >= 0 && wait_mma(it - 1)) epilogue(prev, (it - 1) & 1);
  // Drain the copies in flight, then free the tensor memory.
  cp_wait<0>();
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kUTmemCols));
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
__device__ __forceinline__ float inv_rms(const float* ms, size_t b) {
  const float v = ms[b];
  return v > 0.f ? rsqrtf(v) : 0.f;
}

// incr = B(c) - c and est = incr / Dt - (f(c) + f(B(c))) / 2, formed in T
// and rounded to float, with their squares.
template <class T>
__global__ void base_features(const T* __restrict__ c, const T* __restrict__ base, const T* __restrict__ f0,
                              const T* __restrict__ fb, T inv_dt, size_t n, float* __restrict__ incr,
                              float* __restrict__ est, float* __restrict__ sq_incr, float* __restrict__ sq_est) {
  for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const T d = base[p] - c[p];
    const float u = static_cast<float>(d);
    const float e = static_cast<float>(d * inv_dt - T(0.5) * (f0[p] + fb[p]));
    incr[p] = u;
    est[p] = e;
    sq_incr[p] = u * u;
    sq_est[p] = e * e;
  }
}

// Channel 0 = c, channels 1, 2 = incr and est at unit RMS per sample (0
// without a base step), channels 3..31 = 0.
template <class T>
__global__ void pack_input(const T* __restrict__ c, const float* __restrict__ incr, const float* __restrict__ ms,
                           const float* __restrict__ est, const float* __restrict__ ms_est, int hw, size_t n,
                           __nv_bfloat16* __restrict__ x0) {
  for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<size_t>(gridDim.x) * blockDim.x) {
    uint4* dst = reinterpret_cast<uint4*>(x0 + p * kC);
    uint4 z = make_uint4(0, 0, 0, 0);
    const float u = incr ? incr[p] * inv_rms(ms, p / hw) : 0.f;
    const float e = est ? est[p] * inv_rms(ms_est, p / hw) : 0.f;
    z.x = pack_bf16(static_cast<float>(c[p]), u);
    z.y = pack_bf16(e, 0.f);
    dst[0] = z;
    dst[1] = make_uint4(0, 0, 0, 0);
    dst[2] = make_uint4(0, 0, 0, 0);
    dst[3] = make_uint4(0, 0, 0, 0);
  }
}

// Per-sample mean of f over H*W pixels in two fixed-order passes: kMeanParts
// CTAs per sample sum contiguous chunks in double, then one warp per sample
// adds the partials in order.
constexpr int kMeanParts = 32;

__global__ void sample_sum_parts(const float* __restrict__ f, int hw, double* __restrict__ part) {
  __shared__ double sh[256];
  const int b = blockIdx.y, k = blockIdx.x;
  const int len = (hw + kMeanParts - 1) / kMeanParts;
  const int lo = k * len, hi = min(hw, lo + len);
  const float* s = f + static_cast<size_t>(b) * hw;
  double acc = 0.0;
  for (int i = lo + threadIdx.x; i < hi; i += 256) acc += s[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w >= 1; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[b * kMeanParts + k] = sh[0];
}

__global__ void sample_mean_final(const double* __restrict__ part, int hw, int batch, float* __restrict__ mean) {
  const int b = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (b >= batch) return;
  double v = lane < kMeanParts ? part[b * kMeanParts + lane] : 0.0;
  for (int o = 16; o >= 1; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (lane == 0) mean[b] = static_cast<float>(v / hw);
}


// delta = scale rho_b (z - mean_z), rho_b = sqrt(ms[b]) (1 without ms).
__global__ void project_delta(const float* __restrict__ z, const float* __restrict__ mean,
                              const float* __restrict__ ms, int hw, size_t n, float scale,
                              float* __restrict__ delta) {
  for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const float rho = ms ? sqrtf(ms[p / hw]) : 1.f;
    delta[p] = scale * rho * (z[p] - mean[p / hw]);
  }
}

// out = incr + delta: the whole coarse-step increment.
__global__ void add_increment(const float* __restrict__ incr, const float* __restrict__ delta, size_t n,
                              float* __restrict__ out) {
  for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<size_t>(gridDim.x) * blockDim.x)
    out[p] = incr[p] + delta[p];
}

// (target - start)^2, for the per-sample scale of the normalised loss.
template <class T>
__global__ void step_sq(const T* __restrict__ c, const T* __restrict__ target, size_t n, float* __restrict__ out) {
  for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const float d = static_cast<float>(target[p] - c[p]);
    out[p] = d * d;
  }
}

// r = start + delta - target (start = B(c) with a base step, else c),
// formed in T and stored as float; per-CTA partial sums of r^2 / den[sample]
// (den = 1 for the plain loss; fixed grid).
template <class T>
__global__ void residual_kernel(const T* __restrict__ start, const float* __restrict__ delta,
                                const T* __restrict__ target, size_t n, int hw,
                                const float* __restrict__ den, float* __restrict__ r,
                                double* __restrict__ part) {
  __shared__ double sh[256];
  double acc = 0.0;
  for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const float v = static_cast<float>((start[p] - target[p]) + static_cast<T>(delta[p]));
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

// dz6 (channel 0) = scale rho_b 2/N (r - mean_sample(r)) / den[sample]
// (scale = s_out Dt with a base step, else s_out; `scale` here already
// includes 2/N); other channels 0.
__global__ void last_layer_grad(const float* __restrict__ r, const float* __restrict__ rmean, int hw, size_t n,
                                float scale, const float* __restrict__ den, const float* __restrict__ ms,
                                __nv_bfloat16* __restrict__ dz) {
  for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<size_t>(gridDim.x) * blockDim.x) {
    uint4* dst = reinterpret_cast<uint4*>(dz + p * kC);
    const float w = (den ? 1.0f / den[p / hw] : 1.0f) * (ms ? sqrtf(ms[p / hw]) : 1.f);
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

// cand = start + delta (start = B(psi) with a base step, else psi)
__global__ void apply_delta(const double* __restrict__ psi, const float* __restrict__ delta, size_t n,
                            double* __restrict__ cand) {
  for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<size_t>(gridDim.x) * blockDim.x)
    cand[p] = psi[p] + static_cast<double>(delta[p]);
}

// Acceptance statistics of a coarse step, per CTA (fixed grid, double):
//   [0] sum of the free-energy density of c1, -c^2/2 + c^4/4 + kappa/2 |grad c|^2
//       (order-2 central gradient, the reference's density), times the cell area;
//   [1] sum of ((c1 - c0)/Dt - (f0 + f1)/2)^2 and [2] of ((f0 + f1)/2)^2
//       (the trapezoid residual; skipped when c0 is null).
// 2-D periodic grid; part holds 3 x gridDim.x doubles.
__global__ void accept_stats(const double* __restrict__ c0, const double* __restrict__ c1,
                             const double* __restrict__ f0, const double* __restrict__ f1, int nx, int ny,
                             double inv_2hx, double inv_2hy, double area, double kappa, double inv_dt,
                             double* __restrict__ part) {
  __shared__ double se[256], sr[256], sf[256];
  double ae = 0.0, ar = 0.0, af = 0.0;
  const size_t n = static_cast<size_t>(nx) * ny;
  for (size_t p = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int j = static_cast<int>(p / nx), i = static_cast<int>(p - static_cast<size_t>(j) * nx);
    const double c = c1[p];
    const double gx = (c1[static_cast<size_t>(j) * nx + wrap(i + 1, nx)] -
                       c1[static_cast<size_t>(j) * nx + wrap(i - 1, nx)]) * inv_2hx;
    const double gy = (c1[static_cast<size_t>(wrap(j + 1, ny)) * nx + i] -
                       c1[static_cast<size_t>(wrap(j - 1, ny)) * nx + i]) * inv_2hy;
    const double c2 = c * c;
    ae += -0.5 * c2 + 0.25 * c2 * c2 + 0.5 * kappa * (gx * gx + gy * gy);
    if (c0) {
      const double fm = 0.5 * (f0[p] + f1[p]);
      const double r = (c - c0[p]) * inv_dt - fm;
      ar += r * r;
      af += fm * fm;
    }
  }
  se[threadIdx.x] = ae;
  sr[threadIdx.x] = ar;
  sf[threadIdx.x] = af;
  __syncthreads();
  for (int w = 128; w >= 1; w >>= 1) {
    if (threadIdx.x < w) {
      se[threadIdx.x] += se[threadIdx.x + w];
      sr[threadIdx.x] += sr[threadIdx.x + w];
      sf[threadIdx.x] += sf[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x] = se[0] * area;
    part[3 * blockIdx.x + 1] = sr[0];
    part[3 * blockIdx.x + 2] = sf[0];
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
  double* part = nullptr;           // per-CTA partial sums (3 x kRedBlocks)
  float* wpart = nullptr;           // per-CTA weight-gradient partials
  int wparts = 0;
  double* mpart = nullptr;          // per-sample partial sums (kMeanParts per sample)
  double* adv = nullptr;            // advance scratch: cand, f1 (H x W each)
  double* rkc = nullptr;            // base-step scratch: 4 fields of H x W doubles
  double* host_part = nullptr;      // pinned copy of the acceptance partials
  // Captured graph of one proposed coarse step (forward, candidate,
  // acceptance statistics), rebuilt when anything it bakes in changes.
  cudaGraphExec_t prop_exec = nullptr;
  uint64_t prop_key[8] = {};
  // Base step B = one RKC2 step of dt_coarse with `stages` stages and the
  // Cahn-Hilliard RHS chp (off until gc_corrector_set_base).
  bool base = false;
  gc_ch_params chp{1.0, 1.0, 2};
  double dt_coarse = 0.0;
  int stages = 0;
  double* bbuf = nullptr;           // B(c), max_batch x H x W (double-sized)
  double* f0buf = nullptr;          // f(c)
  double* fbbuf = nullptr;          // f(B(c))
  float* incr = nullptr;            // B(c) - c
  float* est = nullptr;             // trapezoid residual of the base step
  float* ms = nullptr;              // per-sample mean squares of incr, est
  float* ms_est = nullptr;
  float* den = nullptr;             // per-sample scale of the normalised loss
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

gc_status sample_mean(gc_corrector* c, int batch, const float* f, int hw, float* mean) {
  cudaStream_t st = c->ctx->stream;
  sample_sum_parts<<<dim3(kMeanParts, batch), 256, 0, st>>>(f, hw, c->mpart);
  GC_CHECK_LAUNCH("sample_sum_parts");
  sample_mean_final<<<div_up(batch, 8), 256, 0, st>>>(c->mpart, hw, batch, mean);
  GC_CHECK_LAUNCH("sample_mean_final");
  return GC_OK;
}

// Convolution layer on the tcgen05 kernel (NT: output channels the
// epilogue needs -- 32, or 1 for the last layer).
template <int EPI, int NT, bool STORE_Z>
gc_status launch_conv(gc_corrector* c, int batch, const __nv_bfloat16* in, const __nv_bfloat16* w,
                      const float* bias, __nv_bfloat16* oz, __nv_bfloat16* oy, float* of, const __nv_bfloat16* zp) {
  auto kern = conv3x3_umma_kernel<EPI, STORE_Z>;
  GC_TRY(kernel_setup(kern, kUThreads, kUSmem));
  const int tiles_x = div_up(c->W, kUM);
  const int tpi = tiles_x * div_up(c->H, kUR);
  const int n_tiles = batch * tpi;
  const int grid = std::min(n_tiles, 2 * c->ctx->num_sms);  // two CTAs per SM (shared memory)
  kern<<<grid, kUThreads, kUSmem, c->ctx->stream>>>(in, w, bias, oz, oy, of, zp, c->H, c->W, tiles_x, tpi, n_tiles,
                                                    c->ctx->device_status);
  GC_CHECK_LAUNCH("conv3x3_umma_kernel");
  return GC_OK;
}

// Output scale of the network: s_out Dt with a base step (times rho_b =
// rms(est) per sample), else s_out.
float out_scale(const gc_corrector* c) {
  return c->base ? c->s_out * static_cast<float>(c->dt_coarse) : c->s_out;
}

template <class T>
gc_status corr_forward(gc_corrector* c, int batch, const T* in, bool train) {
  GC_TRY(corr_layout(c));
  const int H = c->H, W = c->W;
  const size_t n = static_cast<size_t>(batch) * H * W;
  cudaStream_t st = c->ctx->stream;
  const int grid_ew = c->ctx->num_sms * 8;
  if (c->base) {
    const gc_grid g{W, H, 1, 1.0, 1.0, 1.0};
    const gc_dtype dt = sizeof(T) == 8 ? GC_F64 : GC_F32;
    T* bb = reinterpret_cast<T*>(c->bbuf);
    T* f0 = reinterpret_cast<T*>(c->f0buf);
    T* fb = reinterpret_cast<T*>(c->fbbuf);
    GC_CUDA(cudaMemcpyAsync(bb, in, sizeof(T) * n, cudaMemcpyDeviceToDevice, st));
    const size_t hw = static_cast<size_t>(H) * W;
    void* const scratch[4] = {c->rkc, c->rkc + hw, c->rkc + 2 * hw, c->rkc + 3 * hw};
    for (int b = 0; b < batch; ++b) {
      const size_t o = b * hw;
      GC_TRY(ch_rkc_enqueue(c->ctx, &g, dt, &c->chp, bb + o, c->dt_coarse, c->stages, scratch));
      GC_TRY(ch_rhs_enqueue(c->ctx, &g, dt, &c->chp, in + o, f0 + o));
      GC_TRY(ch_rhs_enqueue(c->ctx, &g, dt, &c->chp, bb + o, fb + o));
    }
    // squares of incr into resid, of est into delta (both overwritten below)
    base_features<T><<<grid_ew, 256, 0, st>>>(in, bb, f0, fb, static_cast<T>(1.0 / c->dt_coarse), n, c->incr,
                                               c->est, c->resid, c->delta);
    GC_CHECK_LAUNCH("base_features");
    GC_TRY(sample_mean(c, batch, c->resid, H * W, c->ms));
    GC_TRY(sample_mean(c, batch, c->delta, H * W, c->ms_est));
  }
  pack_input<T><<<grid_ew, 256, 0, st>>>(in, c->base ? c->incr : nullptr, c->ms, c->base ? c->est : nullptr,
                                         c->ms_est, H * W, n, c->x[0]);
  GC_CHECK_LAUNCH("pack_input");
  for (int l = 0; l < kLayers; ++l) {
    const __nv_bfloat16* wl = c->w_fwd + static_cast<size_t>(l) * kTaps * kC * kC;
    const float* bl = c->params + static_cast<size_t>(l) * kLayerParams + kTaps * kC * kC;
    gc_status s;
    if (l + 1 < kLayers) {
      s = train ? launch_conv<EPI_FWD, 4, true>(c, batch, c->x[l], wl, bl, c->z[l], c->x[l + 1], nullptr, nullptr)
                : launch_conv<EPI_FWD, 4, false>(c, batch, c->x[l], wl, bl, nullptr, c->x[l + 1], nullptr, nullptr);
    } else {
      s = launch_conv<EPI_LAST, 1, false>(c, batch, c->x[l], wl, bl, nullptr, nullptr, c->zlast, nullptr);
    }
    if (s != GC_OK) return s;
  }
  GC_TRY(sample_mean(c, batch, c->zlast, H * W, c->mean));
  project_delta<<<grid_ew, 256, 0, st>>>(c->zlast, c->mean, c->base ? c->ms_est : nullptr, H * W, n, out_scale(c),
                                         c->delta);
  GC_CHECK_LAUNCH("project_delta");
  return GC_OK;
}

// Forward + loss + backward into c->grad (no update).
// loss = sum_b sum_p (start + delta - target)^2 / (N den_b), N = batch H W,
// start = B(c) with a base step else c, den_b = mean((target - start)^2)
// of sample b with the normalised loss else 1 (so with a base step the loss
// is the squared error left relative to the base step's own error).
template <class T>
gc_status corr_backward(gc_corrector* c, int batch, const T* cin, const T* target, double* loss) {
  GC_TRY(corr_forward<T>(c, batch, cin, true));
  const int H = c->H, W = c->W, hw = H * W;
  const size_t n = static_cast<size_t>(batch) * hw;
  cudaStream_t st = c->ctx->stream;
  const int grid_ew = c->ctx->num_sms * 8;
  const T* start = c->base ? reinterpret_cast<const T*>(c->bbuf) : cin;
  const float* den = nullptr;
  if (c->normalized) {
    step_sq<T><<<grid_ew, 256, 0, st>>>(start, target, n, c->resid);
    GC_TRY(sample_mean(c, batch, c->resid, hw, c->den));
    den = c->den;
  }
  residual_kernel<T><<<kRedBlocks, 256, 0, st>>>(start, c->delta, target, n, hw, den, c->resid, c->part);
  GC_CHECK_LAUNCH("residual_kernel");
  GC_TRY(sample_mean(c, batch, c->resid, hw, c->mean2));
  const float scale = out_scale(c) * 2.0f / static_cast<float>(n);
  __nv_bfloat16* dz = c->dz_a;
  __nv_bfloat16* dzn = c->dz_b;
  last_layer_grad<<<grid_ew, 256, 0, st>>>(c->resid, c->mean2, hw, n, scale, den, c->base ? c->ms_est : nullptr, dz);
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
      GC_TRY((launch_conv<EPI_BWD, 4, true>(c, batch, dz, wl, nullptr, dzn, nullptr, nullptr, c->z[l - 1])));
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

gc_status corr_backward_any(gc_corrector* c, int batch, gc_dtype dt, const void* cin, const void* target,
                            double* loss) {
  if (dt == GC_F64)
    return corr_backward<double>(c, batch, static_cast<const double*>(cin), static_cast<const double*>(target), loss);
  return corr_backward<float>(c, batch, static_cast<const float*>(cin), static_cast<const float*>(target), loss);
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
  alloc(reinterpret_cast<void**>(&c->bbuf), sizeof(double) * n);
  alloc(reinterpret_cast<void**>(&c->f0buf), sizeof(double) * n);
  alloc(reinterpret_cast<void**>(&c->fbbuf), sizeof(double) * n);
  alloc(reinterpret_cast<void**>(&c->incr), sizeof(float) * n);
  alloc(reinterpret_cast<void**>(&c->est), sizeof(float) * n);
  alloc(reinterpret_cast<void**>(&c->ms), sizeof(float) * max_batch);
  alloc(reinterpret_cast<void**>(&c->ms_est), sizeof(float) * max_batch);
  alloc(reinterpret_cast<void**>(&c->den), sizeof(float) * max_batch);
  alloc(reinterpret_cast<void**>(&c->mpart), sizeof(double) * kMeanParts * max_batch);
  alloc(reinterpret_cast<void**>(&c->rkc), sizeof(double) * 4 * height * width);
  alloc(reinterpret_cast<void**>(&c->adv), sizeof(double) * 2 * height * width);
  if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&c->host_part), sizeof(double) * 3 * kRedBlocks);
  alloc(reinterpret_cast<void**>(&c->tbuf), sizeof(float) * n);
  alloc(reinterpret_cast<void**>(&c->part), sizeof(double) * 3 * kRedBlocks);
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
                  c->bbuf, c->f0buf, c->fbbuf, c->incr, c->est, c->ms, c->ms_est, c->den, c->mpart, c->rkc};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (auto* p : c->x)
    if (p) cudaFree(p);
  for (auto* p : c->z)
    if (p) cudaFree(p);
  if (c->host_part) cudaFreeHost(c->host_part);
  if (c->prop_exec) cudaGraphExecDestroy(c->prop_exec);
  delete c;
  return GC_OK;
}

GC_API int32_t gc_corrector_num_params(void) { return kParams; }

GC_API gc_status gc_corrector_set_base(gc_corrector* c, const gc_ch_params* p, double dt_coarse, int32_t stages) {
  if (!c) return fail(GC_ERR_INVALID_ARG, "gc_corrector_set_base: null corrector");
  if (!p) {
    c->base = false;
    return GC_OK;
  }
  if (p->order != 2 && p->order != 4 && p->order != 6)
    return fail(GC_ERR_UNSUPPORTED, "gc_corrector_set_base: order must be 2, 4 or 6");
  if (stages < 2 || stages > 64 || !(dt_coarse > 0.0))
    return fail(GC_ERR_INVALID_ARG, "gc_corrector_set_base: need dt_coarse > 0 and 2 <= stages <= 64");
  const gc_grid g{c->W, c->H, 1, 1.0, 1.0, 1.0};
  gc_status s = require_axes(&g, p->order / 2);
  if (s != GC_OK) return s;
  c->base = true;
  c->chp = *p;
  c->dt_coarse = dt_coarse;
  c->stages = stages;
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

// delta_out = the coarse-step increment for each of `batch` fields c (fp32
// or fp64, batch x H x W): B(c) - c + delta with a base step, else delta.
GC_API gc_status gc_corrector_forward(gc_corrector* c, int32_t batch, gc_dtype dt, const void* cin,
                                      float* delta_out) {
  if (!c || !cin || !delta_out) return fail(GC_ERR_INVALID_ARG, "gc_corrector_forward: null pointer");
  Call call(c->ctx);
  if (call.st != GC_OK) return call.st;
  if (batch < 1 || batch > c->max_batch) return fail(GC_ERR_INVALID_ARG, "gc_corrector_forward: batch out of range");
  gc_status s = dt == GC_F64 ? corr_forward<double>(c, batch, static_cast<const double*>(cin), false)
                             : corr_forward<float>(c, batch, static_cast<const float*>(cin), false);
  if (s != GC_OK) return s;
  const size_t n = static_cast<size_t>(batch) * c->H * c->W;
  if (c->base) {
    add_increment<<<c->ctx->num_sms * 8, 256, 0, c->ctx->stream>>>(c->incr, c->delta, n, delta_out);
    GC_CHECK_LAUNCH("add_increment");
  } else {
    GC_CUDA(cudaMemcpyAsync(delta_out, c->delta, sizeof(float) * n, cudaMemcpyDeviceToDevice, c->ctx->stream));
  }
  return GC_OK;
}

// Gradient of the training loss (corr_backward) into grad_host (kParams
// floats), without updating the parameters.
GC_API gc_status gc_corrector_gradient(gc_corrector* c, int32_t batch, gc_dtype dt, const void* cin,
                                       const void* target, float* grad_host, double* loss) {
  if (!c || !cin || !target) return fail(GC_ERR_INVALID_ARG, "gc_corrector_gradient: null pointer");
  Call call(c->ctx);
  if (call.st != GC_OK) return call.st;
  if (batch < 1 || batch > c->max_batch) return fail(GC_ERR_INVALID_ARG, "gc_corrector_gradient: batch out of range");
  gc_status s = corr_backward_any(c, batch, dt, cin, target, loss);
  if (s != GC_OK) return s;
  if (grad_host) {
    GC_CUDA(cudaMemcpyAsync(grad_host, c->grad, sizeof(float) * kParams, cudaMemcpyDeviceToHost, c->ctx->stream));
    GC_CUDA(cudaStreamSynchronize(c->ctx->stream));
  }
  return GC_OK;
}

// One Adam step on the training loss (inputs and targets on the device).
GC_API gc_status gc_corrector_train_step(gc_corrector* c, int32_t batch, gc_dtype dt, const void* cin,
                                         const void* target, float lr, double* loss) {
  NvtxScope nvtx("gc_corrector_train_step");
  if (!c || !cin || !target) return fail(GC_ERR_INVALID_ARG, "gc_corrector_train_step: null pointer");
  Call call(c->ctx);
  if (call.st != GC_OK) return call.st;
  if (batch < 1 || batch > c->max_batch) return fail(GC_ERR_INVALID_ARG, "gc_corrector_train_step: batch out of range");
  gc_status s = corr_backward_any(c, batch, dt, cin, target, loss);
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
// dt_fine * fine_per_coarse.  Each coarse step proposes B(c) + delta(c)
// (c + delta(c) without a base step) and accepts it when the free energy
// does not rise by more than energy_tol + energy_rtol |F| and the trapezoid residual
// |(c1 - c0)/Dt - (f(c0) + f(c1))/2| / |(f(c0) + f(c1))/2| is at most
// residual_tol; otherwise the step is taken by fine_per_coarse plain RK4
// steps.  The proposal (base step, network, candidate, acceptance
// statistics) is one captured CUDA graph; the host reads the statistics
// back once per coarse step to decide.
GC_API gc_status gc_corrector_advance(gc_corrector* c, const gc_grid* g, const gc_ch_params* cp, double* psi,
                                      int32_t n_coarse, const gc_corrector_policy* pol,
                                      gc_corrector_stats* stats) {
  NvtxScope nvtx("gc_corrector_advance");
  if (!c || !g || !cp || !psi || !pol) return fail(GC_ERR_INVALID_ARG, "gc_corrector_advance: null pointer");
  Call call(c->ctx);
  if (call.st != GC_OK) return call.st;
  if (g->nz != 1 || g->ny != c->H || g->nx != c->W)
    return fail(GC_ERR_GRID_MISMATCH, "gc_corrector_advance: grid must be 2-D and match the corrector's size");
  if (n_coarse < 0 || pol->fine_per_coarse < 1 || !(pol->dt_fine > 0.0))
    return fail(GC_ERR_INVALID_ARG, "gc_corrector_advance: bad policy or step count");
  if (cp->order != 2 && cp->order != 4 && cp->order != 6)
    return fail(GC_ERR_UNSUPPORTED, "gc_corrector_advance: order must be 2, 4 or 6");
  gc_status s = require_axes(g, cp->order / 2);
  if (s != GC_OK) return s;
  if (c->base && (g->hx != 1.0 || g->hy != 1.0))
    return fail(GC_ERR_INVALID_ARG, "gc_corrector_advance: the base step works on unit cell spacing");
  gc_context* ctx = c->ctx;
  cudaStream_t st = ctx->stream;
  const size_t n = static_cast<size_t>(c->H) * c->W;
  double* cand = c->adv;
  double* f1 = c->adv + n;
  const double dt_coarse = pol->dt_fine * pol->fine_per_coarse;
  const double inv_2hx = 0.5 / g->hx, inv_2hy = 0.5 / g->hy, area = g->hx * g->hy;

  // Acceptance statistics of c1 (and of the step c0 -> c1 when c0 != null)
  // into c->part.
  auto stats_enqueue = [&](const double* c0, const double* c1) -> gc_status {
    accept_stats<<<kRedBlocks, 256, 0, st>>>(c0, c1, c->f0buf, f1, c->W, c->H, inv_2hx, inv_2hy, area, cp->kappa,
                                              1.0 / dt_coarse, c->part);
    GC_CHECK_LAUNCH("accept_stats");
    return GC_OK;
  };
  double sums[3];
  auto read_stats = [&]() -> gc_status {
    GC_CUDA(cudaMemcpyAsync(c->host_part, c->part, sizeof(double) * 3 * kRedBlocks, cudaMemcpyDeviceToHost, st));
    GC_CUDA(cudaStreamSynchronize(st));
    sums[0] = sums[1] = sums[2] = 0.0;
    for (int b = 0; b < kRedBlocks; ++b)
      for (int q = 0; q < 3; ++q) sums[q] += c->host_part[3 * b + q];
    return GC_OK;
  };
  // One proposal: cand = B(psi) + delta(psi), f1 = f(cand), statistics.
  // The forward pass with a base step leaves f(psi) in f0buf (with chp;
  // it is recomputed with cp when the two differ or without a base step).
  const bool same_rhs = c->base && c->chp.order == cp->order && c->chp.mobility == cp->mobility &&
                        c->chp.kappa == cp->kappa;
  auto propose = [&]() -> gc_status {
    GC_TRY(corr_forward<double>(c, 1, psi, false));
    apply_delta<<<ctx->num_sms * 8, 256, 0, st>>>(c->base ? c->bbuf : psi, c->delta, n, cand);
    GC_CHECK_LAUNCH("apply_delta");
    if (!same_rhs) GC_TRY(ch_rhs_enqueue(ctx, g, GC_F64, cp, psi, c->f0buf));
    GC_TRY(ch_rhs_enqueue(ctx, g, GC_F64, cp, cand, f1));
    return stats_enqueue(psi, cand);
  };
  const uint64_t key[8] = {reinterpret_cast<uint64_t>(psi), bits_of(dt_coarse), bits_of(cp->mobility),
                           bits_of(cp->kappa),
                           (static_cast<uint64_t>(cp->order) << 32) ^ static_cast<uint64_t>(c->stages) ^
                               (c->base ? 1ULL << 40 : 0),
                           bits_of(c->dt_coarse) ^ bits_of(c->chp.kappa) * 3 ^ bits_of(c->chp.mobility) * 5 ^
                               static_cast<uint64_t>(c->chp.order) << 56,
                           bits_of(static_cast<double>(c->s_out)) ^ bits_of(g->hx) * 7, bits_of(g->hy)};

  GC_TRY(stats_enqueue(nullptr, psi));
  GC_TRY(read_stats());
  double F0 = sums[0];
  gc_corrector_stats sres{};
  // The base step alone, B(psi) (left in bbuf by the proposal), under the
  // same test; taken when it passes.  F0 is updated on success.
  gc_status base_st = GC_OK;
  auto tried_base = [&](double& f0) -> bool {
    if ((base_st = ch_rhs_enqueue(ctx, g, GC_F64, cp, c->bbuf, f1)) != GC_OK) return false;
    if ((base_st = stats_enqueue(psi, c->bbuf)) != GC_OK) return false;
    if ((base_st = read_stats()) != GC_OK) return false;
    const double Fb = sums[0];
    const double rb = sums[2] > 0.0 ? std::sqrt(sums[1] / sums[2]) : 0.0;
    if (Fb <= f0 + (pol->energy_tol + pol->energy_rtol * std::fabs(f0)) && rb <= pol->residual_tol) {
      if (cudaMemcpyAsync(psi, c->bbuf, sizeof(double) * n, cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
        base_st = cuda_fail(cudaGetLastError(), "gc_corrector_advance: base step copy");
        return false;
      }
      f0 = Fb;
      return true;
    }
    return false;
  };
  for (int k = 0; k < n_coarse; ++k) {
    GC_TRY(corr_layout(c));
    if (c->prop_exec && std::memcmp(key, c->prop_key, sizeof(key)) == 0) {
      GC_CUDA(cudaGraphLaunch(c->prop_exec, st));
    } else {
      // Run this proposal directly (which also sets up every lazily
      // initialised kernel attribute), then capture the sequence for the
      // following steps.
      GC_TRY(propose());
      if (c->prop_exec) {
        cudaGraphExecDestroy(c->prop_exec);
        c->prop_exec = nullptr;
      }
      cudaGraph_t graph = nullptr;
      GC_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
      const gc_status cs = propose();
      const cudaError_t ce = cudaStreamEndCapture(st, &graph);
      if (cs != GC_OK) {
        if (graph) cudaGraphDestroy(graph);
        return cs;
      }
      if (ce != cudaSuccess) return cuda_fail(ce, "gc_corrector_advance: capture");
      const cudaError_t ie = cudaGraphInstantiate(&c->prop_exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ie != cudaSuccess) {
        c->prop_exec = nullptr;
        return cuda_fail(ie, "gc_corrector_advance: graph instantiation");
      }
      std::memcpy(c->prop_key, key, sizeof(key));
    }
    GC_TRY(read_stats());
    const double F1 = sums[0];
    const double res = sums[2] > 0.0 ? std::sqrt(sums[1] / sums[2]) : 0.0;
    const bool energy_ok = F1 <= F0 + (pol->energy_tol + pol->energy_rtol * std::fabs(F0));
    const bool residual_ok = res <= pol->residual_tol;
    const bool accept = energy_ok && residual_ok;
    sres.last_residual = res;
    if (!energy_ok) ++sres.rejected_energy;
    if (!residual_ok) ++sres.rejected_residual;
    if (accept) {
      GC_CUDA(cudaMemcpyAsync(psi, cand, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
      F0 = F1;
      ++sres.accepted;
    } else if (pol->try_base && c->base && tried_base(F0)) {
      ++sres.accepted_base;
    } else {
      if ((s = gc_ch_integrate(ctx, g, GC_F64, cp, psi, pol->dt_fine, pol->fine_per_coarse, GC_RK4)) != GC_OK)
        return s;
      if (base_st != GC_OK) return base_st;
      GC_TRY(stats_enqueue(nullptr, psi));
      GC_TRY(read_stats());
      F0 = sums[0];
      ++sres.fallbacks;
    }
    if (base_st != GC_OK) return base_st;
  }
  if (stats) {
    stats->accepted += sres.accepted;
    stats->fallbacks += sres.fallbacks;
    stats->rejected_energy += sres.rejected_energy;
    stats->rejected_residual += sres.rejected_residual;
    stats->accepted_base += sres.accepted_base;
    stats->last_residual = sres.last_residual;
  }
  return GC_OK;
}

}  // extern "C"
