// Spectral derivatives on the GPU (spectral/Derivatives.hpp:78-240,
// spectral/Wavenumbers.hpp:50-110): a real-to-complex FFT of the field, one
// kernel applying the derivative's multiplier to the half spectrum, and the
// complex-to-real FFT back, all with this library's own kernels.
//
// Transforms: one CTA per line of one axis, the line staged in shared
// memory.  A power-of-two length runs the iterative radix-2 (Cooley-Tukey,
// decimation in time) butterflies; any other length a direct DFT.  Both take
// their twiddles exp(-2 pi i k / N) from a table computed on the host in
// long double and kept by the context per length.  The x axis is
// real-to-half-complex (the first N/2 + 1 outputs of the line's transform);
// its inverse extends the half spectrum by Hermitian symmetry, transforms
// and keeps the real part -- what a complex-to-real transform computes (the
// imaginary parts of the self-conjugate modes drop out).  The multiplier
// folds in the 1/N normalisation of the inverse transform.
//
// Conventions kept from the reference: wavenumbers k = 2 pi n / (N h) with
// n in [0, N/2] along x (the half spectrum) and the signed range along y
// and z (n - N for 2 n >= N); an odd derivative count along an axis of even
// extent zeroes that axis's Nyquist mode; a degenerate axis (N = 1) has the
// single wavenumber 0.  Results agree with the reference's PocketFFT path to
// rounding (the transforms differ in their operation order).
#include <algorithm>
#include <cmath>
#include <map>
#include <string>
#include <vector>

#include "common.cuh"

namespace gcb {
namespace {

// Twiddle tables of one context, one per transform length: tw[k] =
// exp(-2 pi i k / N), k < N.  A context is driven by one host thread at a
// time, so the cache needs no lock; the tables are freed with the context.
struct TwiddleCache {
  std::map<int, double2*> tables;
};

void release_twiddles(void* p) {
  auto* cache = static_cast<TwiddleCache*>(p);
  for (auto& kv : cache->tables) cudaFree(kv.second);
  delete cache;
}

gc_status twiddles_for(gc_context* ctx, int n, const double2** out) {
  if (!ctx->spectral_plans) {
    ctx->spectral_plans = new TwiddleCache;
    ctx->spectral_release = release_twiddles;
  }
  auto& tables = static_cast<TwiddleCache*>(ctx->spectral_plans)->tables;
  auto it = tables.find(n);
  if (it == tables.end()) {
    std::vector<double2> host(static_cast<size_t>(n));
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int k = 0; k < n; ++k) {
      const long double a = two_pi * static_cast<long double>(k) / static_cast<long double>(n);
      host[static_cast<size_t>(k)] = make_double2(static_cast<double>(std::cos(a)), static_cast<double>(-std::sin(a)));
    }
    double2* dev = nullptr;
    GC_CUDA(cudaMalloc(&dev, sizeof(double2) * static_cast<size_t>(n)));
    const cudaError_t e = cudaMemcpy(dev, host.data(), sizeof(double2) * static_cast<size_t>(n), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cudaFree(dev);
      return cuda_fail(e, "spectral: twiddle table upload");
    }
    it = tables.emplace(n, dev).first;
  }
  *out = it->second;
  return GC_OK;
}

// Transform modes: complex lines in place; a real row to its half spectrum
// (forward, x axis); a half spectrum to a real row (inverse, x axis).
enum FftMode { FFT_C2C = 0, FFT_R2C = 1, FFT_C2R = 2 };
constexpr int kFftThreads = 128;

struct FftLines {
  int n;               // line length
  int nh;              // half-spectrum length (x axis: n / 2 + 1)
  int log2n;           // log2(n) for a power of two, else -1 (direct DFT)
  long long inner;     // line l starts at (l / inner) * outer_stride + (l % inner) * inner_stride (C2C)
  long long inner_stride, outer_stride, elem_stride;
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

template <int MODE, bool INV>
__global__ void __launch_bounds__(kFftThreads) fft_lines(const double* __restrict__ rin, double2* __restrict__ data,
                                                         double* __restrict__ rout, const FftLines f,
                                                         const double2* __restrict__ tw) {
  extern __shared__ double2 sl[];  // the line; a direct DFT also keeps its input (second half)
  const long long l = blockIdx.x;
  const int n = f.n, tid = threadIdx.x;
  double2* x = sl;
  // Load (bit-reversed positions for the radix-2 path).
  auto put = [&](int i, double2 v) {
    if (f.log2n >= 0) x[__brev(static_cast<unsigned>(i)) >> (32 - max(f.log2n, 1)) & (n - 1)] = v;
    else x[n + i] = v;
  };
  long long base = 0;
  if constexpr (MODE == FFT_C2C) base = (l / f.inner) * f.outer_stride + (l % f.inner) * f.inner_stride;
  for (int i = tid; i < n; i += kFftThreads) {
    double2 v;
    if constexpr (MODE == FFT_C2C) {
      v = data[base + i * f.elem_stride];
    } else if constexpr (MODE == FFT_R2C) {
      v = make_double2(rin[l * n + i], 0.0);
    } else {
      v = i < f.nh ? data[l * f.nh + i] : data[l * f.nh + (n - i)];
      if (i >= f.nh) v.y = -v.y;  // X[n - k] = conj(X[k])
    }
    put(i, v);
  }
  __syncthreads();
  if (f.log2n >= 0) {
    for (int half = 1; half < n; half <<= 1) {
      const int step = n / (2 * half);
      for (int j = tid; j < n / 2; j += kFftThreads) {
        const int pos = j & (half - 1);
        const int a = ((j - pos) << 1) + pos, b = a + half;
        double2 w = tw[pos * step];
        if (INV) w.y = -w.y;
        const double2 t = cmul(w, x[b]), u = x[a];
        x[a] = make_double2(u.x + t.x, u.y + t.y);
        x[b] = make_double2(u.x - t.x, u.y - t.y);
      }
      __syncthreads();
    }
  } else {
    for (int k = tid; k < n; k += kFftThreads) {
      double2 acc = make_double2(0.0, 0.0);
      int idx = 0;  // (j k) mod n
      for (int j = 0; j < n; ++j) {
        double2 w = tw[idx];
        if (INV) w.y = -w.y;
        const double2 v = cmul(w, x[n + j]);
        acc.x += v.x;
        acc.y += v.y;
        idx += k;
        if (idx >= n) idx -= n;
      }
      x[k] = acc;
    }
    __syncthreads();
  }
  for (int i = tid; i < n; i += kFftThreads) {
    if constexpr (MODE == FFT_C2C) data[base + i * f.elem_stride] = x[i];
    else if constexpr (MODE == FFT_R2C) {
      if (i < f.nh) data[l * f.nh + i] = x[i];
    } else {
      rout[l * n + i] = x[i].x;
    }
  }
}

int log2_exact(int n) {
  if (n < 1 || (n & (n - 1)) != 0) return -1;
  int k = 0;
  while ((1 << k) < n) ++k;
  return k;
}

template <int MODE, bool INV>
gc_status launch_fft(gc_context* ctx, const double* rin, double2* data, double* rout, FftLines f, long long lines) {
  const double2* tw = nullptr;
  GC_TRY(twiddles_for(ctx, f.n, &tw));
  f.log2n = log2_exact(f.n);
  const size_t smem = sizeof(double2) * static_cast<size_t>(f.n) * (f.log2n >= 0 ? 1 : 2);
  auto kern = fft_lines<MODE, INV>;
  GC_TRY(kernel_setup(kern, kFftThreads, smem));
  kern<<<static_cast<unsigned>(lines), kFftThreads, smem, ctx->stream>>>(rin, data, rout, f, tw);
  GC_CHECK_LAUNCH("fft_lines");
  return GC_OK;
}

// Forward: real field -> half spectrum; inverse: half spectrum -> real field.
gc_status fft3_forward(gc_context* ctx, const gc_grid* g, const double* in, double2* spec) {
  const int nx = g->nx, ny = g->ny, nz = g->nz, nxh = nx / 2 + 1;
  FftLines f{};
  f.n = nx; f.nh = nxh;
  GC_TRY((launch_fft<FFT_R2C, false>(ctx, in, spec, nullptr, f, static_cast<long long>(ny) * nz)));
  if (ny > 1) {
    FftLines fy{};
    fy.n = ny; fy.inner = nxh; fy.inner_stride = 1; fy.outer_stride = static_cast<long long>(ny) * nxh; fy.elem_stride = nxh;
    GC_TRY((launch_fft<FFT_C2C, false>(ctx, nullptr, spec, nullptr, fy, static_cast<long long>(nxh) * nz)));
  }
  if (nz > 1) {
    FftLines fz{};
    fz.n = nz; fz.inner = static_cast<long long>(nxh) * ny; fz.inner_stride = 1; fz.outer_stride = 0;
    fz.elem_stride = static_cast<long long>(nxh) * ny;
    GC_TRY((launch_fft<FFT_C2C, false>(ctx, nullptr, spec, nullptr, fz, static_cast<long long>(nxh) * ny)));
  }
  return GC_OK;
}

gc_status fft3_inverse(gc_context* ctx, const gc_grid* g, double2* spec, double* out) {
  const int nx = g->nx, ny = g->ny, nz = g->nz, nxh = nx / 2 + 1;
  if (nz > 1) {
    FftLines fz{};
    fz.n = nz; fz.inner = static_cast<long long>(nxh) * ny; fz.inner_stride = 1; fz.outer_stride = 0;
    fz.elem_stride = static_cast<long long>(nxh) * ny;
    GC_TRY((launch_fft<FFT_C2C, true>(ctx, nullptr, spec, nullptr, fz, static_cast<long long>(nxh) * ny)));
  }
  if (ny > 1) {
    FftLines fy{};
    fy.n = ny; fy.inner = nxh; fy.inner_stride = 1; fy.outer_stride = static_cast<long long>(ny) * nxh; fy.elem_stride = nxh;
    GC_TRY((launch_fft<FFT_C2C, true>(ctx, nullptr, spec, nullptr, fy, static_cast<long long>(nxh) * nz)));
  }
  FftLines f{};
  f.n = nx; f.nh = nxh;
  return launch_fft<FFT_C2R, true>(ctx, nullptr, spec, out, f, static_cast<long long>(ny) * nz);
}

enum SpecOp { SPEC_PARTIAL = 0, SPEC_LAPLACIAN = 1, SPEC_BIHARMONIC = 2, SPEC_GRADIENT = 3 };

struct SpecParams {
  double2* spec;   // forward spectrum (read; written in place unless out3)
  double2* out3;   // gradient: three spectra
  int nx, ny, nz, nxh;
  int ax, ay, az;             // derivative counts (partial)
  double sx, sy, sz;          // 2 pi / (N h) per axis
  double inv_n;               // 1 / (nx ny nz)
};

__device__ __forceinline__ double pow_int(double v, int n) {
  double r = 1.0;
  for (int i = 0; i < n; ++i) r *= v;
  return r;
}

template <int OP>
__global__ void __launch_bounds__(256) spectral_multiply(const SpecParams p) {
  const long long total = static_cast<long long>(p.nxh) * p.ny * p.nz;
  for (long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int ix = static_cast<int>(idx % p.nxh);
    const long long rest = idx / p.nxh;
    const int iy = static_cast<int>(rest % p.ny);
    const int iz = static_cast<int>(rest / p.ny);
    const double kx = p.sx * ix;
    const double ky = p.sy * (2 * iy < p.ny ? iy : iy - p.ny);
    const double kz = p.sz * (2 * iz < p.nz ? iz : iz - p.nz);
    const bool nyq_x = (p.nx % 2 == 0) && ix == p.nxh - 1;
    const bool nyq_y = (p.ny % 2 == 0) && iy == p.ny / 2;
    const bool nyq_z = (p.nz % 2 == 0) && iz == p.nz / 2;
    const double2 v = p.spec[idx];
    if constexpr (OP == SPEC_GRADIENT) {
      // i k_a * v / N per axis (spectral/Derivatives.hpp:207-240).
      const double m[3] = {nyq_x ? 0.0 : kx * p.inv_n, nyq_y ? 0.0 : ky * p.inv_n, nyq_z ? 0.0 : kz * p.inv_n};
#pragma unroll
      for (int a = 0; a < 3; ++a) p.out3[a * total + idx] = double2{-v.y * m[a], v.x * m[a]};
    } else {
      double r;
      int ipow = 0;
      if constexpr (OP == SPEC_LAPLACIAN) {
        r = -(kx * kx + ky * ky + kz * kz);
      } else if constexpr (OP == SPEC_BIHARMONIC) {
        const double k2 = kx * kx + ky * ky + kz * kz;
        r = k2 * k2;
      } else {
        r = pow_int(kx, p.ax) * pow_int(ky, p.ay) * pow_int(kz, p.az);
        ipow = (p.ax + p.ay + p.az) & 3;
        if (((p.ax & 1) && nyq_x) || ((p.ay & 1) && nyq_y) || ((p.az & 1) && nyq_z)) r = 0.0;
      }
      r *= p.inv_n;
      double2 o;
      switch (ipow) {  // (i^ipow r) * v
        case 0: o = {v.x * r, v.y * r}; break;
        case 1: o = {-v.y * r, v.x * r}; break;
        case 2: o = {-v.x * r, -v.y * r}; break;
        default: o = {v.y * r, -v.x * r}; break;
      }
      p.spec[idx] = o;
    }
  }
}

gc_status run_spectral(gc_context* ctx, const gc_grid* g, gc_dtype dt, int op, int ax, int ay, int az, const void* in,
                       void* out) {
  Call call(ctx);
  gc_status s = call.st;
  if (s != GC_OK) return s;
  if ((s = check_grid(g)) != GC_OK) return s;
  if (!in || !out) return fail(GC_ERR_INVALID_ARG, "spectral: null field pointer");
  if (dt != GC_F64) return fail(GC_ERR_UNSUPPORTED, "spectral: the spectral path computes in double (GC_F64 fields)");
  if (g->nx == 1 && (g->ny > 1 || g->nz > 1))
    return fail(GC_ERR_UNSUPPORTED, "spectral: the half-spectrum axis is x; a grid with Nx = 1 is not supported");
  if (ax < 0 || ay < 0 || az < 0 || ax > 8 || ay > 8 || az > 8)
    return fail(GC_ERR_INVALID_ARG, "spectral: derivative counts must be 0..8");
  const int nxh = g->nx / 2 + 1;
  const long long half = static_cast<long long>(nxh) * g->ny * g->nz;
  const int outs = op == SPEC_GRADIENT ? 3 : 1;
  const int nmax = std::max(g->nx, std::max(g->ny, g->nz));
  if (sizeof(double2) * 2 * static_cast<size_t>(nmax) > 200 * 1024)
    return fail(GC_ERR_UNSUPPORTED, "spectral: an axis of " + std::to_string(nmax) +
                                        " cells is beyond the line length the transform stages (6400)");
  void* buf = nullptr;
  if ((s = scratch_get(ctx, kSlotSpectral, sizeof(double2) * half * (1 + (outs == 3 ? 3 : 0)), &buf)) != GC_OK)
    return s;
  double2* spec = static_cast<double2*>(buf);
  if ((s = fft3_forward(ctx, g, static_cast<const double*>(in), spec)) != GC_OK) return s;
  SpecParams p{};
  p.spec = spec;
  p.out3 = outs == 3 ? spec + half : nullptr;
  p.nx = g->nx; p.ny = g->ny; p.nz = g->nz; p.nxh = nxh;
  p.ax = ax; p.ay = ay; p.az = az;
  const double two_pi = 6.283185307179586476925286766559;
  p.sx = two_pi / (static_cast<double>(g->nx) * g->hx);
  p.sy = two_pi / (static_cast<double>(g->ny) * g->hy);
  p.sz = two_pi / (static_cast<double>(g->nz) * g->hz);
  p.inv_n = 1.0 / (static_cast<double>(g->nx) * g->ny * g->nz);
  const int blocks = static_cast<int>(std::min<long long>((half + 255) / 256, static_cast<long long>(ctx->num_sms) * 16));
  switch (op) {
    case SPEC_PARTIAL: spectral_multiply<SPEC_PARTIAL><<<blocks, 256, 0, ctx->stream>>>(p); break;
    case SPEC_LAPLACIAN: spectral_multiply<SPEC_LAPLACIAN><<<blocks, 256, 0, ctx->stream>>>(p); break;
    case SPEC_BIHARMONIC: spectral_multiply<SPEC_BIHARMONIC><<<blocks, 256, 0, ctx->stream>>>(p); break;
    default: spectral_multiply<SPEC_GRADIENT><<<blocks, 256, 0, ctx->stream>>>(p); break;
  }
  GC_CHECK_LAUNCH("spectral_multiply");
  const size_t cells_n = static_cast<size_t>(g->nx) * g->ny * g->nz;
  for (int c = 0; c < outs; ++c) {
    double2* sp = outs == 3 ? spec + half * (1 + c) : spec;
    if ((s = fft3_inverse(ctx, g, sp, static_cast<double*>(out) + c * cells_n)) != GC_OK) return s;
  }
  return GC_OK;
}

}  // namespace
}  // namespace gcb

using namespace gcb;

extern "C" {

GC_API gc_status gc_spectral_partial(gc_context* ctx, const gc_grid* g, gc_dtype dt, int ax, int ay, int az,
                                     const void* in, void* out) {
  return run_spectral(ctx, g, dt, SPEC_PARTIAL, ax, ay, az, in, out);
}

GC_API gc_status gc_spectral_laplacian(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* in, void* out) {
  return run_spectral(ctx, g, dt, SPEC_LAPLACIAN, 0, 0, 0, in, out);
}

GC_API gc_status gc_spectral_biharmonic(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* in, void* out) {
  return run_spectral(ctx, g, dt, SPEC_BIHARMONIC, 0, 0, 0, in, out);
}

GC_API gc_status gc_spectral_gradient(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* in, void* out3) {
  return run_spectral(ctx, g, dt, SPEC_GRADIENT, 0, 0, 0, in, out3);
}

}  // extern "C"
