// Spectral derivatives on the GPU (spectral/Derivatives.hpp:78-240,
// spectral/Wavenumbers.hpp:50-110): a real-to-complex FFT of the field, one
// kernel applying the derivative's multiplier to the half spectrum, and the
// complex-to-real FFT back.  The FFTs are cuFFT (D2Z / Z2D, double); the
// multiplier kernel is this library's, and folds in the 1/N normalisation
// of the inverse transform.  The gradient writes its three spectra in one
// pass and transforms them back as one batched plan.
//
// Conventions kept from the reference: wavenumbers k = 2 pi n / (N h) with
// n in [0, N/2] along x (the half spectrum) and the signed range along y
// and z (n - N for 2 n >= N); an odd derivative count along an axis of even
// extent zeroes that axis's Nyquist mode; a degenerate axis (N = 1) has the
// single wavenumber 0.  Results agree with the reference's PocketFFT path to
// rounding (the transforms differ in their operation order).
#include <cufft.h>

#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "common.cuh"

namespace gcb {
namespace {

struct PlanKey {
  int device, nx, ny, nz, batch, inverse;
  bool operator<(const PlanKey& o) const {
    return std::tie(device, nx, ny, nz, batch, inverse) < std::tie(o.device, o.nx, o.ny, o.nz, o.batch, o.inverse);
  }
};

// The plans of one context.  A context is driven by one host thread at a time
// and runs everything on its own stream, so its plans need no lock, are bound
// to that stream once, and their work areas are never shared with another
// context's transforms.
struct PlanCache {
  std::map<PlanKey, cufftHandle> plans;
};

void release_plans(void* p) {
  auto* cache = static_cast<PlanCache*>(p);
  for (auto& kv : cache->plans) cufftDestroy(kv.second);
  delete cache;
}

// A D2Z (inverse = 0) or Z2D plan over the grid, `batch` fields laid out
// back to back.  Axes y and z of extent 1 are dropped from the rank; x is
// always the transformed-to-half axis.
gc_status plan_for(gc_context* ctx, const gc_grid* g, int batch, int inverse, cufftHandle* out) {
  if (!ctx->spectral_plans) {
    ctx->spectral_plans = new PlanCache;
    ctx->spectral_release = release_plans;
  }
  auto& plans = static_cast<PlanCache*>(ctx->spectral_plans)->plans;
  const PlanKey key{ctx->device, g->nx, g->ny, g->nz, batch, inverse};
  auto it = plans.find(key);
  if (it == plans.end()) {
    int n[3];
    int rank = 0;
    if (g->nz > 1) n[rank++] = g->nz;
    if (g->ny > 1) n[rank++] = g->ny;
    n[rank++] = g->nx;
    const long long real = static_cast<long long>(g->nx) * g->ny * g->nz;
    const long long half = static_cast<long long>(g->nx / 2 + 1) * g->ny * g->nz;
    cufftHandle h;
    if (cufftCreate(&h) != CUFFT_SUCCESS) return fail(GC_ERR_CUDA, "spectral: cufftCreate failed");
    size_t work = 0;
    long long nn[3] = {n[0], n[1], n[2]};
    const cufftResult r = cufftMakePlanMany64(h, rank, nn, nullptr, 1, inverse ? half : real, nullptr, 1,
                                              inverse ? real : half, inverse ? CUFFT_Z2D : CUFFT_D2Z, batch, &work);
    if (r != CUFFT_SUCCESS) {
      cufftDestroy(h);
      return fail(GC_ERR_CUDA, "spectral: cuFFT plan for " + std::to_string(g->nx) + "x" + std::to_string(g->ny) +
                                   "x" + std::to_string(g->nz) + " failed (" + std::to_string(static_cast<int>(r)) + ")");
    }
    if (cufftSetStream(h, ctx->stream) != CUFFT_SUCCESS) {
      cufftDestroy(h);
      return fail(GC_ERR_CUDA, "spectral: cufftSetStream failed");
    }
    it = plans.emplace(key, h).first;
  }
  *out = it->second;
  return GC_OK;
}

enum SpecOp { SPEC_PARTIAL = 0, SPEC_LAPLACIAN = 1, SPEC_BIHARMONIC = 2, SPEC_GRADIENT = 3 };

struct SpecParams {
  cufftDoubleComplex* spec;   // forward spectrum (read; written in place unless out3)
  cufftDoubleComplex* out3;   // gradient: three spectra
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
    const cufftDoubleComplex v = p.spec[idx];
    if constexpr (OP == SPEC_GRADIENT) {
      // i k_a * v / N per axis (spectral/Derivatives.hpp:207-240).
      const double m[3] = {nyq_x ? 0.0 : kx * p.inv_n, nyq_y ? 0.0 : ky * p.inv_n, nyq_z ? 0.0 : kz * p.inv_n};
#pragma unroll
      for (int a = 0; a < 3; ++a) p.out3[a * total + idx] = cufftDoubleComplex{-v.y * m[a], v.x * m[a]};
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
      cufftDoubleComplex o;
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
  void* buf = nullptr;
  if ((s = scratch_get(ctx, kSlotSpectral, sizeof(cufftDoubleComplex) * half * (1 + (outs == 3 ? 3 : 0)), &buf)) !=
      GC_OK)
    return s;
  cufftDoubleComplex* spec = static_cast<cufftDoubleComplex*>(buf);
  cufftHandle fwd, inv;
  if ((s = plan_for(ctx, g, 1, 0, &fwd)) != GC_OK) return s;
  if ((s = plan_for(ctx, g, outs, 1, &inv)) != GC_OK) return s;
  if (cufftExecD2Z(fwd, static_cast<cufftDoubleReal*>(const_cast<void*>(in)), spec) != CUFFT_SUCCESS)
    return fail(GC_ERR_CUDA, "spectral: forward transform failed");
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
  if (cufftExecZ2D(inv, outs == 3 ? spec + half : spec, static_cast<cufftDoubleReal*>(out)) != CUFFT_SUCCESS)
    return fail(GC_ERR_CUDA, "spectral: inverse transform failed");
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
