// Multi-index partial derivatives d^(ax+ay+az) f / dx^ax dy^ay dz^az
// (diff/detail/MultiIndexDerivative.hpp:96-137): the reference's 31 named
// partials (diff/MixedPartial.hpp, ThirdOrder.hpp, FourthOrder.hpp: dxx ...
// d4dxdydz2) and any other counts 0..4 per axis, orders 2, 4, 6, double
// (reference-exact) and float.
//
// The reference sums, per point, (wx * (wy * wz)) * f over the outer product
// of the three 1-D tables (z taps outermost, x innermost) from 0.0 and
// multiplies by scale = 1 / h_a divided once per derivative on each axis.
// The tap products wx * (wy * wz) are formed on the host in that order and
// passed with the launch, so the device sum has the same operands in the same
// order (zero products are skipped: that changes only the sign of an exact
// zero).  Kernel: a 32 x 8 CTA marches up a chunk of z planes through a ring
// of staged planes (periodic x/y halo of max(rx, ry)) filled by cp.async
// several planes ahead.  The x and y table widths are template parameters
// (one instantiation per pair, so both tap loops unroll); the z radius stays
// a runtime value.
#include <algorithm>

#include "common.cuh"

namespace gcb {
namespace {

constexpr int PX = 32, PY = 8, PT = PX * PY;
constexpr int kPRing = 3;      // planes in flight ahead of the one computed
constexpr int kMaxTaps = 729;  // (2 * 4 + 1)^3

// Passed by value as a __grid_constant__ kernel parameter (about 6 KB: the
// tap products travel with the launch, no copy or synchronisation).
struct PartialParams {
  const void* in;
  void* out;
  int nx, ny, nz;
  int rx, ry, rz, R;   // R = max(rx, ry): staged x/y halo
  int zc;              // planes per CTA chunk
  double scale;
  double coef[kMaxTaps];  // [mz][my][mx], (2rz+1)(2ry+1)(2rx+1) products
};

__device__ __forceinline__ void cp_async_bytes(void* smem, const void* gmem, int bytes) {
  const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  if (bytes == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}

// WX, WY: the x and y extents of the tap table (2 rx + 1, 2 ry + 1),
// compile-time constants so that the two inner loops unroll (shared-memory
// offsets and coefficient indices become immediates); the z extent stays a
// runtime value.
template <class T, int WX, int WY>
__global__ void __launch_bounds__(PT) partial_kernel(const __grid_constant__ PartialParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ring = reinterpret_cast<T*>(smem_raw);  // [NB][PH][PW]
  const int R = p.R, rx = p.rx, ry = p.ry, rz = p.rz;
  const int PW = PX + 2 * R, PH = PY + 2 * R, PS = PW * PH;
  const int NB = 2 * rz + 1 + kPRing;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * PX + tx;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int x0 = blockIdx.x * PX, y0 = blockIdx.y * PY;
  const int z0 = blockIdx.z * p.zc;
  const int z1 = min(z0 + p.zc, nz);
  const size_t plane = static_cast<size_t>(nx) * ny;
  const T* in = static_cast<const T*>(p.in);
  auto slot_of = [&](int z) { return (z - z0 + rz) % NB; };
  auto issue = [&](int z) {  // plane z (wrapped) into its slot, one commit group
    if (z <= z1 - 1 + rz) {
      const size_t zo = static_cast<size_t>(wrap(z, nz)) * plane;
      T* dst = ring + static_cast<size_t>(slot_of(z)) * PS;
      for (int e = tid; e < PS; e += PT) {
        const int r = e / PW, c = e - r * PW;
        cp_async_bytes(dst + e, in + zo + static_cast<size_t>(wrap(y0 - R + r, ny)) * nx + wrap(x0 - R + c, nx),
                       sizeof(T));
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  for (int z = z0 - rz; z < z0 + rz + kPRing; ++z) issue(z);
  const int gx = x0 + tx, gy = y0 + ty;
  const bool active = gx < nx && gy < ny;
  constexpr int wx = WX, wy = WY;
  const int wz = 2 * rz + 1;
  for (int z = z0; z < z1; ++z) {
    asm volatile("cp.async.wait_group %0;" ::"n"(kPRing - 1) : "memory");  // plane z + rz landed
    __syncthreads();
    if (active) {
      T sum = T(0);
      for (int mz = 0; mz < wz; ++mz) {
        const T* pl = ring + static_cast<size_t>(slot_of(z + mz - rz)) * PS;
#pragma unroll
        for (int my = 0; my < wy; ++my) {
          const T* row = pl + (ty + R + my - ry) * PW + tx + R - rx;
          const double* cr = p.coef + (mz * wy + my) * wx;
#pragma unroll
          for (int mx = 0; mx < wx; ++mx) {
            const double c = cr[mx];
            if (c != 0.0) sum = Ar<T>::add(sum, Ar<T>::mul(static_cast<T>(c), row[mx]));
          }
        }
      }
      static_cast<T*>(p.out)[static_cast<size_t>(z) * plane + static_cast<size_t>(gy) * nx + gx] =
          Ar<T>::mul(sum, static_cast<T>(p.scale));
    }
    issue(z + rz + kPRing);
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// Host copy of the 1-D tables: count 0 is the single tap 1.0.
int axis_table(int count, int order, double* w) {
  auto fill = [&](auto tag) {
    using Wk = decltype(tag);
    for (int m = 0; m <= 2 * Wk::R; ++m) w[m] = Wk::w(m);
    return Wk::R;
  };
  if (count == 0) {
    w[0] = 1.0;
    return 0;
  }
  switch (count * 10 + order) {
    case 12: return fill(W<1, 2>{});
    case 14: return fill(W<1, 4>{});
    case 16: return fill(W<1, 6>{});
    case 22: return fill(W<2, 2>{});
    case 24: return fill(W<2, 4>{});
    case 26: return fill(W<2, 6>{});
    case 32: return fill(W<3, 2>{});
    case 34: return fill(W<3, 4>{});
    case 36: return fill(W<3, 6>{});
    case 42: return fill(W<4, 2>{});
    case 44: return fill(W<4, 4>{});
    case 46: return fill(W<4, 6>{});
  }
  return -1;
}

template <class T, int WX>
auto kernel_for_y(int ry) -> void (*)(const PartialParams) {
  switch (ry) {
    case 0: return partial_kernel<T, WX, 1>;
    case 1: return partial_kernel<T, WX, 3>;
    case 2: return partial_kernel<T, WX, 5>;
    case 3: return partial_kernel<T, WX, 7>;
    default: return partial_kernel<T, WX, 9>;
  }
}

template <class T>
auto kernel_for(int rx, int ry) -> void (*)(const PartialParams) {
  switch (rx) {
    case 0: return kernel_for_y<T, 1>(ry);
    case 1: return kernel_for_y<T, 3>(ry);
    case 2: return kernel_for_y<T, 5>(ry);
    case 3: return kernel_for_y<T, 7>(ry);
    default: return kernel_for_y<T, 9>(ry);
  }
}

template <class T>
gc_status launch_partial(gc_context* ctx, PartialParams& p) {
  const int tiles_x = div_up(p.nx, PX), tiles_y = div_up(p.ny, PY);
  const long long tiles = static_cast<long long>(tiles_x) * tiles_y;
  const long long want = 16LL * ctx->num_sms;
  int chunks = static_cast<int>(std::min<long long>((want + tiles - 1) / tiles, std::max(1, p.nz / 16)));
  chunks = std::max(chunks, 1);
  p.zc = div_up(p.nz, chunks);
  chunks = div_up(p.nz, p.zc);
  const size_t smem = sizeof(T) * static_cast<size_t>(2 * p.rz + 1 + kPRing) * (PX + 2 * p.R) * (PY + 2 * p.R);
  // rx, ry <= 4 (axis_table): one instantiation per (WX, WY).
  void (*kern)(const PartialParams) = kernel_for<T>(p.rx, p.ry);
  GC_TRY(kernel_setup(kern, PX * PY, smem));
  kern<<<dim3(tiles_x, tiles_y, chunks), dim3(PX, PY), smem, ctx->stream>>>(p);
  GC_CHECK_LAUNCH("partial_kernel");
  return GC_OK;
}

}  // namespace
}  // namespace gcb

using namespace gcb;

extern "C" {

GC_API gc_status gc_partial(gc_context* ctx, const gc_grid* g, gc_dtype dt, int order, int ax, int ay, int az,
                            const void* in, void* out) {
  Call call(ctx);
  gc_status s = call.st;
  if (s != GC_OK) return s;
  if (ax < 0 || ax > 4 || ay < 0 || ay > 4 || az < 0 || az > 4 || ax + ay + az == 0)
    return fail(GC_ERR_INVALID_ARG, "gc_partial: derivative counts must be 0..4 per axis, not all zero");
  if (order != 2 && order != 4 && order != 6)
    return fail(GC_ERR_UNSUPPORTED, "gridcalc_b200: order must be 2, 4 or 6; got " + std::to_string(order));
  double wx[9], wy[9], wz[9];
  const int rx = axis_table(ax, order, wx), ry = axis_table(ay, order, wy), rz = axis_table(az, order, wz);
  if ((s = require_axes3(g, rx, ry, rz)) != GC_OK) return s;
  if (!in || !out) return fail(GC_ERR_INVALID_ARG, "gc_partial: null field pointer");
  if (dt != GC_F64 && dt != GC_F32) return fail(GC_ERR_INVALID_ARG, "gridcalc_b200: unknown dtype");
  PartialParams p{};
  p.in = in;
  p.out = out;
  p.nx = g->nx; p.ny = g->ny; p.nz = g->nz;
  p.rx = rx; p.ry = ry; p.rz = rz; p.R = std::max(rx, ry);
  // Tap products in the reference's order: wyz = wy * wz, then wx * wyz.
  const int nwx = 2 * rx + 1, nwy = 2 * ry + 1, nwz = 2 * rz + 1;
  for (int mz = 0; mz < nwz; ++mz)
    for (int my = 0; my < nwy; ++my) {
      const double wyz = wy[my] * wz[mz];
      for (int mx = 0; mx < nwx; ++mx) p.coef[(mz * nwy + my) * nwx + mx] = wx[mx] * wyz;
    }
  p.scale = 1.0;
  for (int n = 0; n < ax; ++n) p.scale /= g->hx;
  for (int n = 0; n < ay; ++n) p.scale /= g->hy;
  for (int n = 0; n < az; ++n) p.scale /= g->hz;
  return dt == GC_F64 ? launch_partial<double>(ctx, p) : launch_partial<float>(ctx, p);
}

}  // extern "C"
