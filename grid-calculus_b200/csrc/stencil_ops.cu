// Periodic finite-difference operators: laplacian, gradient, divergence,
// biharmonic at orders 2, 4, 6, in double (reference-exact) and float.
//
// Kernel shape (3-D): a CTA owns a BX x BY column of cells and marches up a
// chunk of z planes.  Each plane is staged once in shared memory with its
// periodic x/y halo (wrapped indices, coalesced rows), into a ring of
// 2*RZ+1 planes, so the z taps, the in-plane taps and the mixed taps of the
// biharmonic all come from shared memory and each input value is read from
// HBM once.  2-D grids (Nz == 1) use the same kernel with a single plane;
// the degenerate z axis then sums the centre value with the z weights, as
// the reference's wrapped access does.
#include <algorithm>

#include "common.cuh"

namespace gcb {
namespace {

constexpr int BX = 32;
constexpr int BY = 8;
constexpr int NT = BX * BY;

enum OpKind { OP_LAP = 0, OP_GRAD = 1, OP_DIV = 2, OP_BIH = 3 };

template <int OP, int ORDER>
struct OpShape;
template <int ORDER>
struct OpShape<OP_LAP, ORDER> { static constexpr int R = W<2, ORDER>::R; static constexpr int NF = 1; };
template <int ORDER>
struct OpShape<OP_GRAD, ORDER> { static constexpr int R = W<1, ORDER>::R; static constexpr int NF = 1; };
template <int ORDER>
struct OpShape<OP_DIV, ORDER> { static constexpr int R = W<1, ORDER>::R; static constexpr int NF = 3; };
template <int ORDER>
struct OpShape<OP_BIH, ORDER> {
  static constexpr int R = W<4, ORDER>::R > W<2, ORDER>::R ? W<4, ORDER>::R : W<2, ORDER>::R;
  static constexpr int NF = 1;
};

template <class T>
struct OpParams {
  const T* in[3];
  T* out;
  int nx, ny, nz;
  int zc;          // planes per CTA chunk
  size_t n;        // cells
  T ihx, ihy, ihz;     // 1/h (first derivative)
  T ihx2, ihy2, ihz2;  // 1/h^2
  T ihx4, ihy4, ihz4;  // 1/h^4
};

template <class T, int OP, int ORDER, bool Z3>
__global__ void __launch_bounds__(NT) stencil_kernel(const OpParams<T> p) {
  constexpr int R = OpShape<OP, ORDER>::R;
  constexpr int NF = OpShape<OP, ORDER>::NF;
  constexpr int RZ = Z3 ? R : 0;
  constexpr int NP = 2 * RZ + 1;
  constexpr int PW = BX + 2 * R;
  constexpr int PH = BY + 2 * R;
  constexpr int PS = PW * PH;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ring = reinterpret_cast<T*>(smem_raw);  // [NF][NP][PS]

  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * BX + tx;
  const int x0 = blockIdx.x * BX, y0 = blockIdx.y * BY;
  const int z0 = blockIdx.z * p.zc;
  const int z1 = min(z0 + p.zc, p.nz);
  const int nx = p.nx, ny = p.ny, nz = p.nz;

  auto load_plane = [&](int z, int slot) {
    const int zw = wrap(z, nz);
    const size_t zoff = static_cast<size_t>(zw) * nx * ny;
    for (int e = tid; e < PS; e += NT) {
      const int sy = e / PW;
      const int sx = e - sy * PW;
      const int gx = wrap(x0 - R + sx, nx);
      const int gy = wrap(y0 - R + sy, ny);
      const size_t gi = zoff + static_cast<size_t>(gy) * nx + gx;
#pragma unroll
      for (int f = 0; f < NF; ++f) ring[(f * NP + slot) * PS + e] = __ldg(p.in[f] + gi);
    }
  };

  // Slot of plane z: planes enter the ring in order starting at z0 - RZ.
  auto slot_of = [&](int z) { return (z - z0 + RZ) % NP; };

  for (int z = z0 - RZ; z < z0 + RZ; ++z) load_plane(z, slot_of(z));

  const int gx = x0 + tx, gy = y0 + ty;
  const bool active = gx < nx && gy < ny;

  for (int z = z0; z < z1; ++z) {
    load_plane(z + RZ, slot_of(z + RZ));
    __syncthreads();
    // Value of field f at offset (dx, dy, dz) from this thread's cell.
    auto at = [&](int f, int dx, int dy, int dz) -> T {
      const int slot = Z3 ? slot_of(z + dz) : 0;
      return ring[(f * NP + slot) * PS + (ty + R + dy) * PW + (tx + R + dx)];
    };
    if (active) {
      const size_t c = static_cast<size_t>(z) * nx * ny + static_cast<size_t>(gy) * nx + gx;
      if constexpr (OP == OP_LAP || OP == OP_GRAD) {
        constexpr int K = OP == OP_LAP ? 2 : 1;
        const T ax = tap_sum<T, K, ORDER>([&](int o) { return at(0, o, 0, 0); });
        const T ay = tap_sum<T, K, ORDER>([&](int o) { return at(0, 0, o, 0); });
        const T az = tap_sum<T, K, ORDER>([&](int o) { return at(0, 0, 0, Z3 ? o : 0); });
        if constexpr (OP == OP_LAP) {
          p.out[c] = Ar<T>::add(Ar<T>::add(Ar<T>::mul(ax, p.ihx2), Ar<T>::mul(ay, p.ihy2)),
                                Ar<T>::mul(az, p.ihz2));
        } else {
          p.out[c] = Ar<T>::mul(ax, p.ihx);
          p.out[p.n + c] = Ar<T>::mul(ay, p.ihy);
          p.out[2 * p.n + c] = Ar<T>::mul(az, p.ihz);
        }
      } else if constexpr (OP == OP_DIV) {
        const T ax = tap_sum<T, 1, ORDER>([&](int o) { return at(0, o, 0, 0); });
        const T ay = tap_sum<T, 1, ORDER>([&](int o) { return at(1, 0, o, 0); });
        const T az = tap_sum<T, 1, ORDER>([&](int o) { return at(2, 0, 0, Z3 ? o : 0); });
        p.out[c] = Ar<T>::add(Ar<T>::add(Ar<T>::mul(ax, p.ihx), Ar<T>::mul(ay, p.ihy)),
                              Ar<T>::mul(az, p.ihz));
      } else {
        // diff/Biharmonic.hpp:70-99: axial fourth derivatives, then the three
        // mixed second-derivative products, outer loop over the second axis.
        const T d4x = tap_sum<T, 4, ORDER>([&](int o) { return at(0, o, 0, 0); });
        const T d4y = tap_sum<T, 4, ORDER>([&](int o) { return at(0, 0, o, 0); });
        const T d4z = tap_sum<T, 4, ORDER>([&](int o) { return at(0, 0, 0, Z3 ? o : 0); });
        constexpr int R2 = W<2, ORDER>::R;
        T xy = T(0), xz = T(0), yz = T(0);
#pragma unroll
        for (int mb = 0; mb <= 2 * R2; ++mb) {
#pragma unroll
          for (int ma = 0; ma <= 2 * R2; ++ma) {
            const double wab_d = W<2, ORDER>::w(ma) * W<2, ORDER>::w(mb);
            const T wab = static_cast<T>(wab_d);
            const int oa = ma - R2, ob = mb - R2;
            const T vxy = at(0, oa, ob, 0);
            const T vxz = at(0, oa, 0, Z3 ? ob : 0);
            const T vyz = at(0, 0, oa, Z3 ? ob : 0);
            if (wab_d == 1.0) {
              xy = Ar<T>::add(xy, vxy);
              xz = Ar<T>::add(xz, vxz);
              yz = Ar<T>::add(yz, vyz);
            } else {
              xy = Ar<T>::mac(xy, wab, vxy);
              xz = Ar<T>::mac(xz, wab, vxz);
              yz = Ar<T>::mac(yz, wab, vyz);
            }
          }
        }
        const T axial = Ar<T>::add(Ar<T>::add(Ar<T>::mul(d4x, p.ihx4), Ar<T>::mul(d4y, p.ihy4)),
                                   Ar<T>::mul(d4z, p.ihz4));
        const T c1 = Ar<T>::mul(Ar<T>::mul(xy, p.ihx2), p.ihy2);
        const T c2 = Ar<T>::mul(Ar<T>::mul(xz, p.ihx2), p.ihz2);
        const T c3 = Ar<T>::mul(Ar<T>::mul(yz, p.ihy2), p.ihz2);
        p.out[c] = Ar<T>::add(axial, Ar<T>::mul(T(2), Ar<T>::add(Ar<T>::add(c1, c2), c3)));
      }
    }
    __syncthreads();
  }
}

template <class T, int OP, int ORDER, bool Z3>
gc_status launch_one(gc_context* ctx, const OpParams<T>& p0) {
  constexpr int R = OpShape<OP, ORDER>::R;
  constexpr int NF = OpShape<OP, ORDER>::NF;
  constexpr int RZ = Z3 ? R : 0;
  constexpr int NP = 2 * RZ + 1;
  constexpr size_t smem = sizeof(T) * NF * NP * (BX + 2 * R) * (BY + 2 * R);
  OpParams<T> p = p0;
  const int tiles_x = div_up(p.nx, BX), tiles_y = div_up(p.ny, BY);
  int chunks = 1;
  if (Z3) {
    // Enough CTAs to fill the GPU several times over, but chunks of at least
    // 8 planes so the 2*RZ prologue planes stay a small overhead.
    const long long want = 8LL * ctx->num_sms;
    const long long tiles = static_cast<long long>(tiles_x) * tiles_y;
    chunks = static_cast<int>(std::min<long long>((want + tiles - 1) / tiles, std::max(1, p.nz / 8)));
    chunks = std::max(chunks, 1);
  }
  p.zc = div_up(p.nz, chunks);
  chunks = div_up(p.nz, p.zc);
  auto kern = stencil_kernel<T, OP, ORDER, Z3>;
  if (smem > 48 * 1024) GC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid(tiles_x, tiles_y, chunks), block(BX, BY);
  kern<<<grid, block, smem, ctx->stream>>>(p);
  GC_CHECK_LAUNCH("stencil_kernel");
  return GC_OK;
}

template <class T, int OP>
gc_status dispatch_order(gc_context* ctx, int order, const OpParams<T>& p) {
  const bool z3 = p.nz > 1;
  switch (order) {
    case 2: return z3 ? launch_one<T, OP, 2, true>(ctx, p) : launch_one<T, OP, 2, false>(ctx, p);
    case 4: return z3 ? launch_one<T, OP, 4, true>(ctx, p) : launch_one<T, OP, 4, false>(ctx, p);
    case 6: return z3 ? launch_one<T, OP, 6, true>(ctx, p) : launch_one<T, OP, 6, false>(ctx, p);
  }
  return fail(GC_ERR_UNSUPPORTED, "gridcalc_b200: order must be 2, 4 or 6; got " + std::to_string(order));
}

int op_radius(int op, int order) {
  const int r2 = order / 2;                 // second derivative: 1, 2, 3
  const int r1 = order / 2;                 // first derivative: 1, 2, 3
  const int r4 = order / 2 + 1;             // fourth derivative: 2, 3, 4
  switch (op) {
    case OP_LAP: return r2;
    case OP_GRAD:
    case OP_DIV: return r1;
    default: return std::max(r4, r2);
  }
}

template <class T>
OpParams<T> make_params(const gc_grid* g) {
  OpParams<T> p{};
  p.nx = g->nx; p.ny = g->ny; p.nz = g->nz;
  p.n = cells(g);
  const double ihx2 = 1.0 / (g->hx * g->hx), ihy2 = 1.0 / (g->hy * g->hy), ihz2 = 1.0 / (g->hz * g->hz);
  p.ihx = static_cast<T>(1.0 / g->hx); p.ihy = static_cast<T>(1.0 / g->hy); p.ihz = static_cast<T>(1.0 / g->hz);
  p.ihx2 = static_cast<T>(ihx2); p.ihy2 = static_cast<T>(ihy2); p.ihz2 = static_cast<T>(ihz2);
  p.ihx4 = static_cast<T>(ihx2 * ihx2); p.ihy4 = static_cast<T>(ihy2 * ihy2); p.ihz4 = static_cast<T>(ihz2 * ihz2);
  return p;
}

template <int OP>
gc_status run_op(gc_context* ctx, const gc_grid* g, gc_dtype dt, int order, const void* in,
                 void* out) {
  Call call(ctx);
  gc_status s = call.st;
  if (s != GC_OK) return s;
  if (order != 2 && order != 4 && order != 6)
    return fail(GC_ERR_UNSUPPORTED, "gridcalc_b200: order must be 2, 4 or 6; got " + std::to_string(order));
  if ((s = require_axes(g, op_radius(OP, order))) != GC_OK) return s;
  if (!in || !out) return fail(GC_ERR_INVALID_ARG, "gridcalc_b200: null field pointer");
  const size_t n = cells(g);
  if (dt == GC_F64) {
    OpParams<double> p = make_params<double>(g);
    const double* base = static_cast<const double*>(in);
    p.in[0] = base; p.in[1] = OP == OP_DIV ? base + n : base; p.in[2] = OP == OP_DIV ? base + 2 * n : base;
    p.out = static_cast<double*>(out);
    return dispatch_order<double, OP>(ctx, order, p);
  } else if (dt == GC_F32) {
    OpParams<float> p = make_params<float>(g);
    const float* base = static_cast<const float*>(in);
    p.in[0] = base; p.in[1] = OP == OP_DIV ? base + n : base; p.in[2] = OP == OP_DIV ? base + 2 * n : base;
    p.out = static_cast<float*>(out);
    return dispatch_order<float, OP>(ctx, order, p);
  }
  return fail(GC_ERR_INVALID_ARG, "gridcalc_b200: unknown dtype");
}

}  // namespace
}  // namespace gcb

using namespace gcb;

extern "C" {

GC_API gc_status gc_laplacian(gc_context* ctx, const gc_grid* g, gc_dtype dt, int order,
                              const void* in, void* out) {
  return run_op<OP_LAP>(ctx, g, dt, order, in, out);
}

GC_API gc_status gc_gradient(gc_context* ctx, const gc_grid* g, gc_dtype dt, int order,
                             const void* in, void* out3) {
  return run_op<OP_GRAD>(ctx, g, dt, order, in, out3);
}

GC_API gc_status gc_divergence(gc_context* ctx, const gc_grid* g, gc_dtype dt, int order,
                               const void* in3, void* out) {
  return run_op<OP_DIV>(ctx, g, dt, order, in3, out);
}

GC_API gc_status gc_biharmonic(gc_context* ctx, const gc_grid* g, gc_dtype dt, int order,
                               const void* in, void* out) {
  return run_op<OP_BIH>(ctx, g, dt, order, in, out);
}

}  // extern "C"
