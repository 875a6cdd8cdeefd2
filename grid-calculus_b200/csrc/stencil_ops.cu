// Periodic finite-difference operators: laplacian, gradient, divergence,
// biharmonic at orders 2, 4, 6, in double (reference-exact) and float.
//
// Kernel shape: a CTA owns a BX x BY column of cells.  Planes are staged in
// shared memory with their periodic x/y halo (wrapped indices, coalesced
// rows), so the z taps, the in-plane taps and the mixed taps of the
// biharmonic all come from shared memory and each input value is read from
// HBM once.  3-D grids march up a chunk of z planes, either with a register
// queue of z taps (zmarch_kernel) or through a ring of whole planes filled
// asynchronously several planes ahead (zring_kernel); 2-D grids (Nz == 1)
// use one staged plane (stencil_kernel), and the degenerate z axis then sums
// the centre value with the z weights, as the reference's wrapped access does.
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

// Output of one cell from the staged values: at(f, dx, dy, dz) is field f
// at that offset from the cell.  The arithmetic follows the reference's
// tap order (diff/Laplacian.hpp:63-69, Gradient.hpp, Divergence.hpp,
// Biharmonic.hpp:70-99), so double results are bit-identical to it.
template <class T, int OP, int ORDER, bool Z3, class At>
__device__ __forceinline__ void cell_op(const OpParams<T>& p, size_t c, const At& at) {
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

  // Plane loads map threads onto rows and columns directly (no division):
  // column wraps are formed once per thread, row wraps once per row.
  const int gxa = wrap(x0 - R + tx, nx);
  const bool has_b = tx < PW - BX;
  const int gxb = wrap(x0 - R + BX + tx, nx);
  (void)tid;
  auto load_plane = [&](int z, int slot) {
    const int zw = wrap(z, nz);
    const size_t zoff = static_cast<size_t>(zw) * nx * ny;
    for (int r = ty; r < PH; r += BY) {
      const size_t rowo = zoff + static_cast<size_t>(wrap(y0 - R + r, ny)) * nx;
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        ring[(f * NP + slot) * PS + r * PW + tx] = __ldg(p.in[f] + rowo + gxa);
        if (has_b) ring[(f * NP + slot) * PS + r * PW + BX + tx] = __ldg(p.in[f] + rowo + gxb);
      }
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
      cell_op<T, OP, ORDER, Z3>(p, c, at);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// z-march kernel for the axis-separable operators (laplacian, gradient,
// divergence) on 3-D grids.  A 32 x 8 CTA owns a column of cells and
// marches up a chunk of z planes; each thread keeps its own column's z taps
// in a register queue, so only the current plane goes through shared memory
// (its interior taken from the queue, its x/y halo strips loaded by a few
// threads).  The next plane's value and halo are loaded one iteration
// ahead into registers, so global latency overlaps the current plane.
// Divergence stages the x component with an x halo and the y component
// with a y halo; the z component only needs the queue.
constexpr int ZM_X = 32, ZM_Y = 8;

// Rows per thread: a CTA's 32 x 8 threads cover 32 x 8 CPT cells, each
// thread CPT cells of its column (rows ty + 8 q), so the plane's barriers,
// halo duties and loop work are shared by CPT cells.  Float divergence takes
// CPT = 2 (512^3: 0.563 -> 0.499 ms per launch, 0.58 -> 0.66 of HBM).
template <class T, int OP>
__host__ __device__ constexpr int zmarch_cpt() {
  return (sizeof(T) == 4 && OP == OP_DIV) ? 2 : 1;
}

template <class T, int OP, int ORDER>
__global__ void __launch_bounds__(ZM_X * ZM_Y) zmarch_kernel(const OpParams<T> p) {
  constexpr int R = OpShape<OP, ORDER>::R;
  constexpr int NQ = 2 * R + 1;
  constexpr int PW = ZM_X + 2 * R, PH = ZM_Y + 2 * R;
  constexpr int K = OP == OP_LAP ? 2 : 1;
  // plane of the field (LAP, GRAD) or of the x component (DIV), and for DIV
  // the y component's plane.
  __shared__ T sp[PH][PW];
  __shared__ T sy[OP == OP_DIV ? PH : 1][OP == OP_DIV ? ZM_X : 1];

  const int tx = threadIdx.x, ty = threadIdx.y;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int x0 = blockIdx.x * ZM_X, y0 = blockIdx.y * ZM_Y;
  const int z0 = blockIdx.z * p.zc;
  const int z1 = min(z0 + p.zc, nz);
  const size_t plane = static_cast<size_t>(nx) * ny;
  const int gx = wrap(x0 + tx, nx), gy = wrap(y0 + ty, ny);
  const size_t col = static_cast<size_t>(gy) * nx + gx;
  const bool active = x0 + tx < nx && y0 + ty < ny;
  // Halo duties: x halo (threads tx < 2R: left for tx < R, right otherwise)
  // for row ty; y halo (threads ty < 2R) for column tx.
  const bool hx = tx < 2 * R;
  const int hx_col = tx < R ? x0 - R + tx : x0 + ZM_X + (tx - R);
  const size_t hx_off = static_cast<size_t>(gy) * nx + wrap(hx_col, nx);
  const int hx_slot = tx < R ? tx : ZM_X + R + (tx - R);
  const bool hy = ty < 2 * R;
  const int hy_row = ty < R ? y0 - R + ty : y0 + ZM_Y + (ty - R);
  const size_t hy_off = static_cast<size_t>(wrap(hy_row, ny)) * nx + gx;
  const int hy_slot = ty < R ? ty : ZM_Y + R + (ty - R);

  const T* fx = p.in[0];                         // LAP/GRAD field, DIV x component
  const T* fy = p.in[1];                         // DIV y component
  const T* fz = OP == OP_DIV ? p.in[2] : p.in[0];  // field whose z taps are queued

  T q[NQ];
#pragma unroll
  for (int k = 0; k < NQ - 1; ++k) q[k + 1] = __ldg(fz + static_cast<size_t>(wrap(z0 - R + k, nz)) * plane + col);
  // Prefetch of plane z0: its queue value (z0 + R), centre and halos.
  T n_q = __ldg(fz + static_cast<size_t>(wrap(z0 + R, nz)) * plane + col);
  size_t zoff = static_cast<size_t>(z0) * plane;
  T n_c = (OP == OP_DIV) ? __ldg(fx + zoff + col) : T(0);
  T n_cy = (OP == OP_DIV) ? __ldg(fy + zoff + col) : T(0);
  T n_hx = hx ? __ldg(fx + zoff + hx_off) : T(0);
  T n_hy = hy ? __ldg((OP == OP_DIV ? fy : fx) + zoff + hy_off) : T(0);

  for (int z = z0; z < z1; ++z) {
#pragma unroll
    for (int k = 0; k + 1 < NQ; ++k) q[k] = q[k + 1];
    q[NQ - 1] = n_q;
    const T c_x = OP == OP_DIV ? n_c : q[R];
    const T c_y = n_cy;
    const T h_x = n_hx, h_y = n_hy;
    if (z + 1 < z1) {  // prefetch plane z + 1
      const size_t zo = static_cast<size_t>(z + 1) * plane;
      n_q = __ldg(fz + static_cast<size_t>(wrap(z + 1 + R, nz)) * plane + col);
      if (OP == OP_DIV) {
        n_c = __ldg(fx + zo + col);
        n_cy = __ldg(fy + zo + col);
      }
      if (hx) n_hx = __ldg(fx + zo + hx_off);
      if (hy) n_hy = __ldg((OP == OP_DIV ? fy : fx) + zo + hy_off);
    }
    sp[ty + R][tx + R] = c_x;
    if (hx) sp[ty + R][hx_slot] = h_x;
    if (OP == OP_DIV) {
      sy[ty + R][tx] = c_y;
      if (hy) sy[hy_slot][tx] = h_y;
    } else {
      if (hy) sp[hy_slot][tx + R] = h_y;
    }
    __syncthreads();
    if (active) {
      const size_t c = static_cast<size_t>(z) * plane + static_cast<size_t>(y0 + ty) * nx + (x0 + tx);
      const T ax = tap_sum<T, K, ORDER>([&](int o) { return sp[ty + R][tx + R + o]; });
      const T az = tap_sum<T, K, ORDER>([&](int o) { return q[R + o]; });
      if constexpr (OP == OP_DIV) {
        const T ay = tap_sum<T, 1, ORDER>([&](int o) { return sy[ty + R + o][tx]; });
        p.out[c] = Ar<T>::add(Ar<T>::add(Ar<T>::mul(ax, p.ihx), Ar<T>::mul(ay, p.ihy)), Ar<T>::mul(az, p.ihz));
      } else {
        const T ay = tap_sum<T, K, ORDER>([&](int o) { return sp[ty + R + o][tx + R]; });
        if constexpr (OP == OP_LAP) {
          p.out[c] = Ar<T>::add(Ar<T>::add(Ar<T>::mul(ax, p.ihx2), Ar<T>::mul(ay, p.ihy2)), Ar<T>::mul(az, p.ihz2));
        } else {
          p.out[c] = Ar<T>::mul(ax, p.ihx);
          p.out[p.n + c] = Ar<T>::mul(ay, p.ihy);
          p.out[2 * p.n + c] = Ar<T>::mul(az, p.ihz);
        }
      }
    }
    __syncthreads();
  }
}

// The same z-march with CPT > 1 rows per thread (float divergence; at one
// row per thread the kernel above measured faster: double gradient order 4
// 0.946 against 1.015 ms at 512^3).
template <class T, int OP, int ORDER>
__global__ void __launch_bounds__(ZM_X * ZM_Y) zmarch_rows_kernel(const OpParams<T> p) {
  constexpr int R = OpShape<OP, ORDER>::R;
  constexpr int NQ = 2 * R + 1;
  constexpr int CPT = zmarch_cpt<T, OP>(), TY = ZM_Y * CPT;
  constexpr int PW = ZM_X + 2 * R, PH = TY + 2 * R;
  constexpr int K = OP == OP_LAP ? 2 : 1;
  // plane of the field (LAP, GRAD) or of the x component (DIV), and for DIV
  // the y component's plane.
  __shared__ T sp[PH][PW];
  __shared__ T sy[OP == OP_DIV ? PH : 1][OP == OP_DIV ? ZM_X : 1];

  const int tx = threadIdx.x, ty = threadIdx.y;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int x0 = blockIdx.x * ZM_X, y0 = blockIdx.y * TY;
  const int z0 = blockIdx.z * p.zc;
  const int z1 = min(z0 + p.zc, nz);
  const size_t plane = static_cast<size_t>(nx) * ny;
  const int gx = wrap(x0 + tx, nx);
  // This thread's cells: rows ty + ZM_Y q of the tile.
  size_t col[CPT];
  bool active[CPT];
  // Halo duties: x halo (threads tx < 2R: left for tx < R, right otherwise)
  // for each of the thread's rows; y halo (threads ty < 2R) for column tx,
  // above the tile for ty < R and below it otherwise.
  const bool hx = tx < 2 * R;
  const int hx_col = tx < R ? x0 - R + tx : x0 + ZM_X + (tx - R);
  const int hx_slot = tx < R ? tx : ZM_X + R + (tx - R);
  size_t hx_off[CPT];
#pragma unroll
  for (int q = 0; q < CPT; ++q) {
    const int gy = wrap(y0 + ty + ZM_Y * q, ny);
    col[q] = static_cast<size_t>(gy) * nx + gx;
    active[q] = x0 + tx < nx && y0 + ty + ZM_Y * q < ny;
    hx_off[q] = static_cast<size_t>(gy) * nx + wrap(hx_col, nx);
  }
  const bool hy = ty < 2 * R;
  const int hy_row = ty < R ? y0 - R + ty : y0 + TY + (ty - R);
  const size_t hy_off = static_cast<size_t>(wrap(hy_row, ny)) * nx + gx;
  const int hy_slot = ty < R ? ty : TY + R + (ty - R);

  const T* fx = p.in[0];                         // LAP/GRAD field, DIV x component
  const T* fy = p.in[1];                         // DIV y component
  const T* fz = OP == OP_DIV ? p.in[2] : p.in[0];  // field whose z taps are queued

  T qz[CPT][NQ];
  T n_q[CPT], n_c[CPT], n_cy[CPT], n_hx[CPT];
  const size_t zoff = static_cast<size_t>(z0) * plane;
#pragma unroll
  for (int q = 0; q < CPT; ++q) {
#pragma unroll
    for (int k = 0; k < NQ - 1; ++k)
      qz[q][k + 1] = __ldg(fz + static_cast<size_t>(wrap(z0 - R + k, nz)) * plane + col[q]);
    // Prefetch of plane z0: its queue value (z0 + R), centre and halos.
    n_q[q] = __ldg(fz + static_cast<size_t>(wrap(z0 + R, nz)) * plane + col[q]);
    n_c[q] = (OP == OP_DIV) ? __ldg(fx + zoff + col[q]) : T(0);
    n_cy[q] = (OP == OP_DIV) ? __ldg(fy + zoff + col[q]) : T(0);
    n_hx[q] = hx ? __ldg(fx + zoff + hx_off[q]) : T(0);
  }
  T n_hy = hy ? __ldg((OP == OP_DIV ? fy : fx) + zoff + hy_off) : T(0);

  for (int z = z0; z < z1; ++z) {
    T c_x[CPT], c_y[CPT], h_x[CPT];
#pragma unroll
    for (int q = 0; q < CPT; ++q) {
#pragma unroll
      for (int k = 0; k + 1 < NQ; ++k) qz[q][k] = qz[q][k + 1];
      qz[q][NQ - 1] = n_q[q];
      c_x[q] = OP == OP_DIV ? n_c[q] : qz[q][R];
      c_y[q] = n_cy[q];
      h_x[q] = n_hx[q];
    }
    const T h_y = n_hy;
    if (z + 1 < z1) {  // prefetch plane z + 1
      const size_t zo = static_cast<size_t>(z + 1) * plane;
#pragma unroll
      for (int q = 0; q < CPT; ++q) {
        n_q[q] = __ldg(fz + static_cast<size_t>(wrap(z + 1 + R, nz)) * plane + col[q]);
        if (OP == OP_DIV) {
          n_c[q] = __ldg(fx + zo + col[q]);
          n_cy[q] = __ldg(fy + zo + col[q]);
        }
        if (hx) n_hx[q] = __ldg(fx + zo + hx_off[q]);
      }
      if (hy) n_hy = __ldg((OP == OP_DIV ? fy : fx) + zo + hy_off);
    }
#pragma unroll
    for (int q = 0; q < CPT; ++q) {
      const int row = ty + ZM_Y * q;
      sp[row + R][tx + R] = c_x[q];
      if (hx) sp[row + R][hx_slot] = h_x[q];
      if (OP == OP_DIV) sy[row + R][tx] = c_y[q];
    }
    if (hy) {
      if (OP == OP_DIV) sy[hy_slot][tx] = h_y;
      else sp[hy_slot][tx + R] = h_y;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < CPT; ++q) {
      if (!active[q]) continue;
      const int row = ty + ZM_Y * q;
      const size_t c = static_cast<size_t>(z) * plane + static_cast<size_t>(y0 + row) * nx + (x0 + tx);
      const T ax = tap_sum<T, K, ORDER>([&](int o) { return sp[row + R][tx + R + o]; });
      const T az = tap_sum<T, K, ORDER>([&](int o) { return qz[q][R + o]; });
      if constexpr (OP == OP_DIV) {
        const T ay = tap_sum<T, 1, ORDER>([&](int o) { return sy[row + R + o][tx]; });
        p.out[c] = Ar<T>::add(Ar<T>::add(Ar<T>::mul(ax, p.ihx), Ar<T>::mul(ay, p.ihy)), Ar<T>::mul(az, p.ihz));
      } else {
        const T ay = tap_sum<T, K, ORDER>([&](int o) { return sp[row + R + o][tx + R]; });
        if constexpr (OP == OP_LAP) {
          p.out[c] = Ar<T>::add(Ar<T>::add(Ar<T>::mul(ax, p.ihx2), Ar<T>::mul(ay, p.ihy2)), Ar<T>::mul(az, p.ihz2));
        } else {
          p.out[c] = Ar<T>::mul(ax, p.ihx);
          p.out[p.n + c] = Ar<T>::mul(ay, p.ihy);
          p.out[2 * p.n + c] = Ar<T>::mul(az, p.ihz);
        }
      }
    }
    __syncthreads();
  }
}

template <class T, int OP, int ORDER>
gc_status launch_zmarch(gc_context* ctx, const OpParams<T>& p0) {
  OpParams<T> p = p0;
  constexpr int TY = ZM_Y * zmarch_cpt<T, OP>();
  const int tiles_x = div_up(p.nx, ZM_X), tiles_y = div_up(p.ny, TY);
  const long long tiles = static_cast<long long>(tiles_x) * tiles_y;
  // Enough CTAs to fill the GPU several times, chunks of at least 16 planes.
  const long long want = 16LL * ctx->num_sms;
  int chunks = static_cast<int>(std::min<long long>((want + tiles - 1) / tiles, std::max(1, p.nz / 16)));
  chunks = std::max(chunks, 1);
  p.zc = div_up(p.nz, chunks);
  chunks = div_up(p.nz, p.zc);
  dim3 grid(tiles_x, tiles_y, chunks), block(ZM_X, ZM_Y);
  if constexpr (zmarch_cpt<T, OP>() > 1) {
    zmarch_rows_kernel<T, OP, ORDER><<<grid, block, 0, ctx->stream>>>(p);
    GC_CHECK_LAUNCH("zmarch_rows_kernel");
  } else {
    zmarch_kernel<T, OP, ORDER><<<grid, block, 0, ctx->stream>>>(p);
    GC_CHECK_LAUNCH("zmarch_kernel");
  }
  return GC_OK;
}

// ---------------------------------------------------------------------------
// 3-D kernel with asynchronous plane staging.  A 32 x 8 CTA owns a column of
// cells and marches up a chunk of z planes.  Every plane (with its periodic
// x/y halo) is copied into a ring of shared-memory slots by cp.async, kRing
// planes ahead of the plane being computed, one commit group per plane, so
// many planes' loads are in flight without holding registers; each thread
// waits for its own copies, one barrier per plane makes them visible, and
// the cell is computed from the ring exactly as in the ring kernel above.
// The ring has 2R + 1 + kRing slots: the slot refilled after computing
// plane z held plane z - R - 1, which no thread reads once all have passed
// plane z's barrier.
constexpr int kRing = 4;

__device__ __forceinline__ void cp_async_n(void* smem, const void* gmem, int bytes) {
  const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  if (bytes == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}

// Tile rows: the 32 x 8 threads cover 8 * CPT rows, each thread CPT cells of
// its column per plane, so the per-plane work (the wait, the barrier, the
// ring-slot arithmetic and the copy bookkeeping) is shared by CPT cells.  One
// cell per thread and plane left the float kernel bound by that work (105
// instructions per cell at 83 % issue).  Measured on B200 at 512^3, ms per
// launch for CPT = 1 / 2 / 4 (float; 8 at radius 1: laplacian order 2 0.291,
// gradient order 2 0.415 against 0.411 at 4) and 1 / 2 (double): float laplacian
// order 2 0.466 / 0.368 / 0.309, order 4 0.583 / 0.478 / 0.443, biharmonic
// 0.726 / 0.669 / 0.642; double laplacian order 2 0.500 / 0.455, order 4
// 0.755 / 0.766, biharmonic 1.041 / 1.074 (at radius 2 the taller double
// ring costs more occupancy than the shared work saves).
template <class T, int R>
__host__ __device__ constexpr int zring_cpt() {
  return sizeof(T) == 4 ? (R == 1 ? 8 : 4) : (R == 1 ? 2 : 1);
}

template <class T, int OP, int ORDER>
__global__ void __launch_bounds__(NT) zring_kernel(const OpParams<T> p) {
  constexpr int R = OpShape<OP, ORDER>::R;
  constexpr int NF = OpShape<OP, ORDER>::NF;
  constexpr int CPT = zring_cpt<T, R>(), TY = BY * CPT;
  constexpr int PW = BX + 2 * R, PH = TY + 2 * R, PS = PW * PH;
  constexpr int NB = 2 * R + 1 + kRing;
  constexpr int EPT = (PS + NT - 1) / NT;  // staged elements per thread per plane and field
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ring = reinterpret_cast<T*>(smem_raw);  // [NF][NB][PS]

  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * BX + tx;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int x0 = blockIdx.x * BX, y0 = blockIdx.y * TY;
  const int z0 = blockIdx.z * p.zc;
  const int z1 = min(z0 + p.zc, nz);
  const size_t plane = static_cast<size_t>(nx) * ny;

  // This thread's staged elements: the same in-plane offsets for every plane.
  size_t goff[EPT];
  int soff[EPT];
#pragma unroll
  for (int e = 0; e < EPT; ++e) {
    const int idx = tid + e * NT;
    soff[e] = idx < PS ? idx : -1;
    const int r = idx / PW, cc = idx - r * PW;
    goff[e] = idx < PS ? static_cast<size_t>(wrap(y0 - R + r, ny)) * nx + wrap(x0 - R + cc, nx) : 0;
  }
  // Slot of plane z + d from the slot s0 of plane z (|d| < NB).
  auto slot_at = [](int s0, int d) {
    int s = s0 + d;
    s += s < 0 ? NB : 0;
    s -= s >= NB ? NB : 0;
    return s;
  };
  auto issue = [&](int z, int sl) {  // plane z (wrapped) into slot sl, as one commit group
    if (z <= z1 - 1 + R) {
      const size_t zo = static_cast<size_t>(wrap(z, nz)) * plane;
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int e = 0; e < EPT; ++e)
          if (soff[e] >= 0) cp_async_n(ring + (f * NB + sl) * PS + soff[e], p.in[f] + zo + goff[e], sizeof(T));
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };

  // Plane z0 - R + j goes to slot j, so plane z sits in slot (z - z0 + R) mod NB.
  for (int j = 0; j < 2 * R + kRing; ++j) issue(z0 - R + j, j);
  const int gx = x0 + tx;
  int s0 = R;  // slot of plane z
  for (int z = z0; z < z1; ++z) {
    // plane z + R landed: the kRing - 1 later groups may still be in flight
    asm volatile("cp.async.wait_group %0;" ::"n"(kRing - 1) : "memory");
    __syncthreads();
    int sl[2 * R + 1];
#pragma unroll
    for (int d = -R; d <= R; ++d) sl[d + R] = slot_at(s0, d);
#pragma unroll
    for (int q = 0; q < CPT; ++q) {
      const int row = ty + q * BY, gy = y0 + row;
      if (gx < nx && gy < ny) {
        auto at = [&](int f, int dx, int dy, int dz) -> T {
          return ring[(f * NB + sl[dz + R]) * PS + (row + R + dy) * PW + (tx + R + dx)];
        };
        cell_op<T, OP, ORDER, true>(p, static_cast<size_t>(z) * plane + static_cast<size_t>(gy) * nx + gx, at);
      }
    }
    // The slot of plane z + R + kRing held plane z - R - 1, read by no one
    // once every thread has passed this plane's barrier.
    issue(z + R + kRing, slot_at(s0, R + kRing));
    s0 = slot_at(s0, 1);
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

template <class T, int OP, int ORDER>
gc_status launch_zring(gc_context* ctx, const OpParams<T>& p0) {
  constexpr int R = OpShape<OP, ORDER>::R;
  constexpr int NF = OpShape<OP, ORDER>::NF;
  constexpr int TY = BY * zring_cpt<T, R>();
  constexpr size_t smem = sizeof(T) * NF * (2 * R + 1 + kRing) * (BX + 2 * R) * (TY + 2 * R);
  OpParams<T> p = p0;
  const int tiles_x = div_up(p.nx, BX), tiles_y = div_up(p.ny, TY);
  const long long tiles = static_cast<long long>(tiles_x) * tiles_y;
  // Enough CTAs to fill the GPU several times, chunks of at least 32 planes
  // so the 2R + kRing prologue planes stay a small overhead.
  const long long want = 16LL * ctx->num_sms;
  int chunks = static_cast<int>(std::min<long long>((want + tiles - 1) / tiles, std::max(1, p.nz / 32)));
  chunks = std::max(chunks, 1);
  p.zc = div_up(p.nz, chunks);
  chunks = div_up(p.nz, p.zc);
  auto kern = zring_kernel<T, OP, ORDER>;
  GC_TRY(kernel_setup(kern, BX * BY, smem));
  dim3 grid(tiles_x, tiles_y, chunks), block(BX, BY);
  kern<<<grid, block, smem, ctx->stream>>>(p);
  GC_CHECK_LAUNCH("zring_kernel");
  return GC_OK;
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
  // 3-D grids.  The divergence, and in double the gradient above order 2
  // and the order-6 laplacian, march with a register queue (one field's
  // value per plane and thread, halo strips by a few threads); everything
  // else stages whole planes through the asynchronous ring with several
  // cells per thread.  Measured on B200 at 512^3, ms per launch (z-march /
  // ring): float gradient order 2 0.521 / 0.411, order 4 0.614 / 0.494,
  // laplacian order 6 0.589 / 0.543; double gradient order 2 0.821 / 0.729,
  // order 4 0.936 / 1.052, laplacian order 6 0.788 / 0.964.  The z-march
  // needs the z extent to exceed the radius; smaller extents take the ring
  // (planes wrap).
  if (z3) {
    if constexpr (OP == OP_GRAD || OP == OP_DIV || OP == OP_LAP) {
      const bool queue = OP == OP_DIV || (sizeof(T) == 8 && (OP == OP_GRAD ? order > 2 : order == 6));
      if (queue && p.nz > 2 * OpShape<OP, 6>::R) {
        switch (order) {
          case 2: return launch_zmarch<T, OP, 2>(ctx, p);
          case 4: return launch_zmarch<T, OP, 4>(ctx, p);
          case 6: return launch_zmarch<T, OP, 6>(ctx, p);
        }
      }
    }
    switch (order) {
      case 2: return launch_zring<T, OP, 2>(ctx, p);
      case 4: return launch_zring<T, OP, 4>(ctx, p);
      case 6: return launch_zring<T, OP, 6>(ctx, p);
    }
  }
  switch (order) {
    case 2: return launch_one<T, OP, 2, false>(ctx, p);
    case 4: return launch_one<T, OP, 4, false>(ctx, p);
    case 6: return launch_one<T, OP, 6, false>(ctx, p);
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

// Rank-2 forms (diff/Gradient.hpp:100-137, diff/Divergence.hpp:100-135).
// A matrix field is nine planes, plane 3*row + col holding M(row, col).
// Row `comp` of grad v is the vector-gradient kernel over plane `comp` of v;
// component `comp` of div M is the vector-divergence kernel over the three
// planes of row `comp`.  Both reproduce the reference's per-component sums
// exactly, and the three passes move exactly the rank-2 operator's bytes
// (every input plane read once, every output plane written once), so a
// fused kernel would save nothing but two launches.
template <int OP>
gc_status run_rank2(gc_context* ctx, const gc_grid* g, gc_dtype dt, int order, const void* in, void* out) {
  static_assert(OP == OP_GRAD || OP == OP_DIV, "rank-2 forms exist for gradient and divergence");
  // The first pass validates the context, grid, order, dtype and pointers.
  gc_status s = run_op<OP>(ctx, g, dt, order, in, out);
  if (s != GC_OK) return s;
  const size_t plane = cells(g) * dtype_size(dt);
  const size_t in_row = (OP == OP_GRAD ? 1 : 3) * plane, out_row = (OP == OP_GRAD ? 3 : 1) * plane;
  for (int comp = 1; comp < 3; ++comp) {
    s = run_op<OP>(ctx, g, dt, order, static_cast<const char*>(in) + comp * in_row,
                   static_cast<char*>(out) + comp * out_row);
    if (s != GC_OK) return s;
  }
  return GC_OK;
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

GC_API gc_status gc_gradient_vec(gc_context* ctx, const gc_grid* g, gc_dtype dt, int order,
                                 const void* in3, void* out9) {
  return run_rank2<OP_GRAD>(ctx, g, dt, order, in3, out9);
}

GC_API gc_status gc_divergence_mat(gc_context* ctx, const gc_grid* g, gc_dtype dt, int order,
                                   const void* in9, void* out3) {
  return run_rank2<OP_DIV>(ctx, g, dt, order, in9, out3);
}

}  // extern "C"
