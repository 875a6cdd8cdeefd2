// Cahn-Hilliard time stepping: fused RK4 / explicit-Euler stage kernels.
//
// RHS (examples/common/cahn_hilliard.hpp:38-59): M lap(mu), mu = -y + y^3 - kappa lap(y).
// RK4 (solve/RK4.hpp:99-154): k1 = f(psi), k2 = f(psi + dt/2 k1),
// k3 = f(psi + dt/2 k2), k4 = f(psi + dt k3),
// psi' = psi + (dt/6 (k1 + k4) + dt/3 (k2 + k3)).
//
// One kernel per stage.  A CTA owns a TX x TY (x TZ) tile of output cells:
//   phase 1  y = psi + a k_prev on the tile plus a 2r halo (wrapped loads),
//            staged in shared memory;
//   phase 2  mu on the tile plus an r halo from the staged y;
//   phase 3  k_s = M lap(mu) on the tile; the last stage instead combines
//            k1, k2, k3 (re-read at the own cell) with k4 and writes psi'.
// Per step each field is read or written once in HBM: 13 field passes
// (stage 1: 2, stages 2-3: 3 each, stage 4: 5); the halo re-reads are L2 hits.
// psi' goes to a second buffer (other CTAs still read psi's halo), so steps
// ping-pong between the caller's buffer and a context buffer; the step
// sequence is captured once into a CUDA graph and replayed.
// Double arithmetic keeps the reference's operation order without FMA, so
// double results match the CPU reference bit for bit.
#include <algorithm>
#include <cstring>

#include "ch_tile.cuh"
#include "common.cuh"
#include "stepper.cuh"
#include "tma.cuh"

namespace gcb {
namespace {

constexpr int kThreads = 256;

template <class T, int ORDER, bool Z3>
struct Tile;
// 2-D tiles: 64 wide rows (512 B of doubles) for coalescing.
template <class T, int ORDER>
struct Tile<T, ORDER, false> { static constexpr int TX = 64, TY = 16, TZ = 1; };
template <class T, int ORDER>
struct Tile<T, ORDER, true> {
  static constexpr int TX = 32, TY = ORDER == 2 ? 8 : 4, TZ = ORDER == 2 ? 8 : 4;
};

template <class T, int ORDER, bool Z3, int MODE>
__global__ void __launch_bounds__(kThreads) ch_stage_kernel(const StageParams<T> p) {
  constexpr int R = W<2, ORDER>::R;
  constexpr int TX = Tile<T, ORDER, Z3>::TX, TY = Tile<T, ORDER, Z3>::TY, TZ = Tile<T, ORDER, Z3>::TZ;
  constexpr int RZ = Z3 ? R : 0;
  // y region: tile + 2R halo; mu region: tile + R halo.
  constexpr int YX = TX + 4 * R, YY = TY + 4 * R, YZ = TZ + 4 * RZ;
  constexpr int MX = TX + 2 * R, MY = TY + 2 * R, MZ = TZ + 2 * RZ;
  constexpr int YN = YX * YY * YZ, MN = MX * MY * MZ, ON = TX * TY * TZ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ys = reinterpret_cast<T*>(smem_raw);
  T* ms = ys + YN;

  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * TZ;
  const size_t plane = static_cast<size_t>(nx) * ny;

  // Phase 1: y on the tile + 2R halo.
  for (int e = threadIdx.x; e < YN; e += kThreads) {
    const int ex = e % YX;
    const int rest = e / YX;
    const int ey = rest % YY;
    const int ez = rest / YY;
    const int gx = wrap(x0 - 2 * R + ex, nx);
    const int gy = wrap(y0 - 2 * R + ey, ny);
    const int gz = Z3 ? wrap(z0 - 2 * RZ + ez, nz) : 0;
    const size_t gi = static_cast<size_t>(gz) * plane + static_cast<size_t>(gy) * nx + gx;
    T v = __ldg(p.psi + gi);
    if (p.kin) v = Ar<T>::add(v, Ar<T>::mul(p.a, __ldg(p.kin + gi)));
    ys[e] = v;
  }
  __syncthreads();

  // Phase 2: mu = -y + y^3 - kappa lap(y) on the tile + R halo.
  for (int e = threadIdx.x; e < MN; e += kThreads) {
    const int ex = e % MX;
    const int rest = e / MX;
    const int ey = rest % MY;
    const int ez = rest / MY;
    const int c = ((ez + RZ) * YY + (ey + R)) * YX + (ex + R);  // same cell in y space
    const T ax = tap_sum<T, 2, ORDER>([&](int o) { return ys[c + o]; });
    const T ay = tap_sum<T, 2, ORDER>([&](int o) { return ys[c + o * YX]; });
    const T az = tap_sum<T, 2, ORDER>([&](int o) { return ys[c + (Z3 ? o : 0) * YX * YY]; });
    const T lap = lap_z(p, lap_xy(p, ax, ay), az);
    const T y = ys[c];
    ms[e] = chem_pot(p, y, lap);
  }
  __syncthreads();

  // Phase 3: k_s = M lap(mu) on the tile.
  for (int e = threadIdx.x; e < ON; e += kThreads) {
    const int ex = e % TX;
    const int rest = e / TX;
    const int ey = rest % TY;
    const int ez = rest / TY;
    const int gx = x0 + ex, gy = y0 + ey, gz = z0 + ez;
    if (gx >= nx || gy >= ny || gz >= nz) continue;
    const int c = ((ez + RZ) * MY + (ey + R)) * MX + (ex + R);
    const T ax = tap_sum<T, 2, ORDER>([&](int o) { return ms[c + o]; });
    const T ay = tap_sum<T, 2, ORDER>([&](int o) { return ms[c + o * MX]; });
    const T az = tap_sum<T, 2, ORDER>([&](int o) { return ms[c + (Z3 ? o : 0) * MX * MY]; });
    const T lap = lap_z(p, lap_xy(p, ax, ay), az);
    const T rhs = mobility(p, lap);
    const size_t gi = static_cast<size_t>(gz) * plane + static_cast<size_t>(gy) * nx + gx;
    if constexpr (MODE == MODE_RHS) {
      p.out[gi] = rhs;
    } else if constexpr (MODE == MODE_RK4_FINAL) {
      const T s14 = Ar<T>::add(__ldg(p.k1 + gi), rhs);
      const T s23 = Ar<T>::add(__ldg(p.k2 + gi), __ldg(p.k3 + gi));
      p.out[gi] = Ar<T>::add(__ldg(p.psi + gi), Ar<T>::add(Ar<T>::mul(p.c6, s14), Ar<T>::mul(p.c3, s23)));
    } else if constexpr (MODE == MODE_RKC_FIRST || MODE == MODE_RKC) {
      const int cy = ((ez + 2 * RZ) * YY + (ey + 2 * R)) * YX + (ex + 2 * R);
      if constexpr (MODE == MODE_RKC_FIRST) {
        p.out[gi] = rhs;
        p.out2[gi] = Ar<T>::add(ys[cy], Ar<T>::mul(p.r[0], rhs));
      } else {
        p.out[gi] = rkc_combine(p, p.k1[gi], ys[cy], p.k2[gi], rhs, p.k3[gi]);
      }
    } else {
      const int cy = ((ez + 2 * RZ) * YY + (ey + 2 * R)) * YX + (ex + 2 * R);
      p.out[gi] = Ar<T>::add(ys[cy], Ar<T>::mul(p.c6, rhs));
    }
  }
}

template <class T, int ORDER, bool Z3, int MODE>
gc_status launch_stage(gc_context* ctx, const StageParams<T>& p) {
  constexpr int R = W<2, ORDER>::R;
  using TL = Tile<T, ORDER, Z3>;
  constexpr int RZ = Z3 ? R : 0;
  constexpr size_t smem =
      sizeof(T) * (static_cast<size_t>(TL::TX + 4 * R) * (TL::TY + 4 * R) * (TL::TZ + 4 * RZ) +
                   static_cast<size_t>(TL::TX + 2 * R) * (TL::TY + 2 * R) * (TL::TZ + 2 * RZ));
  auto kern = ch_stage_kernel<T, ORDER, Z3, MODE>;
  if (smem > 48 * 1024) GC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid(div_up(p.nx, TL::TX), div_up(p.ny, TL::TY), Z3 ? div_up(p.nz, TL::TZ) : 1);
  kern<<<grid, kThreads, smem, ctx->stream>>>(p);
  GC_CHECK_LAUNCH("ch_stage_kernel");
  return GC_OK;
}

// ---------------------------------------------------------------------------
// Persistent TMA-pipelined 2-D stage kernel (double precision, Nz == 1).
// Same tile geometry and the same arithmetic as ch_tile2d_kernel; what
// changes is how the inputs arrive.  Each CTA loops over tiles; while it
// computes tile i, one thread has already issued the TMA loads
// (cp.async.bulk.tensor.2d) of tile i+1 -- psi and k_prev on the y region,
// and k1, k2 on the output tile in the last RK4 stage -- into the other
// half of a double-buffered shared-memory ring, completing an mbarrier
// with the bytes delivered.  Waits on the mbarrier are bounded by a clock
// budget: on expiry the CTA records GC_ERR_TIMEOUT in the context's status
// word and leaves.  TMA has no periodic wrap, so tiles whose y region
// crosses the domain edge (a few percent at large sizes) are loaded with
// ordinary wrapped loads instead; their barrier phase is still completed
// by a plain arrive so the parity sequence stays regular.
constexpr int kTmaThreads = kT2W * kT2TY;
constexpr long long kWaitBudgetCycles = 4000000000LL;  // about 2 s at 2 GHz

template <class T, int ORDER, int MODE, bool KIN>
struct TmaLayout {
  static constexpr int R = W<2, ORDER>::R;
  static constexpr int TX = kT2W - 2 * R, TY = kT2Y;
  static constexpr int YX = TX + 4 * R, YY = TY + 4 * R;
  static constexpr int MX = kT2W, MY = TY + 2 * R;
  // k1, k2 of the last RK4 stage are read once per output cell, so they are
  // fetched into registers rather than staged.
  static constexpr size_t al(size_t b) { return (b + 127) / 128 * 128; }
  static constexpr size_t YB = al(sizeof(T) * YX * YY);   // one y-region field
  static constexpr size_t BUF = YB + (KIN ? YB : 0);
  static constexpr size_t OFF_BUF = 128;                  // after the barriers
  // y = psi + a k_prev is formed in place in the k_prev buffer (no separate
  // y region), which keeps four CTAs per SM in double precision.
  static constexpr size_t OFF_MS = OFF_BUF + 2 * BUF;
  static constexpr size_t BYTES = OFF_MS + al(sizeof(T) * MX * MY) + 128;  // + alignment slack
  static constexpr uint32_t TX_BYTES = static_cast<uint32_t>(sizeof(T) * YX * YY * (KIN ? 2 : 1));
};

template <class T, int ORDER, int MODE, bool KIN>
__global__ void __launch_bounds__(kTmaThreads) ch_tma_kernel(
    const StageParams<T> p, const __grid_constant__ CUtensorMap m_psi, const __grid_constant__ CUtensorMap m_kin,
    const int tiles_x, const int tiles_y, int* status) {
  using L = TmaLayout<T, ORDER, MODE, KIN>;
  constexpr int R = L::R, TX = L::TX, TY = L::TY, YX = L::YX, YY = L::YY, MX = L::MX, MY = L::MY;
  constexpr int NW = 2 * R + 1;
  constexpr int MS = (MY + kT2TY - 1) / kT2TY;
  constexpr int OS = TY / kT2TY;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  uint64_t* bar = reinterpret_cast<uint64_t*>(base);
  int* s_abort = reinterpret_cast<int*>(base + 64);
  auto buf_psi = [&](int b) { return reinterpret_cast<T*>(base + L::OFF_BUF + b * L::BUF); };
  auto buf_kin = [&](int b) { return reinterpret_cast<T*>(base + L::OFF_BUF + b * L::BUF + L::YB); };
  T* ms = reinterpret_cast<T*>(base + L::OFF_MS);

  const int nx = p.nx, ny = p.ny;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kT2W + tx;
  const int ntiles = tiles_x * tiles_y;

  auto tile_origin = [&](int tl, int& x0, int& y0) {
    x0 = (tl % tiles_x) * TX;
    y0 = (tl / tiles_x) * TY;
  };
  auto interior = [&](int x0, int y0) {
    return x0 - 2 * R >= 0 && x0 - 2 * R + YX <= nx && y0 - 2 * R >= 0 && y0 - 2 * R + YY <= ny;
  };
  auto issue = [&](int tl, int b) {  // one thread
    int x0, y0;
    tile_origin(tl, x0, y0);
    if (interior(x0, y0)) {
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&bar[b], L::TX_BYTES);
      tma_load_2d(buf_psi(b), &m_psi, x0 - 2 * R, y0 - 2 * R, &bar[b]);
      if constexpr (KIN) tma_load_2d(buf_kin(b), &m_kin, x0 - 2 * R, y0 - 2 * R, &bar[b]);
    } else {
      mbar_arrive(&bar[b]);
    }
  };

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    *s_abort = 0;
    mbar_init_fence();
  }
  __syncthreads();
  if (tid == 0 && blockIdx.x < ntiles) issue(blockIdx.x, 0);

  int i = 0;
  for (int tl = blockIdx.x; tl < ntiles; tl += gridDim.x, ++i) {
    const int b = i & 1;
    if (tid == 0 && tl + static_cast<int>(gridDim.x) < ntiles) issue(tl + gridDim.x, b ^ 1);
    int x0, y0;
    tile_origin(tl, x0, y0);
    // Last RK4 stage: k1 and k2 at this thread's output cells, issued before
    // the wait so that they travel while the tile's TMA completes.
    T r_k1[OS], r_k2[OS];
    if constexpr (MODE == MODE_RK4_FINAL) {
#pragma unroll
      for (int k = 0; k < OS; ++k) {
        const int oy = ty * OS + k;
        const bool in = tx < TX && x0 + tx < nx && y0 + oy < ny;
        const size_t gi = in ? static_cast<size_t>(y0 + oy) * nx + (x0 + tx) : 0;
        r_k1[k] = in ? __ldg(p.k1 + gi) : T(0);
        r_k2[k] = in ? __ldg(p.k2 + gi) : T(0);
      }
    }
    const long long t_start = clock64();
    while (!mbar_try_wait(&bar[b], (i >> 1) & 1)) {
      if (clock64() - t_start > kWaitBudgetCycles) {
        *s_abort = 1;
        atomicExch(status, static_cast<int>(GC_ERR_TIMEOUT));
        break;
      }
    }
    T* ps = buf_psi(b);
    if (!interior(x0, y0)) {
      // Wrapped y region with ordinary loads.
      T* ks = buf_kin(b);
      for (int e = tid; e < YX * YY; e += kTmaThreads) {
        const int r = e / YX, cc = e - r * YX;
        const size_t gi = static_cast<size_t>(wrap(y0 - 2 * R + r, ny)) * nx + wrap(x0 - 2 * R + cc, nx);
        ps[e] = p.psi[gi];
        if constexpr (KIN) ks[e] = p.kin[gi];
      }
    }
    __syncthreads();
    if (*s_abort) {
      // Let the prefetch of the next tile land (bounded) before leaving.
      if (tid == 0 && tl + static_cast<int>(gridDim.x) < ntiles) {
        const long long t_drain = clock64();
        while (!mbar_try_wait(&bar[b ^ 1], ((i + 1) >> 1) & 1) && clock64() - t_drain < kWaitBudgetCycles) {
        }
      }
      break;
    }

    // y = psi + a k_prev, in place over k_prev (stage 1 and Euler read psi
    // directly).  The last RK4 stage first keeps k3 at its own output cells.
    const T* ys = ps;
    T r_k3[OS];
    if constexpr (KIN) {
      T* ks = buf_kin(b);
      if constexpr (MODE == MODE_RK4_FINAL) {
#pragma unroll
        for (int k = 0; k < OS; ++k) r_k3[k] = ks[(ty * OS + k + 2 * R) * YX + (tx + 2 * R)];
        __syncthreads();
      }
      for (int e = tid; e < YX * YY; e += kTmaThreads) ks[e] = Ar<T>::add(ps[e], Ar<T>::mul(p.a, ks[e]));
      __syncthreads();
      ys = ks;
    }

    // Phase 2: mu at mu-row strip [m0, m1), column tx (y column tx + R).
    {
      const int m0 = ty * MS;
      const int m1 = min(m0 + MS, MY);
      const int cx = tx + R;
      T win[NW];
#pragma unroll
      for (int k = 0; k < 2 * R; ++k) win[k + 1] = ys[(m0 + k) * YX + cx];
#pragma unroll
      for (int k = 0; k < MS; ++k) {
        const int m = m0 + k;
        if (m < m1) {
#pragma unroll
          for (int q = 0; q + 1 < NW; ++q) win[q] = win[q + 1];
          win[NW - 1] = ys[(m + 2 * R) * YX + cx];
          const T yc = win[R];
          const T ax = tap_sum<T, 2, ORDER>([&](int o) { return o == 0 ? yc : ys[(m + R) * YX + cx + o]; });
          const T ay = tap_sum<T, 2, ORDER>([&](int o) { return win[R + o]; });
          T lap = lap_xy(p, ax, ay);
          if constexpr (ORDER != 2) {
            lap = lap_z(p, lap, tap_sum<T, 2, ORDER>([&](int) { return yc; }));
          }
          ms[m * MX + tx] = chem_pot(p, yc, lap);
        }
      }
    }
    __syncthreads();

    // Phase 3: output strip.
    if (tx < TX && x0 + tx < nx) {
      const int o0 = ty * OS;
      const int cx = tx + R;
      T win[NW];
#pragma unroll
      for (int k = 0; k < 2 * R; ++k) win[k + 1] = ms[(o0 + k) * MX + cx];
#pragma unroll
      for (int k = 0; k < OS; ++k) {
        const int oy = o0 + k;
#pragma unroll
        for (int q = 0; q + 1 < NW; ++q) win[q] = win[q + 1];
        win[NW - 1] = ms[(oy + 2 * R) * MX + cx];
        if (y0 + oy >= ny) break;
        const T mc = win[R];
        const T ax = tap_sum<T, 2, ORDER>([&](int o) { return o == 0 ? mc : ms[(oy + R) * MX + cx + o]; });
        const T ay = tap_sum<T, 2, ORDER>([&](int o) { return win[R + o]; });
        T lap = lap_xy(p, ax, ay);
        if constexpr (ORDER != 2) {
          lap = lap_z(p, lap, tap_sum<T, 2, ORDER>([&](int) { return mc; }));
        }
        const T rhs = mobility(p, lap);
        const size_t gi = static_cast<size_t>(y0 + oy) * nx + (x0 + tx);
        const int yc_idx = (oy + 2 * R) * YX + (tx + 2 * R);
        if constexpr (MODE == MODE_RHS) {
          p.out[gi] = rhs;
        } else if constexpr (MODE == MODE_RK4_FINAL) {
          const T s14 = Ar<T>::add(r_k1[k], rhs);
          const T s23 = Ar<T>::add(r_k2[k], r_k3[k]);
          p.out[gi] = Ar<T>::add(ps[yc_idx], Ar<T>::add(Ar<T>::mul(p.c6, s14), Ar<T>::mul(p.c3, s23)));
        } else {
          p.out[gi] = Ar<T>::add(ps[yc_idx], Ar<T>::mul(p.c6, rhs));
        }
      }
    }
    __syncthreads();
  }
}

// Launches the TMA kernel when its layout rules hold; GC_ERR_UNSUPPORTED
// (nothing launched) otherwise, and the caller uses ch_tile2d_kernel.
template <class T, int ORDER, int MODE, bool KIN>
gc_status launch_tma(gc_context* ctx, const StageParams<T>& p) {
  using L = TmaLayout<T, ORDER, MODE, KIN>;
  if (p.nx < L::YX || p.ny < L::YY) return GC_ERR_UNSUPPORTED;
  CUtensorMap mpsi{}, mkin{};
  const int eb = static_cast<int>(sizeof(T));
  if (!make_tensor_map_2d(&mpsi, p.psi, p.nx, p.ny, eb, L::YX, L::YY)) return GC_ERR_UNSUPPORTED;
  if (KIN && !make_tensor_map_2d(&mkin, p.kin, p.nx, p.ny, eb, L::YX, L::YY)) return GC_ERR_UNSUPPORTED;
  auto kern = ch_tma_kernel<T, ORDER, MODE, KIN>;
  int ctas_per_sm = 1;
  GC_TRY(kernel_setup(kern, kTmaThreads, L::BYTES, &ctas_per_sm));
  const int tiles_x = div_up(p.nx, L::TX), tiles_y = div_up(p.ny, L::TY);
  const long long ntiles = static_cast<long long>(tiles_x) * tiles_y;
  const int grid = static_cast<int>(std::min<long long>(ntiles, static_cast<long long>(ctas_per_sm) * ctx->num_sms));
  kern<<<grid, dim3(kT2W, kT2TY), L::BYTES, ctx->stream>>>(p, mpsi, mkin, tiles_x, tiles_y, ctx->device_status);
  GC_CHECK_LAUNCH("ch_tma_kernel");
  return GC_OK;
}

// ---------------------------------------------------------------------------
// Two-column variant of the TMA stage kernel for double grids of even
// width: the RHS stages (RK4 stages 1-3) and the explicit-Euler step.
// 64 threads in x over a 128-column mu region (8 thread rows over 32-row
// tiles at order 2, 4 over 16 rows at order 4); a thread owns a pair of
// adjacent columns in every phase, so shared-memory reads, the in-place y
// pass and the global stores move 16 bytes per instruction, the address
// arithmetic of a row is shared by two cells, and each thread carries two
// independent tap-sum chains.  The single-column kernel is issue-bound, not
// bandwidth-bound, in these stages.  Cell arithmetic is that of
// ch_tma_kernel operation for operation, so results are bit-identical.
//
// Alignment: tile widths (128 - 2R) and tile origins are even, the staged
// rows are YX = 128 + 2R doubles (a multiple of 16 bytes), so the x-tap span
// of a pair (columns 2t .. 2t + 2R + 1 of the y or mu region) and every
// pair store start on 16-byte boundaries.  The centre pair of a y or mu row
// (columns 2t + R, 2t + R + 1) is 16-byte aligned only for even R; for
// R = 1 the whole span (4 doubles) is kept per window row instead.
constexpr int kX2DT = 64;  // threads in x: column pairs of the mu region
constexpr long long kX2MinRounds = 10;  // tiles per persistent CTA for the two-column kernel

// The x-tap span of pair t in a row: sp[j] = row[2 t + j], j < 2R + 2.
template <int R>
__device__ __forceinline__ void x2_span(const double* row, int t, double (&sp)[2 * R + 2]) {
#pragma unroll
  for (int j = 0; j < R + 1; ++j) {
    const double2 v = *reinterpret_cast<const double2*>(row + 2 * t + 2 * j);
    sp[2 * j] = v.x;
    sp[2 * j + 1] = v.y;
  }
}

// The centre pair of pair t in a row (columns 2t + R, 2t + R + 1).
template <int R>
__device__ __forceinline__ double2 x2_centre(const double* row, int t) {
  if constexpr (R % 2 == 0) {
    return *reinterpret_cast<const double2*>(row + 2 * t + R);
  } else {
    return make_double2(row[2 * t + R], row[2 * t + R + 1]);
  }
}

// Laplacian of a pair: x taps from its span, y taps from ya(o), yb(o),
// o = -R .. R; the axes and the 1-cell z axis combined as in ch_tma_kernel.
template <int ORDER, class GA, class GB>
__device__ __forceinline__ void x2_lap_pair(const StageParams<double>& p, const double (&sp)[2 * W<2, ORDER>::R + 2],
                                            GA ya, GB yb, double& la, double& lb) {
  using T = double;
  constexpr int R = W<2, ORDER>::R;
  const T axa = tap_sum<T, 2, ORDER>([&](int o) { return sp[R + o]; });
  const T axb = tap_sum<T, 2, ORDER>([&](int o) { return sp[R + 1 + o]; });
  const T aya = tap_sum<T, 2, ORDER>(ya);
  const T ayb = tap_sum<T, 2, ORDER>(yb);
  la = lap_xy(p, axa, aya);
  lb = lap_xy(p, axb, ayb);
  if constexpr (ORDER != 2) {
    const T ca = sp[R], cb = sp[R + 1];
    la = lap_z(p, la, tap_sum<T, 2, ORDER>([&](int) { return ca; }));
    lb = lap_z(p, lb, tap_sum<T, 2, ORDER>([&](int) { return cb; }));
  }
}

// Runs pair t's window down rows [r0, r1) (at most `count`) of a region
// with row stride `stride`: row r takes rows r .. r + 2R as its y taps and
// row r + R's span as its x taps; emit(r, la, lb, ca, cb) receives the two
// Laplacians and the two centre values.  For R = 1 the window keeps each
// row's whole span (two 16-byte loads per row and pair, nothing else).
template <int ORDER, int COUNT, class Emit>
__device__ __forceinline__ void x2_sweep(const StageParams<double>& p, const double* src, int stride, int t, int r0,
                                         int r1, Emit emit) {
  using T = double;
  constexpr int R = W<2, ORDER>::R;
  constexpr int NS = 2 * R + 2, NW = 2 * R + 1;
  if (r0 >= r1) return;  // an idle thread row: not even the window's first rows
  if constexpr (R == 1) {
    T sw[3][NS];
    x2_span<R>(src + r0 * stride, t, sw[1]);
    x2_span<R>(src + (r0 + 1) * stride, t, sw[2]);
#pragma unroll
    for (int k = 0; k < COUNT; ++k) {
      const int r = r0 + k;
      if (r >= r1) break;
#pragma unroll
      for (int j = 0; j < NS; ++j) {
        sw[0][j] = sw[1][j];
        sw[1][j] = sw[2][j];
      }
      x2_span<R>(src + (r + 2) * stride, t, sw[2]);
      T la, lb;
      x2_lap_pair<ORDER>(p, sw[1], [&](int o) { return sw[1 + o][1]; }, [&](int o) { return sw[1 + o][2]; }, la, lb);
      emit(r, la, lb, sw[1][1], sw[1][2]);
    }
  } else {
    double2 win[NW];
#pragma unroll
    for (int q = 0; q < 2 * R; ++q) win[q + 1] = x2_centre<R>(src + (r0 + q) * stride, t);
#pragma unroll
    for (int k = 0; k < COUNT; ++k) {
      const int r = r0 + k;
      if (r >= r1) break;
#pragma unroll
      for (int q = 0; q + 1 < NW; ++q) win[q] = win[q + 1];
      win[NW - 1] = x2_centre<R>(src + (r + 2 * R) * stride, t);
      T sp[NS];
      x2_span<R>(src + (r + R) * stride, t, sp);
      T la, lb;
      x2_lap_pair<ORDER>(p, sp, [&](int o) { return win[R + o].x; }, [&](int o) { return win[R + o].y; }, la, lb);
      emit(r, la, lb, win[R].x, win[R].y);
    }
  }
}

template <int ORDER, bool KIN>
struct TmaX2Layout {
  static constexpr int R = W<2, ORDER>::R;
  // Order 2: 64 x 8 threads over 32-row tiles (32 warps per SM in both
  // stage kinds, 36 staged rows per 32 output rows); wider stencils keep
  // 64 x 4 threads over 16 rows, whose staged regions fit three CTAs per SM.
  static constexpr int NTY = ORDER == 2 ? 8 : kT2TY;
  static constexpr int MX = 2 * kX2DT, TX = MX - 2 * R, TY = ORDER == 2 ? 32 : kT2Y;
  static constexpr int YX = TX + 4 * R, YY = TY + 4 * R, MY = TY + 2 * R;
  static constexpr size_t al(size_t b) { return (b + 127) / 128 * 128; }
  static constexpr size_t YB = al(sizeof(double) * YX * YY);
  static constexpr size_t BUF = YB * (KIN ? 2 : 1);
  static constexpr size_t OFF_BUF = 128;
  static constexpr size_t MSB = al(sizeof(double) * MX * MY);
  // Input buffers: two (the next tile's TMA lands while this one computes)
  // when two such CTAs fit in an SM's 228 KB of shared memory (each also
  // holds 1 KB reserved by the hardware); otherwise one, where the next
  // tile's TMA is issued once the y region is consumed (after phase 2) and
  // an L2 prefetch of that tile at the start of this one covers its
  // latency.  Order 2: two buffers without k_prev and one with it, 108 KB
  // and two 512-thread CTAs per SM either way; order 4 with k_prev: one
  // buffer, 71 KB, three CTAs per SM instead of one.
  static constexpr int NB = 2 * (OFF_BUF + 2 * BUF + MSB + 128 + 1024) <= 228 * 1024 ? 2 : 1;
  static constexpr size_t OFF_MS = OFF_BUF + NB * BUF;
  static constexpr size_t BYTES = OFF_MS + MSB + 128;
  static constexpr uint32_t TX_BYTES = static_cast<uint32_t>(sizeof(double) * YX * YY * (KIN ? 2 : 1));
  static_assert(YX % 2 == 0 && TX % 2 == 0 && (YX * YY) % 2 == 0, "pairs must stay 16-byte aligned");
};

template <int ORDER, int MODE, bool KIN>
__global__ void __launch_bounds__(kX2DT * TmaX2Layout<ORDER, KIN>::NTY) ch_tma_x2_kernel(
    const StageParams<double> p, const __grid_constant__ CUtensorMap m_psi,
    const __grid_constant__ CUtensorMap m_kin, const int tiles_x, const int tiles_y, int* status) {
  using T = double;
  using L = TmaX2Layout<ORDER, KIN>;
  static_assert(MODE == MODE_RHS || L::NB == 2, "a single input buffer holds psi only until phase 2");
  constexpr int R = L::R, TX = L::TX, TY = L::TY, YX = L::YX, YY = L::YY, MX = L::MX, MY = L::MY;
  constexpr int NTY = L::NTY, NT = kX2DT * NTY;
  constexpr int NB = L::NB;
  constexpr int MS = (MY + NTY - 1) / NTY;
  constexpr int OS = TY / NTY;
  static_assert(TY % NTY == 0, "output rows split evenly over thread rows");
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  uint64_t* bar = reinterpret_cast<uint64_t*>(base);
  int* s_abort = reinterpret_cast<int*>(base + 64);
  auto buf_psi = [&](int b) { return reinterpret_cast<T*>(base + L::OFF_BUF + b * L::BUF); };
  auto buf_kin = [&](int b) { return reinterpret_cast<T*>(base + L::OFF_BUF + b * L::BUF + L::YB); };
  T* ms = reinterpret_cast<T*>(base + L::OFF_MS);

  const int nx = p.nx, ny = p.ny;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kX2DT + tx;
  const int ntiles = tiles_x * tiles_y;

  auto tile_origin = [&](int tl, int& x0, int& y0) {
    x0 = (tl % tiles_x) * TX;
    y0 = (tl / tiles_x) * TY;
  };
  auto interior = [&](int x0, int y0) {
    return x0 - 2 * R >= 0 && x0 - 2 * R + YX <= nx && y0 - 2 * R >= 0 && y0 - 2 * R + YY <= ny;
  };
  auto issue = [&](int tl, int b) {  // one thread
    int x0, y0;
    tile_origin(tl, x0, y0);
    if (interior(x0, y0)) {
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&bar[b], L::TX_BYTES);
      tma_load_2d(buf_psi(b), &m_psi, x0 - 2 * R, y0 - 2 * R, &bar[b]);
      if constexpr (KIN) tma_load_2d(buf_kin(b), &m_kin, x0 - 2 * R, y0 - 2 * R, &bar[b]);
    } else {
      mbar_arrive(&bar[b]);
    }
  };
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    *s_abort = 0;
    mbar_init_fence();
  }
  __syncthreads();
  if (tid == 0 && blockIdx.x < ntiles) issue(blockIdx.x, 0);

  int i = 0;
  for (int tl = blockIdx.x; tl < ntiles; tl += gridDim.x, ++i) {
    const int b = NB == 2 ? (i & 1) : 0;
    const uint32_t parity = NB == 2 ? (i >> 1) & 1 : i & 1;
    const int next = tl + static_cast<int>(gridDim.x);
    if (tid == 0 && next < ntiles) {
      if constexpr (NB == 2) {
        issue(next, b ^ 1);
      } else {
        int nx0, ny0;
        tile_origin(next, nx0, ny0);
        if (interior(nx0, ny0)) {
          tma_prefetch_2d(&m_psi, nx0 - 2 * R, ny0 - 2 * R);
          tma_prefetch_2d(&m_kin, nx0 - 2 * R, ny0 - 2 * R);
        }
      }
    }
    int x0, y0;
    tile_origin(tl, x0, y0);
    const long long t_start = clock64();
    while (!mbar_try_wait(&bar[b], parity)) {
      if (clock64() - t_start > kWaitBudgetCycles) {
        *s_abort = 1;
        atomicExch(status, static_cast<int>(GC_ERR_TIMEOUT));
        break;
      }
    }
    T* ps = buf_psi(b);
    if (!interior(x0, y0)) {
      T* ks = buf_kin(b);
      for (int e = tid; e < YX * YY; e += NT) {
        const int r = e / YX, cc = e - r * YX;
        const size_t gi = static_cast<size_t>(wrap(y0 - 2 * R + r, ny)) * nx + wrap(x0 - 2 * R + cc, nx);
        ps[e] = p.psi[gi];
        if constexpr (KIN) ks[e] = p.kin[gi];
      }
    }
    __syncthreads();
    if (*s_abort) {
      if (NB == 2 && tid == 0 && next < ntiles) {
        const long long t_drain = clock64();
        while (!mbar_try_wait(&bar[b ^ 1], ((i + 1) >> 1) & 1) && clock64() - t_drain < kWaitBudgetCycles) {
        }
      }
      break;
    }

    // y = psi + a k_prev, in place over k_prev, a pair per thread and step.
    const T* ys = ps;
    if constexpr (KIN) {
      double2* k2 = reinterpret_cast<double2*>(buf_kin(b));
      const double2* p2 = reinterpret_cast<const double2*>(ps);
      for (int e = tid; e < YX * YY / 2; e += NT) {
        const double2 v = p2[e];
        double2 w = k2[e];
        w.x = Ar<T>::add(v.x, Ar<T>::mul(p.a, w.x));
        w.y = Ar<T>::add(v.y, Ar<T>::mul(p.a, w.y));
        k2[e] = w;
      }
      __syncthreads();
      ys = buf_kin(b);
    }

    // Phase 2: mu on mu columns 2 tx, 2 tx + 1 of the mu-row strip.
    {
      const int m0 = ty * MS;
      x2_sweep<ORDER, MS>(p, ys, YX, tx, m0, min(m0 + MS, MY), [&](int m, T la, T lb, T ya, T yb) {
        *reinterpret_cast<double2*>(ms + m * MX + 2 * tx) = make_double2(chem_pot(p, ya, la), chem_pot(p, yb, lb));
      });
    }
    __syncthreads();
    // One buffer: the y region is consumed, the next tile may land in it.
    if (NB == 1 && tid == 0 && next < ntiles) issue(next, 0);

    // Phase 3: output pair (2 tx, 2 tx + 1) of each of this thread's rows.
    if (2 * tx < TX && x0 + 2 * tx < nx) {
      const int o0 = ty * OS;
      const int o1 = min(o0 + OS, ny - y0);
      x2_sweep<ORDER, OS>(p, ms, MX, tx, o0, o1, [&](int oy, T la, T lb, T, T) {
        const double2 rhs = make_double2(mobility(p, la), mobility(p, lb));
        const size_t gi = static_cast<size_t>(y0 + oy) * nx + (x0 + 2 * tx);
        double2* out = reinterpret_cast<double2*>(p.out + gi);
        if constexpr (MODE == MODE_RHS) {
          *out = rhs;
        } else {  // MODE_EULER_FINAL
          const double2 pc = *reinterpret_cast<const double2*>(ps + (oy + 2 * R) * YX + 2 * tx + 2 * R);
          *out = make_double2(Ar<T>::add(pc.x, Ar<T>::mul(p.c6, rhs.x)), Ar<T>::add(pc.y, Ar<T>::mul(p.c6, rhs.y)));
        }
      });
    }
    __syncthreads();
  }
}

// Launches the two-column kernel when its rules hold (even width, 16-byte
// aligned output, the staged region fits the grid, enough tiles to fill
// ten rounds of persistent CTAs); GC_ERR_UNSUPPORTED (nothing launched)
// otherwise, and the caller uses ch_tma_kernel.
template <int ORDER, int MODE, bool KIN>
gc_status launch_tma_x2(gc_context* ctx, const StageParams<double>& p) {
  using L = TmaX2Layout<ORDER, KIN>;
  if (p.nx % 2 != 0 || p.nx < L::YX || p.ny < L::YY || reinterpret_cast<uintptr_t>(p.out) % 16 != 0) {
    return GC_ERR_UNSUPPORTED;
  }
  CUtensorMap mpsi{}, mkin{};
  if (!make_tensor_map_2d(&mpsi, p.psi, p.nx, p.ny, 8, L::YX, L::YY)) return GC_ERR_UNSUPPORTED;
  if (KIN && !make_tensor_map_2d(&mkin, p.kin, p.nx, p.ny, 8, L::YX, L::YY)) return GC_ERR_UNSUPPORTED;
  auto kern = ch_tma_x2_kernel<ORDER, MODE, KIN>;
  int ctas_per_sm = 1;
  GC_TRY(kernel_setup(kern, kX2DT * L::NTY, L::BYTES, &ctas_per_sm));
  const int tiles_x = div_up(p.nx, L::TX), tiles_y = div_up(p.ny, L::TY);
  const long long ntiles = static_cast<long long>(tiles_x) * tiles_y;
  const long long slots = static_cast<long long>(ctas_per_sm) * ctx->num_sms;
  // The two-column tiles hold 4x (order 2) or 2x (order 4) the cells of the
  // one-column kernel's: with fewer than ten rounds of them per persistent
  // CTA, idle SMs and the partly filled last round cost more than the two
  // columns save (measured on B200, RK4 per step at order 2: 512^2 31 vs 24 us,
  // 3072^2 273 vs 240 us, 4096^2 424 vs 430 us, 8192^2 1.54 vs 1.70 ms; order 4:
  // 2048^2 equal, 3072^2 370 vs 389 us).
  if (ntiles < kX2MinRounds * slots) return GC_ERR_UNSUPPORTED;
  const int grid = static_cast<int>(std::min<long long>(ntiles, slots));
  kern<<<grid, dim3(kX2DT, L::NTY), L::BYTES, ctx->stream>>>(p, mpsi, mkin, tiles_x, tiles_y, ctx->device_status);
  GC_CHECK_LAUNCH("ch_tma_x2_kernel");
  return GC_OK;
}

// Single-grid work source for the cp.async-pipelined persistent loop.
template <class T>
struct GridSource {
  StageParams<T> p;
  int tiles_x, n_tiles, tile_w, tile_h;
  __device__ int count() const { return n_tiles; }
  __device__ void get(int k, StageParams<T>& q, int& x0, int& y0) const {
    q = p;
    x0 = (k % tiles_x) * tile_w;
    y0 = (k / tiles_x) * tile_h;
  }
};

template <class T, int ORDER, int MODE>
__global__ void __launch_bounds__(kT2W * kT2TY) ch_pipe_kernel(const StageParams<T> p, int tiles_x, int n_tiles) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int TX = kT2W - 2 * W<2, ORDER>::R;
  const GridSource<T> src{p, tiles_x, n_tiles, TX, kT2Y};
  pipelined_tiles<T, ORDER, MODE, kT2W, kT2Y, kT2TY>(src, smem_raw);
}

template <class T, int ORDER, int MODE>
gc_status launch_pipe(gc_context* ctx, const StageParams<T>& p) {
  constexpr int TX = kT2W - 2 * W<2, ORDER>::R;
  constexpr size_t smem = pipe_smem<T, ORDER, kT2W, kT2Y>();
  auto kern = ch_pipe_kernel<T, ORDER, MODE>;
  int per_sm = 1;
  GC_TRY(kernel_setup(kern, kT2W * kT2TY, smem, &per_sm));
  const int tiles_x = div_up(p.nx, TX), tiles_y = div_up(p.ny, kT2Y);
  const int n_tiles = tiles_x * tiles_y;
  const int grid = std::max(1, std::min(n_tiles, per_sm * ctx->num_sms));
  kern<<<grid, dim3(kT2W, kT2TY), smem, ctx->stream>>>(p, tiles_x, n_tiles);
  GC_CHECK_LAUNCH("ch_pipe_kernel");
  return GC_OK;
}

// Two-column float variant (even grid widths): 64 x 4 threads over a
// 128-column mu region.
constexpr int kX2T = 64;

template <int ORDER, int MODE>
__global__ void __launch_bounds__(kX2T * kT2TY) ch_pipe_x2_kernel(const StageParams<float> p, int tiles_x,
                                                                  int n_tiles) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int TX = 2 * kX2T - 2 * W<2, ORDER>::R;
  const GridSource<float> src{p, tiles_x, n_tiles, TX, kT2Y};
  pipelined_tiles_x2<ORDER, MODE, kX2T, kT2Y, kT2TY>(src, smem_raw);
}

template <int ORDER, int MODE>
gc_status launch_pipe_x2(gc_context* ctx, const StageParams<float>& p) {
  constexpr int TX = 2 * kX2T - 2 * W<2, ORDER>::R;
  constexpr size_t smem = pipe_smem_x2<ORDER, kX2T, kT2Y>();
  auto kern = ch_pipe_x2_kernel<ORDER, MODE>;
  int per_sm = 1;
  GC_TRY(kernel_setup(kern, kX2T * kT2TY, smem, &per_sm));
  const int tiles_x = div_up(p.nx, TX), tiles_y = div_up(p.ny, kT2Y);
  const int n_tiles = tiles_x * tiles_y;
  const int grid = std::max(1, std::min(n_tiles, per_sm * ctx->num_sms));
  kern<<<grid, dim3(kX2T, kT2TY), smem, ctx->stream>>>(p, tiles_x, n_tiles);
  GC_CHECK_LAUNCH("ch_pipe_x2_kernel");
  return GC_OK;
}

// 2-D dispatch: TMA pipeline for double when its rules hold, the
// cp.async-pipelined persistent loop otherwise (two columns per thread for
// float on even widths).
template <class T, int ORDER, int MODE>
gc_status launch_2d(gc_context* ctx, const StageParams<T>& p) {
  if constexpr (sizeof(T) == 8 && (MODE == MODE_RHS || MODE == MODE_EULER_FINAL)) {
    gc_status s = GC_ERR_UNSUPPORTED;
    if constexpr (ORDER != 6) {  // order 6: 118 registers in two columns, slower than one
      if (!p.kin) {
        s = launch_tma_x2<ORDER, MODE, false>(ctx, p);
      } else if constexpr (MODE == MODE_RHS) {
        s = launch_tma_x2<ORDER, MODE, true>(ctx, p);
      }
    }
    if (s != GC_ERR_UNSUPPORTED) return s;
  }
  if constexpr (sizeof(T) == 8 && MODE != MODE_RKC_FIRST && MODE != MODE_RKC) {
    gc_status s;
    if constexpr (MODE == MODE_RHS) {
      s = p.kin ? launch_tma<T, ORDER, MODE, true>(ctx, p) : launch_tma<T, ORDER, MODE, false>(ctx, p);
    } else if constexpr (MODE == MODE_RK4_FINAL) {
      s = launch_tma<T, ORDER, MODE, true>(ctx, p);
    } else {
      s = launch_tma<T, ORDER, MODE, false>(ctx, p);
    }
    if (s != GC_ERR_UNSUPPORTED) return s;
  }
  if constexpr (sizeof(T) == 4) {
    if (p.nx % 2 == 0) return launch_pipe_x2<ORDER, MODE>(ctx, p);
  }
  return launch_pipe<T, ORDER, MODE>(ctx, p);
}

template <class T, int MODE>
gc_status launch_mode(gc_context* ctx, int order, const StageParams<T>& p) {
  const bool z3 = p.nz > 1;
  switch (order) {
    case 2: return z3 ? launch_stage<T, 2, true, MODE>(ctx, p) : launch_2d<T, 2, MODE>(ctx, p);
    case 4: return z3 ? launch_stage<T, 4, true, MODE>(ctx, p) : launch_2d<T, 4, MODE>(ctx, p);
    case 6: return z3 ? launch_stage<T, 6, true, MODE>(ctx, p) : launch_2d<T, 6, MODE>(ctx, p);
  }
  return fail(GC_ERR_UNSUPPORTED, "gridcalc_b200: Cahn-Hilliard order must be 2, 4 or 6");
}

template <class T>
StageParams<T> base_params(const gc_grid* g, const gc_ch_params* cp) {
  StageParams<T> p{};
  p.nx = g->nx; p.ny = g->ny; p.nz = g->nz;
  p.ihx2 = static_cast<T>(1.0 / (g->hx * g->hx));
  p.ihy2 = static_cast<T>(1.0 / (g->hy * g->hy));
  p.ihz2 = static_cast<T>(1.0 / (g->hz * g->hz));
  p.mob = static_cast<T>(cp->mobility);
  p.kappa = static_cast<T>(cp->kappa);
  p.unit_h = p.ihx2 == T(1) && p.ihy2 == T(1) && p.ihz2 == T(1);
  p.unit_m = p.mob == T(1);
  p.unit_k = p.kappa == T(1);
  return p;
}

// Enqueues one time step from `src` into `dst` (src != dst).
template <class T>
gc_status enqueue_step(gc_context* ctx, const gc_grid* g, const gc_ch_params* cp, const T* src,
                       T* dst, T* k1, T* k2, T* k3, double dt, gc_integrator integ) {
  if (integ == GC_RK4 && ctx->fused_step) {
    bool done = false;
    if constexpr (sizeof(T) == 8) GC_TRY(ch_fused_step(ctx, g, cp, src, dst, dt, &done));
    else GC_TRY(ch_fused_step_f32(ctx, g, cp, src, dst, dt, &done));
    if (done) return GC_OK;
  }
  StageParams<T> p = base_params<T>(g, cp);
  p.psi = src;
  const int order = cp->order;
  gc_status s;
  if (integ == GC_EXPLICIT_EULER) {
    p.kin = nullptr;
    p.out = dst;
    p.c6 = static_cast<T>(dt);
    return launch_mode<T, MODE_EULER_FINAL>(ctx, order, p);
  }
  const double half_dt = 0.5 * dt, sixth_dt = dt / 6.0, third_dt = dt / 3.0;
  p.kin = nullptr; p.out = k1;
  if ((s = launch_mode<T, MODE_RHS>(ctx, order, p)) != GC_OK) return s;
  p.kin = k1; p.a = static_cast<T>(half_dt); p.out = k2;
  if ((s = launch_mode<T, MODE_RHS>(ctx, order, p)) != GC_OK) return s;
  p.kin = k2; p.a = static_cast<T>(half_dt); p.out = k3;
  if ((s = launch_mode<T, MODE_RHS>(ctx, order, p)) != GC_OK) return s;
  p.kin = k3; p.a = static_cast<T>(dt); p.out = dst;
  p.k1 = k1; p.k2 = k2; p.k3 = k3;
  p.c6 = static_cast<T>(sixth_dt); p.c3 = static_cast<T>(third_dt);
  return launch_mode<T, MODE_RK4_FINAL>(ctx, order, p);
}

template <class T>
gc_status integrate_t(gc_context* ctx, const gc_grid* g, const gc_ch_params* cp, T* psi,
                      double dt, int n_steps, gc_integrator integ) {
  if (ctx->cluster_stepping && g->nz == 1) {
    bool done = false;
    GC_TRY(ch_cluster_integrate(ctx, g, sizeof(T) == 8 ? GC_F64 : GC_F32, cp, psi, dt, n_steps, integ, &done));
    if (done) return GC_OK;
  }
  const size_t n = cells(g);
  const size_t bytes = n * sizeof(T);
  void *vb = nullptr, *v1 = nullptr, *v2 = nullptr, *v3 = nullptr;
  gc_status s;
  if ((s = scratch_get(ctx, kSlotPsiB, bytes, &vb)) != GC_OK) return s;
  if (integ == GC_RK4) {
    if ((s = scratch_get(ctx, kSlotK1, bytes, &v1)) != GC_OK) return s;
    if ((s = scratch_get(ctx, kSlotK2, bytes, &v2)) != GC_OK) return s;
    if ((s = scratch_get(ctx, kSlotK3, bytes, &v3)) != GC_OK) return s;
  }
  T* pb = static_cast<T*>(vb);
  T *k1 = static_cast<T*>(v1), *k2 = static_cast<T*>(v2), *k3 = static_cast<T*>(v3);
  const uint64_t key[8] = {reinterpret_cast<uint64_t>(psi) ^ 0x1ULL,
                           reinterpret_cast<uint64_t>(pb),
                           reinterpret_cast<uint64_t>(k1) ^ (reinterpret_cast<uint64_t>(k3) << 1),
                           (static_cast<uint64_t>(g->nx) << 40) ^ (static_cast<uint64_t>(g->ny) << 20) ^
                               static_cast<uint64_t>(g->nz) ^ (bits_of(g->hx) * 3) ^ (bits_of(g->hy) * 5) ^
                               (bits_of(g->hz) * 7),
                           bits_of(dt),
                           bits_of(cp->mobility),
                           bits_of(cp->kappa),
                           (static_cast<uint64_t>(cp->order) << 8) | (static_cast<uint64_t>(integ) << 4) |
                               (sizeof(T) == 8 ? 1u : 2u) | (ctx->fused_step ? 1ULL << 16 : 0) | (0xC4ULL << 56)};
  return run_steps<T>(ctx, psi, pb, bytes, n_steps, key, [&](const T* src, T* dst) {
    return enqueue_step<T>(ctx, g, cp, src, dst, k1, k2, k3, dt, integ);
  });
}

// ---------------------------------------------------------------------------
// RKC2: the damped second-order Runge-Kutta-Chebyshev method (Sommeijer,
// Shampine & Verwer, "RKC: an explicit solver for parabolic PDEs", 1998;
// Hundsdorfer & Verwer, 2003, ch. V.1), damping eps = 2/13.  With
// w0 = 1 + eps/s^2 and Chebyshev polynomials T_j (and derivatives) at w0:
//   w1 = T_s'/T_s'', b_j = T_j''/T_j'^2 (j >= 2), b_0 = b_1 = b_2,
//   a_j = 1 - b_j T_j;
//   Y1 = Y0 + mu~1 dt F0,                                   mu~1 = b1 w1
//   Yj = (1 - mu_j - nu_j) Y0 + mu_j Y_{j-1} + nu_j Y_{j-2}
//        + mu~_j dt F(Y_{j-1}) + gamma~_j dt F0,
//   mu_j = 2 b_j w0 / b_{j-1}, nu_j = -b_j / b_{j-2},
//   mu~_j = 2 b_j w1 / b_{j-1}, gamma~_j = -a_{j-1} mu~_j;   y' = Y_s.
// All coefficients come from three-term recurrences (no transcendental
// calls).  Real stability interval [-beta, 0], beta = (w0 + 1) T_s''/T_s'
// (about 0.65 s^2): s stages reach s^2 / 4 times the RK4 step limit.
struct RkcCoeffs {
  int s = 0;
  double mt1 = 0.0;                       // mu~_1
  double mu[65], nu[65], mt[65], gt[65];  // j = 2..s
  double beta = 0.0;
};

RkcCoeffs rkc_coeffs(int s) {
  RkcCoeffs c;
  c.s = s;
  const double eps = 2.0 / 13.0;
  const double w0 = 1.0 + eps / (static_cast<double>(s) * s);
  double T[65], d1[65], d2[65];
  T[0] = 1.0; T[1] = w0;
  d1[0] = 0.0; d1[1] = 1.0;
  d2[0] = 0.0; d2[1] = 0.0;
  for (int j = 2; j <= s; ++j) {
    T[j] = 2.0 * w0 * T[j - 1] - T[j - 2];
    d1[j] = 2.0 * T[j - 1] + 2.0 * w0 * d1[j - 1] - d1[j - 2];
    d2[j] = 4.0 * d1[j - 1] + 2.0 * w0 * d2[j - 1] - d2[j - 2];
  }
  const double w1 = d1[s] / d2[s];
  double b[65], a[65];
  for (int j = 2; j <= s; ++j) b[j] = d2[j] / (d1[j] * d1[j]);
  b[0] = b[1] = b[2];
  for (int j = 0; j <= s; ++j) a[j] = 1.0 - b[j] * T[j];
  c.mt1 = b[1] * w1;
  for (int j = 2; j <= s; ++j) {
    c.mu[j] = 2.0 * b[j] * w0 / b[j - 1];
    c.nu[j] = -b[j] / b[j - 2];
    c.mt[j] = 2.0 * b[j] * w1 / b[j - 1];
    c.gt[j] = -a[j - 1] * c.mt[j];
  }
  c.beta = (w0 + 1.0) * d2[s] / d1[s];
  return c;
}

// One RKC2 step of psi in place.  Scratch: F0 and three rotating stage
// buffers; the last stage writes psi (it reads Y0 only at its own cell).
template <class T>
gc_status rkc_step(gc_context* ctx, const gc_grid* g, const gc_ch_params* cp, T* psi, double dt, const RkcCoeffs& c,
                   T* f0, T* const (&yb)[3]) {
  StageParams<T> p = base_params<T>(g, cp);
  const int order = cp->order;
  p.psi = psi;
  p.kin = nullptr;
  p.out = f0;
  p.out2 = yb[0];
  p.r[0] = static_cast<T>(c.mt1 * dt);
  GC_TRY((launch_mode<T, MODE_RKC_FIRST>(ctx, order, p)));
  const T* ym2 = psi;    // Y_{j-2}
  const T* ym1 = yb[0];  // Y_{j-1}
  for (int j = 2; j <= c.s; ++j) {
    T* out = j == c.s ? psi : yb[(j - 1) % 3];
    p.psi = ym1;
    p.out = out;
    p.k1 = psi;
    p.k2 = ym2;
    p.k3 = f0;
    p.r[0] = static_cast<T>(1.0 - c.mu[j] - c.nu[j]);
    p.r[1] = static_cast<T>(c.mu[j]);
    p.r[2] = static_cast<T>(c.nu[j]);
    p.r[3] = static_cast<T>(c.mt[j] * dt);
    p.r[4] = static_cast<T>(c.gt[j] * dt);
    GC_TRY((launch_mode<T, MODE_RKC>(ctx, order, p)));
    ym2 = ym1;
    ym1 = out;
  }
  return GC_OK;
}

template <class T>
gc_status rhs_t(gc_context* ctx, const gc_grid* g, const gc_ch_params* cp, const T* psi, T* out) {
  StageParams<T> p = base_params<T>(g, cp);
  p.psi = psi;
  p.out = out;
  return launch_mode<T, MODE_RHS>(ctx, cp->order, p);
}

template <class T>
gc_status rkc_t(gc_context* ctx, const gc_grid* g, const gc_ch_params* cp, T* psi, double dt, int n_steps,
                int stages) {
  const size_t bytes = cells(g) * sizeof(T);
  void *vf = nullptr, *va = nullptr, *vb = nullptr, *vc = nullptr;
  GC_TRY(scratch_get(ctx, kSlotK1, bytes, &vf));
  GC_TRY(scratch_get(ctx, kSlotK2, bytes, &va));
  GC_TRY(scratch_get(ctx, kSlotK3, bytes, &vb));
  GC_TRY(scratch_get(ctx, kSlotPsiB, bytes, &vc));
  T* const yb[3] = {static_cast<T*>(va), static_cast<T*>(vb), static_cast<T*>(vc)};
  const RkcCoeffs c = rkc_coeffs(stages);
  for (int k = 0; k < n_steps; ++k) GC_TRY(rkc_step<T>(ctx, g, cp, psi, dt, c, static_cast<T*>(vf), yb));
  return GC_OK;
}

}  // namespace

gc_status ch_rhs_enqueue(gc_context* ctx, const gc_grid* g, gc_dtype dt, const gc_ch_params* cp, const void* psi,
                         void* out) {
  if (dt == GC_F64) return rhs_t<double>(ctx, g, cp, static_cast<const double*>(psi), static_cast<double*>(out));
  return rhs_t<float>(ctx, g, cp, static_cast<const float*>(psi), static_cast<float*>(out));
}

gc_status ch_rkc_enqueue(gc_context* ctx, const gc_grid* g, gc_dtype dt, const gc_ch_params* cp, void* psi,
                         double dt_step, int stages, void* const (&scratch)[4]) {
  const RkcCoeffs c = rkc_coeffs(stages);
  if (dt == GC_F64) {
    double* const yb[3] = {static_cast<double*>(scratch[1]), static_cast<double*>(scratch[2]),
                           static_cast<double*>(scratch[3])};
    return rkc_step<double>(ctx, g, cp, static_cast<double*>(psi), dt_step, c, static_cast<double*>(scratch[0]), yb);
  }
  float* const yb[3] = {static_cast<float*>(scratch[1]), static_cast<float*>(scratch[2]),
                        static_cast<float*>(scratch[3])};
  return rkc_step<float>(ctx, g, cp, static_cast<float*>(psi), dt_step, c, static_cast<float*>(scratch[0]), yb);
}

namespace {

gc_status check_ch(gc_context* ctx, const gc_grid* g, gc_dtype dt, const gc_ch_params* cp) {
  Call call(ctx);
  gc_status s = call.st;
  if (s != GC_OK) return s;
  if ((s = check_grid(g)) != GC_OK) return s;
  if (!cp) return fail(GC_ERR_INVALID_ARG, "gridcalc_b200: null Cahn-Hilliard parameters");
  if (cp->order != 2 && cp->order != 4 && cp->order != 6)
    return fail(GC_ERR_UNSUPPORTED, "gridcalc_b200: Cahn-Hilliard order must be 2, 4 or 6; got " +
                                        std::to_string(cp->order));
  if (dt != GC_F64 && dt != GC_F32) return fail(GC_ERR_INVALID_ARG, "gridcalc_b200: unknown dtype");
  return GC_OK;
}

}  // namespace
}  // namespace gcb

using namespace gcb;

extern "C" {

GC_API gc_status gc_ch_rhs(gc_context* ctx, const gc_grid* g, gc_dtype dt, const gc_ch_params* cp,
                           const void* psi, void* out) {
  Call call(ctx);
  if (call.st != GC_OK) return call.st;
  gc_status s = check_ch(ctx, g, dt, cp);
  if (s != GC_OK) return s;
  if ((s = require_axes(g, cp->order / 2)) != GC_OK) return s;
  if (!psi || !out) return fail(GC_ERR_INVALID_ARG, "gc_ch_rhs: null field pointer");
  return ch_rhs_enqueue(ctx, g, dt, cp, psi, out);
}

GC_API gc_status gc_ch_integrate(gc_context* ctx, const gc_grid* g, gc_dtype dt,
                                 const gc_ch_params* cp, void* psi, double dt_step, int n_steps,
                                 gc_integrator integ) {
  NvtxScope nvtx("gc_ch_integrate");
  Call call(ctx);
  if (call.st != GC_OK) return call.st;
  gc_status s = check_ch(ctx, g, dt, cp);
  if (s != GC_OK) return s;
  const char* who = integ == GC_RK4 ? "solve::integrate(... RK4)" : "solve::integrate(... ExplicitEuler)";
  if (integ != GC_RK4 && integ != GC_EXPLICIT_EULER)
    return fail(GC_ERR_INVALID_ARG, "gridcalc_b200: unknown integrator");
  if (n_steps < 0)
    return fail(GC_ERR_INVALID_ARG, std::string(who) + ": n_steps must be >= 0; got " + std::to_string(n_steps));
  if (dt_step < 0.0)
    return fail(GC_ERR_INVALID_ARG, std::string(who) + ": dt must be >= 0; got " + std::to_string(dt_step));
  if (n_steps == 0) return GC_OK;
  if ((s = require_axes(g, cp->order / 2)) != GC_OK) return s;
  if (!psi) return fail(GC_ERR_INVALID_ARG, "gc_ch_integrate: null psi");
  if (dt == GC_F64)
    return integrate_t<double>(ctx, g, cp, static_cast<double*>(psi), dt_step, n_steps, integ);
  return integrate_t<float>(ctx, g, cp, static_cast<float*>(psi), dt_step, n_steps, integ);
}

GC_API gc_status gc_ch_rkc(gc_context* ctx, const gc_grid* g, gc_dtype dt, const gc_ch_params* cp, void* psi,
                           double dt_step, int32_t n_steps, int32_t stages) {
  Call call(ctx);
  if (call.st != GC_OK) return call.st;
  gc_status s = check_ch(ctx, g, dt, cp);
  if (s != GC_OK) return s;
  if (n_steps < 0 || !(dt_step >= 0.0))
    return fail(GC_ERR_INVALID_ARG, "gc_ch_rkc: n_steps and dt must be >= 0");
  if (stages < 2 || stages > 64) return fail(GC_ERR_INVALID_ARG, "gc_ch_rkc: stages must be in [2, 64]");
  if (n_steps == 0) return GC_OK;
  if ((s = require_axes(g, cp->order / 2)) != GC_OK) return s;
  if (!psi) return fail(GC_ERR_INVALID_ARG, "gc_ch_rkc: null psi");
  if (dt == GC_F64) return rkc_t<double>(ctx, g, cp, static_cast<double*>(psi), dt_step, n_steps, stages);
  return rkc_t<float>(ctx, g, cp, static_cast<float*>(psi), dt_step, n_steps, stages);
}

GC_API double gc_rkc_stability_bound(int32_t stages) {
  if (stages < 2 || stages > 64) return 0.0;
  return rkc_coeffs(stages).beta;
}

}  // extern "C"
