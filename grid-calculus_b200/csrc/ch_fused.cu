// Fused RK4 step for 2-D double Cahn-Hilliard at Laplacian order 2: all
// four stages of one step in one kernel, with psi read from and psi' written
// to HBM once.
//
// solve::integrate(psi, computeRhs, dt, n, RK4{}) (solve/RK4.hpp:99-154,
// examples/common/cahn_hilliard.hpp:38-59):
//   k1 = f(psi), k2 = f(psi + dt/2 k1), k3 = f(psi + dt/2 k2),
//   k4 = f(psi + dt k3), psi' = psi + (dt/6 (k1 + k4) + dt/3 (k2 + k3)),
//   f(y) = M lap(mu), mu = -y + y^3 - kappa lap(y).
// The stage kernels (ch.cu) move 13 field passes per step through HBM and
// are bound by it.  Here a persistent CTA owns a TX x TY output tile and
// stages psi on the tile plus a halo of H = 8R cells (R = 1, the stencil
// radius): each stage's f needs its input y on 2R more cells than it
// produces, so stage s produces k_s on a halo of H - 2R s and the last
// stage exactly the tile.  Per stage, in shared memory:
//   mu pass  mu = -y + y^3 - kappa lap(y) on halo H - 2R s + R
//            (y = psi in stage 1, else the y buffer)
//   k pass   k = M lap(mu) on halo H - 2R s; y of the next stage
//            (psi + dt/2 k, psi + dt/2 k, psi + dt k) overwrites the y
//            buffer; on the tile k1 is kept, k2 kept and then replaced by
//            k2 + k3, and stage 4 writes psi' to global memory.
// HBM traffic per step is psi once (the halo's overlap with neighbouring
// tiles comes from L2) and psi' once: 16 B per cell instead of 104.  The
// price is the halo's extra arithmetic (about 1.4x at 64 x 28 tiles): the
// kernel is bound by instruction issue (FP64 arithmetic and shared-memory
// accesses), not by HBM.  Every stage is its own template instance with
// compile-time regions, and each thread walks a column strip keeping three
// rows in registers, so a cell costs three shared-memory reads.
//
// Interior tiles arrive by one TMA box (x offset a multiple of 8 doubles);
// tiles touching the grid edge load their wrapped frame with plain loads.
// The next tile's box is prefetched into L2 while this one computes.  Every
// operation is the stage kernels' (tap_sum, lap_xy, chem_pot, mobility,
// the same RK4 combination), so results are bit-identical to them and to
// the CPU reference.  The single TMA wait is bounded: on expiry the CTA
// records GC_ERR_TIMEOUT in the context's status word and leaves.
#include <algorithm>

#include "ch_tile.cuh"
#include "common.cuh"
#include "tma.cuh"

namespace gcb {
namespace {

constexpr int kFzThreads = 512;
constexpr long long kFzWaitCycles = 4000000000LL;  // about 2 s at 2 GHz

constexpr size_t fz_al(size_t b) { return (b + 127) / 128 * 128; }

// Tile of TX_ x TY_ output cells: 64 x 28 (two CTAs per SM) for grids with
// enough tiles, 64 x 16 (three CTAs per SM, more tiles) for small grids,
// 32 x 16 for grids that 64 x 16 tiles would not spread over every SM and
// 32 x 8 where 32 x 16 tiles would fill under half of them.
template <int TY_, int TX_ = 64>
struct FzLayout {
  static constexpr int R = 1;
  static constexpr int H = 8 * R;         // four stages x 2R
  static constexpr int TX = TX_, TY = TY_;  // output tile
  static constexpr int CTAS_PER_SM = TY_ <= 16 ? 3 : 2;
  static constexpr int SX = TX + 2 * H;   // frame row (80 doubles = 640 B at TX = 64)
  static constexpr int SY = TY + 2 * H;   // frame rows
  static constexpr int YR0 = 2 * R;       // first frame row the y buffer holds (halo 6R)
  static constexpr int YROWS = SY - 2 * YR0;
  static constexpr int MR0 = R;           // first frame row the mu buffer holds (halo 7R)
  static constexpr int MROWS = SY - 2 * MR0;
  static constexpr size_t OFF_PSI = 128;  // after the mbarrier
  static constexpr size_t OFF_Y = OFF_PSI + fz_al(sizeof(double) * SX * SY);
  static constexpr size_t OFF_MU = OFF_Y + fz_al(sizeof(double) * SX * YROWS);
  static constexpr size_t OFF_K1 = OFF_MU + fz_al(sizeof(double) * SX * MROWS);
  static constexpr size_t OFF_K23 = OFF_K1 + fz_al(sizeof(double) * TX * TY);
  static constexpr size_t BYTES = OFF_K23 + fz_al(sizeof(double) * TX * TY) + 128;  // + alignment slack
  static constexpr uint32_t TX_BYTES = static_cast<uint32_t>(sizeof(double) * SX * SY);
};
static_assert(FzLayout<28>::BYTES <= 113 * 1024, "two CTAs per SM");
static_assert(FzLayout<16>::BYTES <= 74 * 1024 && FzLayout<16, 32>::BYTES <= 74 * 1024 &&
                  FzLayout<8, 32>::BYTES <= 74 * 1024,
              "three CTAs per SM");
static_assert((FzLayout<16, 32>::SX * 8) % 16 == 0 && FzLayout<16, 32>::TX % 8 == 0,
              "TMA box rows and x offsets stay 16-byte multiples");
static_assert((FzLayout<28>::SX * 8) % 16 == 0 && FzLayout<28>::H % 2 == 0,
              "TMA box rows and x offsets stay 16-byte multiples");

struct FzParams {
  StageParams<double> p;   // RHS constants, nx, ny
  const double* psi;       // state in
  double* out;             // state out (another buffer)
  double half_dt, dt, c6, c3;
  int tiles_x, tiles_y;
};

// The cells of a W x NR region (frame offset of its first cell: base) in
// column strips: thread t takes column t % W and rows [j RP, j RP + RP) of
// it, j = t / W < NS, with NS = 512 / W strips of RP = ceil(NR / NS) rows.
// f(off, rr, cc, k) for each of its cells in order down the column (k the
// cell's index within the strip, for the caller's register window).
template <int SX, int W, int NR, class F>
__device__ __forceinline__ void fz_strips(int base, F&& f) {
  constexpr int NS = kFzThreads / W;
  constexpr int RP = (NR + NS - 1) / NS;
  const int t = threadIdx.x, j = t / W, cc = t - j * W;
  if (j < NS) {
    const int r0 = j * RP;
    int off = base + r0 * SX + cc;
#pragma unroll
    for (int k = 0; k < RP; ++k) {
      if (RP * NS == NR || r0 + k < NR) f(off, r0 + k, cc, k);
      off += SX;
    }
  }
}

// One stage S (0..3) of the fused step on the tile at (x0, y0).  Regions and
// the stage's update are compile-time constants: the mu pass covers the
// tile plus hm = H - 2R S - R cells, the k pass the tile plus hk = hm - R.
// Each thread walks a column strip and keeps the centre column's three rows
// in registers, so a cell reads three values from shared memory (the new
// row below, the two x neighbours).  UNIT: unit spacing, mobility and kappa
// (the multiplies by 1 are skipped, as the stage kernels' exact shortcuts do).
template <int TYT, int TXT, int S, bool UNIT>
__device__ __forceinline__ void fz_stage(const FzParams& a, const double* __restrict__ ps, double* __restrict__ ys,
                                         double* __restrict__ ms, double* __restrict__ k1s,
                                         double* __restrict__ k23s, int x0, int y0) {
  using L = FzLayout<TYT, TXT>;
  using T = double;
  constexpr int R = L::R, H = L::H, TX = L::TX, TY = L::TY, SX = L::SX;
  constexpr int hy = H - 2 * R * S, hm = hy - R, hk = hm - R;
  constexpr int YOFF = L::YR0 * SX, MOFF = L::MR0 * SX;  // frame offset of each buffer's first row
  const StageParams<T>& p = a.p;

  // mu = -y + y^3 - kappa lap(y)
  {
    constexpr int W = TX + 2 * hm, NR = TY + 2 * hm, B = H - hm;
    const T* yb = S == 0 ? ps : ys - YOFF;  // indexed by frame offset (valid rows only)
    T w0 = 0.0, w1 = 0.0;
    fz_strips<SX, W, NR>(B * SX + B, [&](int off, int, int, int k) {
      if (k == 0) {
        w0 = yb[off - SX];
        w1 = yb[off];
      }
      const T w2 = yb[off + SX];
      const T yc = w1;
      const T ax = Ar<T>::add(Ar<T>::add(yb[off - 1], Ar<T>::mul(-2.0, yc)), yb[off + 1]);
      const T ay = Ar<T>::add(Ar<T>::add(w0, Ar<T>::mul(-2.0, yc)), w2);
      w0 = w1;
      w1 = w2;
      T mu;
      if constexpr (UNIT) {
        mu = Ar<T>::sub(Ar<T>::add(-yc, Ar<T>::mul(Ar<T>::mul(yc, yc), yc)), Ar<T>::add(ax, ay));
      } else {
        mu = chem_pot(p, yc, lap_xy(p, ax, ay));
      }
      ms[off - MOFF] = mu;
    });
  }
  __syncthreads();
  // k = M lap(mu), then the stage's update
  {
    constexpr int W = TX + 2 * hk, NR = TY + 2 * hk, B = H - hk;
    const T* mb = ms - MOFF;
    T w0 = 0.0, w1 = 0.0;
    fz_strips<SX, W, NR>(B * SX + B, [&](int off, int rr, int cc, int k) {
      if (k == 0) {
        w0 = mb[off - SX];
        w1 = mb[off];
      }
      const T w2 = mb[off + SX];
      const T mc = w1;
      const T ax = Ar<T>::add(Ar<T>::add(mb[off - 1], Ar<T>::mul(-2.0, mc)), mb[off + 1]);
      const T ay = Ar<T>::add(Ar<T>::add(w0, Ar<T>::mul(-2.0, mc)), w2);
      w0 = w1;
      w1 = w2;
      T rhs;
      if constexpr (UNIT) {
        rhs = Ar<T>::add(ax, ay);
      } else {
        rhs = mobility(p, lap_xy(p, ax, ay));
      }
      const T pc = ps[off];
      if constexpr (S < 3) {
        ys[off - YOFF] = Ar<T>::add(pc, Ar<T>::mul(S < 2 ? a.half_dt : a.dt, rhs));
        const int tr = rr - hk, tc = cc - hk;
        if (static_cast<unsigned>(tr) < static_cast<unsigned>(TY) && static_cast<unsigned>(tc) < static_cast<unsigned>(TX)) {
          const int t = tr * TX + tc;
          if constexpr (S == 0) k1s[t] = rhs;
          else if constexpr (S == 1) k23s[t] = rhs;
          else k23s[t] = Ar<T>::add(k23s[t], rhs);
        }
      } else {  // the region is the tile
        const int t = rr * TX + cc;
        if (y0 + rr < p.ny && x0 + cc < p.nx) {
          const T s14 = Ar<T>::add(k1s[t], rhs);
          a.out[static_cast<size_t>(y0 + rr) * p.nx + (x0 + cc)] =
              Ar<T>::add(pc, Ar<T>::add(Ar<T>::mul(a.c6, s14), Ar<T>::mul(a.c3, k23s[t])));
        }
      }
    });
  }
  __syncthreads();
}

template <int TYT, int TXT, bool UNIT>
__global__ void __launch_bounds__(kFzThreads, FzLayout<TYT, TXT>::CTAS_PER_SM)
    ch_fused_rk4_kernel(const FzParams a, const __grid_constant__ CUtensorMap m_psi, int* status) {
  using L = FzLayout<TYT, TXT>;
  using T = double;
  constexpr int H = L::H, TX = L::TX, TY = L::TY, SX = L::SX, SY = L::SY;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  uint64_t* bar = reinterpret_cast<uint64_t*>(base);
  int* s_abort = reinterpret_cast<int*>(base + 64);
  T* ps = reinterpret_cast<T*>(base + L::OFF_PSI);
  T* ys = reinterpret_cast<T*>(base + L::OFF_Y);
  T* ms = reinterpret_cast<T*>(base + L::OFF_MU);
  T* k1s = reinterpret_cast<T*>(base + L::OFF_K1);
  T* k23s = reinterpret_cast<T*>(base + L::OFF_K23);
  const int nx = a.p.nx, ny = a.p.ny, tid = threadIdx.x;
  const int ntiles = a.tiles_x * a.tiles_y;

  auto origin = [&](int tl, int& x0, int& y0) {
    x0 = (tl % a.tiles_x) * TX;
    y0 = (tl / a.tiles_x) * TY;
  };
  auto interior = [&](int x0, int y0) { return x0 - H >= 0 && x0 - H + SX <= nx && y0 - H >= 0 && y0 - H + SY <= ny; };
  if (tid == 0) {
    mbar_init(bar, 1);
    *s_abort = 0;
    mbar_init_fence();
  }
  __syncthreads();

  uint32_t phase = 0;
  for (int tl = blockIdx.x; tl < ntiles; tl += gridDim.x) {
    int x0, y0;
    origin(tl, x0, y0);
    const bool in = interior(x0, y0);
    if (tid == 0) {
      const int next = tl + static_cast<int>(gridDim.x);
      if (in) {
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(bar, L::TX_BYTES);
        tma_load_2d(ps, &m_psi, x0 - H, y0 - H, bar);
      }
      if (next < ntiles) {
        int nx0, ny0;
        origin(next, nx0, ny0);
        if (interior(nx0, ny0)) tma_prefetch_2d(&m_psi, nx0 - H, ny0 - H);
      }
    }
    if (in) {
      const long long t0 = clock64();
      while (!mbar_try_wait(bar, phase)) {
        if (clock64() - t0 > kFzWaitCycles) {
          *s_abort = 1;
          atomicExch(status, static_cast<int>(GC_ERR_TIMEOUT));
          break;
        }
      }
      phase ^= 1u;
    } else {
      for (int e = tid; e < SX * SY; e += kFzThreads) {
        const int r = e / SX, c = e - r * SX;
        ps[e] = __ldg(a.psi + static_cast<size_t>(wrap(y0 - H + r, ny)) * nx + wrap(x0 - H + c, nx));
      }
    }
    __syncthreads();
    if (*s_abort) break;
    fz_stage<TYT, TXT, 0, UNIT>(a, ps, ys, ms, k1s, k23s, x0, y0);
    fz_stage<TYT, TXT, 1, UNIT>(a, ps, ys, ms, k1s, k23s, x0, y0);
    fz_stage<TYT, TXT, 2, UNIT>(a, ps, ys, ms, k1s, k23s, x0, y0);
    fz_stage<TYT, TXT, 3, UNIT>(a, ps, ys, ms, k1s, k23s, x0, y0);
  }
}

}  // namespace

namespace {

template <int TYT, int TXT>
gc_status fz_launch(gc_context* ctx, const gc_grid* g, FzParams a, bool unit) {
  using L = FzLayout<TYT, TXT>;
  CUtensorMap m{};
  if (!make_tensor_map_2d(&m, a.psi, g->nx, g->ny, 8, L::SX, L::SY)) return GC_ERR_UNSUPPORTED;
  a.tiles_x = div_up(g->nx, L::TX);
  a.tiles_y = div_up(g->ny, L::TY);
  auto kern = unit ? ch_fused_rk4_kernel<TYT, TXT, true> : ch_fused_rk4_kernel<TYT, TXT, false>;
  int per_sm = 1;
  GC_TRY(kernel_setup(kern, kFzThreads, L::BYTES, &per_sm));
  const long long ntiles = static_cast<long long>(a.tiles_x) * a.tiles_y;
  const int grid = static_cast<int>(std::min<long long>(ntiles, static_cast<long long>(per_sm) * ctx->num_sms));
  kern<<<grid, kFzThreads, L::BYTES, ctx->stream>>>(a, m, ctx->device_status);
  GC_CHECK_LAUNCH("ch_fused_rk4_kernel");
  return GC_OK;
}

}  // namespace

gc_status ch_fused_step(gc_context* ctx, const gc_grid* g, const gc_ch_params* cp, const double* src, double* dst,
                        double dt, bool* done) {
  *done = false;
  if (g->nz != 1 || cp->order != 2 || g->nx < FzLayout<16, 32>::SX || g->ny < FzLayout<16, 32>::SY) return GC_OK;
  // Measured on B200 per RK4 step (fused with 64 x 28 tiles / fused with
  // 64 x 16 tiles / four stage kernels): 256^2 9.2 / 7.2 / 24.5 us, 512^2
  // 13.3 / 10.0 / 24.4, 1024^2 22.8 / 28.2 / 45.7, 4096^2 311 / 362 / 427,
  // 8192^2 1196 / 1415 / 1553.  The taller tiles halve the halo's share of
  // the work; the shorter ones make more tiles and fit three CTAs per SM,
  // which pays while 64 x 28 tiles would fill fewer than two rounds of the
  // persistent CTAs.  32 x 16 tiles, on grids that 64 x 16 tiles would not
  // spread over every SM: 128^2 6.8 -> 5.5 us, 256^2 7.1 -> 5.4 us; 32 x 8
  // tiles where 32 x 16 ones would fill under half the SMs: 128^2 5.5 ->
  // 4.5 us.
  FzParams a{};
  StageParams<double>& p = a.p;
  p.nx = g->nx; p.ny = g->ny; p.nz = 1;
  p.ihx2 = 1.0 / (g->hx * g->hx);
  p.ihy2 = 1.0 / (g->hy * g->hy);
  p.ihz2 = 1.0 / (g->hz * g->hz);
  p.mob = cp->mobility;
  p.kappa = cp->kappa;
  p.unit_h = p.ihx2 == 1.0 && p.ihy2 == 1.0 && p.ihz2 == 1.0;
  p.unit_m = p.mob == 1.0;
  p.unit_k = p.kappa == 1.0;
  a.psi = src;
  a.out = dst;
  a.half_dt = 0.5 * dt;
  a.dt = dt;
  a.c6 = dt / 6.0;
  a.c3 = dt / 3.0;
  const bool unit = p.unit_h && p.unit_m && p.unit_k;
  const long long tiles28 = static_cast<long long>(div_up(g->nx, 64)) * div_up(g->ny, 28);
  const long long tiles16 = static_cast<long long>(div_up(g->nx, 64)) * div_up(g->ny, 16);
  const bool tall = g->ny >= FzLayout<28>::SY && tiles28 >= 2LL * FzLayout<28>::CTAS_PER_SM * ctx->num_sms;
  const long long tiles16n = static_cast<long long>(div_up(g->nx, 32)) * div_up(g->ny, 16);
  const bool narrow = g->nx < FzLayout<16>::SX || tiles16 < ctx->num_sms;
  const bool flat = narrow && 2 * tiles16n < ctx->num_sms;  // 32 x 16 tiles would fill under half the SMs
  const gc_status s = tall     ? fz_launch<28, 64>(ctx, g, a, unit)
                      : flat   ? fz_launch<8, 32>(ctx, g, a, unit)
                      : narrow ? fz_launch<16, 32>(ctx, g, a, unit)
                               : fz_launch<16, 64>(ctx, g, a, unit);
  if (s == GC_ERR_UNSUPPORTED) return GC_OK;  // layout unfit for TMA: the stage kernels run
  if (s != GC_OK) return s;
  *done = true;
  return GC_OK;
}

}  // namespace gcb
