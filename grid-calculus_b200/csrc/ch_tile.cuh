// Cahn-Hilliard stage building blocks shared by the single-grid drivers
// (ch.cu) and the batched ensemble (ch_batch.cu): stage parameters, the
// reference-ordered RHS arithmetic, the 2-D strip-tile geometry and the
// cp.async-pipelined persistent tile loop.
#pragma once

#include "common.cuh"

namespace gcb {
namespace {

// MODE_RKC_FIRST: out = f(psi), out2 = psi + r[0] f(psi)    (stage 1 of RKC2)
// MODE_RKC:       out = r[0] Y0 + r[1] y + r[2] Yjm2 + r[3] f(y) + r[4] F0
//                 with Y0 = k1, Yjm2 = k2, F0 = k3, summed left to right
enum StageMode { MODE_RHS = 0, MODE_RK4_FINAL = 1, MODE_EULER_FINAL = 2, MODE_RKC_FIRST = 3, MODE_RKC = 4 };

template <class T>
struct StageParams {
  const T* psi;    // state
  const T* kin;    // previous stage (y = psi + a kin), nullptr for y = psi
  T a;             // stage coefficient
  T* out;          // k_s (MODE_RHS) or psi' (final modes)
  const T* k1;     // MODE_RK4_FINAL only
  const T* k2;
  const T* k3;
  T c6, c3;        // dt/6, dt/3 (RK4 final) ; c6 = dt (Euler final)
  T* out2;         // MODE_RKC_FIRST second output
  T r[5];          // RKC stage coefficients
  T mob, kappa;
  T ihx2, ihy2, ihz2;
  int nx, ny, nz;
  // Exact shortcuts: x * 1 == x, so a unit spacing, mobility or kappa
  // skips its multiply without changing a bit.
  bool unit_h, unit_m, unit_k;
};

// (ax / hx^2 + ay / hy^2) [+ az / hz^2], as the reference combines the axes.
template <class T>
__device__ __forceinline__ T lap_xy(const StageParams<T>& p, T ax, T ay) {
  return p.unit_h ? Ar<T>::add(ax, ay) : Ar<T>::add(Ar<T>::mul(ax, p.ihx2), Ar<T>::mul(ay, p.ihy2));
}
template <class T>
__device__ __forceinline__ T lap_z(const StageParams<T>& p, T lap, T az) {
  return Ar<T>::add(lap, p.unit_h ? az : Ar<T>::mul(az, p.ihz2));
}
// mu = -y + y^3 - kappa lap(y)
template <class T>
__device__ __forceinline__ T chem_pot(const StageParams<T>& p, T y, T lap) {
  return Ar<T>::sub(Ar<T>::add(-y, Ar<T>::mul(Ar<T>::mul(y, y), y)), p.unit_k ? lap : Ar<T>::mul(p.kappa, lap));
}
template <class T>
__device__ __forceinline__ T mobility(const StageParams<T>& p, T lap) {
  return p.unit_m ? lap : Ar<T>::mul(lap, p.mob);
}

// r0 Y0 + r1 y + r2 Yjm2 + r3 f + r4 F0, products rounded and summed left to
// right (the order the RKC restatement in the tests uses).
template <class T>
__device__ __forceinline__ T rkc_combine(const StageParams<T>& p, T y0, T y, T yjm2, T f, T f0) {
  T acc = Ar<T>::mul(p.r[0], y0);
  acc = Ar<T>::add(acc, Ar<T>::mul(p.r[1], y));
  acc = Ar<T>::add(acc, Ar<T>::mul(p.r[2], yjm2));
  acc = Ar<T>::add(acc, Ar<T>::mul(p.r[3], f));
  return Ar<T>::add(acc, Ar<T>::mul(p.r[4], f0));
}

// ---------------------------------------------------------------------------
// 2-D strip-tile geometry (Nz == 1), used by the TMA kernel (ch.cu), the
// cp.async-pipelined loop below and the ensemble.  64 x 4 threads; the mu
// region is exactly 64 columns wide (output tile 64 - 2R columns by 16
// rows).  In the mu and output phases a thread owns one column and a strip
// of consecutive rows: y-direction taps come from a register window of its
// own column (one new shared-memory value per row), only the x taps are
// read from neighbouring columns -- in double precision every warp-wide
// shared read is two wavefronts, and this halves the shared-memory reads
// per cell that bounded a plain tiled layout.
constexpr int kT2W = 64;   // mu-region columns = threads in x
constexpr int kT2Y = 16;   // output rows
constexpr int kT2TY = 4;   // thread rows

// ---------------------------------------------------------------------------
// Software-pipelined persistent tile loop.  A CTA walks a list of work
// items (a grid tile, or a (member, tile) of an ensemble); before computing
// item k it issues cp.async copies of item k+1's y-region inputs (psi and
// k_prev, wrapped per element) into the other half of a double buffer, so
// global-memory latency overlaps the previous item's arithmetic.  Each
// thread forms y from exactly the elements it copied, so its own
// cp.async.wait_group suffices before that pass.  Arithmetic as strip_tile.
__device__ __forceinline__ void cp_async_elem(void* smem, const void* gmem, int bytes) {
  const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  if (bytes == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <class T, int ORDER, int TW, int TY>
constexpr size_t pipe_smem() {
  constexpr int R = W<2, ORDER>::R;
  constexpr size_t yn = static_cast<size_t>(TW + 2 * R) * (TY + 4 * R);
  return sizeof(T) * (4 * yn + yn + static_cast<size_t>(TW) * (TY + 2 * R));
}

// Source: get(k, p, x0, y0) fills the stage parameters and tile origin of
// item k; count() is the number of items.
template <class T, int ORDER, int MODE, int TW, int TY, int NTY, class Source>
__device__ __forceinline__ void pipelined_tiles(const Source& src, unsigned char* smem) {
  constexpr int R = W<2, ORDER>::R;
  constexpr int TX = TW - 2 * R;
  constexpr int YX = TX + 4 * R, YY = TY + 4 * R;
  constexpr int MX = TW, MY = TY + 2 * R;
  constexpr int NW = 2 * R + 1;
  constexpr int MS = (MY + NTY - 1) / NTY;
  constexpr int OS = (TY + NTY - 1) / NTY;
  constexpr int YN = YX * YY;
  T* raw = reinterpret_cast<T*>(smem);            // [2 buffers][psi, kin][YY][YX]
  T* ysb = raw + 4 * YN;                          // y region
  T* ms = ysb + YN;                               // mu region [MY][MX]
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int n_items = src.count();

  auto issue = [&](int k, int b) {
    StageParams<T> p;
    int x0, y0;
    src.get(k, p, x0, y0);
    T* rp = raw + (2 * b) * YN;
    T* rk = raw + (2 * b + 1) * YN;
    const int gxa = wrap(x0 - 2 * R + tx, p.nx);
    const bool has_b = tx < YX - TW;
    const int gxb = wrap(x0 - 2 * R + TW + tx, p.nx);
#pragma unroll
    for (int ry = ty; ry < YY; ry += NTY) {
      const size_t row = static_cast<size_t>(wrap(y0 - 2 * R + ry, p.ny)) * p.nx;
      cp_async_elem(rp + ry * YX + tx, p.psi + row + gxa, sizeof(T));
      if (p.kin) cp_async_elem(rk + ry * YX + tx, p.kin + row + gxa, sizeof(T));
      if (has_b) {
        cp_async_elem(rp + ry * YX + TW + tx, p.psi + row + gxb, sizeof(T));
        if (p.kin) cp_async_elem(rk + ry * YX + TW + tx, p.kin + row + gxb, sizeof(T));
      }
    }
    if constexpr (MODE == MODE_RK4_FINAL) {
      // k1, k2 at this thread's output cells of item k: into L2 now.
      if (tx < TX && x0 + tx < p.nx) {
#pragma unroll
        for (int q = 0; q < OS; ++q) {
          const int oy = ty * OS + q;
          if (oy < TY && y0 + oy < p.ny) {
            const size_t gi = static_cast<size_t>(y0 + oy) * p.nx + (x0 + tx);
            asm volatile("prefetch.global.L2 [%0];" ::"l"(p.k1 + gi));
            asm volatile("prefetch.global.L2 [%0];" ::"l"(p.k2 + gi));
          }
        }
      }
    }
  };

  if (blockIdx.x < n_items) issue(blockIdx.x, 0);
  cp_async_commit();
  int i = 0;
  for (int k = blockIdx.x; k < n_items; k += gridDim.x, ++i) {
    const int b = i & 1;
    if (k + static_cast<int>(gridDim.x) < n_items) issue(k + gridDim.x, b ^ 1);
    cp_async_commit();
    cp_async_wait<1>();  // this item's copies (this thread's) have landed
    StageParams<T> p;
    int x0, y0;
    src.get(k, p, x0, y0);
    const T* rp = raw + (2 * b) * YN;
    const T* rk = raw + (2 * b + 1) * YN;
    const T* ys = rp;
    if (p.kin) {
      const bool has_b = tx < YX - TW;
#pragma unroll
      for (int ry = ty; ry < YY; ry += NTY) {
        const int e = ry * YX + tx;
        ysb[e] = Ar<T>::add(rp[e], Ar<T>::mul(p.a, rk[e]));
        if (has_b) ysb[e + TW] = Ar<T>::add(rp[e + TW], Ar<T>::mul(p.a, rk[e + TW]));
      }
      ys = ysb;
    }
    __syncthreads();

    // Phase 2: mu.
    {
      const int m0 = ty * MS;
      const int m1 = min(m0 + MS, MY);
      const int cx = tx + R;
      T win[NW];
      if (m0 < MY) {
#pragma unroll
        for (int q = 0; q < 2 * R; ++q) win[q + 1] = ys[(m0 + q) * YX + cx];
      }
#pragma unroll
      for (int q = 0; q < MS; ++q) {
        const int m = m0 + q;
        if (m < m1) {
#pragma unroll
          for (int z = 0; z + 1 < NW; ++z) win[z] = win[z + 1];
          win[NW - 1] = ys[(m + 2 * R) * YX + cx];
          const T yc = win[R];
          const T ax = tap_sum<T, 2, ORDER>([&](int o) { return o == 0 ? yc : ys[(m + R) * YX + cx + o]; });
          const T ay = tap_sum<T, 2, ORDER>([&](int o) { return win[R + o]; });
          T lap = lap_xy(p, ax, ay);
          if constexpr (ORDER != 2) lap = lap_z(p, lap, tap_sum<T, 2, ORDER>([&](int) { return yc; }));
          ms[m * MX + tx] = chem_pot(p, yc, lap);
        }
      }
    }
    __syncthreads();

    // Phase 3: output strip.
    const int o0 = ty * OS;
    if (tx < TX && x0 + tx < p.nx && o0 < TY) {
      const int cx = tx + R;
      T win[NW];
#pragma unroll
      for (int q = 0; q < 2 * R; ++q) win[q + 1] = ms[(o0 + q) * MX + cx];
#pragma unroll
      for (int q = 0; q < OS; ++q) {
        const int oy = o0 + q;
        if (oy >= TY) break;
#pragma unroll
        for (int z = 0; z + 1 < NW; ++z) win[z] = win[z + 1];
        win[NW - 1] = ms[(oy + 2 * R) * MX + cx];
        if (y0 + oy >= p.ny) break;
        const T mc = win[R];
        const T ax = tap_sum<T, 2, ORDER>([&](int o) { return o == 0 ? mc : ms[(oy + R) * MX + cx + o]; });
        const T ay = tap_sum<T, 2, ORDER>([&](int o) { return win[R + o]; });
        T lap = lap_xy(p, ax, ay);
        if constexpr (ORDER != 2) lap = lap_z(p, lap, tap_sum<T, 2, ORDER>([&](int) { return mc; }));
        const T rhs = mobility(p, lap);
        const size_t gi = static_cast<size_t>(y0 + oy) * p.nx + (x0 + tx);
        const int yc_idx = (oy + 2 * R) * YX + (tx + 2 * R);
        if constexpr (MODE == MODE_RHS) {
          p.out[gi] = rhs;
        } else if constexpr (MODE == MODE_RK4_FINAL) {
          const T s14 = Ar<T>::add(__ldg(p.k1 + gi), rhs);
          const T s23 = Ar<T>::add(__ldg(p.k2 + gi), rk[yc_idx]);
          p.out[gi] = Ar<T>::add(rp[yc_idx], Ar<T>::add(Ar<T>::mul(p.c6, s14), Ar<T>::mul(p.c3, s23)));
        } else if constexpr (MODE == MODE_RKC_FIRST) {
          p.out[gi] = rhs;
          p.out2[gi] = Ar<T>::add(ys[yc_idx], Ar<T>::mul(p.r[0], rhs));
        } else if constexpr (MODE == MODE_RKC) {
          p.out[gi] = rkc_combine(p, p.k1[gi], ys[yc_idx], p.k2[gi], rhs, p.k3[gi]);
        } else {
          p.out[gi] = Ar<T>::add(rp[yc_idx], Ar<T>::mul(p.c6, rhs));
        }
      }
    }
    __syncthreads();
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// Two-column variant of the pipelined tile loop for float on grids of even
// width.  A thread owns a pair of adjacent columns in every phase, so
// copies, shared-memory traffic, address arithmetic and global stores move
// 8 bytes per instruction -- the float loop above is bound by instruction
// issue, not by bandwidth.  TWT threads in x cover a mu region of 2 TWT
// columns.  Tile origins and grid widths are even, so a pair never
// straddles the periodic wrap.  y and mu rows are stored with a one-column
// shift when R is odd, so each thread's centre pair is 8-byte aligned.
template <int ORDER, int TWT, int TY>
constexpr size_t pipe_smem_x2() {
  constexpr int R = W<2, ORDER>::R;
  constexpr size_t YX = 2 * TWT + 2 * R, YY = TY + 4 * R;
  constexpr size_t YS = YX + 2, MY = TY + 2 * R, MS = 2 * TWT + 2;
  return sizeof(float) * (4 * YX * YY + YS * YY + MS * MY);
}

__device__ __forceinline__ void st_pair(float* p, float2 v, bool aligned) {
  if (aligned) {
    *reinterpret_cast<float2*>(p) = v;
  } else {
    p[0] = v.x;
    p[1] = v.y;
  }
}

template <int ORDER, int MODE, int TWT, int TY, int NTY, class Source>
__device__ __forceinline__ void pipelined_tiles_x2(const Source& src, unsigned char* smem) {
  using T = float;
  constexpr int R = W<2, ORDER>::R;
  constexpr int TW = 2 * TWT;           // mu-region columns
  constexpr int TX = TW - 2 * R;        // output columns
  constexpr int YX = TX + 4 * R;        // staged columns (even)
  constexpr int YY = TY + 4 * R;
  constexpr int MY = TY + 2 * R;
  constexpr int PAD = R & 1;
  constexpr int YS = YX + 2;            // padded row strides (even)
  constexpr int MSW = TW + 2;
  constexpr int RE = (R + 1) / 2 * 2;   // R rounded up to even: the x-tap span start
  constexpr int NSP = (2 * RE + 2) / 2; // float2 loads covering cb - RE .. cb + 1 + RE
  constexpr int NW = 2 * R + 1;
  constexpr int MSR = (MY + NTY - 1) / NTY;
  constexpr int OSR = (TY + NTY - 1) / NTY;
  constexpr int YN = YX * YY;
  T* raw = reinterpret_cast<T*>(smem);  // [2 buffers][psi, kin][YY][YX]
  T* ysb = raw + 4 * YN;                // [YY][YS], column c at c + PAD
  T* ms = ysb + YY * YS;                // [MY][MSW], column c at c + PAD
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int n_items = src.count();
  const bool has_b = tx < R;            // pairs TWT .. TWT + R - 1

  auto issue = [&](int k, int b) {
    StageParams<T> p;
    int x0, y0;
    src.get(k, p, x0, y0);
    T* rp = raw + (2 * b) * YN;
    T* rk = raw + (2 * b + 1) * YN;
    const int ga = wrap(x0 - 2 * R + 2 * tx, p.nx);
    const int gb = wrap(x0 - 2 * R + 2 * (TWT + tx), p.nx);
#pragma unroll
    for (int ry = ty; ry < YY; ry += NTY) {
      const size_t row = static_cast<size_t>(wrap(y0 - 2 * R + ry, p.ny)) * p.nx;
      cp_async_elem(rp + ry * YX + 2 * tx, p.psi + row + ga, 8);
      if (p.kin) cp_async_elem(rk + ry * YX + 2 * tx, p.kin + row + ga, 8);
      if (has_b) {
        cp_async_elem(rp + ry * YX + 2 * (TWT + tx), p.psi + row + gb, 8);
        if (p.kin) cp_async_elem(rk + ry * YX + 2 * (TWT + tx), p.kin + row + gb, 8);
      }
    }
    if constexpr (MODE == MODE_RK4_FINAL) {
      if (2 * tx < TX && x0 + 2 * tx < p.nx) {
#pragma unroll
        for (int q = 0; q < OSR; ++q) {
          const int oy = ty * OSR + q;
          if (oy < TY && y0 + oy < p.ny) {
            const size_t gi = static_cast<size_t>(y0 + oy) * p.nx + (x0 + 2 * tx);
            asm volatile("prefetch.global.L2 [%0];" ::"l"(p.k1 + gi));
            asm volatile("prefetch.global.L2 [%0];" ::"l"(p.k2 + gi));
          }
        }
      }
    }
  };

  // x taps around the pair (cb, cb + 1) of a row: sp[j] = row[cb - RE + j].
  auto span = [&](const T* row, int cb, T (&sp)[2 * NSP]) {
#pragma unroll
    for (int j = 0; j < NSP; ++j) {
      const float2 v = *reinterpret_cast<const float2*>(row + cb - RE + 2 * j);
      sp[2 * j] = v.x;
      sp[2 * j + 1] = v.y;
    }
  };

  if (blockIdx.x < n_items) issue(blockIdx.x, 0);
  cp_async_commit();
  int i = 0;
  for (int k = blockIdx.x; k < n_items; k += gridDim.x, ++i) {
    const int b = i & 1;
    if (k + static_cast<int>(gridDim.x) < n_items) issue(k + gridDim.x, b ^ 1);
    cp_async_commit();
    cp_async_wait<1>();  // this item's copies (this thread's) have landed
    StageParams<T> p;
    int x0, y0;
    src.get(k, p, x0, y0);
    const T* rp = raw + (2 * b) * YN;
    const T* rk = raw + (2 * b + 1) * YN;
    // Phase 1: y = psi + a k_prev into the padded layout (own pairs only).
#pragma unroll
    for (int ry = ty; ry < YY; ry += NTY) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (h == 1 && !has_b) break;
        const int c = 2 * (h == 0 ? tx : TWT + tx);
        float2 v = *reinterpret_cast<const float2*>(rp + ry * YX + c);
        if (p.kin) {
          const float2 w = *reinterpret_cast<const float2*>(rk + ry * YX + c);
          v.x = Ar<T>::add(v.x, Ar<T>::mul(p.a, w.x));
          v.y = Ar<T>::add(v.y, Ar<T>::mul(p.a, w.y));
        }
        st_pair(ysb + ry * YS + c + PAD, v, PAD == 0);
      }
    }
    __syncthreads();

    // Phase 2: mu on columns 2 tx, 2 tx + 1 of the mu region.
    {
      const int m0 = ty * MSR;
      const int m1 = min(m0 + MSR, MY);
      const int cb = 2 * tx + R + PAD;
      float2 win[NW];
      if (m0 < MY) {
#pragma unroll
        for (int q = 0; q < 2 * R; ++q) win[q + 1] = *reinterpret_cast<const float2*>(ysb + (m0 + q) * YS + cb);
      }
#pragma unroll
      for (int q = 0; q < MSR; ++q) {
        const int m = m0 + q;
        if (m < m1) {
#pragma unroll
          for (int z = 0; z + 1 < NW; ++z) win[z] = win[z + 1];
          win[NW - 1] = *reinterpret_cast<const float2*>(ysb + (m + 2 * R) * YS + cb);
          T sp[2 * NSP];
          span(ysb + (m + R) * YS, cb, sp);
          const T ya = win[R].x, yb = win[R].y;
          const T axa = tap_sum<T, 2, ORDER>([&](int o) { return o == 0 ? ya : sp[RE + o]; });
          const T axb = tap_sum<T, 2, ORDER>([&](int o) { return o == 0 ? yb : sp[RE + 1 + o]; });
          const T aya = tap_sum<T, 2, ORDER>([&](int o) { return win[R + o].x; });
          const T ayb = tap_sum<T, 2, ORDER>([&](int o) { return win[R + o].y; });
          T la = lap_xy(p, axa, aya), lb = lap_xy(p, axb, ayb);
          if constexpr (ORDER != 2) {
            la = lap_z(p, la, tap_sum<T, 2, ORDER>([&](int) { return ya; }));
            lb = lap_z(p, lb, tap_sum<T, 2, ORDER>([&](int) { return yb; }));
          }
          st_pair(ms + m * MSW + 2 * tx + PAD, make_float2(chem_pot(p, ya, la), chem_pot(p, yb, lb)), PAD == 0);
        }
      }
    }
    __syncthreads();

    // Phase 3: output pair (2 tx, 2 tx + 1) of each of this thread's rows.
    const int o0 = ty * OSR;
    if (2 * tx < TX && x0 + 2 * tx < p.nx && o0 < TY) {
      const int cb = 2 * tx + R + PAD;
      float2 win[NW];
#pragma unroll
      for (int q = 0; q < 2 * R; ++q) win[q + 1] = *reinterpret_cast<const float2*>(ms + (o0 + q) * MSW + cb);
#pragma unroll
      for (int q = 0; q < OSR; ++q) {
        const int oy = o0 + q;
        if (oy >= TY) break;
#pragma unroll
        for (int z = 0; z + 1 < NW; ++z) win[z] = win[z + 1];
        win[NW - 1] = *reinterpret_cast<const float2*>(ms + (oy + 2 * R) * MSW + cb);
        if (y0 + oy >= p.ny) break;
        T sp[2 * NSP];
        span(ms + (oy + R) * MSW, cb, sp);
        const T ma = win[R].x, mb = win[R].y;
        const T axa = tap_sum<T, 2, ORDER>([&](int o) { return o == 0 ? ma : sp[RE + o]; });
        const T axb = tap_sum<T, 2, ORDER>([&](int o) { return o == 0 ? mb : sp[RE + 1 + o]; });
        const T aya = tap_sum<T, 2, ORDER>([&](int o) { return win[R + o].x; });
        const T ayb = tap_sum<T, 2, ORDER>([&](int o) { return win[R + o].y; });
        T la = lap_xy(p, axa, aya), lb = lap_xy(p, axb, ayb);
        if constexpr (ORDER != 2) {
          la = lap_z(p, la, tap_sum<T, 2, ORDER>([&](int) { return ma; }));
          lb = lap_z(p, lb, tap_sum<T, 2, ORDER>([&](int) { return mb; }));
        }
        const float2 rhs = make_float2(mobility(p, la), mobility(p, lb));
        const size_t gi = static_cast<size_t>(y0 + oy) * p.nx + (x0 + 2 * tx);
        const int own = (oy + 2 * R) * YX + 2 * tx + 2 * R;  // own pair in the raw buffers (even)
        float2* out = reinterpret_cast<float2*>(p.out + gi);
        if constexpr (MODE == MODE_RHS) {
          *out = rhs;
        } else if constexpr (MODE == MODE_RK4_FINAL) {
          const float2 k1 = __ldg(reinterpret_cast<const float2*>(p.k1 + gi));
          const float2 k2 = __ldg(reinterpret_cast<const float2*>(p.k2 + gi));
          const float2 ps = *reinterpret_cast<const float2*>(rp + own);
          const float2 k3 = *reinterpret_cast<const float2*>(rk + own);
          *out = make_float2(
              Ar<T>::add(ps.x, Ar<T>::add(Ar<T>::mul(p.c6, Ar<T>::add(k1.x, rhs.x)),
                                          Ar<T>::mul(p.c3, Ar<T>::add(k2.x, k3.x)))),
              Ar<T>::add(ps.y, Ar<T>::add(Ar<T>::mul(p.c6, Ar<T>::add(k1.y, rhs.y)),
                                          Ar<T>::mul(p.c3, Ar<T>::add(k2.y, k3.y)))));
        } else if constexpr (MODE == MODE_RKC_FIRST) {
          const float2 ps = *reinterpret_cast<const float2*>(rp + own);
          *out = rhs;
          *reinterpret_cast<float2*>(p.out2 + gi) =
              make_float2(Ar<T>::add(ps.x, Ar<T>::mul(p.r[0], rhs.x)), Ar<T>::add(ps.y, Ar<T>::mul(p.r[0], rhs.y)));
        } else if constexpr (MODE == MODE_RKC) {
          const float2 ps = *reinterpret_cast<const float2*>(rp + own);
          const float2 y0v = *reinterpret_cast<const float2*>(p.k1 + gi);
          const float2 ym2 = *reinterpret_cast<const float2*>(p.k2 + gi);
          const float2 f0 = *reinterpret_cast<const float2*>(p.k3 + gi);
          *out = make_float2(rkc_combine(p, y0v.x, ps.x, ym2.x, rhs.x, f0.x),
                             rkc_combine(p, y0v.y, ps.y, ym2.y, rhs.y, f0.y));
        } else {
          const float2 ps = *reinterpret_cast<const float2*>(rp + own);
          *out = make_float2(Ar<T>::add(ps.x, Ar<T>::mul(p.c6, rhs.x)), Ar<T>::add(ps.y, Ar<T>::mul(p.c6, rhs.y)));
        }
      }
    }
    __syncthreads();
  }
  cp_async_wait<0>();
}

}  // namespace
}  // namespace gcb
