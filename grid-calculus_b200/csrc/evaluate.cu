// func::evaluate with a general integrand (func/Functional.hpp:88-148 for a
// scalar psi, :183-220 for a Vec3d field u).
//
// The reference materialises the derivative fields the callable's arity asks
// for (order-2 gradient, Laplacian, biharmonic; for a vector field the
// order-2 rank-2 gradient), evaluates the callable per cell into an integrand
// field and reduces it with func::integrate.  Here the callable arrives as a
// straight-line register program (gc_program), which is turned into CUDA
// source, compiled once per distinct program with NVRTC for sm_100a and
// cached: the integrand becomes a device functor inlined into the
// reduction.  One kernel walks the reduction's chunks, forms at every cell
// the derivatives of the arity from its neighbours (read through L1/L2; one
// HBM read per value), evaluates the integrand and reduces it in place, so
// neither a derivative field nor the integrand field is ever written.
//
// Exactness: every sum, product, quotient and square root in the generated
// code is an explicitly rounded intrinsic (__dadd_rn ...), the derivative
// sums run in the reference's tap order from 0.0, and the reduction is the
// reference's pairwise tree (the chunk walk of pairwise_chunks), so double
// results are bit-identical to the reference when the program performs the
// callable's operations in the callable's order.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <nvrtc.h>

#include <algorithm>
#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"

namespace gcb {
namespace {

constexpr int kChunkCells = 8192;   // pairwise chunk bound (pairwise.cuh kChunkMax)
constexpr int kEvalThreads = 512;

// Kernel argument; the device source declares the same layout.
struct EvalGrid {
  const void* field;
  long long n;
  int nx, ny, nz;
  int step_i, step_j, step_k;     // 2 kEvalThreads cells (one chunk-walk iteration) as (di, dj, dk)
  int kstep_i, kstep_j, kstep_k;  // the compensated sum's stride as (di, dj, dk)
  int pad;
  double ihx, ihy, ihz;     // 1 / h
  double ihx2, ihy2, ihz2;  // 1 / h^2
  double ihx4, ihy4, ihz4;  // (1 / h^2)^2
};

// Device code shared by every program.  gc_cell forms the inputs of the
// arity at one cell and calls the generated gc_integrand; the two kernels are
// the pairwise chunk walk (as pairwise_chunks) and the compensated block sum
// (as kahan_blocks) with the summand computed in place.
const char kDeviceSource[] = R"GCSRC(
typedef long long gc_i64;
struct EvalGrid {
  const void* field;
  gc_i64 n;
  int nx, ny, nz;
  int step_i, step_j, step_k;
  int kstep_i, kstep_j, kstep_k;
  int pad;
  double ihx, ihy, ihz, ihx2, ihy2, ihz2, ihx4, ihy4, ihz4;
};

__device__ __forceinline__ double gc_integrand(const double* in);

// Tap offsets in elements: 32-bit when every offset of the field fits
// (GC_IDX32, set when components x cells < 2^31), else 64-bit.
#ifdef GC_IDX32
typedef int gc_ix;
#else
typedef gc_i64 gc_ix;
#endif

#define GC_R (GC_COMPS == 1 ? (GC_ARITY >= 4 ? 2 : GC_ARITY >= 2 ? 1 : 0) : (GC_ARITY >= 2 ? 1 : 0))
#define GC_NIN (GC_COMPS == 1 ? (GC_ARITY == 1 ? 1 : GC_ARITY + 2) : (GC_ARITY == 1 ? 3 : 12))

// Order-2 first derivative: taps (-1, 0, 1), weights (-0.5, 0, 0.5), from
// 0.0.  The zero-weight centre tap changes the sum only when the centre is
// not finite (0 * inf is NaN; for a finite centre s + (+-0) == s, since s
// is never -0 here), so it is only added then.
template <class Tap>
__device__ __forceinline__ double gc_d1(const Tap& tap, double centre) {
  double s = __dadd_rn(0.0, __dmul_rn(-0.5, tap(-1)));
  if (!isfinite(centre)) s = __dadd_rn(s, __dmul_rn(0.0, centre));
  return __dadd_rn(s, __dmul_rn(0.5, tap(1)));
}

// wrap(i + o, n) - i.  The extent checks leave n >= 2 R + 1 or n == 1, so
// one correction suffices.
__device__ __forceinline__ int gc_off(int i, int o, int n) {
  if (n == 1) return 0;
  const int t = i + o;
  return o + (t < 0 ? n : 0) - (t >= n ? n : 0);
}

// Inputs of the arity and the integrand of one cell; v(comp, ox, oy, oz)
// is the value of component comp at tap (ox, oy, oz) from the cell.
template <class V>
__device__ __forceinline__ double gc_eval_with(const EvalGrid& g, const V& v) {
  double in[GC_NIN];
#if GC_COMPS == 1
  in[0] = v(0, 0, 0, 0);
#if GC_ARITY >= 2
  in[1] = __dmul_rn(gc_d1([&](int o) { return v(0, o, 0, 0); }, in[0]), g.ihx);
  in[2] = __dmul_rn(gc_d1([&](int o) { return v(0, 0, o, 0); }, in[0]), g.ihy);
  in[3] = __dmul_rn(gc_d1([&](int o) { return v(0, 0, 0, o); }, in[0]), g.ihz);
#endif
#if GC_ARITY >= 3
  {  // Laplacian, taps (1, -2, 1) from 0.0 (diff/Laplacian.hpp:60-69)
    const double w2[3] = {1.0, -2.0, 1.0};
    double dxx = 0.0, dyy = 0.0, dzz = 0.0;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      dxx = __dadd_rn(dxx, __dmul_rn(w2[m], v(0, m - 1, 0, 0)));
      dyy = __dadd_rn(dyy, __dmul_rn(w2[m], v(0, 0, m - 1, 0)));
      dzz = __dadd_rn(dzz, __dmul_rn(w2[m], v(0, 0, 0, m - 1)));
    }
    in[4] = __dadd_rn(__dadd_rn(__dmul_rn(dxx, g.ihx2), __dmul_rn(dyy, g.ihy2)), __dmul_rn(dzz, g.ihz2));
  }
#endif
#if GC_ARITY >= 4
  {  // biharmonic (diff/Biharmonic.hpp:70-99)
    const double w4[5] = {1.0, -4.0, 6.0, -4.0, 1.0};
    const double w2[3] = {1.0, -2.0, 1.0};
    double dx4 = 0.0, dy4 = 0.0, dz4 = 0.0;
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      dx4 = __dadd_rn(dx4, __dmul_rn(w4[m], v(0, m - 2, 0, 0)));
      dy4 = __dadd_rn(dy4, __dmul_rn(w4[m], v(0, 0, m - 2, 0)));
      dz4 = __dadd_rn(dz4, __dmul_rn(w4[m], v(0, 0, 0, m - 2)));
    }
    double xy = 0.0, xz = 0.0, yz = 0.0;
#pragma unroll
    for (int mb = 0; mb < 3; ++mb) {
#pragma unroll
      for (int ma = 0; ma < 3; ++ma) {
        const double wab = __dmul_rn(w2[ma], w2[mb]);
        xy = __dadd_rn(xy, __dmul_rn(wab, v(0, ma - 1, mb - 1, 0)));
        xz = __dadd_rn(xz, __dmul_rn(wab, v(0, ma - 1, 0, mb - 1)));
        yz = __dadd_rn(yz, __dmul_rn(wab, v(0, 0, ma - 1, mb - 1)));
      }
    }
    const double axial = __dadd_rn(__dadd_rn(__dmul_rn(dx4, g.ihx4), __dmul_rn(dy4, g.ihy4)), __dmul_rn(dz4, g.ihz4));
    const double c1 = __dmul_rn(__dmul_rn(xy, g.ihx2), g.ihy2);
    const double c2 = __dmul_rn(__dmul_rn(xz, g.ihx2), g.ihz2);
    const double c3 = __dmul_rn(__dmul_rn(yz, g.ihy2), g.ihz2);
    in[5] = __dadd_rn(axial, __dmul_rn(2.0, __dadd_rn(__dadd_rn(c1, c2), c3)));
  }
#endif
#else
#pragma unroll
  for (int c = 0; c < 3; ++c) in[c] = v(c, 0, 0, 0);
#if GC_ARITY >= 2
#pragma unroll
  for (int r = 0; r < 3; ++r) {  // M(r, c) = d_c u_r (diff/Gradient.hpp:115-131)
    in[3 + 3 * r + 0] = __dmul_rn(gc_d1([&](int o) { return v(r, o, 0, 0); }, in[r]), g.ihx);
    in[3 + 3 * r + 1] = __dmul_rn(gc_d1([&](int o) { return v(r, 0, o, 0); }, in[r]), g.ihy);
    in[3 + 3 * r + 2] = __dmul_rn(gc_d1([&](int o) { return v(r, 0, 0, o); }, in[r]), g.ihz);
  }
#endif
#endif
  return gc_integrand(in);
}

// The integrand at the cell p points to; xo / yo / zo are the flat offsets
// of its x, y and z taps.
__device__ __forceinline__ double gc_eval_at(const EvalGrid& g, const GC_T* __restrict__ p, const gc_ix* xo,
                                             const gc_ix* yo, const gc_ix* zo) {
  return gc_eval_with(g, [&](int comp, int ox, int oy, int oz) -> double {
    gc_ix off = (gc_ix)comp * (gc_ix)g.n;
    if (ox) off += xo[ox + GC_R];
    if (oy) off += yo[oy + GC_R];
    if (oz) off += zo[oz + GC_R];
    return (double)__ldg(p + off);
  });
}

__device__ __forceinline__ void gc_yz_offsets(const EvalGrid& g, int j, int k, gc_ix* yo, gc_ix* zo) {
  const gc_ix plane = (gc_ix)g.nx * (gc_ix)g.ny;
#pragma unroll
  for (int m = 0; m <= 2 * GC_R; ++m) {
    yo[m] = (gc_ix)gc_off(j, m - GC_R, g.ny) * (gc_ix)g.nx;
    zo[m] = (gc_ix)gc_off(k, m - GC_R, g.nz) * plane;
  }
}

__device__ __forceinline__ double gc_cell(const EvalGrid& g, gc_i64 c, int i, int j, int k) {
  gc_ix xo[2 * GC_R + 1], yo[2 * GC_R + 1], zo[2 * GC_R + 1];
#pragma unroll
  for (int m = 0; m <= 2 * GC_R; ++m) xo[m] = gc_off(i, m - GC_R, g.nx);
  gc_yz_offsets(g, j, k, yo, zo);
  return gc_eval_at(g, (const GC_T*)g.field + c, xo, yo, zo);
}

// Cells (i, j, k) and (i + 1, j, k) of one row (i + 1 < nx): the y and z
// offsets are formed once.
__device__ __forceinline__ void gc_cell_pair(const EvalGrid& g, gc_i64 c, int i, int j, int k, double& a,
                                             double& b) {
  gc_ix xa[2 * GC_R + 1], xb[2 * GC_R + 1], yo[2 * GC_R + 1], zo[2 * GC_R + 1];
#pragma unroll
  for (int m = 0; m <= 2 * GC_R; ++m) {
    xa[m] = gc_off(i, m - GC_R, g.nx);
    xb[m] = gc_off(i + 1, m - GC_R, g.nx);
  }
  gc_yz_offsets(g, j, k, yo, zo);
  const GC_T* p = (const GC_T*)g.field + c;
  a = gc_eval_at(g, p, xa, yo, zo);
  b = gc_eval_at(g, p + 1, xb, yo, zo);
}

#ifdef GC_PAIRS
// The same pair when cell c is even, nx is even and the field is aligned to
// two elements (GC_PAIRS): both cells' taps with the same (oy, oz) form one
// aligned two-element load, so the pair reads each such tap once; only the
// x taps outside the pair are single loads.
__device__ __forceinline__ void gc_cell_pair_aligned(const EvalGrid& g, gc_i64 c, int i, int j, int k, double& a,
                                                     double& b) {
  gc_ix xa[2 * GC_R + 1], xb[2 * GC_R + 1], yo[2 * GC_R + 1], zo[2 * GC_R + 1];
#pragma unroll
  for (int m = 0; m <= 2 * GC_R; ++m) {
    xa[m] = gc_off(i, m - GC_R, g.nx);
    xb[m] = gc_off(i + 1, m - GC_R, g.nx);
  }
  gc_yz_offsets(g, j, k, yo, zo);
  const GC_T* p = (const GC_T*)g.field + c;
  auto yz = [&](int comp, int oy, int oz) -> gc_ix {
    gc_ix off = (gc_ix)comp * (gc_ix)g.n;
    if (oy) off += yo[oy + GC_R];
    if (oz) off += zo[oz + GC_R];
    return off;
  };
  auto pr = [&](int comp, int oy, int oz) -> GC_T2 { return __ldg((const GC_T2*)(p + yz(comp, oy, oz))); };
  a = gc_eval_with(g, [&](int comp, int ox, int oy, int oz) -> double {
    if (ox == 0) return (double)pr(comp, oy, oz).x;
    if (ox == 1) return (double)pr(comp, oy, oz).y;
    return (double)__ldg(p + yz(comp, oy, oz) + xa[ox + GC_R]);
  });
  b = gc_eval_with(g, [&](int comp, int ox, int oy, int oz) -> double {
    if (ox == 0) return (double)pr(comp, oy, oz).y;
    if (ox == -1) return (double)pr(comp, oy, oz).x;
    return (double)__ldg(p + 1 + yz(comp, oy, oz) + xb[ox + GC_R]);
  });
}
#endif

// (i, j, k) += a step given as (di, dj, dk) with di < nx, dj < ny.
__device__ __forceinline__ void gc_advance(int& i, int& j, int& k, int nx, int ny, int di, int dj, int dk) {
  i += di;
  if (i >= nx) { i -= nx; ++j; }
  j += dj;
  if (j >= ny) { j -= ny; ++k; }
  k += dk;
}

__device__ __forceinline__ void gc_locate(const EvalGrid& g, gc_i64 c, int& i, int& j, int& k) {
  i = (int)(c % g.nx);
  const gc_i64 rest = c / g.nx;
  j = (int)(rest % g.ny);
  k = (int)(rest / g.ny);
}

__device__ __forceinline__ int gc_padpos(int e) { return e + (e >> 6); }

// Bulk prefetch into L2 of cells [first, first + count) of every component:
// the 16-byte-aligned bytes inside that range (the bulk copy's alignment
// rule; the few bytes at either end are left out, so nothing outside the
// field is touched).
__device__ __forceinline__ void gc_prefetch_l2(const EvalGrid& g, gc_i64 first, gc_i64 count) {
  for (int comp = 0; comp < GC_COMPS; ++comp) {
    const unsigned long long a = (unsigned long long)((const GC_T*)g.field + (gc_i64)comp * g.n + first);
    const unsigned long long b = a + (unsigned long long)count * sizeof(GC_T);
    const unsigned long long a16 = (a + 15) & ~15ull, b16 = b & ~15ull;
    if (b16 > a16)
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a16), "r"((unsigned)(b16 - a16)) : "memory");
  }
}

__device__ __forceinline__ void gc_descend(gc_i64& lo, gc_i64& hi, gc_i64 idx, int depth) {
  for (int b = depth - 1; b >= 0; --b) {
    const gc_i64 mid = lo + (hi - lo) / 2;
    if ((idx >> b) & 1) lo = mid;
    else hi = mid;
  }
}

__device__ __forceinline__ double gc_seq_sum(const double* s, int a, int b) {
  double acc = 0.0;
  for (int e = a; e < b; ++e) acc = __dadd_rn(acc, s[gc_padpos(e)]);
  return acc;
}

// 512 threads (16 warps) per CTA.  With the 68.7 KB chunk stage three CTAs fit
// on an SM (48 warps to hide the neighbour loads' latency) where the program
// fits in 40 registers: GC_MIN_CTAS is 3 for scalar integrands of arity 1
// and 2, 2 (64 registers) for vector integrands and 1 (no register cap) for
// scalar arity 3 and 4, the caps under which the programs do not spill.
extern "C" __global__ void __launch_bounds__(512, GC_MIN_CTAS) gc_eval_pairwise(const EvalGrid g, int depth, gc_i64 nchunks,
                                                                      double* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* s = (double*)smem_raw;
  double* ns = s + gc_padpos(8192) + 8;   // 128 half-node sums, then the node tree
  for (gc_i64 c = blockIdx.x; c < nchunks; c += gridDim.x) {
    gc_i64 lo = 0, hi = g.n;
    gc_descend(lo, hi, c, depth);
    const int len = (int)(hi - lo);
    // The next chunk of this CTA streams into L2 while this one is formed.
    if (threadIdx.x == 0 && c + gridDim.x < nchunks) {
      gc_i64 nlo = 0, nhi = g.n;
      gc_descend(nlo, nhi, c + gridDim.x, depth);
      gc_prefetch_l2(g, nlo, nhi - nlo);
    }
    // Two consecutive cells per thread and iteration.
    int i, j, k;
    gc_locate(g, lo + 2 * threadIdx.x, i, j, k);
#ifdef GC_PAIRS
    const bool aligned = (lo & 1) == 0;
#endif
    for (int e = 2 * threadIdx.x; e < len; e += 1024) {
      if (e + 1 < len && i + 1 < g.nx) {
        double a, b;
#ifdef GC_PAIRS
        if (aligned) gc_cell_pair_aligned(g, lo + e, i, j, k, a, b);
        else
#endif
          gc_cell_pair(g, lo + e, i, j, k, a, b);
        s[gc_padpos(e)] = a;
        s[gc_padpos(e + 1)] = b;
      } else {
        s[gc_padpos(e)] = gc_cell(g, lo + e, i, j, k);
        if (e + 1 < len) {
          int i1 = i + 1, j1 = j, k1 = k;
          if (i1 == g.nx) {
            i1 = 0;
            if (++j1 == g.ny) {
              j1 = 0;
              ++k1;
            }
          }
          s[gc_padpos(e + 1)] = gc_cell(g, lo + e + 1, i1, j1, k1);
        }
      }
      gc_advance(i, j, k, g.nx, g.ny, g.step_i, g.step_j, g.step_k);
    }
    int d2 = 0;
    while (((len + (1 << d2) - 1) >> d2) > 128) ++d2;
    const int nodes = 1 << d2;
    __syncthreads();
    // A leaf node of m <= 128 values is summed in order from 0.0, and one of
    // m > 64 as its two halves [0, m/2) and [m/2, m) summed that way and then
    // added: threads 2n and 2n + 1 take node n's halves at the same time.
    if (threadIdx.x < 2 * nodes) {
      const int node = threadIdx.x >> 1, half = threadIdx.x & 1;
      gc_i64 a = 0, b = len;
      gc_descend(a, b, node, d2);
      const int m = (int)(b - a);
      double v = 0.0;
      if (m <= 64) {
        if (half == 0) v = gc_seq_sum(s, (int)a, (int)b);
      } else {
        const int h = m / 2;
        v = half == 0 ? gc_seq_sum(s, (int)a, (int)a + h) : gc_seq_sum(s, (int)a + h, (int)b);
      }
      ns[threadIdx.x] = v;
    }
    __syncthreads();
    {
      double v = 0.0;
      if (threadIdx.x < nodes) {
        gc_i64 a = 0, b = len;
        gc_descend(a, b, threadIdx.x, d2);
        const double v0 = ns[2 * threadIdx.x], v1 = ns[2 * threadIdx.x + 1];
        v = (b - a) <= 64 ? v0 : __dadd_rn(v0, v1);
      }
      __syncthreads();
      if (threadIdx.x < nodes) ns[threadIdx.x] = v;
      __syncthreads();
    }
    for (int w = nodes >> 1; w >= 1; w >>= 1) {
      double v = 0.0;
      if (threadIdx.x < w) v = __dadd_rn(ns[2 * threadIdx.x], ns[2 * threadIdx.x + 1]);
      __syncthreads();
      if (threadIdx.x < w) ns[threadIdx.x] = v;
      __syncthreads();
    }
    if (threadIdx.x == 0) partial[c] = ns[0];
    __syncthreads();
  }
}

struct GcSumC { double s, c; };

__device__ __forceinline__ GcSumC gc_neumaier_add(GcSumC a, double v) {
  const double t = __dadd_rn(a.s, v);
  if (fabs(a.s) >= fabs(v)) a.c = __dadd_rn(a.c, __dadd_rn(__dsub_rn(a.s, t), v));
  else a.c = __dadd_rn(a.c, __dadd_rn(__dsub_rn(v, t), a.s));
  a.s = t;
  return a;
}

__device__ __forceinline__ GcSumC gc_merge(GcSumC a, GcSumC b) {
  const double t = __dadd_rn(a.s, b.s);
  const double bp = __dsub_rn(t, a.s);
  const double err = __dadd_rn(__dsub_rn(a.s, __dsub_rn(t, bp)), __dsub_rn(b.s, bp));
  GcSumC r;
  r.s = t;
  r.c = __dadd_rn(__dadd_rn(a.c, b.c), err);
  return r;
}

extern "C" __global__ void __launch_bounds__(256) gc_eval_kahan(const EvalGrid g, double* __restrict__ out) {
  __shared__ GcSumC sh[256];
  GcSumC acc;
  acc.s = 0.0;
  acc.c = 0.0;
  const gc_i64 first = (gc_i64)blockIdx.x * 256 + threadIdx.x;
  if (first < g.n) {
    int i, j, k;
    gc_locate(g, first, i, j, k);
    for (gc_i64 c = first; c < g.n; c += (gc_i64)1024 * 256) {
      acc = gc_neumaier_add(acc, gc_cell(g, c, i, j, k));
      gc_advance(i, j, k, g.nx, g.ny, g.kstep_i, g.kstep_j, g.kstep_k);
    }
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w >= 1; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] = gc_merge(sh[threadIdx.x], sh[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[2 * blockIdx.x] = sh[0].s;
    out[2 * blockIdx.x + 1] = sh[0].c;
  }
}
)GCSRC";

static_assert(kKahanBlocks == 1024 && kKahanThreads == 256, "the device source bakes in the compensated sum's shape");
static_assert(kEvalThreads == 512, "the device source bakes in 512 threads per block");

constexpr int n_inputs(int comps, int arity) {
  return comps == 1 ? (arity == 1 ? 1 : arity + 2) : (arity == 1 ? 3 : 12);
}

// Checks the program's shape and that every register is written before it
// is read.
gc_status check_program(const gc_program* f) {
  auto bad = [](const std::string& m) { return fail(GC_ERR_INVALID_ARG, "gc_evaluate_program: " + m); };
  if (f->components != 1 && f->components != 3) return bad("components must be 1 (scalar) or 3 (vector)");
  const int max_arity = f->components == 1 ? 4 : 2;
  if (f->arity < 1 || f->arity > max_arity)
    return bad("arity must be 1.." + std::to_string(max_arity) + " for " + std::to_string(f->components) +
               " component(s); got " + std::to_string(f->arity));
  if (f->n_instr < 1 || f->n_instr > GC_PROGRAM_MAX_INSTR)
    return bad("n_instr must be 1.." + std::to_string(GC_PROGRAM_MAX_INSTR) + "; got " + std::to_string(f->n_instr));
  const int inputs = n_inputs(f->components, f->arity);
  uint32_t defined = 0;
  for (int pc = 0; pc < f->n_instr; ++pc) {
    const gc_instr& I = f->instr[pc];
    const std::string at = "instruction " + std::to_string(pc) + ": ";
    if (I.op < GC_OPC_CONST || I.op > GC_OPC_MAX) return bad(at + "unknown opcode " + std::to_string(I.op));
    if (I.dst < 0 || I.dst >= GC_PROGRAM_REGS) return bad(at + "destination register out of range");
    const int reads = I.op <= GC_OPC_INPUT ? 0 : (I.op >= GC_OPC_NEG && I.op <= GC_OPC_SQRT) ? 1 : 2;
    if (I.op == GC_OPC_INPUT && (I.a < 0 || I.a >= inputs))
      return bad(at + "input " + std::to_string(I.a) + " is not available at arity " + std::to_string(f->arity));
    const int16_t src[2] = {I.a, I.b};
    for (int q = 0; q < reads; ++q) {
      if (src[q] < 0 || src[q] >= GC_PROGRAM_REGS || !(defined >> src[q] & 1u))
        return bad(at + "register " + std::to_string(src[q]) + " is read before it is written");
    }
    defined |= 1u << I.dst;
  }
  return GC_OK;
}

// The program as a device function: one named value per instruction, each
// an explicitly rounded operation on the values its registers held.
std::string integrand_source(const gc_program* f) {
  std::string out = "__device__ __forceinline__ double gc_integrand(const double* in) {\n";
  std::string reg[GC_PROGRAM_REGS];
  char buf[96];
  for (int pc = 0; pc < f->n_instr; ++pc) {
    const gc_instr& I = f->instr[pc];
    const std::string A = I.op > GC_OPC_INPUT ? reg[I.a] : "";
    const std::string B = I.op > GC_OPC_INPUT ? reg[I.b] : "";
    std::string e;
    switch (I.op) {
      case GC_OPC_CONST: {
        uint64_t bits;
        std::memcpy(&bits, &I.value, sizeof bits);
        std::snprintf(buf, sizeof buf, "__longlong_as_double(0x%016" PRIx64 "LL)", bits);
        e = buf;
        break;
      }
      case GC_OPC_INPUT: e = "in[" + std::to_string(I.a) + "]"; break;
      case GC_OPC_ADD: e = "__dadd_rn(" + A + ", " + B + ")"; break;
      case GC_OPC_SUB: e = "__dsub_rn(" + A + ", " + B + ")"; break;
      case GC_OPC_MUL: e = "__dmul_rn(" + A + ", " + B + ")"; break;
      case GC_OPC_DIV: e = "__ddiv_rn(" + A + ", " + B + ")"; break;
      case GC_OPC_NEG: e = "-" + A; break;
      case GC_OPC_ABS: e = "fabs(" + A + ")"; break;
      case GC_OPC_SQRT: e = "__dsqrt_rn(" + A + ")"; break;
      case GC_OPC_MIN: e = "(" + B + " < " + A + " ? " + B + " : " + A + ")"; break;
      default: e = "(" + A + " < " + B + " ? " + B + " : " + A + ")"; break;  // GC_OPC_MAX
    }
    const std::string name = "v" + std::to_string(pc);
    out += "  const double " + name + " = " + e + ";\n";
    reg[I.dst] = name;
  }
  out += "  return " + reg[f->instr[f->n_instr - 1].dst] + ";\n}\n";
  return out;
}

// idx32: every tap offset of the field fits in 32 bits; pairs: two-element
// loads of cell pairs are aligned (even nx, field aligned to two elements).
std::string program_source(const gc_program* f, gc_dtype dt, bool idx32, bool pairs) {
  std::string s = "#define GC_T " + std::string(dt == GC_F64 ? "double" : "float") + "\n";
  s += "#define GC_T2 " + std::string(dt == GC_F64 ? "double2" : "float2") + "\n";
  if (idx32) s += "#define GC_IDX32 1\n";
  if (pairs) s += "#define GC_PAIRS 1\n";
  s += "#define GC_COMPS " + std::to_string(f->components) + "\n";
  s += "#define GC_ARITY " + std::to_string(f->arity) + "\n";
  s += "#define GC_MIN_CTAS " +
       std::string(f->components == 1 ? (f->arity <= 2 ? "3" : "1") : "2") + "\n";
  s += kDeviceSource;
  s += integrand_source(f);
  return s;
}

// ---- NVRTC compilation and the module cache ------------------------------
// Driver entry points are fetched through the runtime, so the library does
// not link libcuda itself.
struct Driver {
  PFN_cuModuleLoadData load = nullptr;
  PFN_cuModuleGetFunction get = nullptr;
  PFN_cuFuncSetAttribute attr = nullptr;
  PFN_cuLaunchKernel launch = nullptr;
};

struct Compiled {
  CUfunction pairwise = nullptr;
  CUfunction kahan = nullptr;
};

std::mutex g_jit_mu;
std::map<std::pair<int, std::string>, Compiled> g_jit;  // (device, source) -> kernels; modules live for the process

gc_status driver(Driver* d) {
  static Driver drv;
  static bool ok = false;
  if (!ok) {
    cudaDriverEntryPointQueryResult q;
    auto get = [&](const char* name, void** slot) -> bool {
      return cudaGetDriverEntryPoint(name, slot, cudaEnableDefault, &q) == cudaSuccess &&
             q == cudaDriverEntryPointSuccess && *slot;
    };
    if (!get("cuModuleLoadData", reinterpret_cast<void**>(&drv.load)) ||
        !get("cuModuleGetFunction", reinterpret_cast<void**>(&drv.get)) ||
        !get("cuFuncSetAttribute", reinterpret_cast<void**>(&drv.attr)) ||
        !get("cuLaunchKernel", reinterpret_cast<void**>(&drv.launch)))
      return fail(GC_ERR_CUDA, "gc_evaluate_program: CUDA driver entry points unavailable");
    ok = true;
  }
  *d = drv;
  return GC_OK;
}

gc_status compile(gc_context* ctx, const std::string& src, Compiled* out) {
  std::lock_guard<std::mutex> lock(g_jit_mu);
  const auto key = std::make_pair(ctx->device, src);
  auto it = g_jit.find(key);
  if (it != g_jit.end()) {
    *out = it->second;
    return GC_OK;
  }
  Driver drv;
  gc_status s = driver(&drv);
  if (s != GC_OK) return s;
  nvrtcProgram prog;
  if (nvrtcCreateProgram(&prog, src.c_str(), "gc_integrand.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS)
    return fail(GC_ERR_CUDA, "gc_evaluate_program: nvrtcCreateProgram failed");
  const char* opts[] = {"--gpu-architecture=sm_100a", "--fmad=false", "-std=c++17"};
  const nvrtcResult rc = nvrtcCompileProgram(prog, 3, opts);
  if (rc != NVRTC_SUCCESS) {
    size_t n = 0;
    nvrtcGetProgramLogSize(prog, &n);
    std::string log(n, '\0');
    if (n) nvrtcGetProgramLog(prog, &log[0]);
    nvrtcDestroyProgram(&prog);
    return fail(GC_ERR_CUDA, std::string("gc_evaluate_program: NVRTC: ") + nvrtcGetErrorString(rc) + "\n" + log);
  }
  size_t cubin_size = 0;
  nvrtcGetCUBINSize(prog, &cubin_size);
  std::vector<char> cubin(cubin_size);
  nvrtcGetCUBIN(prog, cubin.data());
  nvrtcDestroyProgram(&prog);
  CUmodule mod;
  Compiled c;
  if (drv.load(&mod, cubin.data()) != CUDA_SUCCESS || drv.get(&c.pairwise, mod, "gc_eval_pairwise") != CUDA_SUCCESS ||
      drv.get(&c.kahan, mod, "gc_eval_kahan") != CUDA_SUCCESS)
    return fail(GC_ERR_CUDA, "gc_evaluate_program: loading the compiled integrand failed");
  const int smem = static_cast<int>(sizeof(double) * (kChunkCells + kChunkCells / 64 + 8 + 2 * 128));
  if (drv.attr(c.pairwise, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, smem) != CUDA_SUCCESS)
    return fail(GC_ERR_CUDA, "gc_evaluate_program: shared-memory attribute refused");
  g_jit.emplace(key, c);
  *out = c;
  return GC_OK;
}

// A step of `cells` flat cells as (di, dj, dk) with di < nx, dj < ny.
void split_step(long long cells, int nx, int ny, int* di, int* dj, int* dk) {
  *di = static_cast<int>(cells % nx);
  const long long rows = cells / nx;
  *dj = static_cast<int>(rows % ny);
  *dk = static_cast<int>(rows / ny);
}

}  // namespace
}  // namespace gcb

using namespace gcb;

extern "C" {

GC_API gc_status gc_evaluate_program(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* field,
                                     const gc_program* f, gc_sum sum, double* result) {
  NvtxScope nvtx("gc_evaluate_program");
  Call call(ctx);
  gc_status s = call.st;
  if (s != GC_OK) return s;
  if ((s = check_grid(g)) != GC_OK) return s;
  if (!field || !f || !result) return fail(GC_ERR_INVALID_ARG, "gc_evaluate_program: null pointer");
  if (dt != GC_F64 && dt != GC_F32) return fail(GC_ERR_INVALID_ARG, "gc_evaluate_program: unknown dtype");
  if ((s = check_program(f)) != GC_OK) return s;
  // The derivative fields of the arity, checked in the reference's order:
  // gradient (radius 1), Laplacian (radius 1), biharmonic (radius 2).
  if (f->arity >= 2 && (s = require_axes(g, 1)) != GC_OK) return s;
  if (f->components == 1 && f->arity >= 4 && (s = require_axes(g, 2)) != GC_OK) return s;
  return run_program(ctx, g, dt, field, f, sum, result);
}

GC_API size_t gc_program_source(const gc_program* f, gc_dtype dt, char* buf, size_t cap) {
  if (!f || check_program(f) != GC_OK) return 0;
  const std::string src = program_source(f, dt, false, false);
  if (buf && cap) {
    const size_t n = std::min(cap - 1, src.size());
    std::memcpy(buf, src.data(), n);
    buf[n] = '\0';
  }
  return src.size() + 1;
}

}  // extern "C"

namespace gcb {

gc_status run_program(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* field, const gc_program* f,
                      gc_sum sum, double* result) {
  gc_status s;
  const long long n = static_cast<long long>(cells(g));
  const size_t esize = dt == GC_F64 ? sizeof(double) : sizeof(float);
  const bool idx32 = static_cast<long long>(f->components) * n < (1ll << 31);
  const bool pairs = g->nx % 2 == 0 && reinterpret_cast<uintptr_t>(field) % (2 * esize) == 0;
  Compiled k;
  if ((s = compile(ctx, program_source(f, dt, idx32, pairs), &k)) != GC_OK) return s;
  Driver drv;
  if ((s = driver(&drv)) != GC_OK) return s;

  EvalGrid a{};
  a.field = field;
  a.n = n;
  a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
  split_step(2 * kEvalThreads, g->nx, g->ny, &a.step_i, &a.step_j, &a.step_k);
  split_step(static_cast<long long>(kKahanBlocks) * kKahanThreads, g->nx, g->ny, &a.kstep_i, &a.kstep_j, &a.kstep_k);
  a.ihx = 1.0 / g->hx; a.ihy = 1.0 / g->hy; a.ihz = 1.0 / g->hz;
  a.ihx2 = 1.0 / (g->hx * g->hx); a.ihy2 = 1.0 / (g->hy * g->hy); a.ihz2 = 1.0 / (g->hz * g->hz);
  a.ihx4 = a.ihx2 * a.ihx2; a.ihy4 = a.ihy2 * a.ihy2; a.ihz4 = a.ihz2 * a.ihz2;
  const double vol = g->hx * g->hy * g->hz;
  double total = 0.0;
  void* buf = nullptr;
  if (sum == GC_SUM_KAHAN) {
    if ((s = scratch_get(ctx, kSlotReduce, kKahanScratchBytes, &buf)) != GC_OK) return s;
    double* part = static_cast<double*>(buf);
    void* args[] = {&a, &part};
    if (drv.launch(k.kahan, kKahanBlocks, 1, 1, kKahanThreads, 1, 1, 0, ctx->stream, args, nullptr) != CUDA_SUCCESS)
      return fail(GC_ERR_CUDA, "gc_evaluate_program: launch failed");
    if ((s = kahan_finish(ctx, part, &total)) != GC_OK) return s;
  } else {
    const PairwisePlan plan = pairwise_plan(n);
    if ((s = scratch_get(ctx, kSlotReduce, plan.scratch_bytes, &buf)) != GC_OK) return s;
    double* partial = static_cast<double*>(buf);
    int depth = plan.depth;
    long long nchunks = plan.nchunks;
    void* args[] = {&a, &depth, &nchunks, &partial};
    const unsigned grid = static_cast<unsigned>(std::min<long long>(nchunks, static_cast<long long>(ctx->num_sms) * 3));
    const unsigned smem = static_cast<unsigned>(sizeof(double) * (kChunkCells + kChunkCells / 64 + 8 + 2 * 128));
    if (drv.launch(k.pairwise, grid, 1, 1, kEvalThreads, 1, 1, smem, ctx->stream, args, nullptr) != CUDA_SUCCESS)
      return fail(GC_ERR_CUDA, "gc_evaluate_program: launch failed");
    if ((s = pairwise_finish(ctx, partial, nchunks, &total)) != GC_OK) return s;
  }
  *result = vol * total;
  return GC_OK;
}

}  // namespace gcb
