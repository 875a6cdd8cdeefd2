// Shared device/host helpers for the gridcalc_b200 kernels.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <cstring>
#include <string>

#include "gridcalc_b200.h"

namespace gcb {

// ---------------------------------------------------------------------------
// Error plumbing: thread-local message + status (never throws across the ABI).
void set_error(const std::string& msg);
gc_status fail(gc_status s, const std::string& msg);
gc_status cuda_fail(cudaError_t e, const char* what);

#define GC_CUDA(call)                                            \
  do {                                                           \
    cudaError_t gc_e_ = (call);                                  \
    if (gc_e_ != cudaSuccess) return ::gcb::cuda_fail(gc_e_, #call); \
  } while (0)

#define GC_CHECK_LAUNCH(what)                                    \
  do {                                                           \
    cudaError_t gc_e_ = cudaGetLastError();                      \
    if (gc_e_ != cudaSuccess) return ::gcb::cuda_fail(gc_e_, what); \
  } while (0)

#define GC_TRY(expr)                                             \
  do {                                                           \
    gc_status gc_s_ = (expr);                                    \
    if (gc_s_ != GC_OK) return gc_s_;                            \
  } while (0)

// ---------------------------------------------------------------------------
// Context: stream + cached scratch.
struct Scratch {
  void* ptr = nullptr;
  size_t bytes = 0;
};

}  // namespace gcb

struct gc_context {
  int device = 0;
  // All work runs on `stream`, owned by the context (capturable); each call
  // first waits for the caller's stream and makes the caller's stream wait
  // for it on return, so the call is ordered like a launch on that stream.
  cudaStream_t stream = nullptr;
  cudaStream_t user_stream = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  int num_sms = 148;
  // Named scratch slots, grown on demand and kept for the context's life.
  gcb::Scratch scratch[16];
  // Pinned host word(s) for small device->host results.
  void* host_pinned = nullptr;
  // Device status word: kernels with bounded waits set it when a wait gives
  // up (GC_ERR_TIMEOUT); gc_synchronize() reports and clears it.
  int* device_status = nullptr;
  // Small cache of captured step graphs, keyed by everything the captured
  // kernels bake in; least recently used entry is replaced.
  static constexpr int kGraphSlots = 6;
  cudaGraphExec_t graph_exec[kGraphSlots] = {};
  uint64_t graph_key[kGraphSlots][8] = {};
  uint64_t graph_used[kGraphSlots] = {};
  uint64_t graph_clock = 0;
  // FFT plans of the spectral entry points: one set per context, so each
  // context's transforms run on its own stream with their own work area;
  // released by gc_context_destroy through spectral_release.
  void* spectral_plans = nullptr;
  void (*spectral_release)(void*) = nullptr;
  // gc_context_set_option switches.
  bool cluster_stepping = false;
  bool fused_step = true;
};

namespace gcb {

enum ScratchSlot {
  kSlotK1 = 0,
  kSlotK2,
  kSlotK3,
  kSlotPsiB,
  kSlotReduce,
  kSlotFlags,
  kSlotMisc,
  kSlotSpectral,
  kSlotFaces,
};

gc_status scratch_get(gc_context* ctx, int slot, size_t bytes, void** out);

// Validation helpers mirroring the reference contracts.
gc_status check_grid(const gc_grid* g);
gc_status require_axes(const gc_grid* g, int radius);
// Per-axis radii (an axis with radius 0 accepts any extent).
gc_status require_axes3(const gc_grid* g, int rx, int ry, int rz);
gc_status check_ctx(gc_context* ctx);

// Whole-integration fast path for 2-D grids whose state fits in one
// thread-block cluster's shared memory (ch_cluster.cu): *done reports whether
// it ran (false: the grid does not fit, take the multi-launch path).
gc_status ch_cluster_integrate(gc_context* ctx, const gc_grid* g, gc_dtype dt, const gc_ch_params* cp, void* psi,
                               double dt_step, int n_steps, gc_integrator integ, bool* done);

// One RK4 step of a 2-D double grid at order 2 in one fused kernel
// (ch_fused.cu), src -> dst; *done reports whether it ran (false: the grid
// or its layout does not suit it, use the stage kernels).
gc_status ch_fused_step(gc_context* ctx, const gc_grid* g, const gc_ch_params* cp, const double* src, double* dst,
                        double dt, bool* done);
// The same for a 2-D float grid at order 2 or 4 (ch_batch.cu: the ensemble's
// fused tile walk over one grid).
gc_status ch_fused_step_f32(gc_context* ctx, const gc_grid* g, const gc_ch_params* cp, const float* src, float* dst,
                            double dt, bool* done);

// Opts kernel `kern` into `smem` bytes of dynamic shared memory on the
// current device and, with ctas_per_sm, returns how many CTAs of `threads`
// threads and `smem` bytes fit on one SM (at least 1).  The attribute belongs
// to one device's context, so it is set once per (kernel, device) -- not once
// per process -- under a lock, since contexts may be driven from several host
// threads.
gc_status kernel_setup_raw(const void* kern, int threads, size_t smem, int* ctas_per_sm);
template <class K>
inline gc_status kernel_setup(K* kern, int threads, size_t smem, int* ctas_per_sm = nullptr) {
  return kernel_setup_raw(reinterpret_cast<const void*>(kern), threads, smem, ctas_per_sm);
}

// Stream-ordered building blocks for other parts of the library (no
// validation, no Call scope, no allocation): enqueue on ctx->stream only, so
// they can be captured into a CUDA graph.
// f(psi) of the Cahn-Hilliard RHS into out.
gc_status ch_rhs_enqueue(gc_context* ctx, const gc_grid* g, gc_dtype dt, const gc_ch_params* cp, const void* psi,
                         void* out);
// One RKC2 step of psi in place; scratch = four fields of the grid's size
// (F0 and three stage buffers).
gc_status ch_rkc_enqueue(gc_context* ctx, const gc_grid* g, gc_dtype dt, const gc_ch_params* cp, void* psi,
                         double dt_step, int stages, void* const (&scratch)[4]);

// The reduction's building blocks, for kernels that produce the summands
// themselves.  Pairwise: 2^depth chunks of at most 8192 values, reduced per
// chunk into partial[0, nchunks) and finished by pairwise_finish (which uses
// the rest of scratch_bytes after the chunk sums).  Compensated: kKahanBlocks
// blocks of kKahanThreads threads, each thread over the values
// i = block * kKahanThreads + thread + m * kKahanBlocks * kKahanThreads, the
// block's (sum, compensation) at part[2 * block]; kahan_finish merges them.
struct PairwisePlan {
  int depth = 0;
  long long nchunks = 1;
  size_t scratch_bytes = 0;
};
PairwisePlan pairwise_plan(long long n);
gc_status pairwise_finish(gc_context* ctx, double* partial, long long nchunks, double* result);
constexpr int kKahanBlocks = 1024;
constexpr int kKahanThreads = 256;
constexpr size_t kKahanScratchBytes = sizeof(double) * (2 * kKahanBlocks + 8);
gc_status kahan_finish(gc_context* ctx, double* part, double* result);

// Sum of n values (double or float, as dt) on ctx->stream, exactly the
// reference's pairwise tree (GC_SUM_PAIRWISE) or the deterministic
// compensated sum (GC_SUM_KAHAN); synchronises and returns it on the host.
gc_status sum_any(gc_context* ctx, gc_dtype dt, const void* x, long long n, gc_sum sum, double* result);

// func::evaluate of a checked integrand program over a field whose axis
// extents were checked: the NVRTC-compiled chunk walk forms the integrand
// from the field and its neighbours and reduces it (no integrand field in
// HBM); returns volume x sum on the host.
gc_status run_program(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* field, const gc_program* f,
                      gc_sum sum, double* result);

// A named NVTX range for the duration of a scope: the long-running entry
// points show up by name on an Nsight Systems / NVTX timeline (no cost when
// no tool is attached).
struct NvtxScope {
  explicit NvtxScope(const char* name) { nvtxRangePushA(name); }
  ~NvtxScope() { nvtxRangePop(); }
  NvtxScope(const NvtxScope&) = delete;
  NvtxScope& operator=(const NvtxScope&) = delete;
};

// Scope of one API call: validates the context, orders the context stream
// after the caller's stream on entry and the caller's stream after the
// context stream on exit.
struct Call {
  gc_context* ctx;
  gc_status st;
  explicit Call(gc_context* c);
  ~Call();
};
inline uint64_t bits_of(double d) {
  uint64_t b;
  std::memcpy(&b, &d, sizeof b);
  return b;
}
inline size_t cells(const gc_grid* g) {
  return static_cast<size_t>(g->nx) * static_cast<size_t>(g->ny) * static_cast<size_t>(g->nz);
}
inline size_t dtype_size(gc_dtype d) { return d == GC_F64 ? 8 : 4; }

// ---------------------------------------------------------------------------
// Arithmetic policy.  Double follows the reference exactly: every product
// and sum is rounded on its own (__dmul_rn/__dadd_rn are never fused into
// an FMA), so tap-by-tap accumulation reproduces the CPU result bit for bit.
// Float is the precision variant: the compiler may contract into FMAs.
template <class T>
struct Ar;

template <>
struct Ar<double> {
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
  // acc + w * x, rounded twice (no FMA).
  static __device__ __forceinline__ double mac(double acc, double w, double x) {
    return __dadd_rn(acc, __dmul_rn(w, x));
  }
};

template <>
struct Ar<float> {
  static __device__ __forceinline__ float mul(float a, float b) { return a * b; }
  static __device__ __forceinline__ float add(float a, float b) { return a + b; }
  static __device__ __forceinline__ float sub(float a, float b) { return a - b; }
  static __device__ __forceinline__ float div(float a, float b) { return a / b; }
  static __device__ __forceinline__ float mac(float acc, float w, float x) { return fmaf(w, x, acc); }
};

// Periodic wrap, ((i % N) + N) % N (reference core/IndexPolicy.hpp:28), with
// a branch for the common in-range case.
__device__ __forceinline__ int wrap(int i, int n) {
  if (i >= 0 && i < n) return i;
  int r = i % n;
  return r < 0 ? r + n : r;
}

// ---------------------------------------------------------------------------
// Stencil weight tables (unscaled), as compile-time constants.
// Kind 1: first derivative; kind 2: second derivative; kind 4: fourth.
// Orders 2 and 4 are the reference tables (stencil/CentralDifference.hpp:41-74,
// stencil/FirstDerivative.hpp:51-86, stencil/FourthDerivative.hpp:49-83);
// order 6 is the standard central-difference set (radius 3, 3, 4).
template <int Kind, int Order>
struct W;

template <> struct W<2, 2> {
  static constexpr int R = 1;
  static __host__ __device__ constexpr double w(int m) { return m == 1 ? -2.0 : 1.0; }
};
template <> struct W<2, 4> {
  static constexpr int R = 2;
  static __host__ __device__ constexpr double w(int m) {
    return m == 0 || m == 4 ? -1.0 / 12.0 : (m == 1 || m == 3 ? 4.0 / 3.0 : -5.0 / 2.0);
  }
};
template <> struct W<2, 6> {
  static constexpr int R = 3;
  static __host__ __device__ constexpr double w(int m) {
    return m == 0 || m == 6 ? 1.0 / 90.0
         : m == 1 || m == 5 ? -3.0 / 20.0
         : m == 2 || m == 4 ? 3.0 / 2.0
                            : -49.0 / 18.0;
  }
};
template <> struct W<1, 2> {
  static constexpr int R = 1;
  static __host__ __device__ constexpr double w(int m) { return m == 0 ? -0.5 : (m == 2 ? 0.5 : 0.0); }
};
template <> struct W<1, 4> {
  static constexpr int R = 2;
  static __host__ __device__ constexpr double w(int m) {
    return m == 0 ? 1.0 / 12.0 : m == 1 ? -2.0 / 3.0 : m == 2 ? 0.0 : m == 3 ? 2.0 / 3.0 : -1.0 / 12.0;
  }
};
template <> struct W<1, 6> {
  static constexpr int R = 3;
  static __host__ __device__ constexpr double w(int m) {
    return m == 0 ? -1.0 / 60.0 : m == 1 ? 3.0 / 20.0 : m == 2 ? -3.0 / 4.0 : m == 3 ? 0.0
         : m == 4 ? 3.0 / 4.0 : m == 5 ? -3.0 / 20.0 : 1.0 / 60.0;
  }
};
template <> struct W<4, 2> {
  static constexpr int R = 2;
  static __host__ __device__ constexpr double w(int m) {
    return m == 0 || m == 4 ? 1.0 : (m == 1 || m == 3 ? -4.0 : 6.0);
  }
};
template <> struct W<4, 4> {
  static constexpr int R = 3;
  static __host__ __device__ constexpr double w(int m) {
    return m == 0 || m == 6 ? -1.0 / 6.0
         : m == 1 || m == 5 ? 2.0
         : m == 2 || m == 4 ? -13.0 / 2.0
                            : 28.0 / 3.0;
  }
};
template <> struct W<4, 6> {
  static constexpr int R = 4;
  static __host__ __device__ constexpr double w(int m) {
    return m == 0 || m == 8 ? 7.0 / 240.0
         : m == 1 || m == 7 ? -2.0 / 5.0
         : m == 2 || m == 6 ? 169.0 / 60.0
         : m == 3 || m == 5 ? -122.0 / 15.0
                            : 91.0 / 8.0;
  }
};

// Kind 3 (third derivative): the reference tables for orders 2 and 4
// (stencil/ThirdDerivative.hpp:49-84), order 6 the standard central set.
template <> struct W<3, 2> {
  static constexpr int R = 2;
  static __host__ __device__ constexpr double w(int m) {
    return m == 0 ? -1.0 / 2.0 : m == 1 ? 1.0 : m == 2 ? 0.0 : m == 3 ? -1.0 : 1.0 / 2.0;
  }
};
template <> struct W<3, 4> {
  static constexpr int R = 3;
  static __host__ __device__ constexpr double w(int m) {
    return m == 0 ? 1.0 / 8.0 : m == 1 ? -1.0 : m == 2 ? 13.0 / 8.0 : m == 3 ? 0.0
         : m == 4 ? -13.0 / 8.0 : m == 5 ? 1.0 : -1.0 / 8.0;
  }
};
template <> struct W<3, 6> {
  static constexpr int R = 4;
  static __host__ __device__ constexpr double w(int m) {
    return m == 0 ? -7.0 / 240.0 : m == 1 ? 3.0 / 10.0 : m == 2 ? -169.0 / 120.0 : m == 3 ? 61.0 / 30.0
         : m == 4 ? 0.0 : m == 5 ? -61.0 / 30.0 : m == 6 ? 169.0 / 120.0 : m == 7 ? -3.0 / 10.0 : 7.0 / 240.0;
  }
};

// Weight as the storage type T (float tables are the double ones rounded).
template <class T, int Kind, int Order>
__device__ __forceinline__ T wt(int m) {
  return static_cast<T>(W<Kind, Order>::w(m));
}

// True when the weight is exactly 1 (the product w*x == x needs no multiply).
template <int Kind, int Order>
__host__ __device__ constexpr bool unit_weight(int m) {
  return W<Kind, Order>::w(m) == 1.0;
}
template <int Kind, int Order>
__host__ __device__ constexpr bool zero_weight(int m) {
  return W<Kind, Order>::w(m) == 0.0;
}

// Tap-ordered 1-D stencil sum over values v[0..2R] (v[m] = f(x + m - R)):
// acc = ((w0 v0 + w1 v1) + ...) accumulated left to right, as the reference
// loops `acc += w[m] * field(...)`.  Zero-weight taps are skipped (that only
// changes the sign of an exactly-zero sum) and unit weights skip the multiply.
// The reference starts from 0.0; starting from the first tap instead
// differs only when that tap is -0 (the sum's sign of zero).
template <class T, int Kind, int Order, class Get>
__device__ __forceinline__ T tap_sum(Get get) {
  constexpr int R = W<Kind, Order>::R;
  T acc = T(0);
  bool first = true;
#pragma unroll
  for (int m = 0; m <= 2 * R; ++m) {
    if (zero_weight<Kind, Order>(m)) continue;
    const T v = get(m - R);
    const T term = unit_weight<Kind, Order>(m) ? v : Ar<T>::mul(wt<T, Kind, Order>(m), v);
    acc = first ? term : Ar<T>::add(acc, term);
    first = false;
  }
  return acc;
}

inline int div_up(long long a, long long b) { return static_cast<int>((a + b - 1) / b); }

}  // namespace gcb
