// Integrals: func::integrate (pairwise / Kahan), func::evaluate integrands,
// the largest harmonic face D, and the D > 0 precondition.
//
// Pairwise sum, reproduced exactly.  The reference sums recursively
// (func/Integrate.hpp:65-74): a range of n > 64 values splits at n/2, a range
// of n <= 64 is summed left to right from 0.0.  Every node at depth d has
// n/2^d rounded down or up values, so the tree is cut in two layers:
//   1. the first D levels split the field into 2^D "chunks" of at most 8192
//      values (every node above them is larger than 64, so it is a plain
//      split); one CTA stages a chunk in shared memory and walks the next
//      levels down to per-thread nodes of at most 128 values, which a thread
//      sums exactly as the reference's base case (one extra split when the
//      node holds 65..128 values); the node sums are combined up the perfect
//      binary tree they form;
//   2. the 2^D chunk sums form a perfect binary tree too, reduced in groups
//      of 1024 (a perfect subtree each) until one value is left.
// Because every addition happens between the same two operands as in the
// reference, the double result is bit-identical.  Staging: a chunk is
// loaded with coalesced loads and stored padded by one double every 64, so
// that the 32 lanes walking 64-value nodes hit distinct banks.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "pairwise.cuh"

namespace gcb {
namespace {

// ---- deterministic compensated sum (GC_SUM_KAHAN) -------------------------
// Each thread runs Neumaier's update over a fixed strided subset, then the
// (sum, compensation) pairs merge up a fixed tree with an error-free
// two-sum.  Grid and block sizes are constants, so the result does not
// depend on the device.
struct SumC { double s, c; };

__device__ __forceinline__ SumC neumaier_add(SumC a, double v) {
  const double t = __dadd_rn(a.s, v);
  if (fabs(a.s) >= fabs(v)) a.c = __dadd_rn(a.c, __dadd_rn(__dsub_rn(a.s, t), v));
  else a.c = __dadd_rn(a.c, __dadd_rn(__dsub_rn(v, t), a.s));
  a.s = t;
  return a;
}

__device__ __forceinline__ SumC merge(SumC a, SumC b) {
  const double t = __dadd_rn(a.s, b.s);
  const double bp = __dsub_rn(t, a.s);
  const double err = __dadd_rn(__dsub_rn(a.s, __dsub_rn(t, bp)), __dsub_rn(b.s, bp));
  return SumC{t, __dadd_rn(__dadd_rn(a.c, b.c), err)};
}

template <class T>
__global__ void __launch_bounds__(kKahanThreads) kahan_blocks(const T* __restrict__ x, long long n,
                                                              double* __restrict__ out) {
  __shared__ SumC sh[kKahanThreads];
  SumC acc{0.0, 0.0};
  const long long stride = static_cast<long long>(kKahanBlocks) * kKahanThreads;
  for (long long i = static_cast<long long>(blockIdx.x) * kKahanThreads + threadIdx.x; i < n; i += stride)
    acc = neumaier_add(acc, static_cast<double>(x[i]));
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = kKahanThreads / 2; w >= 1; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] = merge(sh[threadIdx.x], sh[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[2 * blockIdx.x] = sh[0].s;
    out[2 * blockIdx.x + 1] = sh[0].c;
  }
}

__global__ void __launch_bounds__(1024) kahan_final(const double* __restrict__ in, double* __restrict__ out) {
  __shared__ SumC sh[kKahanBlocks];
  sh[threadIdx.x] = SumC{in[2 * threadIdx.x], in[2 * threadIdx.x + 1]};
  __syncthreads();
  for (int w = kKahanBlocks / 2; w >= 1; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] = merge(sh[threadIdx.x], sh[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = __dadd_rn(sh[0].s, sh[0].c);
}

// ---- largest harmonic face D (solve/Diffusion.hpp:187-207) -----------------
template <class T>
__global__ void d_max_face_kernel(const T* __restrict__ D, int nx, int ny, int nz,
                                  unsigned long long* __restrict__ best_bits) {
  const size_t n = static_cast<size_t>(nx) * ny * nz;
  double m = 0.0;
  for (size_t c = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < n;
       c += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(c % nx);
    const size_t rest = c / nx;
    const int j = static_cast<int>(rest % ny);
    const int k = static_cast<int>(rest / ny);
    const int ip = i + 1 == nx ? 0 : i + 1, jp = j + 1 == ny ? 0 : j + 1, kp = k + 1 == nz ? 0 : k + 1;
    const double dc = static_cast<double>(D[c]);
    const double nb[3] = {static_cast<double>(D[c - i + ip]),
                          static_cast<double>(D[c + static_cast<size_t>(jp - j) * nx]),
                          static_cast<double>(D[c + (static_cast<long long>(kp) - k) * static_cast<long long>(nx) * ny])};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double f = __ddiv_rn(__dmul_rn(__dmul_rn(2.0, dc), nb[a]), __dadd_rn(dc, nb[a]));
      if (f > m) m = f;  // NaN and non-positive faces never win, as in the reference
    }
  }
  // Non-negative doubles order like their bit patterns.
  if (m > 0.0) atomicMax(best_bits, static_cast<unsigned long long>(__double_as_longlong(m)));
}

// First flat index with !(D > 0) (fvm/CellLaplacian.hpp:100-109).
template <class T>
__global__ void first_nonpositive_kernel(const T* __restrict__ D, long long n,
                                         unsigned long long* __restrict__ first) {
  for (long long c = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; c < n;
       c += static_cast<long long>(gridDim.x) * blockDim.x) {
    if (!(static_cast<double>(D[c]) > 0.0)) {
      atomicMin(first, static_cast<unsigned long long>(c));
      return;
    }
  }
}

// First flat index holding a NaN or an infinity.
template <class T>
__global__ void first_nonfinite_kernel(const T* __restrict__ x, long long n, unsigned long long* __restrict__ first) {
  for (long long c = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; c < n;
       c += static_cast<long long>(gridDim.x) * blockDim.x) {
    if (!isfinite(static_cast<double>(x[c]))) {
      atomicMin(first, static_cast<unsigned long long>(c));
      return;
    }
  }
}

}  // namespace

PairwisePlan pairwise_plan(long long n) {
  PairwisePlan p;
  while (((n + (1LL << p.depth) - 1) >> p.depth) > kChunkMax) ++p.depth;
  p.nchunks = 1LL << p.depth;
  // Chunk sums, then the group-reduction levels.
  p.scratch_bytes = sizeof(double) * static_cast<size_t>(p.nchunks + p.nchunks / 1024 + 64);
  return p;
}

gc_status pairwise_finish(gc_context* ctx, double* partial, long long nchunks, double* result) {
  long long count = nchunks;
  double* src = partial;
  double* dst = partial + nchunks;
  while (count > 1) {
    const int group = static_cast<int>(std::min<long long>(count, 1024));
    const long long blocks = count / group;
    tree_groups<<<static_cast<unsigned>(blocks), 1024, 0, ctx->stream>>>(src, count, group, dst);
    GC_CHECK_LAUNCH("tree_groups");
    count = blocks;
    std::swap(src, dst);
  }
  double* host = static_cast<double*>(ctx->host_pinned);
  GC_CUDA(cudaMemcpyAsync(host, src, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  GC_CUDA(cudaStreamSynchronize(ctx->stream));
  *result = host[0];
  return GC_OK;
}

gc_status kahan_finish(gc_context* ctx, double* part, double* result) {
  kahan_final<<<1, kKahanBlocks, 0, ctx->stream>>>(part, part + 2 * kKahanBlocks);
  GC_CHECK_LAUNCH("kahan_final");
  double* host = static_cast<double*>(ctx->host_pinned);
  GC_CUDA(cudaMemcpyAsync(host, part + 2 * kKahanBlocks, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  GC_CUDA(cudaStreamSynchronize(ctx->stream));
  *result = host[0];
  return GC_OK;
}

// Exact pairwise sum of n values on the context's stream; result on the host.
template <class T>
gc_status pairwise_sum(gc_context* ctx, const T* x, long long n, double* result) {
  if (n == 0) {
    *result = 0.0;
    return GC_OK;
  }
  const PairwisePlan plan = pairwise_plan(n);
  void* buf = nullptr;
  gc_status s = scratch_get(ctx, kSlotReduce, plan.scratch_bytes, &buf);
  if (s != GC_OK) return s;
  double* a = static_cast<double*>(buf);
  const size_t smem = sizeof(double) * (padpos(kChunkMax) + 8 + kNodeMax);
  auto kern = pairwise_chunks<T>;
  GC_TRY(kernel_setup(kern, kSumThreads, smem));
  const long long grid = std::min<long long>(plan.nchunks, static_cast<long long>(ctx->num_sms) * 3);
  kern<<<static_cast<unsigned>(grid), kSumThreads, smem, ctx->stream>>>(x, n, plan.depth, plan.nchunks, a);
  GC_CHECK_LAUNCH("pairwise_chunks");
  return pairwise_finish(ctx, a, plan.nchunks, result);
}

template <class T>
gc_status kahan_sum(gc_context* ctx, const T* x, long long n, double* result) {
  void* buf = nullptr;
  gc_status s = scratch_get(ctx, kSlotReduce, kKahanScratchBytes, &buf);
  if (s != GC_OK) return s;
  double* part = static_cast<double*>(buf);
  kahan_blocks<T><<<kKahanBlocks, kKahanThreads, 0, ctx->stream>>>(x, n, part);
  GC_CHECK_LAUNCH("kahan_blocks");
  return kahan_finish(ctx, part, result);
}

template gc_status pairwise_sum<double>(gc_context*, const double*, long long, double*);
template gc_status pairwise_sum<float>(gc_context*, const float*, long long, double*);

gc_status sum_any(gc_context* ctx, gc_dtype dt, const void* x, long long n, gc_sum sum,
                  double* result) {
  if (dt == GC_F64) {
    const double* p = static_cast<const double*>(x);
    return sum == GC_SUM_KAHAN ? kahan_sum(ctx, p, n, result) : pairwise_sum(ctx, p, n, result);
  }
  const float* p = static_cast<const float*>(x);
  return sum == GC_SUM_KAHAN ? kahan_sum(ctx, p, n, result) : pairwise_sum(ctx, p, n, result);
}

gc_status d_max_face_any(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* D, double* result) {
  void* buf = nullptr;
  gc_status s = scratch_get(ctx, kSlotFlags, 64, &buf);
  if (s != GC_OK) return s;
  unsigned long long* bits = static_cast<unsigned long long*>(buf);
  GC_CUDA(cudaMemsetAsync(bits, 0, sizeof(unsigned long long), ctx->stream));
  const int blocks = ctx->num_sms * 8;
  if (dt == GC_F64)
    d_max_face_kernel<double><<<blocks, 256, 0, ctx->stream>>>(static_cast<const double*>(D), g->nx, g->ny, g->nz, bits);
  else
    d_max_face_kernel<float><<<blocks, 256, 0, ctx->stream>>>(static_cast<const float*>(D), g->nx, g->ny, g->nz, bits);
  GC_CHECK_LAUNCH("d_max_face_kernel");
  unsigned long long* host = static_cast<unsigned long long*>(ctx->host_pinned);
  GC_CUDA(cudaMemcpyAsync(host, bits, sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
  GC_CUDA(cudaStreamSynchronize(ctx->stream));
  std::memcpy(result, &host[0], sizeof(double));
  return GC_OK;
}

gc_status first_nonpositive(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* D, long long* first) {
  void* buf = nullptr;
  gc_status s = scratch_get(ctx, kSlotFlags, 64, &buf);
  if (s != GC_OK) return s;
  unsigned long long* word = static_cast<unsigned long long*>(buf) + 1;
  GC_CUDA(cudaMemsetAsync(word, 0xff, sizeof(unsigned long long), ctx->stream));
  const long long n = static_cast<long long>(cells(g));
  const int blocks = ctx->num_sms * 8;
  if (dt == GC_F64)
    first_nonpositive_kernel<double><<<blocks, 256, 0, ctx->stream>>>(static_cast<const double*>(D), n, word);
  else
    first_nonpositive_kernel<float><<<blocks, 256, 0, ctx->stream>>>(static_cast<const float*>(D), n, word);
  GC_CHECK_LAUNCH("first_nonpositive_kernel");
  unsigned long long* host = static_cast<unsigned long long*>(ctx->host_pinned) + 1;
  GC_CUDA(cudaMemcpyAsync(host, word, sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
  GC_CUDA(cudaStreamSynchronize(ctx->stream));
  *first = host[0] == ~0ULL ? -1 : static_cast<long long>(host[0]);
  return GC_OK;
}

// The hot-path integrands (cahn_hilliard.hpp:64-77, heterogeneous_diffusion.hpp:82)
// as integrand programs: the operations of the reference's expressions in
// its order, so the fused evaluation gives its values bit for bit.
// -psi^2/2 + psi^4/4 + kappa/2 |grad psi|^2 is ((-0.5 p) p + (((0.25 p) p) p) p)
// + (0.5 kappa) ((gx gx + gy gy) + gz gz).
gc_program fixed_program(int kind, double kappa) {
  gc_program f{};
  f.components = 1;
  auto op = [&](int code, int dst, int a, int b, double v = 0.0) {
    f.instr[f.n_instr++] = gc_instr{static_cast<int16_t>(code), static_cast<int16_t>(dst), static_cast<int16_t>(a),
                                    static_cast<int16_t>(b), v};
  };
  switch (kind) {
    case GC_INTEGRAND_PSI:
      f.arity = 1;
      op(GC_OPC_INPUT, 0, GC_IN_PSI, 0);
      break;
    case GC_INTEGRAND_PSI_SQUARED:
      f.arity = 1;
      op(GC_OPC_INPUT, 0, GC_IN_PSI, 0);
      op(GC_OPC_MUL, 0, 0, 0);
      break;
    case GC_INTEGRAND_GRAD_SQUARED:  // (gx gx + gy gy) + gz gz in r0..r2, as the recorder lays it out
      f.arity = 2;
      op(GC_OPC_INPUT, 0, GC_IN_GRAD_X, 0);
      op(GC_OPC_INPUT, 1, GC_IN_GRAD_Y, 0);
      op(GC_OPC_INPUT, 2, GC_IN_GRAD_Z, 0);
      op(GC_OPC_MUL, 0, 0, 0);
      op(GC_OPC_MUL, 1, 1, 1);
      op(GC_OPC_ADD, 1, 0, 1);
      op(GC_OPC_MUL, 2, 2, 2);
      op(GC_OPC_ADD, 2, 1, 2);
      break;
    default:  // GC_INTEGRAND_CH_FREE_ENERGY
      f.arity = 2;
      op(GC_OPC_INPUT, 0, GC_IN_PSI, 0);
      op(GC_OPC_INPUT, 1, GC_IN_GRAD_X, 0);
      op(GC_OPC_INPUT, 2, GC_IN_GRAD_Y, 0);
      op(GC_OPC_INPUT, 3, GC_IN_GRAD_Z, 0);
      op(GC_OPC_CONST, 4, 0, 0, -0.5);
      op(GC_OPC_MUL, 4, 4, 0);
      op(GC_OPC_MUL, 4, 4, 0);
      op(GC_OPC_CONST, 5, 0, 0, 0.25);
      for (int q = 0; q < 4; ++q) op(GC_OPC_MUL, 5, 5, 0);
      op(GC_OPC_ADD, 5, 4, 5);
      op(GC_OPC_MUL, 1, 1, 1);  // |grad psi|^2 = (gx gx + gy gy) + gz gz into r3
      op(GC_OPC_MUL, 2, 2, 2);
      op(GC_OPC_ADD, 1, 1, 2);
      op(GC_OPC_MUL, 3, 3, 3);
      op(GC_OPC_ADD, 3, 1, 3);
      op(GC_OPC_CONST, 1, 0, 0, 0.5 * kappa);
      op(GC_OPC_MUL, 1, 1, 3);
      op(GC_OPC_ADD, 5, 5, 1);
      break;
  }
  return f;
}

gc_status evaluate_any(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* psi,
                       const gc_integrand* f, gc_sum sum, double* result) {
  if (f->kind == GC_INTEGRAND_PSI && dt == GC_F64) {  // the field itself: a plain sum
    double s = 0.0;
    const gc_status st = sum_any(ctx, dt, psi, static_cast<long long>(cells(g)), sum, &s);
    *result = g->hx * g->hy * g->hz * s;
    return st;
  }
  const gc_program prog = fixed_program(f->kind, f->kappa);
  return run_program(ctx, g, dt, psi, &prog, sum, result);
}

}  // namespace gcb

using namespace gcb;

extern "C" {

GC_API gc_status gc_integrate(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* in,
                              gc_sum sum, double* result) {
  Call call(ctx);
  gc_status s = call.st;
  if (s != GC_OK) return s;
  if ((s = check_grid(g)) != GC_OK) return s;
  if (!in || !result) return fail(GC_ERR_INVALID_ARG, "gc_integrate: null pointer");
  if (dt != GC_F64 && dt != GC_F32) return fail(GC_ERR_INVALID_ARG, "gc_integrate: unknown dtype");
  double total = 0.0;
  s = sum_any(ctx, dt, in, static_cast<long long>(cells(g)), sum, &total);
  if (s != GC_OK) return s;
  *result = (g->hx * g->hy * g->hz) * total;
  return GC_OK;
}

GC_API gc_status gc_check_finite(gc_context* ctx, const gc_grid* g, gc_dtype dt, int32_t components,
                                 const void* field, int64_t* first_bad) {
  Call call(ctx);
  gc_status s = call.st;
  if (s != GC_OK) return s;
  if ((s = check_grid(g)) != GC_OK) return s;
  if (!field) return fail(GC_ERR_INVALID_ARG, "gc_check_finite: null field pointer");
  if (dt != GC_F64 && dt != GC_F32) return fail(GC_ERR_INVALID_ARG, "gc_check_finite: unknown dtype");
  if (components < 1) return fail(GC_ERR_INVALID_ARG, "gc_check_finite: components must be >= 1");
  void* buf = nullptr;
  if ((s = scratch_get(ctx, kSlotFlags, 64, &buf)) != GC_OK) return s;
  unsigned long long* word = static_cast<unsigned long long*>(buf) + 2;
  GC_CUDA(cudaMemsetAsync(word, 0xff, sizeof(unsigned long long), ctx->stream));
  const long long n = static_cast<long long>(cells(g)) * components;
  const int blocks = ctx->num_sms * 8;
  if (dt == GC_F64)
    first_nonfinite_kernel<double><<<blocks, 256, 0, ctx->stream>>>(static_cast<const double*>(field), n, word);
  else
    first_nonfinite_kernel<float><<<blocks, 256, 0, ctx->stream>>>(static_cast<const float*>(field), n, word);
  GC_CHECK_LAUNCH("first_nonfinite_kernel");
  unsigned long long* host = static_cast<unsigned long long*>(ctx->host_pinned) + 2;
  GC_CUDA(cudaMemcpyAsync(host, word, sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
  GC_CUDA(cudaStreamSynchronize(ctx->stream));
  const long long first = host[0] == ~0ULL ? -1 : static_cast<long long>(host[0]);
  if (first_bad) *first_bad = first;
  if (first < 0) return GC_OK;
  double v = 0.0;
  if (dt == GC_F64) {
    GC_CUDA(cudaMemcpy(&v, static_cast<const double*>(field) + first, sizeof(double), cudaMemcpyDeviceToHost));
  } else {
    float f = 0.f;
    GC_CUDA(cudaMemcpy(&f, static_cast<const float*>(field) + first, sizeof(float), cudaMemcpyDeviceToHost));
    v = f;
  }
  const long long nc = static_cast<long long>(cells(g));
  const long long cell = first % nc;
  const long long i = cell % g->nx, j = (cell / g->nx) % g->ny, k = cell / (static_cast<long long>(g->nx) * g->ny);
  return fail(GC_ERR_NONFINITE, "gc_check_finite: non-finite value " + std::to_string(v) + " at flat index " +
                                    std::to_string(first) + " (component " + std::to_string(first / nc) + ", cell (" +
                                    std::to_string(i) + ", " + std::to_string(j) + ", " + std::to_string(k) + "))");
}

GC_API gc_status gc_integrand_program(const gc_integrand* f, gc_program* out) {
  if (!f || !out) return fail(GC_ERR_INVALID_ARG, "gc_integrand_program: null pointer");
  if (f->kind < GC_INTEGRAND_PSI || f->kind > GC_INTEGRAND_GRAD_SQUARED)
    return fail(GC_ERR_INVALID_ARG, "gc_integrand_program: unknown integrand kind");
  *out = fixed_program(f->kind, f->kappa);
  return GC_OK;
}

GC_API gc_status gc_evaluate(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* psi,
                             const gc_integrand* f, gc_sum sum, double* result) {
  Call call(ctx);
  gc_status s = call.st;
  if (s != GC_OK) return s;
  if ((s = check_grid(g)) != GC_OK) return s;
  if (!psi || !f || !result) return fail(GC_ERR_INVALID_ARG, "gc_evaluate: null pointer");
  if (f->kind < GC_INTEGRAND_PSI || f->kind > GC_INTEGRAND_GRAD_SQUARED)
    return fail(GC_ERR_INVALID_ARG, "gc_evaluate: unknown integrand kind");
  if (f->kind >= GC_INTEGRAND_CH_FREE_ENERGY && (s = require_axes(g, 1)) != GC_OK) return s;
  return evaluate_any(ctx, g, dt, psi, f, sum, result);
}

GC_API gc_status gc_d_max_face(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* D,
                               double* result) {
  Call call(ctx);
  gc_status s = call.st;
  if (s != GC_OK) return s;
  if ((s = check_grid(g)) != GC_OK) return s;
  if (!D || !result) return fail(GC_ERR_INVALID_ARG, "gc_d_max_face: null pointer");
  return d_max_face_any(ctx, g, dt, D, result);
}

}  // extern "C"
