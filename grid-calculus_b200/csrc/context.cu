// Context, error state, scratch and memory helpers of the C ABI.
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "common.cuh"

namespace gcb {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }

gc_status fail(gc_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

gc_status cuda_fail(cudaError_t e, const char* what) {
  g_last_error = std::string("gridcalc_b200: CUDA error in ") + what + ": " + cudaGetErrorString(e);
  return GC_ERR_CUDA;
}

gc_status check_ctx(gc_context* ctx) {
  if (!ctx) return fail(GC_ERR_INVALID_ARG, "gridcalc_b200: null context");
  GC_CUDA(cudaSetDevice(ctx->device));
  return GC_OK;
}

Call::Call(gc_context* c) : ctx(c), st(check_ctx(c)) {
  if (st != GC_OK) return;
  cudaError_t e = cudaEventRecord(ctx->ev_in, ctx->user_stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->stream, ctx->ev_in, 0);
  if (e != cudaSuccess) st = cuda_fail(e, "joining the caller stream");
}

Call::~Call() {
  if (!ctx || !ctx->ev_out) return;
  if (cudaEventRecord(ctx->ev_out, ctx->stream) == cudaSuccess)
    cudaStreamWaitEvent(ctx->user_stream, ctx->ev_out, 0);
}

gc_status kernel_setup_raw(const void* kern, int threads, size_t smem, int* ctas_per_sm) {
  int dev = 0;
  GC_CUDA(cudaGetDevice(&dev));
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> smem_set;             // (kernel, device) -> bytes
  static std::map<std::tuple<const void*, int, int, size_t>, int> occupancy;  // (kernel, device, threads, bytes)
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair(kern, dev);
  auto it = smem_set.find(key);
  if (smem > 48 * 1024 && (it == smem_set.end() || it->second < smem)) {
    GC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    smem_set[key] = smem;
  }
  if (ctas_per_sm) {
    const auto okey = std::make_tuple(kern, dev, threads, smem);
    auto ot = occupancy.find(okey);
    if (ot == occupancy.end()) {
      int n = 0;
      GC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, threads, smem));
      ot = occupancy.emplace(okey, n < 1 ? 1 : n).first;
    }
    *ctas_per_sm = ot->second;
  }
  return GC_OK;
}

// core::Grid constructor preconditions (core/Grid.hpp:39-52).
gc_status check_grid(const gc_grid* g) {
  if (!g) return fail(GC_ERR_INVALID_ARG, "gridcalc_b200: null grid");
  if (g->nx <= 0 || g->ny <= 0 || g->nz <= 0) {
    return fail(GC_ERR_INVALID_ARG, "Grid: extents (Nx, Ny, Nz) must be > 0; got (" +
                                        std::to_string(g->nx) + ", " + std::to_string(g->ny) +
                                        ", " + std::to_string(g->nz) + ")");
  }
  if (!(g->hx > 0.0) || !(g->hy > 0.0) || !(g->hz > 0.0)) {
    return fail(GC_ERR_INVALID_ARG, "Grid: cell_size components must be > 0; got (" +
                                        std::to_string(g->hx) + ", " + std::to_string(g->hy) +
                                        ", " + std::to_string(g->hz) + ")");
  }
  return GC_OK;
}

// diff::detail::requireAxisExtent (diff/detail/PreconditionAxisExtent.hpp:64-79).
static gc_status require_axis(const char* axis, int n, int radius) {
  if (radius == 0 || n == 1) return GC_OK;
  const int min_n = 2 * radius + 1;
  if (n < min_n) {
    return fail(GC_ERR_AXIS_EXTENT,
                std::string("gridcalc: axis ") + axis + " has N=" + std::to_string(n) +
                    " but the requested stencil has radius " + std::to_string(radius) +
                    ", which requires N>=" + std::to_string(min_n) +
                    " on a periodic grid (or N=1 for a degenerate axis); intermediate extents "
                    "alias the [-r, r] offsets under the periodic wrap and the stencil silently "
                    "degrades. Use a larger grid or a lower-Order stencil.");
  }
  return GC_OK;
}

gc_status require_axes(const gc_grid* g, int radius) {
  gc_status s = check_grid(g);
  if (s != GC_OK) return s;
  if ((s = require_axis("x", g->nx, radius)) != GC_OK) return s;
  if ((s = require_axis("y", g->ny, radius)) != GC_OK) return s;
  return require_axis("z", g->nz, radius);
}

gc_status require_axes3(const gc_grid* g, int rx, int ry, int rz) {
  gc_status s = check_grid(g);
  if (s != GC_OK) return s;
  if ((s = require_axis("x", g->nx, rx)) != GC_OK) return s;
  if ((s = require_axis("y", g->ny, ry)) != GC_OK) return s;
  return require_axis("z", g->nz, rz);
}

gc_status scratch_get(gc_context* ctx, int slot, size_t bytes, void** out) {
  Scratch& s = ctx->scratch[slot];
  if (s.bytes < bytes) {
    if (s.ptr) GC_CUDA(cudaFree(s.ptr));
    s.ptr = nullptr;
    s.bytes = 0;
    // Round up to 2 MiB so that nearby sizes reuse one allocation.
    const size_t rounded = (bytes + (size_t(2) << 20) - 1) & ~((size_t(2) << 20) - 1);
    GC_CUDA(cudaMalloc(&s.ptr, rounded));
    s.bytes = rounded;
  }
  *out = s.ptr;
  return GC_OK;
}

}  // namespace gcb

using namespace gcb;

extern "C" {

GC_API const char* gc_last_error(void) { return g_last_error.c_str(); }

GC_API const char* gc_version(void) { return "0.15.1-b200"; }

GC_API const char* gc_status_string(gc_status s) {
  switch (s) {
    case GC_OK: return "GC_OK";
    case GC_ERR_INVALID_ARG: return "GC_ERR_INVALID_ARG";
    case GC_ERR_AXIS_EXTENT: return "GC_ERR_AXIS_EXTENT";
    case GC_ERR_GRID_MISMATCH: return "GC_ERR_GRID_MISMATCH";
    case GC_ERR_NONPOSITIVE_D: return "GC_ERR_NONPOSITIVE_D";
    case GC_ERR_CFL: return "GC_ERR_CFL";
    case GC_ERR_CUDA: return "GC_ERR_CUDA";
    case GC_ERR_TIMEOUT: return "GC_ERR_TIMEOUT";
    case GC_ERR_NONFINITE: return "GC_ERR_NONFINITE";
    case GC_ERR_UNSUPPORTED: return "GC_ERR_UNSUPPORTED";
    case GC_ERR_IO: return "GC_ERR_IO";
  }
  return "GC_ERR_UNKNOWN";
}

GC_API gc_status gc_context_create(gc_context** out, int device, void* stream) {
  if (!out) return fail(GC_ERR_INVALID_ARG, "gc_context_create: null out");
  *out = nullptr;
  int count = 0;
  GC_CUDA(cudaGetDeviceCount(&count));
  if (device < 0 || device >= count) {
    return fail(GC_ERR_INVALID_ARG, "gc_context_create: device " + std::to_string(device) +
                                        " out of range (" + std::to_string(count) + " devices)");
  }
  GC_CUDA(cudaSetDevice(device));
  gc_context* ctx = new gc_context();
  ctx->device = device;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) ctx->num_sms = prop.multiProcessorCount;
  ctx->user_stream = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_in, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_out, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMallocHost(&ctx->host_pinned, 4096);
  if (e == cudaSuccess) e = cudaMalloc(&ctx->device_status, 256);
  if (e == cudaSuccess) e = cudaMemset(ctx->device_status, 0, 256);
  if (e != cudaSuccess) {
    if (ctx->device_status) cudaFree(ctx->device_status);
    if (ctx->host_pinned) cudaFreeHost(ctx->host_pinned);
    if (ctx->ev_in) cudaEventDestroy(ctx->ev_in);
    if (ctx->ev_out) cudaEventDestroy(ctx->ev_out);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return cuda_fail(e, "gc_context_create");
  }
  *out = ctx;
  return GC_OK;
}

GC_API gc_status gc_context_set_option(gc_context* ctx, int32_t option, int32_t value) {
  if (!ctx) return fail(GC_ERR_INVALID_ARG, "gridcalc_b200: null context");
  switch (option) {
    case GC_OPT_CLUSTER_STEPPING: ctx->cluster_stepping = value != 0; return GC_OK;
    case GC_OPT_FUSED_STEP: ctx->fused_step = value != 0; return GC_OK;
  }
  return fail(GC_ERR_INVALID_ARG, "gc_context_set_option: unknown option " + std::to_string(option));
}

GC_API gc_status gc_context_destroy(gc_context* ctx) {
  if (!ctx) return GC_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto& ge : ctx->graph_exec)
    if (ge) cudaGraphExecDestroy(ge);
  if (ctx->spectral_release) ctx->spectral_release(ctx->spectral_plans);
  for (auto& s : ctx->scratch)
    if (s.ptr) cudaFree(s.ptr);
  if (ctx->host_pinned) cudaFreeHost(ctx->host_pinned);
  if (ctx->device_status) cudaFree(ctx->device_status);
  if (ctx->ev_in) cudaEventDestroy(ctx->ev_in);
  if (ctx->ev_out) cudaEventDestroy(ctx->ev_out);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return GC_OK;
}

namespace gcb {
// Waits on a device flag that nothing sets, for at most `budget` clock
// cycles, then records GC_ERR_TIMEOUT in the status word and returns: the
// same bounded-wait path the TMA pipeline takes when a tile never arrives.
__global__ void bounded_wait_selftest(const volatile int* flag, long long budget, int* status) {
  const long long t0 = clock64();
  while (*flag == 0) {
    if (clock64() - t0 > budget) {
      atomicExch(status, static_cast<int>(GC_ERR_TIMEOUT));
      return;
    }
  }
}
}  // namespace gcb

GC_API gc_status gc_selftest_bounded_wait(gc_context* ctx, int64_t budget_cycles) {
  Call call(ctx);
  gc_status s = call.st;
  if (s != GC_OK) return s;
  if (budget_cycles < 0 || budget_cycles > 4000000000LL)
    return fail(GC_ERR_INVALID_ARG, "gc_selftest_bounded_wait: budget must be in [0, 4e9] cycles");
  // ints 32..63 of the 256-byte status block are never written after creation
  gcb::bounded_wait_selftest<<<1, 1, 0, ctx->stream>>>(ctx->device_status + 32, budget_cycles, ctx->device_status);
  GC_CHECK_LAUNCH("bounded_wait_selftest");
  return GC_OK;
}

GC_API gc_status gc_synchronize(gc_context* ctx) {
  Call call(ctx);
  gc_status s = call.st;
  if (s != GC_OK) return s;
  int* host = static_cast<int*>(ctx->host_pinned) + 64;
  GC_CUDA(cudaMemcpyAsync(host, ctx->device_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  GC_CUDA(cudaStreamSynchronize(ctx->stream));
  if (*host != 0) {
    GC_CUDA(cudaMemsetAsync(ctx->device_status, 0, sizeof(int), ctx->stream));
    GC_CUDA(cudaStreamSynchronize(ctx->stream));
    return fail(GC_ERR_TIMEOUT, "gridcalc_b200: a bounded device wait gave up (TMA tile not delivered); "
                                "the results of the affected calls are undefined");
  }
  return GC_OK;
}

GC_API gc_status gc_malloc(gc_context* ctx, size_t bytes, void** dev) {
  Call call(ctx);
  gc_status s = call.st;
  if (s != GC_OK) return s;
  if (!dev) return fail(GC_ERR_INVALID_ARG, "gc_malloc: null out");
  GC_CUDA(cudaMalloc(dev, bytes));
  return GC_OK;
}

GC_API gc_status gc_free(gc_context* ctx, void* dev) {
  Call call(ctx);
  gc_status s = call.st;
  if (s != GC_OK) return s;
  GC_CUDA(cudaFree(dev));
  return GC_OK;
}

GC_API gc_status gc_memcpy_h2d(gc_context* ctx, void* dev, const void* host, size_t bytes) {
  Call call(ctx);
  gc_status s = call.st;
  if (s != GC_OK) return s;
  GC_CUDA(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, ctx->stream));
  return GC_OK;
}

GC_API gc_status gc_memcpy_d2h(gc_context* ctx, void* host, const void* dev, size_t bytes) {
  Call call(ctx);
  gc_status s = call.st;
  if (s != GC_OK) return s;
  GC_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  GC_CUDA(cudaStreamSynchronize(ctx->stream));
  return GC_OK;
}

}  // extern "C"
