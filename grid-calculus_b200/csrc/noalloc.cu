// gc_integrate_noalloc: func::integrate (Pairwise tag) for callers that
// cannot allocate device memory.
//
// Who needs it: applications whose device memory is owned entirely by
// another allocator (a framework's caching allocator or a solver that
// reserves the whole device up front), plug-in hosts that hand a library
// only the buffers it is given, and real-time loops that forbid allocation
// once they are running.  Such callers cannot create a gc_context (that
// allocates a stream, events, pinned host memory and scratch on demand).
//
// How: the same kernels as gc_integrate (pairwise.cuh), with the chunk
// partials in the file-scope device array below instead of context scratch,
// launched on the caller's stream, and the result (cell volume times the
// sum) written to a device double the caller passes.  No cudaMalloc,
// cudaFree or allocating library routine is called.
//
// The array is 65600 doubles (525 KB) and every GPU that loads this library
// holds it until the process exits.  It bounds the field to
// kNoAllocMaxCells = 2^29 values (65536 chunks of 8192).  All calls share
// it: calls whose work overlaps on the GPU (different streams, or different
// host threads on one device) race on it, so order them on one stream.
// Nothing in it needs to start at zero: every call writes each partial it
// later reads.
//
// Host code must not pass the array's name to a kernel: in host code it is
// a host-side stand-in, not a device address.  The first call on each
// device, with that device current, looks up the device address with
// cudaGetSymbolAddress (and sets the chunk kernel's shared-memory limit) and
// keeps both for the life of the process; make that first call before any
// stream capture, and do not reset the device after it (cudaDeviceReset
// unloads the module, which would leave the kept address stale).
#include <mutex>
#include <string>

#include "common.cuh"
#include "pairwise.cuh"

namespace gcb {
namespace {

constexpr long long kNoAllocMaxChunks = 65536;
constexpr long long kNoAllocMaxCells = kNoAllocMaxChunks * kChunkMax;  // 2^29
// Chunk partials (65536) plus the first group-reduction level (64).
constexpr int kNoAllocSlots = static_cast<int>(kNoAllocMaxChunks + kNoAllocMaxChunks / 1024);

static __device__ __align__(256) double g_noalloc_partials[kNoAllocSlots];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_partials_ptr[kMaxDevices] = {};

__global__ void scale_store(const double* __restrict__ sum, double vol, double* __restrict__ out) {
  out[0] = __dmul_rn(vol, sum[0]);
}

// Per-device set-up with the device current: the array's device address and
// the dynamic shared-memory limit of the chunk kernels.
gc_status setup(int device, double** partials) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (g_partials_ptr[device]) {
    *partials = g_partials_ptr[device];
    return GC_OK;
  }
  void* ptr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_partials);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_partials)");
  const int smem = static_cast<int>(sizeof(double) * (padpos(kChunkMax) + 8 + kNodeMax));
  e = cudaFuncSetAttribute(pairwise_chunks<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(pairwise_chunks<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(pairwise_chunks)");
  g_partials_ptr[device] = static_cast<double*>(ptr);
  *partials = g_partials_ptr[device];
  return GC_OK;
}

template <class T>
gc_status run(const T* x, long long n, double vol, double* result, cudaStream_t stream, double* a, int sms) {
  int depth = 0;
  while (((n + (1LL << depth) - 1) >> depth) > kChunkMax) ++depth;
  const long long nchunks = 1LL << depth;
  double* b = a + kNoAllocMaxChunks;
  const size_t smem = sizeof(double) * (padpos(kChunkMax) + 8 + kNodeMax);
  const long long grid = nchunks < 3LL * sms ? nchunks : 3LL * sms;
  pairwise_chunks<T><<<static_cast<unsigned>(grid), kSumThreads, smem, stream>>>(x, n, depth, nchunks, a);
  GC_CHECK_LAUNCH("pairwise_chunks (noalloc)");
  long long count = nchunks;
  double* src = a;
  double* dst = b;
  while (count > 1) {
    const int group = static_cast<int>(count < 1024 ? count : 1024);
    const long long blocks = count / group;
    tree_groups<<<static_cast<unsigned>(blocks), 1024, 0, stream>>>(src, count, group, dst);
    GC_CHECK_LAUNCH("tree_groups (noalloc)");
    count = blocks;
    double* t = src;
    src = dst;
    dst = t;
  }
  scale_store<<<1, 1, 0, stream>>>(src, vol, result);
  GC_CHECK_LAUNCH("scale_store (noalloc)");
  return GC_OK;
}

}  // namespace
}  // namespace gcb

using namespace gcb;

extern "C" {

GC_API gc_status gc_integrate_noalloc(const gc_grid* g, gc_dtype dt, const void* in,
                                      double* result_dev, void* stream) {
  gc_status s = check_grid(g);
  if (s != GC_OK) return s;
  if (!in || !result_dev) return fail(GC_ERR_INVALID_ARG, "gc_integrate_noalloc: null pointer");
  if (dt != GC_F64 && dt != GC_F32) return fail(GC_ERR_INVALID_ARG, "gc_integrate_noalloc: unknown dtype");
  const long long n = static_cast<long long>(cells(g));
  if (n > kNoAllocMaxCells) {
    return fail(GC_ERR_INVALID_ARG,
                "gc_integrate_noalloc: the field has " + std::to_string(n) +
                    " cells, more than the fixed scratch of this entry point allows (" +
                    std::to_string(kNoAllocMaxCells) + " = 2^29); use gc_integrate");
  }
  int device = 0;
  GC_CUDA(cudaGetDevice(&device));
  if (device < 0 || device >= kMaxDevices)
    return fail(GC_ERR_INVALID_ARG, "gc_integrate_noalloc: device index out of range");
  int sms = 148;
  GC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  double* partials = nullptr;
  if ((s = setup(device, &partials)) != GC_OK) return s;
  const double vol = g->hx * g->hy * g->hz;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dt == GC_F64) return run(static_cast<const double*>(in), n, vol, result_dev, st, partials, sms);
  return run(static_cast<const float*>(in), n, vol, result_dev, st, partials, sms);
}

}  // extern "C"
