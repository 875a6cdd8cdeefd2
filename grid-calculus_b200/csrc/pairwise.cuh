// Exact pairwise-sum kernels (func::integrate with the Pairwise tag,
// func/Integrate.hpp:65-74), shared by the context entry point (reduce.cu)
// and the allocation-free entry point (noalloc.cu).  See reduce.cu for how
// the reference's recursion tree is reproduced.
#pragma once

#include "common.cuh"

namespace gcb {
namespace {

constexpr int kChunkMax = 8192;   // values per chunk (layer 1)
constexpr int kNodeMax = 128;     // values per thread node
constexpr int kSumThreads = 256;

__host__ __device__ constexpr int padpos(int e) { return e + (e >> 6); }

// [lo, hi) of node `idx` at depth `depth` below the range [lo, hi).
__device__ __forceinline__ void descend(long long& lo, long long& hi, long long idx, int depth) {
  for (int b = depth - 1; b >= 0; --b) {
    const long long mid = lo + (hi - lo) / 2;
    if ((idx >> b) & 1) lo = mid;
    else hi = mid;
  }
}

__device__ __forceinline__ double seq_sum(const double* s, int a, int b) {
  double acc = 0.0;
  for (int e = a; e < b; ++e) acc = __dadd_rn(acc, s[padpos(e)]);
  return acc;
}

template <class T>
__global__ void __launch_bounds__(kSumThreads) pairwise_chunks(const T* __restrict__ x, long long n,
                                                               int depth, long long nchunks,
                                                               double* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* s = reinterpret_cast<double*>(smem_raw);                 // padded chunk
  double* ns = s + padpos(kChunkMax) + 8;                           // node sums
  for (long long c = blockIdx.x; c < nchunks; c += gridDim.x) {
    long long lo = 0, hi = n;
    descend(lo, hi, c, depth);
    const int len = static_cast<int>(hi - lo);
    const T* src = x + lo;
#pragma unroll 8
    for (int e = threadIdx.x; e < len; e += kSumThreads) s[padpos(e)] = static_cast<double>(src[e]);
    // Depth below the chunk at which every node holds <= kNodeMax values.
    int d2 = 0;
    while (((len + (1 << d2) - 1) >> d2) > kNodeMax) ++d2;
    const int nodes = 1 << d2;
    __syncthreads();
    if (threadIdx.x < nodes) {
      long long a = 0, b = len;
      descend(a, b, threadIdx.x, d2);
      const int m = static_cast<int>(b - a);
      double v;
      if (m <= 64) {
        v = seq_sum(s, static_cast<int>(a), static_cast<int>(b));
      } else {
        const int h = m / 2;
        v = __dadd_rn(seq_sum(s, static_cast<int>(a), static_cast<int>(a) + h),
                      seq_sum(s, static_cast<int>(a) + h, static_cast<int>(b)));
      }
      ns[threadIdx.x] = v;
    }
    __syncthreads();
    // Adjacent pairs (2i, 2i+1) at every level, as the recursion pairs them;
    // read and write are separated by a barrier (in place would race).
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

// Reduces each group of `group` (a power of two) consecutive values to one,
// as a perfect binary tree.
__global__ void __launch_bounds__(1024) tree_groups(const double* __restrict__ in, long long count,
                                                    int group, double* __restrict__ out) {
  __shared__ double t[1024];
  const long long base = static_cast<long long>(blockIdx.x) * group;
  for (int i = threadIdx.x; i < group; i += blockDim.x) t[i] = (base + i < count) ? in[base + i] : 0.0;
  __syncthreads();
  for (int w = group >> 1; w >= 1; w >>= 1) {
    double v = 0.0;
    if (threadIdx.x < w) v = __dadd_rn(t[2 * threadIdx.x], t[2 * threadIdx.x + 1]);
    __syncthreads();
    if (threadIdx.x < w) t[threadIdx.x] = v;
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = t[0];
}

}  // namespace
}  // namespace gcb
