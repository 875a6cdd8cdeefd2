// Ping-pong time stepping with CUDA-graph replay, shared by the
// Cahn-Hilliard and diffusion drivers.
//
// Each step reads the state from one buffer and writes the next state to
// the other (stencil halos of neighbouring CTAs still read the old state).
// A captured graph holds an even number of steps (caller buffer -> context
// buffer -> caller buffer ...), so every replay leaves the state where the
// caller expects it; leftover steps launch directly and an odd count ends
// with one device-to-device copy.
#pragma once

#include <algorithm>
#include <cstring>

#include "common.cuh"

namespace gcb {

// step(src, dst) enqueues one time step on ctx->stream.  `key` identifies
// everything the captured kernels bake in (pointers, sizes, coefficients).
constexpr int kStepsPerGraph = 16;

template <class T, class StepFn>
gc_status run_steps(gc_context* ctx, T* psi, T* other, size_t bytes, int n_steps,
                    const uint64_t (&key_in)[8], StepFn&& step) {
  // A fixed graph unit (16 steps, or the largest even count below n_steps)
  // keeps the key independent of n_steps, so repeated calls replay.
  const int per_graph = n_steps >= kStepsPerGraph ? kStepsPerGraph : n_steps - (n_steps & 1);
  int done = 0;
  if (per_graph >= 2) {
    uint64_t key[8];
    std::memcpy(key, key_in, sizeof key);
    key[0] ^= static_cast<uint64_t>(per_graph) * 0x9E3779B97F4A7C15ULL;
    int slot = -1;
    for (int i = 0; i < gc_context::kGraphSlots; ++i)
      if (ctx->graph_exec[i] && std::memcmp(key, ctx->graph_key[i], sizeof key) == 0) slot = i;
    if (slot < 0) {
      slot = 0;
      for (int i = 1; i < gc_context::kGraphSlots; ++i)
        if (ctx->graph_used[i] < ctx->graph_used[slot]) slot = i;
      if (ctx->graph_exec[slot]) {
        cudaGraphExecDestroy(ctx->graph_exec[slot]);
        ctx->graph_exec[slot] = nullptr;
      }
      cudaGraph_t graph;
      GC_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
      gc_status cs = GC_OK;
      for (int i = 0; i < per_graph && cs == GC_OK; i += 2) {
        cs = step(psi, other);
        if (cs == GC_OK) cs = step(other, psi);
      }
      cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
      if (cs != GC_OK) {
        if (ce == cudaSuccess) cudaGraphDestroy(graph);
        return cs;
      }
      if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
      ce = cudaGraphInstantiate(&ctx->graph_exec[slot], graph, 0);
      cudaGraphDestroy(graph);
      if (ce != cudaSuccess) return cuda_fail(ce, "cudaGraphInstantiate");
      std::memcpy(ctx->graph_key[slot], key, sizeof key);
    }
    ctx->graph_used[slot] = ++ctx->graph_clock;
    for (; done + per_graph <= n_steps; done += per_graph)
      GC_CUDA(cudaGraphLaunch(ctx->graph_exec[slot], ctx->stream));
  }
  T* cur = psi;
  T* nxt = other;
  for (; done < n_steps; ++done) {
    gc_status s = step(cur, nxt);
    if (s != GC_OK) return s;
    std::swap(cur, nxt);
  }
  if (cur != psi) GC_CUDA(cudaMemcpyAsync(psi, cur, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  return GC_OK;
}

}  // namespace gcb
