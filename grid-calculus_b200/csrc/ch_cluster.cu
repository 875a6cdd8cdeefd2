// Cahn-Hilliard time stepping for small 2-D grids: the whole integration in
// ONE launch of one thread-block cluster, with the state resident in shared
// memory.
//
// solve::integrate(psi, computeRhs, dt, n, RK4|ExplicitEuler)
// (solve/RK4.hpp:99-154, solve/ExplicitEuler.hpp:79-112,
// examples/common/cahn_hilliard.hpp:38-59) on a grid of a few ten thousand
// cells (the plain method's 128 x 128 configuration) is bound by launch and
// grid-synchronisation latency, not by memory: the four stage kernels of
// the multi-launch path spend most of each step waiting for the previous
// stage.  Here the grid is split into C horizontal slabs, one per CTA of a
// cluster (C <= 16, one CTA per SM); each CTA keeps its slab of psi, k1, k2,
// k3, the stage input y (two buffers) and mu in shared memory for all
// n_steps steps.  Per stage:
//   cluster barrier            every CTA's y rows of this stage are written
//   pull the 2R halo rows of y above and below the slab from the neighbour
//                              CTAs' shared memory (distributed shared memory)
//   mu = -y + y^3 - kappa lap(y) on the slab plus R halo rows (the halo's mu
//                              is recomputed locally, so mu needs no exchange)
//   k  = M lap(mu) on the slab; the next stage's y = psi + a k goes to the
//                              other y buffer, the last stage forms psi'
// One cluster barrier per stage: y alternates between two buffers, so a CTA
// writing the next stage's y can never overwrite rows a neighbour is still
// pulling (every pull of a buffer ends before its puller reaches the barrier
// after which that buffer is written again).  psi is read from and written
// to global memory once per launch.
//
// Arithmetic: the same reference-ordered helpers as the stage kernels
// (tap_sum, lap_xy, chem_pot, mobility from ch_tile.cuh) and the same RK4
// combination psi + (dt/6 (k1 + k4) + dt/3 (k2 + k3)), so double results are
// bit-identical to the multi-launch path and to the CPU reference.
// The cluster barrier is the hardware barrier.cluster; nothing here spins.
#include <cooperative_groups.h>

#include <algorithm>

#include "ch_tile.cuh"
#include "common.cuh"

namespace cg = cooperative_groups;

namespace gcb {
namespace {

constexpr int kClThreads = 512;
constexpr int kClMaxCtas = 16;
constexpr size_t kClusterSmemMax = 227 * 1024;  // dynamic shared memory one CTA may opt into

template <class T>
struct ClusterArgs {
  StageParams<T> p;  // constants of the RHS (mob, kappa, spacings, nx, ny)
  T* psi;            // global state, read at the start, written at the end
  T half_dt, dt, c6, c3;
  int n_steps;
  int ctas;          // slabs (cluster size)
  int rows_max;      // ceil(ny / ctas)
};

// First row of slab r: r ny / C (slabs differ by at most one row).
__device__ __forceinline__ int slab_start(int r, int ny, int c) {
  return static_cast<int>((static_cast<long long>(r) * ny) / c);
}
// Slab holding global row g: the largest r with slab_start(r) <= g.
__device__ __forceinline__ int slab_of(int g, int ny, int c) {
  return static_cast<int>(((static_cast<long long>(g) + 1) * c + ny - 1) / ny) - 1;
}
// x index i + o wrapped into the row (|o| <= R < nx, or nx == 1).
__device__ __forceinline__ int xwrap(int i, int nx) { return nx == 1 ? 0 : (i < 0 ? i + nx : (i >= nx ? i - nx : i)); }

// Shared-memory bytes of one CTA: psi, (k1, k2, k3), two y buffers of
// rows + 4R rows and mu of rows + 2R rows.
template <class T>
size_t cluster_smem(int order, bool rk4, int rows, int nx) {
  const int R = order / 2;
  const size_t own = static_cast<size_t>(rk4 ? 4 : 1) * rows;
  return sizeof(T) * static_cast<size_t>(nx) * (own + 2 * static_cast<size_t>(rows + 4 * R) + (rows + 2 * R));
}

template <class T, int ORDER, bool RK4>
__global__ void __launch_bounds__(kClThreads, 1) ch_cluster_kernel(const ClusterArgs<T> a) {
  constexpr int R = W<2, ORDER>::R;
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = static_cast<int>(cluster.block_rank());
  const StageParams<T>& p = a.p;
  const int nx = p.nx, ny = p.ny, C = a.ctas, HM = a.rows_max;
  const int j0 = slab_start(rank, ny, C);
  const int rows = slab_start(rank + 1, ny, C) - j0;
  const int tid = threadIdx.x;
  const int own = rows * nx;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ps = reinterpret_cast<T*>(smem_raw);              // [HM][nx]
  T* k1 = ps + static_cast<size_t>(HM) * nx;            // RK4 only
  T* k2 = k1 + static_cast<size_t>(HM) * nx;
  T* k3 = k2 + static_cast<size_t>(HM) * nx;
  T* ybuf0 = RK4 ? k3 + static_cast<size_t>(HM) * nx : k1;  // [HM + 4R][nx], row r at (r + 2R)
  T* ybuf1 = ybuf0 + static_cast<size_t>(HM + 4 * R) * nx;
  T* mu = ybuf1 + static_cast<size_t>(HM + 4 * R) * nx;     // [HM + 2R][nx], row r at (r + R)

  // Load the slab; y of the first stage is psi.
  for (int e = tid; e < own; e += kClThreads) {
    const T v = a.psi[static_cast<size_t>(j0) * nx + e];
    ps[e] = v;
    ybuf0[2 * R * nx + e] = v;
  }

  constexpr int kStages = RK4 ? 4 : 1;
  int cur = 0;
  for (int step = 0; step < a.n_steps; ++step) {
#pragma unroll 1
    for (int s = 0; s < kStages; ++s) {
      T* y = cur ? ybuf1 : ybuf0;
      T* yn = cur ? ybuf0 : ybuf1;
      cluster.sync();  // y rows of this stage written everywhere (and this CTA's own loads/stores)
      // Halo rows of y: 2R above and 2R below the slab, from their owners.
      for (int e = tid; e < 4 * R * nx; e += kClThreads) {
        const int q = e / nx, i = e - q * nx;
        const int lr = q < 2 * R ? q - 2 * R : rows + (q - 2 * R);
        int g = j0 + lr;
        g = ((g % ny) + ny) % ny;
        const int owner = slab_of(g, ny, C);
        const T* src = cluster.map_shared_rank(cur ? ybuf1 : ybuf0, owner);
        y[(lr + 2 * R) * nx + i] = src[(g - slab_start(owner, ny, C) + 2 * R) * nx + i];
      }
      __syncthreads();
      // mu on rows -R .. rows + R - 1.
      for (int e = tid; e < (rows + 2 * R) * nx; e += kClThreads) {
        const int q = e / nx, i = e - q * nx;  // q = local row + R
        const T* yr = y + (q + R) * nx;        // row q - R, at index (q - R) + 2R
        const T yc = yr[i];
        const T ax = tap_sum<T, 2, ORDER>([&](int o) { return o == 0 ? yc : yr[xwrap(i + o, nx)]; });
        const T ay = tap_sum<T, 2, ORDER>([&](int o) { return yr[o * nx + i]; });
        T lap = lap_xy(p, ax, ay);
        if constexpr (ORDER != 2) lap = lap_z(p, lap, tap_sum<T, 2, ORDER>([&](int) { return yc; }));
        mu[q * nx + i] = chem_pot(p, yc, lap);
      }
      __syncthreads();
      // k = M lap(mu) on the slab, then this stage's update.
      for (int e = tid; e < own; e += kClThreads) {
        const int r = e / nx, i = e - r * nx;
        const T* mr = mu + (r + R) * nx;
        const T mc = mr[i];
        const T ax = tap_sum<T, 2, ORDER>([&](int o) { return o == 0 ? mc : mr[xwrap(i + o, nx)]; });
        const T ay = tap_sum<T, 2, ORDER>([&](int o) { return mr[o * nx + i]; });
        T lap = lap_xy(p, ax, ay);
        if constexpr (ORDER != 2) lap = lap_z(p, lap, tap_sum<T, 2, ORDER>([&](int) { return mc; }));
        const T rhs = mobility(p, lap);
        const int yo = (r + 2 * R) * nx + i;
        if constexpr (RK4) {
          if (s == 0) {
            k1[e] = rhs;
            yn[yo] = Ar<T>::add(ps[e], Ar<T>::mul(a.half_dt, rhs));
          } else if (s == 1) {
            k2[e] = rhs;
            yn[yo] = Ar<T>::add(ps[e], Ar<T>::mul(a.half_dt, rhs));
          } else if (s == 2) {
            k3[e] = rhs;
            yn[yo] = Ar<T>::add(ps[e], Ar<T>::mul(a.dt, rhs));
          } else {
            const T s14 = Ar<T>::add(k1[e], rhs);
            const T s23 = Ar<T>::add(k2[e], k3[e]);
            const T v = Ar<T>::add(ps[e], Ar<T>::add(Ar<T>::mul(a.c6, s14), Ar<T>::mul(a.c3, s23)));
            ps[e] = v;
            yn[yo] = v;
          }
        } else {
          const T v = Ar<T>::add(ps[e], Ar<T>::mul(a.dt, rhs));
          ps[e] = v;
          yn[yo] = v;
        }
      }
      cur ^= 1;
    }
  }
  __syncthreads();
  for (int e = tid; e < own; e += kClThreads) a.psi[static_cast<size_t>(j0) * nx + e] = ps[e];
  // No CTA may exit while a neighbour could still read its shared memory.
  cluster.sync();
}

template <class T, int ORDER, bool RK4>
gc_status launch_cluster(gc_context* ctx, const ClusterArgs<T>& a, size_t smem, bool* launched) {
  auto kern = ch_cluster_kernel<T, ORDER, RK4>;
  if (a.ctas > 8) GC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  GC_TRY(kernel_setup(kern, kClThreads, smem));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(a.ctas, 1, 1);
  cfg.blockDim = dim3(kClThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = a.ctas;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  // A cluster of this size with this much shared memory per CTA must be
  // schedulable; otherwise the caller takes the multi-launch path.
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) != cudaSuccess || clusters < 1) {
    cudaGetLastError();
    *launched = false;
    return GC_OK;
  }
  GC_CUDA(cudaLaunchKernelEx(&cfg, kern, a));
  GC_CHECK_LAUNCH("ch_cluster_kernel");
  *launched = true;
  return GC_OK;
}

// Cluster size for a 2-D grid: the fewest CTAs (at least 8 where the grid
// has the rows, for parallel arithmetic) whose slab fits in one SM's shared
// memory; 0 when even 16 slabs do not fit.
int cluster_plan(const gc_grid* g, size_t elem, int order, bool rk4, size_t* smem) {
  if (g->nz != 1 || g->nx < 1 || g->ny < 1) return 0;
  for (int c = std::min(8, g->ny); c <= std::min(kClMaxCtas, g->ny); ++c) {
    const int rows = (g->ny + c - 1) / c;
    const size_t b = elem == 8 ? cluster_smem<double>(order, rk4, rows, g->nx)
                               : cluster_smem<float>(order, rk4, rows, g->nx);
    if (b <= kClusterSmemMax) {
      if (smem) *smem = b;
      return c;
    }
  }
  return 0;
}

template <class T>
gc_status cluster_integrate_t(gc_context* ctx, const gc_grid* g, const gc_ch_params* cp, T* psi, double dt,
                              int n_steps, gc_integrator integ, bool* done) {
  *done = false;
  const bool rk4 = integ == GC_RK4;
  size_t smem = 0;
  const int ctas = cluster_plan(g, sizeof(T), cp->order, rk4, &smem);
  if (ctas == 0) return GC_OK;
  ClusterArgs<T> a{};
  StageParams<T>& p = a.p;
  p.nx = g->nx; p.ny = g->ny; p.nz = 1;
  p.ihx2 = static_cast<T>(1.0 / (g->hx * g->hx));
  p.ihy2 = static_cast<T>(1.0 / (g->hy * g->hy));
  p.ihz2 = static_cast<T>(1.0 / (g->hz * g->hz));
  p.mob = static_cast<T>(cp->mobility);
  p.kappa = static_cast<T>(cp->kappa);
  p.unit_h = p.ihx2 == T(1) && p.ihy2 == T(1) && p.ihz2 == T(1);
  p.unit_m = p.mob == T(1);
  p.unit_k = p.kappa == T(1);
  a.psi = psi;
  a.half_dt = static_cast<T>(0.5 * dt);
  a.dt = static_cast<T>(dt);
  a.c6 = static_cast<T>(dt / 6.0);
  a.c3 = static_cast<T>(dt / 3.0);
  a.n_steps = n_steps;
  a.ctas = ctas;
  a.rows_max = (g->ny + ctas - 1) / ctas;
  switch (cp->order) {
    case 2: return rk4 ? launch_cluster<T, 2, true>(ctx, a, smem, done) : launch_cluster<T, 2, false>(ctx, a, smem, done);
    case 4: return rk4 ? launch_cluster<T, 4, true>(ctx, a, smem, done) : launch_cluster<T, 4, false>(ctx, a, smem, done);
    case 6: return rk4 ? launch_cluster<T, 6, true>(ctx, a, smem, done) : launch_cluster<T, 6, false>(ctx, a, smem, done);
  }
  return GC_OK;
}

}  // namespace

gc_status ch_cluster_integrate(gc_context* ctx, const gc_grid* g, gc_dtype dt, const gc_ch_params* cp, void* psi,
                               double dt_step, int n_steps, gc_integrator integ, bool* done) {
  *done = false;
  if (g->nz != 1 || n_steps < 1) return GC_OK;
  if (dt == GC_F64)
    return cluster_integrate_t<double>(ctx, g, cp, static_cast<double*>(psi), dt_step, n_steps, integ, done);
  return cluster_integrate_t<float>(ctx, g, cp, static_cast<float*>(psi), dt_step, n_steps, integ, done);
}

}  // namespace gcb

GC_API int32_t gc_ch_cluster_ctas(const gc_grid* g, gc_dtype dt, int32_t order, gc_integrator integ) {
  if (!g || (order != 2 && order != 4 && order != 6) || (dt != GC_F64 && dt != GC_F32)) return 0;
  return gcb::cluster_plan(g, dt == GC_F64 ? 8 : 4, order, integ == GC_RK4, nullptr);
}
