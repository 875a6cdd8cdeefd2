// Finite-volume heterogeneous diffusion and the constant-D heat equation.
//
// RHS kinds:
//   KIND_FVM  fvm::cellLaplacian (fvm/CellLaplacian.hpp:91-143):
//             sum over axes of [D+ (psi+ - psi) - D- (psi - psi-)] / h^2 with
//             harmonic-mean faces D = 2ab/(a+b) (fvm/CellLaplacian.hpp:48-50);
//   KIND_LAP  diff::laplacian<2> (diff/Laplacian.hpp:44-75), the RHS of
//             solve::diffuse(psi, double D, ...) (solve/Diffusion.hpp:106-111).
// A stage kernel stages y = psi + a k_prev (and D) with a one-cell periodic
// halo in shared memory and writes k_s, or psi' on the last stage.  A single
// cellLaplacian, and float stepping, form the face coefficients on the fly
// from the staged D; 3-D double stepping computes the three face fields once
// per call (D is constant) and its z-march stages read faces instead of D:
// RK4 then costs 13 field passes plus 4 x 3 face reads per step, and no
// division.
#include <algorithm>
#include <type_traits>

#include "common.cuh"
#include "stepper.cuh"

namespace gcb {

gc_status d_max_face_any(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* D, double* result);
gc_status first_nonpositive(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* D, long long* first);

namespace {

constexpr int kThreads = 256;
enum RhsKind { KIND_FVM = 0, KIND_LAP = 1 };
enum StageMode { MODE_RHS = 0, MODE_RK4_FINAL = 1, MODE_EULER_FINAL = 2 };

template <class T>
struct FvmParams {
  const T* psi;
  const T* kin;
  T a;
  T* out;
  const T* D;
  const T* k1;
  const T* k2;
  const T* k3;
  // Precomputed faces (z-march stepping): f*[c] = hmean(D[c], D[c + e_axis]),
  // the +x / +y / +z face of cell c and the - face of its neighbour.
  const T* fx;
  const T* fy;
  const T* fz;
  T c6, c3;
  T ihx2, ihy2, ihz2;
  int nx, ny, nz;
};

template <bool Z3>
struct FvmTile;
template <> struct FvmTile<false> { static constexpr int TX = 64, TY = 16, TZ = 1; };
template <> struct FvmTile<true> { static constexpr int TX = 32, TY = 16, TZ = 8; };

// Face coefficient 2ab / (a + b) (reference fvm/CellLaplacian.hpp:48-50).  Double
// keeps the reference's rounding; float, the precision variant, uses the fast
// division intrinsic (2 ulp for the positive, normal-range coefficients the
// positivity check admits): six IEEE divisions per cell would otherwise
// dominate the kernel's issue slots.
template <class T>
__device__ __forceinline__ T hmean(T a, T b) {
  return Ar<T>::div(Ar<T>::mul(Ar<T>::mul(T(2), a), b), Ar<T>::add(a, b));
}
template <>
__device__ __forceinline__ float hmean<float>(float a, float b) {
  return __fdividef(2.0f * a * b, a + b);
}

// The three face fields of D for a whole stepping call: D is constant over
// the call, so every face is computed once instead of twice per RHS
// evaluation (and the stage kernels read faces, not D and its neighbours).
template <class T>
__global__ void __launch_bounds__(kThreads) fvm_faces_kernel(const T* __restrict__ D, T* __restrict__ fx,
                                                             T* __restrict__ fy, T* __restrict__ fz, int nx, int ny,
                                                             int nz) {
  const size_t plane = static_cast<size_t>(nx) * ny;
  const size_t n = plane * nz;
  for (size_t c = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < n;
       c += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(c % nx);
    const size_t rest = c / nx;
    const int j = static_cast<int>(rest % ny);
    const int k = static_cast<int>(rest / ny);
    const T dc = D[c];
    fx[c] = hmean(dc, D[c - i + (i + 1 == nx ? 0 : i + 1)]);
    fy[c] = hmean(dc, D[static_cast<size_t>(k) * plane + static_cast<size_t>(j + 1 == ny ? 0 : j + 1) * nx + i]);
    fz[c] = hmean(dc, D[static_cast<size_t>(k + 1 == nz ? 0 : k + 1) * plane + static_cast<size_t>(j) * nx + i]);
  }
}

template <class T, int KIND, bool Z3, int MODE>
__global__ void __launch_bounds__(kThreads) fvm_stage_kernel(const FvmParams<T> p) {
  constexpr int TX = FvmTile<Z3>::TX, TY = FvmTile<Z3>::TY, TZ = FvmTile<Z3>::TZ;
  constexpr int RZ = Z3 ? 1 : 0;
  constexpr int YX = TX + 2, YY = TY + 2, YZ = TZ + 2 * RZ;
  constexpr int YN = YX * YY * YZ, ON = TX * TY * TZ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ys = reinterpret_cast<T*>(smem_raw);
  T* ds = ys + YN;

  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * TZ;
  const size_t plane = static_cast<size_t>(nx) * ny;

  for (int e = threadIdx.x; e < YN; e += kThreads) {
    const int ex = e % YX;
    const int rest = e / YX;
    const int ey = rest % YY;
    const int ez = rest / YY;
    const int gx = wrap(x0 - 1 + ex, nx);
    const int gy = wrap(y0 - 1 + ey, ny);
    const int gz = Z3 ? wrap(z0 - 1 + ez, nz) : 0;
    const size_t gi = static_cast<size_t>(gz) * plane + static_cast<size_t>(gy) * nx + gx;
    T v = __ldg(p.psi + gi);
    if (p.kin) v = Ar<T>::add(v, Ar<T>::mul(p.a, __ldg(p.kin + gi)));
    ys[e] = v;
    if constexpr (KIND == KIND_FVM) ds[e] = __ldg(p.D + gi);
  }
  __syncthreads();

  for (int e = threadIdx.x; e < ON; e += kThreads) {
    const int ex = e % TX;
    const int rest = e / TX;
    const int ey = rest % TY;
    const int ez = rest / TY;
    const int gx = x0 + ex, gy = y0 + ey, gz = z0 + ez;
    if (gx >= nx || gy >= ny || gz >= nz) continue;
    const int c = ((ez + RZ) * YY + (ey + 1)) * YX + (ex + 1);
    constexpr int SX = 1, SY = YX, SZ = Z3 ? YX * YY : 0;
    const T pc = ys[c];
    T rhs;
    if constexpr (KIND == KIND_FVM) {
      const T dc = ds[c];
      const T dxp = hmean(dc, ds[c + SX]), dxm = hmean(ds[c - SX], dc);
      const T dyp = hmean(dc, ds[c + SY]), dym = hmean(ds[c - SY], dc);
      const T dzp = hmean(dc, ds[c + SZ]), dzm = hmean(ds[c - SZ], dc);
      const T rx = Ar<T>::mul(Ar<T>::sub(Ar<T>::mul(dxp, Ar<T>::sub(ys[c + SX], pc)),
                                         Ar<T>::mul(dxm, Ar<T>::sub(pc, ys[c - SX]))), p.ihx2);
      const T ry = Ar<T>::mul(Ar<T>::sub(Ar<T>::mul(dyp, Ar<T>::sub(ys[c + SY], pc)),
                                         Ar<T>::mul(dym, Ar<T>::sub(pc, ys[c - SY]))), p.ihy2);
      const T rz = Ar<T>::mul(Ar<T>::sub(Ar<T>::mul(dzp, Ar<T>::sub(ys[c + SZ], pc)),
                                         Ar<T>::mul(dzm, Ar<T>::sub(pc, ys[c - SZ]))), p.ihz2);
      rhs = Ar<T>::add(Ar<T>::add(rx, ry), rz);
    } else {
      const T ax = tap_sum<T, 2, 2>([&](int o) { return ys[c + o * SX]; });
      const T ay = tap_sum<T, 2, 2>([&](int o) { return ys[c + o * SY]; });
      const T az = tap_sum<T, 2, 2>([&](int o) { return ys[c + o * SZ]; });
      rhs = Ar<T>::add(Ar<T>::add(Ar<T>::mul(ax, p.ihx2), Ar<T>::mul(ay, p.ihy2)), Ar<T>::mul(az, p.ihz2));
    }
    const size_t gi = static_cast<size_t>(gz) * plane + static_cast<size_t>(gy) * nx + gx;
    if constexpr (MODE == MODE_RHS) {
      p.out[gi] = rhs;
    } else if constexpr (MODE == MODE_RK4_FINAL) {
      const T s14 = Ar<T>::add(__ldg(p.k1 + gi), rhs);
      const T s23 = Ar<T>::add(__ldg(p.k2 + gi), __ldg(p.k3 + gi));
      p.out[gi] = Ar<T>::add(__ldg(p.psi + gi), Ar<T>::add(Ar<T>::mul(p.c6, s14), Ar<T>::mul(p.c3, s23)));
    } else {
      p.out[gi] = Ar<T>::add(pc, Ar<T>::mul(p.c6, rhs));
    }
  }
}

template <class T, int KIND, bool Z3, int MODE>
gc_status launch_fvm(gc_context* ctx, const FvmParams<T>& p) {
  using TL = FvmTile<Z3>;
  constexpr int RZ = Z3 ? 1 : 0;
  constexpr size_t yn = static_cast<size_t>(TL::TX + 2) * (TL::TY + 2) * (TL::TZ + 2 * RZ);
  constexpr size_t smem = sizeof(T) * yn * (KIND == KIND_FVM ? 2 : 1);
  auto kern = fvm_stage_kernel<T, KIND, Z3, MODE>;
  if (smem > 48 * 1024) GC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid(div_up(p.nx, TL::TX), div_up(p.ny, TL::TY), Z3 ? div_up(p.nz, TL::TZ) : 1);
  kern<<<grid, kThreads, smem, ctx->stream>>>(p);
  GC_CHECK_LAUNCH("fvm_stage_kernel");
  return GC_OK;
}

// ---------------------------------------------------------------------------
// 3-D z-march stage kernel.  A 32 x 8 CTA owns a column of cells and
// marches up a chunk of z planes.  Each thread keeps its own column's psi,
// k_prev, y = psi + a k_prev and D at planes z-1, z, z+1 in registers; the
// current plane of y and D goes to shared memory with a one-cell x/y halo
// (strips loaded by a few threads).  Every global load of plane z+1 is
// issued while plane z is computed.  Same arithmetic as fvm_stage_kernel.
constexpr int FZ_X = 32, FZ_Y = 8;

// FACES: the FVM coefficients come from the precomputed face fields (the
// thread's own +x/+y/+z faces and its -x/-y neighbours' +faces, the -z face
// carried from the plane below); otherwise D is staged like y and the six
// harmonic means are formed per cell.
template <class T, int KIND, int MODE, bool FACES>
__global__ void __launch_bounds__(FZ_X * FZ_Y) fvm_zmarch_kernel(const FvmParams<T> p, int zc) {
  constexpr bool FVM = KIND == KIND_FVM;
  constexpr bool DST = FVM && !FACES;  // D staged in shared memory
  constexpr bool FF = FVM && FACES;
  __shared__ T sy[FZ_Y + 2][FZ_X + 2];
  __shared__ T sd[DST ? FZ_Y + 2 : 1][DST ? FZ_X + 2 : 1];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int x0 = blockIdx.x * FZ_X, y0 = blockIdx.y * FZ_Y;
  const int z0 = blockIdx.z * zc;
  const int z1 = min(z0 + zc, nz);
  const size_t plane = static_cast<size_t>(nx) * ny;
  const int gx = wrap(x0 + tx, nx), gy = wrap(y0 + ty, ny);
  const size_t col = static_cast<size_t>(gy) * nx + gx;
  const size_t col_xm = static_cast<size_t>(gy) * nx + wrap(gx - 1, nx);
  const size_t col_ym = static_cast<size_t>(wrap(gy - 1, ny)) * nx + gx;
  const bool active = x0 + tx < nx && y0 + ty < ny;
  const bool hx = tx < 2;
  const size_t hx_off = static_cast<size_t>(gy) * nx + wrap(tx == 0 ? x0 - 1 : x0 + FZ_X, nx);
  const int hx_slot = tx == 0 ? 0 : FZ_X + 1;
  const bool hy = ty < 2;
  const size_t hy_off = static_cast<size_t>(wrap(ty == 0 ? y0 - 1 : y0 + FZ_Y, ny)) * nx + gx;
  const int hy_slot = ty == 0 ? 0 : FZ_Y + 1;
  const bool has_kin = p.kin != nullptr;

  auto yval = [&](size_t gi) -> T {
    T v = __ldg(p.psi + gi);
    if (has_kin) v = Ar<T>::add(v, Ar<T>::mul(p.a, __ldg(p.kin + gi)));
    return v;
  };
  auto dval = [&](size_t gi) -> T { return DST ? __ldg(p.D + gi) : T(0); };

  // Queues: index 0 = plane z-1, 1 = z, 2 = z+1.
  T qy[3], qd[3], qp[3], qk[3];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const size_t gi = static_cast<size_t>(wrap(z0 - 1 + k, nz)) * plane + col;
    qp[k + 1] = __ldg(p.psi + gi);
    qk[k + 1] = has_kin ? __ldg(p.kin + gi) : T(0);
    qy[k + 1] = has_kin ? Ar<T>::add(qp[k + 1], Ar<T>::mul(p.a, qk[k + 1])) : qp[k + 1];
    qd[k + 1] = dval(gi);
  }
  // Prefetch registers for plane z0: queue entry (z0 + 1), halos of z0, k1/k2 of z0.
  auto qaddr = [&](int z) { return static_cast<size_t>(wrap(z, nz)) * plane + col; };
  T n_p = __ldg(p.psi + qaddr(z0 + 1));
  T n_k = has_kin ? __ldg(p.kin + qaddr(z0 + 1)) : T(0);
  T n_d = dval(qaddr(z0 + 1));
  T n_hxy = hx ? yval(static_cast<size_t>(z0) * plane + hx_off) : T(0);
  T n_hxd = hx ? dval(static_cast<size_t>(z0) * plane + hx_off) : T(0);
  T n_hyy = hy ? yval(static_cast<size_t>(z0) * plane + hy_off) : T(0);
  T n_hyd = hy ? dval(static_cast<size_t>(z0) * plane + hy_off) : T(0);
  T n_k1 = T(0), n_k2 = T(0);
  if (MODE == MODE_RK4_FINAL && active) {
    n_k1 = __ldg(p.k1 + static_cast<size_t>(z0) * plane + col);
    n_k2 = __ldg(p.k2 + static_cast<size_t>(z0) * plane + col);
  }
  // Faces of plane z0 and the -z face (the +z face of plane z0 - 1).
  T n_fx = T(0), n_fxm = T(0), n_fy = T(0), n_fym = T(0), n_fz = T(0), fz_below = T(0);
  if constexpr (FF) {
    const size_t zo = static_cast<size_t>(z0) * plane;
    n_fx = __ldg(p.fx + zo + col);
    n_fxm = __ldg(p.fx + zo + col_xm);
    n_fy = __ldg(p.fy + zo + col);
    n_fym = __ldg(p.fy + zo + col_ym);
    n_fz = __ldg(p.fz + zo + col);
    fz_below = __ldg(p.fz + static_cast<size_t>(wrap(z0 - 1, nz)) * plane + col);
  }

  for (int z = z0; z < z1; ++z) {
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      qy[k] = qy[k + 1];
      qd[k] = qd[k + 1];
      qp[k] = qp[k + 1];
      qk[k] = qk[k + 1];
    }
    qp[2] = n_p;
    qk[2] = n_k;
    qy[2] = has_kin ? Ar<T>::add(n_p, Ar<T>::mul(p.a, n_k)) : n_p;
    qd[2] = n_d;
    const T hxy = n_hxy, hxd = n_hxd, hyy = n_hyy, hyd = n_hyd, k1c = n_k1, k2c = n_k2;
    const T fxp = n_fx, fxm = n_fxm, fyp = n_fy, fym = n_fym, fzp = n_fz;
    if (z + 1 < z1) {
      const size_t zo = static_cast<size_t>(z + 1) * plane;
      n_p = __ldg(p.psi + qaddr(z + 2));
      if (has_kin) n_k = __ldg(p.kin + qaddr(z + 2));
      n_d = dval(qaddr(z + 2));
      if (hx) {
        n_hxy = yval(zo + hx_off);
        n_hxd = dval(zo + hx_off);
      }
      if (hy) {
        n_hyy = yval(zo + hy_off);
        n_hyd = dval(zo + hy_off);
      }
      if (MODE == MODE_RK4_FINAL && active) {
        n_k1 = __ldg(p.k1 + zo + col);
        n_k2 = __ldg(p.k2 + zo + col);
      }
      if constexpr (FF) {
        n_fx = __ldg(p.fx + zo + col);
        n_fxm = __ldg(p.fx + zo + col_xm);
        n_fy = __ldg(p.fy + zo + col);
        n_fym = __ldg(p.fy + zo + col_ym);
        n_fz = __ldg(p.fz + zo + col);
      }
    }
    sy[ty + 1][tx + 1] = qy[1];
    if (DST) sd[ty + 1][tx + 1] = qd[1];
    if (hx) {
      sy[ty + 1][hx_slot] = hxy;
      if (DST) sd[ty + 1][hx_slot] = hxd;
    }
    if (hy) {
      sy[hy_slot][tx + 1] = hyy;
      if (DST) sd[hy_slot][tx + 1] = hyd;
    }
    __syncthreads();
    if (active) {
      const T pc = qy[1];
      T rhs;
      if constexpr (FVM) {
        T dxp, dxm, dyp, dym, dzp, dzm;
        if constexpr (FF) {
          dxp = fxp; dxm = fxm; dyp = fyp; dym = fym; dzp = fzp; dzm = fz_below;
        } else {
          const T dc = qd[1];
          dxp = hmean(dc, sd[ty + 1][tx + 2]); dxm = hmean(sd[ty + 1][tx], dc);
          dyp = hmean(dc, sd[ty + 2][tx + 1]); dym = hmean(sd[ty][tx + 1], dc);
          dzp = hmean(dc, qd[2]); dzm = hmean(qd[0], dc);
        }
        const T rx = Ar<T>::mul(Ar<T>::sub(Ar<T>::mul(dxp, Ar<T>::sub(sy[ty + 1][tx + 2], pc)),
                                           Ar<T>::mul(dxm, Ar<T>::sub(pc, sy[ty + 1][tx]))), p.ihx2);
        const T ry = Ar<T>::mul(Ar<T>::sub(Ar<T>::mul(dyp, Ar<T>::sub(sy[ty + 2][tx + 1], pc)),
                                           Ar<T>::mul(dym, Ar<T>::sub(pc, sy[ty][tx + 1]))), p.ihy2);
        const T rz = Ar<T>::mul(Ar<T>::sub(Ar<T>::mul(dzp, Ar<T>::sub(qy[2], pc)),
                                           Ar<T>::mul(dzm, Ar<T>::sub(pc, qy[0]))), p.ihz2);
        rhs = Ar<T>::add(Ar<T>::add(rx, ry), rz);
      } else {
        const T ax = tap_sum<T, 2, 2>([&](int o) { return sy[ty + 1][tx + 1 + o]; });
        const T ay = tap_sum<T, 2, 2>([&](int o) { return sy[ty + 1 + o][tx + 1]; });
        const T az = tap_sum<T, 2, 2>([&](int o) { return qy[1 + o]; });
        rhs = Ar<T>::add(Ar<T>::add(Ar<T>::mul(ax, p.ihx2), Ar<T>::mul(ay, p.ihy2)), Ar<T>::mul(az, p.ihz2));
      }
      const size_t gi = static_cast<size_t>(z) * plane + static_cast<size_t>(y0 + ty) * nx + (x0 + tx);
      if constexpr (MODE == MODE_RHS) {
        p.out[gi] = rhs;
      } else if constexpr (MODE == MODE_RK4_FINAL) {
        const T s14 = Ar<T>::add(k1c, rhs);
        const T s23 = Ar<T>::add(k2c, qk[1]);
        p.out[gi] = Ar<T>::add(qp[1], Ar<T>::add(Ar<T>::mul(p.c6, s14), Ar<T>::mul(p.c3, s23)));
      } else {
        p.out[gi] = Ar<T>::add(pc, Ar<T>::mul(p.c6, rhs));
      }
    }
    if constexpr (FF) fz_below = fzp;
    __syncthreads();
  }
}

// Two-column float variant of the FVM z-march (even nx): a 32 x 8 CTA owns a
// 64 x 8 column block, each thread two adjacent cells loaded and stored as
// float2, so the per-plane index arithmetic, queue rotation and barriers are
// paid once per two cells (the single-column float kernel was issue-bound).
// Row layout in shared memory: halo column at 1, the block at 2 .. 65, halo
// at 66, so each thread's pair sits on an 8-byte boundary.
template <int MODE>
__global__ void __launch_bounds__(FZ_X * FZ_Y) fvm_zmarch_x2_kernel(const FvmParams<float> p, int zc) {
  constexpr int RW = 2 * FZ_X + 4;
  // Two plane buffers: plane z's rows go to buffer z & 1, so the one barrier
  // per plane suffices (a buffer is rewritten two planes later, after every
  // thread has passed the barrier of the plane in between).
  __shared__ __align__(8) float sy2[2][FZ_Y + 2][RW];
  __shared__ __align__(8) float sd2[2][FZ_Y + 2][RW];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int x0 = blockIdx.x * (2 * FZ_X), y0 = blockIdx.y * FZ_Y;
  const int z0 = blockIdx.z * zc;
  const int z1 = min(z0 + zc, nz);
  const size_t plane = static_cast<size_t>(nx) * ny;
  const int gx = wrap(x0 + 2 * tx, nx), gy = wrap(y0 + ty, ny);  // gx even (nx even)
  const size_t col = static_cast<size_t>(gy) * nx + gx;
  const bool active = x0 + 2 * tx < nx && y0 + ty < ny;
  const bool hx = tx < 2;
  const size_t hx_off = static_cast<size_t>(gy) * nx + wrap(tx == 0 ? x0 - 1 : x0 + 2 * FZ_X, nx);
  const int hx_slot = tx == 0 ? 1 : 2 * FZ_X + 2;
  const bool hy = ty < 2;
  const size_t hy_off = static_cast<size_t>(wrap(ty == 0 ? y0 - 1 : y0 + FZ_Y, ny)) * nx + gx;
  const int hy_slot = ty == 0 ? 0 : FZ_Y + 1;
  const bool has_kin = p.kin != nullptr;
  const int sc = 2 * tx + 2;  // this thread's first cell in a shared row

  auto ld2 = [](const float* base, size_t gi) { return __ldg(reinterpret_cast<const float2*>(base + gi)); };
  auto y2 = [&](float2 ps, float2 ks) {
    return has_kin ? make_float2(ps.x + p.a * ks.x, ps.y + p.a * ks.y) : ps;
  };
  auto yval = [&](size_t gi) -> float {
    float v = __ldg(p.psi + gi);
    if (has_kin) v = v + p.a * __ldg(p.kin + gi);
    return v;
  };
  auto qaddr = [&](int z) { return static_cast<size_t>(wrap(z, nz)) * plane + col; };

  float2 qy[3], qd[3], qp[3], qk[3];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const size_t gi = qaddr(z0 - 1 + k);
    qp[k + 1] = ld2(p.psi, gi);
    qk[k + 1] = has_kin ? ld2(p.kin, gi) : make_float2(0.f, 0.f);
    qy[k + 1] = y2(qp[k + 1], qk[k + 1]);
    qd[k + 1] = ld2(p.D, gi);
  }
  float2 n_p = ld2(p.psi, qaddr(z0 + 1));
  float2 n_k = has_kin ? ld2(p.kin, qaddr(z0 + 1)) : make_float2(0.f, 0.f);
  float2 n_d = ld2(p.D, qaddr(z0 + 1));
  float n_hxy = hx ? yval(static_cast<size_t>(z0) * plane + hx_off) : 0.f;
  float n_hxd = hx ? __ldg(p.D + static_cast<size_t>(z0) * plane + hx_off) : 0.f;
  float2 n_hyy = make_float2(0.f, 0.f), n_hyd = make_float2(0.f, 0.f);
  if (hy) {
    const size_t gi = static_cast<size_t>(z0) * plane + hy_off;
    n_hyy = y2(ld2(p.psi, gi), has_kin ? ld2(p.kin, gi) : make_float2(0.f, 0.f));
    n_hyd = ld2(p.D, gi);
  }
  float2 n_k1 = make_float2(0.f, 0.f), n_k2 = make_float2(0.f, 0.f);
  if (MODE == MODE_RK4_FINAL && active) {
    n_k1 = ld2(p.k1, static_cast<size_t>(z0) * plane + col);
    n_k2 = ld2(p.k2, static_cast<size_t>(z0) * plane + col);
  }

  for (int z = z0; z < z1; ++z) {
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      qy[k] = qy[k + 1];
      qd[k] = qd[k + 1];
      qp[k] = qp[k + 1];
      qk[k] = qk[k + 1];
    }
    qp[2] = n_p;
    qk[2] = n_k;
    qy[2] = y2(n_p, n_k);
    qd[2] = n_d;
    float(&sy)[FZ_Y + 2][RW] = sy2[(z - z0) & 1];
    float(&sd)[FZ_Y + 2][RW] = sd2[(z - z0) & 1];
    const float hxy = n_hxy, hxd = n_hxd;
    const float2 hyy = n_hyy, hyd = n_hyd, k1c = n_k1, k2c = n_k2;
    if (z + 1 < z1) {
      const size_t zo = static_cast<size_t>(z + 1) * plane;
      n_p = ld2(p.psi, qaddr(z + 2));
      if (has_kin) n_k = ld2(p.kin, qaddr(z + 2));
      n_d = ld2(p.D, qaddr(z + 2));
      if (hx) {
        n_hxy = yval(zo + hx_off);
        n_hxd = __ldg(p.D + zo + hx_off);
      }
      if (hy) {
        n_hyy = y2(ld2(p.psi, zo + hy_off), has_kin ? ld2(p.kin, zo + hy_off) : make_float2(0.f, 0.f));
        n_hyd = ld2(p.D, zo + hy_off);
      }
      if (MODE == MODE_RK4_FINAL && active) {
        n_k1 = ld2(p.k1, zo + col);
        n_k2 = ld2(p.k2, zo + col);
      }
    }
    *reinterpret_cast<float2*>(&sy[ty + 1][sc]) = qy[1];
    *reinterpret_cast<float2*>(&sd[ty + 1][sc]) = qd[1];
    if (hx) {
      sy[ty + 1][hx_slot] = hxy;
      sd[ty + 1][hx_slot] = hxd;
    }
    if (hy) {
      *reinterpret_cast<float2*>(&sy[hy_slot][sc]) = hyy;
      *reinterpret_cast<float2*>(&sd[hy_slot][sc]) = hyd;
    }
    __syncthreads();
    if (active) {
      float out[2];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int c = sc + q;
        const float pc = q == 0 ? qy[1].x : qy[1].y;
        const float dc = q == 0 ? qd[1].x : qd[1].y;
        const float dzu = q == 0 ? qd[2].x : qd[2].y, dzd = q == 0 ? qd[0].x : qd[0].y;
        const float yzu = q == 0 ? qy[2].x : qy[2].y, yzd = q == 0 ? qy[0].x : qy[0].y;
        const float dxp = hmean(dc, sd[ty + 1][c + 1]), dxm = hmean(sd[ty + 1][c - 1], dc);
        const float dyp = hmean(dc, sd[ty + 2][c]), dym = hmean(sd[ty][c], dc);
        const float dzp = hmean(dc, dzu), dzm = hmean(dzd, dc);
        const float rx = (dxp * (sy[ty + 1][c + 1] - pc) - dxm * (pc - sy[ty + 1][c - 1])) * p.ihx2;
        const float ry = (dyp * (sy[ty + 2][c] - pc) - dym * (pc - sy[ty][c])) * p.ihy2;
        const float rz = (dzp * (yzu - pc) - dzm * (pc - yzd)) * p.ihz2;
        const float rhs = (rx + ry) + rz;
        if constexpr (MODE == MODE_RHS) {
          out[q] = rhs;
        } else if constexpr (MODE == MODE_RK4_FINAL) {
          const float s14 = (q == 0 ? k1c.x : k1c.y) + rhs;
          const float s23 = (q == 0 ? k2c.x : k2c.y) + (q == 0 ? qk[1].x : qk[1].y);
          out[q] = (q == 0 ? qp[1].x : qp[1].y) + (p.c6 * s14 + p.c3 * s23);
        } else {
          out[q] = pc + p.c6 * rhs;
        }
      }
      const size_t gi = static_cast<size_t>(z) * plane + static_cast<size_t>(y0 + ty) * nx + (x0 + 2 * tx);
      *reinterpret_cast<float2*>(p.out + gi) = make_float2(out[0], out[1]);
    }
  }
}

template <class T, int KIND, int MODE>
gc_status launch_fvm_zmarch(gc_context* ctx, const FvmParams<T>& p) {
  bool x2 = false;
  if constexpr (std::is_same_v<T, float> && KIND == KIND_FVM)
    x2 = !p.fx && p.nx % 2 == 0 &&
         (reinterpret_cast<uintptr_t>(p.psi) | reinterpret_cast<uintptr_t>(p.kin) | reinterpret_cast<uintptr_t>(p.D) |
          reinterpret_cast<uintptr_t>(p.out) | reinterpret_cast<uintptr_t>(p.k1) | reinterpret_cast<uintptr_t>(p.k2)) %
                 8 == 0;
  const int tiles_x = div_up(p.nx, x2 ? 2 * FZ_X : FZ_X), tiles_y = div_up(p.ny, FZ_Y);
  const long long tiles = static_cast<long long>(tiles_x) * tiles_y;
  const long long want = 16LL * ctx->num_sms;
  int chunks = static_cast<int>(std::min<long long>((want + tiles - 1) / tiles, std::max(1, p.nz / 16)));
  chunks = std::max(chunks, 1);
  const int zc = div_up(p.nz, chunks);
  chunks = div_up(p.nz, zc);
  dim3 grid(tiles_x, tiles_y, chunks), block(FZ_X, FZ_Y);
  if constexpr (std::is_same_v<T, float> && KIND == KIND_FVM) {
    if (x2) {
      fvm_zmarch_x2_kernel<MODE><<<grid, block, 0, ctx->stream>>>(p, zc);
      GC_CHECK_LAUNCH("fvm_zmarch_x2_kernel");
      return GC_OK;
    }
  }
  if (KIND == KIND_FVM && p.fx)
    fvm_zmarch_kernel<T, KIND, MODE, true><<<grid, block, 0, ctx->stream>>>(p, zc);
  else
    fvm_zmarch_kernel<T, KIND, MODE, false><<<grid, block, 0, ctx->stream>>>(p, zc);
  GC_CHECK_LAUNCH("fvm_zmarch_kernel");
  return GC_OK;
}

template <class T, int KIND, int MODE>
gc_status launch_kind(gc_context* ctx, const FvmParams<T>& p) {
  if (p.nz > 2) return launch_fvm_zmarch<T, KIND, MODE>(ctx, p);
  return p.nz > 1 ? launch_fvm<T, KIND, true, MODE>(ctx, p) : launch_fvm<T, KIND, false, MODE>(ctx, p);
}

template <class T>
FvmParams<T> fvm_params(const gc_grid* g) {
  FvmParams<T> p{};
  p.nx = g->nx; p.ny = g->ny; p.nz = g->nz;
  p.ihx2 = static_cast<T>(1.0 / (g->hx * g->hx));
  p.ihy2 = static_cast<T>(1.0 / (g->hy * g->hy));
  p.ihz2 = static_cast<T>(1.0 / (g->hz * g->hz));
  return p;
}

template <class T, int KIND>
gc_status enqueue_step(gc_context* ctx, const gc_grid* g, const T* D, const T* faces, const T* src, T* dst,
                       T* k1, T* k2, T* k3, double dt, gc_integrator integ) {
  FvmParams<T> p = fvm_params<T>(g);
  p.psi = src;
  p.D = D;
  if (faces) {
    const size_t n = cells(g);
    p.fx = faces;
    p.fy = faces + n;
    p.fz = faces + 2 * n;
  }
  gc_status s;
  if (integ == GC_EXPLICIT_EULER) {
    p.out = dst;
    p.c6 = static_cast<T>(dt);
    return launch_kind<T, KIND, MODE_EULER_FINAL>(ctx, p);
  }
  const double half_dt = 0.5 * dt, sixth_dt = dt / 6.0, third_dt = dt / 3.0;
  p.out = k1;
  if ((s = launch_kind<T, KIND, MODE_RHS>(ctx, p)) != GC_OK) return s;
  p.kin = k1; p.a = static_cast<T>(half_dt); p.out = k2;
  if ((s = launch_kind<T, KIND, MODE_RHS>(ctx, p)) != GC_OK) return s;
  p.kin = k2; p.out = k3;
  if ((s = launch_kind<T, KIND, MODE_RHS>(ctx, p)) != GC_OK) return s;
  p.kin = k3; p.a = static_cast<T>(dt); p.out = dst;
  p.k1 = k1; p.k2 = k2; p.k3 = k3;
  p.c6 = static_cast<T>(sixth_dt); p.c3 = static_cast<T>(third_dt);
  return launch_kind<T, KIND, MODE_RK4_FINAL>(ctx, p);
}

template <class T, int KIND>
gc_status diffuse_t(gc_context* ctx, const gc_grid* g, const T* D, T* psi, double dt, int n_steps,
                    gc_integrator integ) {
  const size_t bytes = cells(g) * sizeof(T);
  void *vb = nullptr, *v1 = nullptr, *v2 = nullptr, *v3 = nullptr;
  gc_status s;
  if ((s = scratch_get(ctx, kSlotPsiB, bytes, &vb)) != GC_OK) return s;
  if (integ == GC_RK4) {
    if ((s = scratch_get(ctx, kSlotK1, bytes, &v1)) != GC_OK) return s;
    if ((s = scratch_get(ctx, kSlotK2, bytes, &v2)) != GC_OK) return s;
    if ((s = scratch_get(ctx, kSlotK3, bytes, &v3)) != GC_OK) return s;
  }
  T* pb = static_cast<T*>(vb);
  T *k1 = static_cast<T*>(v1), *k2 = static_cast<T*>(v2), *k3 = static_cast<T*>(v3);
  // Double z-march stages read precomputed faces (one pass over D per call)
  // instead of forming six correctly rounded divisions per cell and stage;
  // float keeps the on-the-fly faces, whose fast division costs less than
  // the five extra face loads (measured: 2.07 vs 2.21 ms per 384^3 step).
  T* faces = nullptr;
  if (KIND == KIND_FVM && g->nz > 2 && sizeof(T) == 8) {
    void* vf = nullptr;
    if ((s = scratch_get(ctx, kSlotFaces, 3 * bytes, &vf)) != GC_OK) return s;
    faces = static_cast<T*>(vf);
    const size_t n = cells(g);
    const int blocks = static_cast<int>(std::min<size_t>((n + kThreads - 1) / kThreads, static_cast<size_t>(ctx->num_sms) * 16));
    fvm_faces_kernel<T><<<blocks, kThreads, 0, ctx->stream>>>(D, faces, faces + n, faces + 2 * n, g->nx, g->ny, g->nz);
    GC_CHECK_LAUNCH("fvm_faces_kernel");
  }
  const uint64_t key[8] = {reinterpret_cast<uint64_t>(psi) ^ 0x2ULL,
                           reinterpret_cast<uint64_t>(pb),
                           reinterpret_cast<uint64_t>(k1) ^ (reinterpret_cast<uint64_t>(k3) << 1),
                           (static_cast<uint64_t>(g->nx) << 40) ^ (static_cast<uint64_t>(g->ny) << 20) ^
                               static_cast<uint64_t>(g->nz) ^ (bits_of(g->hx) * 3) ^ (bits_of(g->hy) * 5) ^
                               (bits_of(g->hz) * 7),
                           bits_of(dt),
                           reinterpret_cast<uint64_t>(D),
                           reinterpret_cast<uint64_t>(faces),
                           (static_cast<uint64_t>(KIND) << 8) | (static_cast<uint64_t>(integ) << 4) |
                               (sizeof(T) == 8 ? 1u : 2u) | (0xD1ULL << 56)};
  return run_steps<T>(ctx, psi, pb, bytes, n_steps, key, [&](const T* src, T* dst) {
    return enqueue_step<T, KIND>(ctx, g, D, faces, src, dst, k1, k2, k3, dt, integ);
  });
}

gc_status cfl_check(const gc_grid* g, double D, double dt, gc_integrator integ) {
  const double limit = integ == GC_RK4 ? 0.6963 : 0.5;
  const double inv_sum = 1.0 / (g->hx * g->hx) + 1.0 / (g->hy * g->hy) + 1.0 / (g->hz * g->hz);
  const double cfl = D * dt * inv_sum;
  if (cfl > limit) {
    return fail(GC_ERR_CFL, std::string("solve::diffuse: explicit-diffusion CFL violated for ") +
                                (integ == GC_RK4 ? "RK4" : "ExplicitEuler") + ": D=" + std::to_string(D) +
                                ", dt=" + std::to_string(dt) + ", h=(" + std::to_string(g->hx) + ", " +
                                std::to_string(g->hy) + ", " + std::to_string(g->hz) +
                                "); D*dt*(1/hx^2 + 1/hy^2 + 1/hz^2) = " + std::to_string(cfl) + " > " +
                                std::to_string(limit));
  }
  return GC_OK;
}

gc_status d_positive(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* D, int64_t* bad,
                     const char* who) {
  long long first = -1;
  gc_status s = first_nonpositive(ctx, g, dt, D, &first);
  if (s != GC_OK) return s;
  if (first >= 0) {
    double v = 0.0;
    if (dt == GC_F64) {
      GC_CUDA(cudaMemcpy(&v, static_cast<const double*>(D) + first, sizeof(double), cudaMemcpyDeviceToHost));
    } else {
      float f = 0.f;
      GC_CUDA(cudaMemcpy(&f, static_cast<const float*>(D) + first, sizeof(float), cudaMemcpyDeviceToHost));
      v = f;
    }
    if (bad) *bad = first;
    return fail(GC_ERR_NONPOSITIVE_D,
                std::string(who) + ": D must be strictly positive at every cell (the harmonic-mean face-D "
                                   "averaging is undefined otherwise); first violation at flat index " +
                    std::to_string(first) + " with D=" + std::to_string(v));
  }
  return GC_OK;
}

}  // namespace
}  // namespace gcb

using namespace gcb;

extern "C" {

GC_API gc_status gc_cell_laplacian(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* psi,
                                   const void* D, void* out, int64_t* bad_index) {
  Call call(ctx);
  gc_status s = call.st;
  if (s != GC_OK) return s;
  if ((s = require_axes(g, 1)) != GC_OK) return s;
  if (!psi || !D || !out) return fail(GC_ERR_INVALID_ARG, "gc_cell_laplacian: null field pointer");
  if (dt != GC_F64 && dt != GC_F32) return fail(GC_ERR_INVALID_ARG, "gc_cell_laplacian: unknown dtype");
  if ((s = d_positive(ctx, g, dt, D, bad_index, "fvm::cellLaplacian")) != GC_OK) return s;
  if (dt == GC_F64) {
    FvmParams<double> p = fvm_params<double>(g);
    p.psi = static_cast<const double*>(psi);
    p.D = static_cast<const double*>(D);
    p.out = static_cast<double*>(out);
    return launch_kind<double, KIND_FVM, MODE_RHS>(ctx, p);
  }
  FvmParams<float> p = fvm_params<float>(g);
  p.psi = static_cast<const float*>(psi);
  p.D = static_cast<const float*>(D);
  p.out = static_cast<float*>(out);
  return launch_kind<float, KIND_FVM, MODE_RHS>(ctx, p);
}

GC_API gc_status gc_diffuse(gc_context* ctx, const gc_grid* g, gc_dtype dt, void* psi, double D,
                            double dt_step, int n_steps, gc_integrator integ) {
  NvtxScope nvtx("gc_diffuse");
  Call call(ctx);
  gc_status s = call.st;
  if (s != GC_OK) return s;
  if ((s = check_grid(g)) != GC_OK) return s;
  if (integ != GC_RK4 && integ != GC_EXPLICIT_EULER) return fail(GC_ERR_INVALID_ARG, "gc_diffuse: unknown integrator");
  if (D < 0.0) return fail(GC_ERR_INVALID_ARG, "solve::diffuse: D must be >= 0; got " + std::to_string(D));
  if (dt_step < 0.0) return fail(GC_ERR_INVALID_ARG, "solve::diffuse: dt must be >= 0; got " + std::to_string(dt_step));
  if (n_steps < 0) return fail(GC_ERR_INVALID_ARG, "solve::diffuse: n_steps must be >= 0; got " + std::to_string(n_steps));
  if ((s = cfl_check(g, D, dt_step, integ)) != GC_OK) return s;
  if (n_steps == 0) return GC_OK;
  if ((s = require_axes(g, 1)) != GC_OK) return s;
  if (!psi) return fail(GC_ERR_INVALID_ARG, "gc_diffuse: null psi");
  // The reference integrates lap(psi) with step D*dt (solve/Diffusion.hpp:106-111).
  if (dt == GC_F64) return diffuse_t<double, KIND_LAP>(ctx, g, nullptr, static_cast<double*>(psi), D * dt_step, n_steps, integ);
  if (dt == GC_F32) return diffuse_t<float, KIND_LAP>(ctx, g, nullptr, static_cast<float*>(psi), D * dt_step, n_steps, integ);
  return fail(GC_ERR_INVALID_ARG, "gc_diffuse: unknown dtype");
}

GC_API gc_status gc_diffuse_fvm(gc_context* ctx, const gc_grid* g, gc_dtype dt, void* psi, const void* D,
                                double dt_step, int n_steps, gc_integrator integ, int64_t* bad_index) {
  NvtxScope nvtx("gc_diffuse_fvm");
  Call call(ctx);
  gc_status s = call.st;
  if (s != GC_OK) return s;
  if ((s = check_grid(g)) != GC_OK) return s;
  if (integ != GC_RK4 && integ != GC_EXPLICIT_EULER) return fail(GC_ERR_INVALID_ARG, "gc_diffuse_fvm: unknown integrator");
  if (dt != GC_F64 && dt != GC_F32) return fail(GC_ERR_INVALID_ARG, "gc_diffuse_fvm: unknown dtype");
  if (dt_step < 0.0) return fail(GC_ERR_INVALID_ARG, "solve::diffuse: dt must be >= 0; got " + std::to_string(dt_step));
  if (n_steps < 0) return fail(GC_ERR_INVALID_ARG, "solve::diffuse: n_steps must be >= 0; got " + std::to_string(n_steps));
  if (!psi || !D) return fail(GC_ERR_INVALID_ARG, "gc_diffuse_fvm: null field pointer");
  double dmax = 0.0;
  if ((s = d_max_face_any(ctx, g, dt, D, &dmax)) != GC_OK) return s;
  if ((s = cfl_check(g, dmax, dt_step, integ)) != GC_OK) return s;
  if (n_steps == 0) return GC_OK;
  // cellLaplacian's own preconditions, checked once instead of on every RHS
  // call: D is constant over the call (fvm/CellLaplacian.hpp:95-109).
  if ((s = require_axes(g, 1)) != GC_OK) return s;
  if ((s = d_positive(ctx, g, dt, D, bad_index, "solve::diffuse: fvm::cellLaplacian")) != GC_OK) return s;
  if (dt == GC_F64)
    return diffuse_t<double, KIND_FVM>(ctx, g, static_cast<const double*>(D), static_cast<double*>(psi), dt_step, n_steps, integ);
  return diffuse_t<float, KIND_FVM>(ctx, g, static_cast<const float*>(D), static_cast<float*>(psi), dt_step, n_steps, integ);
}

}  // extern "C"
