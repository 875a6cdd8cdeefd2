// func::evaluate with a general integrand (func/Functional.hpp:88-148 for a
// scalar psi, :183-220 for a Vec3d field u).
//
// The reference materialises the derivative fields the callable's arity asks
// for (order-2 gradient, Laplacian, biharmonic; for a vector field the
// order-2 rank-2 gradient), evaluates the callable per cell into an integrand
// field and reduces it with func::integrate.  Here one kernel forms every
// derivative a cell needs from its neighbours (read through L1/L2; one HBM
// read per value), runs the integrand program on them and writes the
// integrand; the reduction is the exact pairwise tree of gc_integrate (or
// its compensated sum).  No derivative field is materialised.
//
// The program is a straight-line list of register instructions passed by
// value as a kernel parameter, so every thread of a warp reads the same
// instruction from the constant bank and the interpreter's branches are
// uniform.  Every sum, product and quotient is rounded on its own, in the
// reference's order, so double results are bit-identical to the reference
// when the program performs the callable's operations in the callable's
// order.
#include <algorithm>
#include <cstring>
#include <string>

#include "common.cuh"

namespace gcb {
namespace {

constexpr int kEvX = 32;
constexpr int kEvY = 8;

struct EvalArgs {
  const void* field;
  double* out;
  int nx, ny, nz, zc;
  size_t n;
  double ihx, ihy, ihz;     // 1 / h
  double ihx2, ihy2, ihz2;  // 1 / h^2
  double ihx4, ihy4, ihz4;  // (1 / h^2)^2
  int n_instr, result_reg;
  gc_instr prog[GC_PROGRAM_MAX_INSTR];
};

constexpr int n_inputs(int comps, int arity) {
  return comps == 1 ? (arity == 1 ? 1 : arity == 2 ? 4 : arity == 3 ? 5 : 6) : (arity == 1 ? 3 : 12);
}

__device__ __forceinline__ double run_program(const EvalArgs& a, const double* in) {
  double r[GC_PROGRAM_REGS];
  for (int pc = 0; pc < a.n_instr; ++pc) {
    const gc_instr& I = a.prog[pc];
    double v;
    switch (I.op) {
      case GC_OPC_CONST: v = I.value; break;
      case GC_OPC_INPUT: v = in[I.a]; break;
      case GC_OPC_ADD: v = __dadd_rn(r[I.a], r[I.b]); break;
      case GC_OPC_SUB: v = __dsub_rn(r[I.a], r[I.b]); break;
      case GC_OPC_MUL: v = __dmul_rn(r[I.a], r[I.b]); break;
      case GC_OPC_DIV: v = __ddiv_rn(r[I.a], r[I.b]); break;
      case GC_OPC_NEG: v = -r[I.a]; break;
      case GC_OPC_ABS: v = fabs(r[I.a]); break;
      case GC_OPC_SQRT: v = __dsqrt_rn(r[I.a]); break;
      case GC_OPC_MIN: v = r[I.b] < r[I.a] ? r[I.b] : r[I.a]; break;
      default: v = r[I.a] < r[I.b] ? r[I.b] : r[I.a]; break;  // GC_OPC_MAX (validated on the host)
    }
    r[I.dst] = v;
  }
  return r[a.result_reg];
}

// Order-2 first derivative along one axis: every tap of (-1, 0, 1) with
// weights (-0.5, 0, 0.5) summed from 0.0 (diff/Gradient.hpp:59-66).
template <class Tap>
__device__ __forceinline__ double d1(const Tap& tap) {
  double s = 0.0;
#pragma unroll
  for (int m = 0; m < 3; ++m) s = __dadd_rn(s, __dmul_rn(W<1, 2>::w(m), tap(m - 1)));
  return s;
}

// A thread walks a column of cells (i, j, z0..z1).  R is the largest stencil
// radius the arity needs: 0 (values only), 1 (gradient, Laplacian) or 2
// (biharmonic).
template <class T, int COMPS, int ARITY>
__global__ void __launch_bounds__(kEvX * kEvY) evaluate_kernel(const __grid_constant__ EvalArgs a) {
  constexpr int R = COMPS == 1 ? (ARITY >= 4 ? 2 : ARITY >= 2 ? 1 : 0) : (ARITY >= 2 ? 1 : 0);
  const int i = blockIdx.x * kEvX + threadIdx.x;
  const int j = blockIdx.y * kEvY + threadIdx.y;
  if (i >= a.nx || j >= a.ny) return;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const T* __restrict__ f = static_cast<const T*>(a.field);
  int xs[2 * R + 1];
  size_t ys[2 * R + 1];
#pragma unroll
  for (int m = 0; m <= 2 * R; ++m) {
    xs[m] = wrap(i + m - R, nx);
    ys[m] = static_cast<size_t>(wrap(j + m - R, ny)) * nx;
  }
  const size_t plane = static_cast<size_t>(nx) * ny;
  const int z0 = blockIdx.z * a.zc;
  const int z1 = min(z0 + a.zc, nz);
  for (int k = z0; k < z1; ++k) {
    size_t zs[2 * R + 1];
#pragma unroll
    for (int m = 0; m <= 2 * R; ++m) zs[m] = static_cast<size_t>(wrap(k + m - R, nz)) * plane;
    auto v = [&](int comp, int ox, int oy, int oz) -> double {
      return static_cast<double>(__ldg(f + comp * a.n + zs[oz + R] + ys[oy + R] + xs[ox + R]));
    };
    double in[n_inputs(COMPS, ARITY)];
    if constexpr (COMPS == 1) {
      in[GC_IN_PSI] = v(0, 0, 0, 0);
      if constexpr (ARITY >= 2) {
        in[GC_IN_GRAD_X] = __dmul_rn(d1([&](int o) { return v(0, o, 0, 0); }), a.ihx);
        in[GC_IN_GRAD_Y] = __dmul_rn(d1([&](int o) { return v(0, 0, o, 0); }), a.ihy);
        in[GC_IN_GRAD_Z] = __dmul_rn(d1([&](int o) { return v(0, 0, 0, o); }), a.ihz);
      }
      if constexpr (ARITY >= 3) {
        // diff/Laplacian.hpp:60-69 at order 2.
        double dxx = 0.0, dyy = 0.0, dzz = 0.0;
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          const double w = W<2, 2>::w(m);
          dxx = __dadd_rn(dxx, __dmul_rn(w, v(0, m - 1, 0, 0)));
          dyy = __dadd_rn(dyy, __dmul_rn(w, v(0, 0, m - 1, 0)));
          dzz = __dadd_rn(dzz, __dmul_rn(w, v(0, 0, 0, m - 1)));
        }
        in[GC_IN_LAP] = __dadd_rn(__dadd_rn(__dmul_rn(dxx, a.ihx2), __dmul_rn(dyy, a.ihy2)), __dmul_rn(dzz, a.ihz2));
      }
      if constexpr (ARITY >= 4) {
        // diff/Biharmonic.hpp:70-99 at order 2.
        double dx4 = 0.0, dy4 = 0.0, dz4 = 0.0;
#pragma unroll
        for (int m = 0; m < 5; ++m) {
          const double w = W<4, 2>::w(m);
          dx4 = __dadd_rn(dx4, __dmul_rn(w, v(0, m - 2, 0, 0)));
          dy4 = __dadd_rn(dy4, __dmul_rn(w, v(0, 0, m - 2, 0)));
          dz4 = __dadd_rn(dz4, __dmul_rn(w, v(0, 0, 0, m - 2)));
        }
        double xy = 0.0, xz = 0.0, yz = 0.0;
#pragma unroll
        for (int mb = 0; mb < 3; ++mb) {
#pragma unroll
          for (int ma = 0; ma < 3; ++ma) {
            const double wab = W<2, 2>::w(ma) * W<2, 2>::w(mb);  // exact: products of 1 and -2
            xy = __dadd_rn(xy, __dmul_rn(wab, v(0, ma - 1, mb - 1, 0)));
            xz = __dadd_rn(xz, __dmul_rn(wab, v(0, ma - 1, 0, mb - 1)));
            yz = __dadd_rn(yz, __dmul_rn(wab, v(0, 0, ma - 1, mb - 1)));
          }
        }
        const double axial =
            __dadd_rn(__dadd_rn(__dmul_rn(dx4, a.ihx4), __dmul_rn(dy4, a.ihy4)), __dmul_rn(dz4, a.ihz4));
        const double c1 = __dmul_rn(__dmul_rn(xy, a.ihx2), a.ihy2);
        const double c2 = __dmul_rn(__dmul_rn(xz, a.ihx2), a.ihz2);
        const double c3 = __dmul_rn(__dmul_rn(yz, a.ihy2), a.ihz2);
        in[GC_IN_BIH] = __dadd_rn(axial, __dmul_rn(2.0, __dadd_rn(__dadd_rn(c1, c2), c3)));
      }
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c) in[GC_IN_U_X + c] = v(c, 0, 0, 0);
      if constexpr (ARITY >= 2) {
        // diff/Gradient.hpp:115-131: row = component, column = axis.
#pragma unroll
        for (int row = 0; row < 3; ++row) {
          in[GC_IN_DU + 3 * row + 0] = __dmul_rn(d1([&](int o) { return v(row, o, 0, 0); }), a.ihx);
          in[GC_IN_DU + 3 * row + 1] = __dmul_rn(d1([&](int o) { return v(row, 0, o, 0); }), a.ihy);
          in[GC_IN_DU + 3 * row + 2] = __dmul_rn(d1([&](int o) { return v(row, 0, 0, o); }), a.ihz);
        }
      }
    }
    a.out[static_cast<size_t>(k) * plane + static_cast<size_t>(j) * nx + i] = run_program(a, in);
  }
}

template <class T, int COMPS, int ARITY>
gc_status launch(gc_context* ctx, const EvalArgs& a) {
  const int gx = (a.nx + kEvX - 1) / kEvX, gy = (a.ny + kEvY - 1) / kEvY;
  const int gz = (a.nz + a.zc - 1) / a.zc;
  evaluate_kernel<T, COMPS, ARITY><<<dim3(gx, gy, gz), dim3(kEvX, kEvY), 0, ctx->stream>>>(a);
  GC_CHECK_LAUNCH("evaluate_kernel");
  return GC_OK;
}

template <class T>
gc_status dispatch(gc_context* ctx, int comps, int arity, const EvalArgs& a) {
  if (comps == 1) {
    switch (arity) {
      case 1: return launch<T, 1, 1>(ctx, a);
      case 2: return launch<T, 1, 2>(ctx, a);
      case 3: return launch<T, 1, 3>(ctx, a);
      default: return launch<T, 1, 4>(ctx, a);
    }
  }
  return arity == 1 ? launch<T, 3, 1>(ctx, a) : launch<T, 3, 2>(ctx, a);
}

// Checks the program's shape and that every register is written before it
// is read; returns the result register.
gc_status check_program(const gc_program* f, int* result_reg) {
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
  *result_reg = f->instr[f->n_instr - 1].dst;
  return GC_OK;
}

}  // namespace
}  // namespace gcb

using namespace gcb;

extern "C" {

GC_API gc_status gc_evaluate_program(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* field,
                                     const gc_program* f, gc_sum sum, double* result) {
  Call call(ctx);
  gc_status s = call.st;
  if (s != GC_OK) return s;
  if ((s = check_grid(g)) != GC_OK) return s;
  if (!field || !f || !result) return fail(GC_ERR_INVALID_ARG, "gc_evaluate_program: null pointer");
  if (dt != GC_F64 && dt != GC_F32) return fail(GC_ERR_INVALID_ARG, "gc_evaluate_program: unknown dtype");
  EvalArgs a{};
  if ((s = check_program(f, &a.result_reg)) != GC_OK) return s;
  // The derivative fields of the arity, checked in the reference's order:
  // gradient (radius 1), Laplacian (radius 1), biharmonic (radius 2).
  if (f->arity >= 2 && (s = require_axes(g, 1)) != GC_OK) return s;
  if (f->components == 1 && f->arity >= 4 && (s = require_axes(g, 2)) != GC_OK) return s;
  const size_t n = cells(g);
  void* buf = nullptr;
  if ((s = scratch_get(ctx, kSlotIntegrand, sizeof(double) * n, &buf)) != GC_OK) return s;
  a.field = field;
  a.out = static_cast<double*>(buf);
  a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
  a.n = n;
  a.ihx = 1.0 / g->hx; a.ihy = 1.0 / g->hy; a.ihz = 1.0 / g->hz;
  a.ihx2 = 1.0 / (g->hx * g->hx); a.ihy2 = 1.0 / (g->hy * g->hy); a.ihz2 = 1.0 / (g->hz * g->hz);
  a.ihx4 = a.ihx2 * a.ihx2; a.ihy4 = a.ihy2 * a.ihy2; a.ihz4 = a.ihz2 * a.ihz2;
  a.n_instr = f->n_instr;
  std::memcpy(a.prog, f->instr, sizeof(gc_instr) * static_cast<size_t>(f->n_instr));
  // Enough z chunks for about eight CTAs per SM.
  const long long columns = static_cast<long long>((g->nx + kEvX - 1) / kEvX) * ((g->ny + kEvY - 1) / kEvY);
  const long long want = std::max<long long>(1, (static_cast<long long>(ctx->num_sms) * 8 + columns - 1) / columns);
  a.zc = static_cast<int>((g->nz + std::min<long long>(want, g->nz) - 1) / std::min<long long>(want, g->nz));
  s = dt == GC_F64 ? dispatch<double>(ctx, f->components, f->arity, a)
                   : dispatch<float>(ctx, f->components, f->arity, a);
  if (s != GC_OK) return s;
  double total = 0.0;
  if ((s = sum_any(ctx, GC_F64, a.out, static_cast<long long>(n), sum, &total)) != GC_OK) return s;
  *result = (g->hx * g->hy * g->hz) * total;
  return GC_OK;
}

}  // extern "C"
