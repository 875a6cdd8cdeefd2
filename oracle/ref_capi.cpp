// Test infrastructure: a C harness over the reference gridcalc headers,
// compiled from the reference tree where it lies (never copied) by
// oracle/Makefile into oracle/_ref/libgcref.so.  It pins the C restatement
// in oracle/gc_oracle.c and serves as the timed CPU baseline.  Nothing on
// the product path links or loads it.
//
// Every function takes a raw buffer in the reference memory layout
// (i fastest, core/Grid.hpp:132-137), builds a reference Field from it,
// calls the reference function and copies the result out.  Vector fields
// cross this boundary as three planes (x, y, z components, N values each).
// std::invalid_argument is caught and turned into return code 1 with the
// message available from ref_last_error().
#include <algorithm>
#include <cmath>
#include <array>
#include <cstdint>
#include <utility>
#include <cstring>
#include <stdexcept>
#include <string>

#include <gridcalc/core/Field.hpp>
#include <gridcalc/core/Grid.hpp>
#include <gridcalc/diff/Biharmonic.hpp>
#include <gridcalc/diff/Divergence.hpp>
#include <gridcalc/diff/Gradient.hpp>
#include <gridcalc/diff/FourthOrder.hpp>
#include <gridcalc/diff/Laplacian.hpp>
#include <gridcalc/diff/MixedPartial.hpp>
#include <gridcalc/diff/ThirdOrder.hpp>
#include <gridcalc/func/Functional.hpp>
#include <gridcalc/func/Integrate.hpp>
#include <gridcalc/fvm/CellLaplacian.hpp>
#include <gridcalc/solve/Diffusion.hpp>
#include <gridcalc/solve/Integrator.hpp>
#include <gridcalc/spectral/Derivatives.hpp>

#include <common/cahn_hilliard.hpp>
#include <common/vtk_writer.hpp>

namespace {

using gridcalc::core::Field;
using gridcalc::core::Grid;
using gridcalc::core::Mat3d;
using gridcalc::core::Vec3d;
namespace ch = gridcalc::examples::cahn_hilliard;

thread_local std::string g_err;

// spectral::partial<A, B, C> for every count triple 0..4 (runtime dispatch).
template <int A, int B, int C>
void spectralPartial(const Field<double>& f, double* out) {
  const Field<double> r = gridcalc::spectral::partial<A, B, C>(f);
  std::memcpy(out, r.data(), sizeof(double) * r.getSize());
}
using SpectralFn = void (*)(const Field<double>&, double*);
template <int... I>
constexpr std::array<SpectralFn, sizeof...(I)> spectralTable(std::integer_sequence<int, I...>) {
  return {&spectralPartial<I / 25, (I / 5) % 5, I % 5>...};
}
const std::array<SpectralFn, 125> kSpectral = spectralTable(std::make_integer_sequence<int, 125>{});

// A straight-line register program standing in for a callable (the layout
// of gc_instr / oc_instr): r[dst] = op(r[a], r[b]), a constant or input a.
struct RefInstr {
  int16_t op, dst, a, b;
  double value;
};

double runProgram(const RefInstr* prog, int n, const double* in) {
  double r[32];
  for (int pc = 0; pc < n; ++pc) {
    const RefInstr& I = prog[pc];
    double v;
    switch (I.op) {
      case 0: v = I.value; break;
      case 1: v = in[I.a]; break;
      case 2: v = r[I.a] + r[I.b]; break;
      case 3: v = r[I.a] - r[I.b]; break;
      case 4: v = r[I.a] * r[I.b]; break;
      case 5: v = r[I.a] / r[I.b]; break;
      case 6: v = -r[I.a]; break;
      case 7: v = std::fabs(r[I.a]); break;
      case 8: v = std::sqrt(r[I.a]); break;
      case 9: v = std::min(r[I.a], r[I.b]); break;
      default: v = std::max(r[I.a], r[I.b]); break;
    }
    r[I.dst] = v;
  }
  return r[prog[n - 1].dst];
}

Grid makeGrid(int nx, int ny, int nz, double hx, double hy, double hz) {
  return Grid(nx, ny, nz, Vec3d(hx, hy, hz));
}

Field<double> load(const Grid& g, const double* p) {
  Field<double> f(g);
  std::memcpy(f.data(), p, sizeof(double) * g.getSize());
  return f;
}

void store(const Field<double>& f, double* p) {
  std::memcpy(p, f.data(), sizeof(double) * f.getSize());
}

template <class Fn>
int guarded(Fn&& fn) {
  try {
    fn();
    return 0;
  } catch (const std::invalid_argument& e) {
    g_err = e.what();
    return 1;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 2;
  }
}

// Cahn-Hilliard RHS at a selectable Laplacian order.  Order 2 calls the
// reference function itself (examples/common/cahn_hilliard.hpp:38-59);
// order 4 is the same three statements with laplacian<4>, because the
// reference hard-codes the default order there.
template <int Order>
Field<double> chRhs(const Field<double>& psi, double M, double kappa) {
  if constexpr (Order == 2) {
    return ch::computeRhs(psi, M, kappa);
  } else {
    auto lap_psi = gridcalc::diff::laplacian<Order>(psi);
    Field<double> mu(psi.getGrid());
    const std::size_t n = psi.getSize();
    const double* p_psi = psi.data();
    const double* p_lap = lap_psi.data();
    double* p_mu = mu.data();
    for (std::size_t idx = 0; idx < n; ++idx) {
      const double p = p_psi[idx];
      p_mu[idx] = -p + p * p * p - kappa * p_lap[idx];
    }
    auto rhs = gridcalc::diff::laplacian<Order>(mu);
    double* p_rhs = rhs.data();
    for (std::size_t idx = 0; idx < n; ++idx) p_rhs[idx] *= M;
    return rhs;
  }
}

// The 31 named partials of diff/MixedPartial.hpp, ThirdOrder.hpp and
// FourthOrder.hpp, keyed by their per-axis derivative counts.
template <int O>
Field<double> namedPartial(int ax, int ay, int az, const Field<double>& f) {
  namespace d = gridcalc::diff;
  const int key = ax * 100 + ay * 10 + az;
  switch (key) {
    case 200: return d::dxx<O>(f);
    case 20: return d::dyy<O>(f);
    case 2: return d::dzz<O>(f);
    case 110: return d::dxy<O>(f);
    case 101: return d::dxz<O>(f);
    case 11: return d::dyz<O>(f);
    case 300: return d::d3dx3<O>(f);
    case 30: return d::d3dy3<O>(f);
    case 3: return d::d3dz3<O>(f);
    case 210: return d::d3dx2dy<O>(f);
    case 120: return d::d3dxdy2<O>(f);
    case 201: return d::d3dx2dz<O>(f);
    case 102: return d::d3dxdz2<O>(f);
    case 21: return d::d3dy2dz<O>(f);
    case 12: return d::d3dydz2<O>(f);
    case 111: return d::d3dxdydz<O>(f);
    case 400: return d::d4dx4<O>(f);
    case 40: return d::d4dy4<O>(f);
    case 4: return d::d4dz4<O>(f);
    case 310: return d::d4dx3dy<O>(f);
    case 130: return d::d4dxdy3<O>(f);
    case 301: return d::d4dx3dz<O>(f);
    case 103: return d::d4dxdz3<O>(f);
    case 31: return d::d4dy3dz<O>(f);
    case 13: return d::d4dydz3<O>(f);
    case 220: return d::d4dx2dy2<O>(f);
    case 202: return d::d4dx2dz2<O>(f);
    case 22: return d::d4dy2dz2<O>(f);
    case 211: return d::d4dx2dydz<O>(f);
    case 121: return d::d4dxdy2dz<O>(f);
    case 112: return d::d4dxdydz2<O>(f);
  }
  throw std::invalid_argument("ref: no named partial with these derivative counts");
}

}  // namespace

extern "C" {

int ref_mixed(int ax, int ay, int az, int order, int nx, int ny, int nz, double hx, double hy, double hz,
              const double* in, double* out) {
  return guarded([&] {
    const Grid g = makeGrid(nx, ny, nz, hx, hy, hz);
    const Field<double> f = load(g, in);
    if (order == 2) store(namedPartial<2>(ax, ay, az, f), out);
    else if (order == 4) store(namedPartial<4>(ax, ay, az, f), out);
    else throw std::invalid_argument("ref: partial order must be 2 or 4");
  });
}

const char* ref_last_error(void) { return g_err.c_str(); }

int ref_laplacian(int order, int nx, int ny, int nz, double hx, double hy, double hz,
                  const double* in, double* out) {
  return guarded([&] {
    const Grid g = makeGrid(nx, ny, nz, hx, hy, hz);
    const Field<double> f = load(g, in);
    if (order == 2) store(gridcalc::diff::laplacian<2>(f), out);
    else if (order == 4) store(gridcalc::diff::laplacian<4>(f), out);
    else throw std::invalid_argument("ref: laplacian order must be 2 or 4");
  });
}

int ref_gradient(int order, int nx, int ny, int nz, double hx, double hy, double hz,
                 const double* in, double* out3) {
  return guarded([&] {
    const Grid g = makeGrid(nx, ny, nz, hx, hy, hz);
    const Field<double> f = load(g, in);
    Field<Vec3d> r(g);
    if (order == 2) r = gridcalc::diff::gradient<2>(f);
    else if (order == 4) r = gridcalc::diff::gradient<4>(f);
    else throw std::invalid_argument("ref: gradient order must be 2 or 4");
    const std::size_t n = g.getSize();
    for (std::size_t i = 0; i < n; ++i) {
      const Vec3d& v = r.data()[i];
      out3[i] = v(0);
      out3[n + i] = v(1);
      out3[2 * n + i] = v(2);
    }
  });
}

int ref_divergence(int order, int nx, int ny, int nz, double hx, double hy, double hz,
                   const double* in3, double* out) {
  return guarded([&] {
    const Grid g = makeGrid(nx, ny, nz, hx, hy, hz);
    Field<Vec3d> v(g);
    const std::size_t n = g.getSize();
    for (std::size_t i = 0; i < n; ++i) v.data()[i] = Vec3d(in3[i], in3[n + i], in3[2 * n + i]);
    if (order == 2) store(gridcalc::diff::divergence<2>(v), out);
    else if (order == 4) store(gridcalc::diff::divergence<4>(v), out);
    else throw std::invalid_argument("ref: divergence order must be 2 or 4");
  });
}

// Matrix fields cross this boundary as nine planes, plane 3*row + col
// holding M(row, col); diff::gradient(Field<Vec3d>) puts d_col v_row there.
int ref_gradient_vec(int order, int nx, int ny, int nz, double hx, double hy, double hz,
                     const double* in3, double* out9) {
  return guarded([&] {
    const Grid g = makeGrid(nx, ny, nz, hx, hy, hz);
    Field<Vec3d> v(g);
    const std::size_t n = g.getSize();
    for (std::size_t i = 0; i < n; ++i) v.data()[i] = Vec3d(in3[i], in3[n + i], in3[2 * n + i]);
    Field<Mat3d> r(g);
    if (order == 2) r = gridcalc::diff::gradient<2>(v);
    else if (order == 4) r = gridcalc::diff::gradient<4>(v);
    else throw std::invalid_argument("ref: gradient order must be 2 or 4");
    for (std::size_t i = 0; i < n; ++i)
      for (int row = 0; row < 3; ++row)
        for (int col = 0; col < 3; ++col) out9[(3 * row + col) * n + i] = r.data()[i](row, col);
  });
}

int ref_divergence_mat(int order, int nx, int ny, int nz, double hx, double hy, double hz,
                       const double* in9, double* out3) {
  return guarded([&] {
    const Grid g = makeGrid(nx, ny, nz, hx, hy, hz);
    Field<Mat3d> m(g);
    const std::size_t n = g.getSize();
    for (std::size_t i = 0; i < n; ++i)
      for (int row = 0; row < 3; ++row)
        for (int col = 0; col < 3; ++col) m.data()[i](row, col) = in9[(3 * row + col) * n + i];
    Field<Vec3d> r(g);
    if (order == 2) r = gridcalc::diff::divergence<2>(m);
    else if (order == 4) r = gridcalc::diff::divergence<4>(m);
    else throw std::invalid_argument("ref: divergence order must be 2 or 4");
    for (std::size_t i = 0; i < n; ++i) {
      out3[i] = r.data()[i](0);
      out3[n + i] = r.data()[i](1);
      out3[2 * n + i] = r.data()[i](2);
    }
  });
}

// func::evaluate (func/Functional.hpp:88-148, :183-220) with a callable of
// the program's arity; the reference materialises the derivative fields and
// integrates the integrand itself.
int ref_evaluate_program(int components, int arity, int nx, int ny, int nz, double hx, double hy, double hz,
                         const double* field, const RefInstr* prog, int n_instr, int kahan, double* result) {
  return guarded([&] {
    const Grid g = makeGrid(nx, ny, nz, hx, hy, hz);
    auto run = [&](const double* in) { return runProgram(prog, n_instr, in); };
    if (components == 1) {
      const Field<double> f = load(g, field);
      auto ev = [&](auto&& fn) {
        *result = kahan ? gridcalc::func::evaluate(f, fn, gridcalc::func::Kahan{}) : gridcalc::func::evaluate(f, fn);
      };
      if (arity == 1) {
        ev([&](double p) { const double in[1] = {p}; return run(in); });
      } else if (arity == 2) {
        ev([&](double p, const Vec3d& d) { const double in[4] = {p, d(0), d(1), d(2)}; return run(in); });
      } else if (arity == 3) {
        ev([&](double p, const Vec3d& d, double l) { const double in[5] = {p, d(0), d(1), d(2), l}; return run(in); });
      } else if (arity == 4) {
        ev([&](double p, const Vec3d& d, double l, double b) {
          const double in[6] = {p, d(0), d(1), d(2), l, b};
          return run(in);
        });
      } else {
        throw std::invalid_argument("ref: scalar arity must be 1..4");
      }
    } else if (components == 3) {
      Field<Vec3d> u(g);
      const std::size_t n = g.getSize();
      for (std::size_t i = 0; i < n; ++i) u.data()[i] = Vec3d(field[i], field[n + i], field[2 * n + i]);
      auto ev = [&](auto&& fn) {
        *result = kahan ? gridcalc::func::evaluate(u, fn, gridcalc::func::Kahan{}) : gridcalc::func::evaluate(u, fn);
      };
      if (arity == 1) {
        ev([&](const Vec3d& v) { const double in[3] = {v(0), v(1), v(2)}; return run(in); });
      } else if (arity == 2) {
        ev([&](const Vec3d& v, const Mat3d& M) {
          double in[12] = {v(0), v(1), v(2)};
          for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) in[3 + 3 * r + c] = M(r, c);
          return run(in);
        });
      } else {
        throw std::invalid_argument("ref: vector arity must be 1 or 2");
      }
    } else {
      throw std::invalid_argument("ref: components must be 1 or 3");
    }
  });
}

// examples/common/vtk_writer.hpp:34-66, the reference's snapshot writer.
int ref_write_vtk(int nx, int ny, int nz, double hx, double hy, double hz, const double* f, const char* path,
                  const char* name) {
  return guarded([&] {
    const Grid g = makeGrid(nx, ny, nz, hx, hy, hz);
    gridcalc::examples::writeVtkStructuredPoints(load(g, f), path, name);
  });
}

// spectral/Derivatives.hpp: the reference's PocketFFT path.  op: 0 partial
// (counts ax, ay, az in 0..4), 1 laplacian, 2 biharmonic, 3 gradient (out: 3 planes).
int ref_spectral(int op, int ax, int ay, int az, int nx, int ny, int nz, double hx, double hy, double hz,
                 const double* in, double* out) {
  return guarded([&] {
    const Grid g = makeGrid(nx, ny, nz, hx, hy, hz);
    const Field<double> f = load(g, in);
    if (op == 0) {
      if (ax < 0 || ay < 0 || az < 0 || ax > 4 || ay > 4 || az > 4)
        throw std::invalid_argument("ref: spectral counts must be 0..4");
      kSpectral[static_cast<std::size_t>(25 * ax + 5 * ay + az)](f, out);
    } else if (op == 1) {
      store(gridcalc::spectral::laplacian(f), out);
    } else if (op == 2) {
      store(gridcalc::spectral::biharmonic(f), out);
    } else {
      const Field<Vec3d> r = gridcalc::spectral::gradient(f);
      const std::size_t n = g.getSize();
      for (std::size_t i = 0; i < n; ++i) {
        out[i] = r.data()[i](0);
        out[n + i] = r.data()[i](1);
        out[2 * n + i] = r.data()[i](2);
      }
    }
  });
}

int ref_biharmonic(int order, int nx, int ny, int nz, double hx, double hy, double hz,
                   const double* in, double* out) {
  return guarded([&] {
    const Grid g = makeGrid(nx, ny, nz, hx, hy, hz);
    const Field<double> f = load(g, in);
    if (order == 2) store(gridcalc::diff::biharmonic<2>(f), out);
    else if (order == 4) store(gridcalc::diff::biharmonic<4>(f), out);
    else throw std::invalid_argument("ref: biharmonic order must be 2 or 4");
  });
}

int ref_cell_laplacian(int nx, int ny, int nz, double hx, double hy, double hz,
                       const double* psi, const double* D, double* out) {
  return guarded([&] {
    const Grid g = makeGrid(nx, ny, nz, hx, hy, hz);
    store(gridcalc::fvm::cellLaplacian(load(g, psi), load(g, D)), out);
  });
}

double ref_integrate(int nx, int ny, int nz, double hx, double hy, double hz,
                     const double* in, int kahan) {
  const Grid g = makeGrid(nx, ny, nz, hx, hy, hz);
  const Field<double> f = load(g, in);
  return kahan ? gridcalc::func::integrate(f, gridcalc::func::Kahan{})
               : gridcalc::func::integrate(f, gridcalc::func::Pairwise{});
}

int ref_ch_rhs(int order, double M, double kappa, int nx, int ny, int nz, double hx,
               double hy, double hz, const double* psi, double* out) {
  return guarded([&] {
    const Grid g = makeGrid(nx, ny, nz, hx, hy, hz);
    const Field<double> f = load(g, psi);
    if (order == 2) store(chRhs<2>(f, M, kappa), out);
    else if (order == 4) store(chRhs<4>(f, M, kappa), out);
    else throw std::invalid_argument("ref: CH order must be 2 or 4");
  });
}

// integrator: 0 = ExplicitEuler, 1 = RK4 (solve/ExplicitEuler.hpp:79,
// solve/RK4.hpp:99).  psi is advanced in place.
int ref_ch_integrate(int order, double M, double kappa, int nx, int ny, int nz, double hx,
                     double hy, double hz, double* psi, double dt, int n_steps,
                     int integrator) {
  return guarded([&] {
    const Grid g = makeGrid(nx, ny, nz, hx, hy, hz);
    Field<double> f = load(g, psi);
    auto run = [&](auto rhs) {
      if (integrator == 1) gridcalc::solve::integrate(f, rhs, dt, n_steps, gridcalc::solve::RK4{});
      else gridcalc::solve::integrate(f, rhs, dt, n_steps, gridcalc::solve::ExplicitEuler{});
    };
    if (order == 2) run([&](const Field<double>& p) { return chRhs<2>(p, M, kappa); });
    else if (order == 4) run([&](const Field<double>& p) { return chRhs<4>(p, M, kappa); });
    else throw std::invalid_argument("ref: CH order must be 2 or 4");
    store(f, psi);
  });
}

double ref_ch_free_energy(int nx, int ny, int nz, double hx, double hy, double hz,
                          const double* psi, double kappa) {
  const Grid g = makeGrid(nx, ny, nz, hx, hy, hz);
  return ch::computeFreeEnergy(load(g, psi), kappa);
}

double ref_ch_gradient_energy(int nx, int ny, int nz, double hx, double hy, double hz,
                              const double* psi) {
  const Grid g = makeGrid(nx, ny, nz, hx, hy, hz);
  return ch::computeGradientEnergy(load(g, psi));
}

double ref_ch_mean(int nx, int ny, int nz, double hx, double hy, double hz, const double* psi) {
  const Grid g = makeGrid(nx, ny, nz, hx, hy, hz);
  return ch::computeMean(load(g, psi));
}

void ref_make_random_ic(int nx, int ny, int nz, double hx, double hy, double hz,
                        uint64_t seed, double amplitude, double* out) {
  const Grid g = makeGrid(nx, ny, nz, hx, hy, hz);
  store(ch::makeRandomIc(g, seed, amplitude), out);
}

// The draws of makeRandomIc before its mean subtraction
// (examples/common/cahn_hilliard.hpp:89-95): std::mt19937_64(seed) through
// std::uniform_real_distribution<double>(-amplitude, amplitude), one per
// value, in order.  Pins the product's generator when it keeps raw draws.
void ref_uniform_draws(uint64_t seed, double amplitude, size_t n, double* out) {
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> dist(-amplitude, amplitude);
  for (size_t i = 0; i < n; ++i) out[i] = dist(rng);
}

// Constant-D heat equation, solve/Diffusion.hpp:89-112.
int ref_diffuse_const(int nx, int ny, int nz, double hx, double hy, double hz, double* psi,
                      double D, double dt, int n_steps, int integrator) {
  return guarded([&] {
    const Grid g = makeGrid(nx, ny, nz, hx, hy, hz);
    Field<double> f = load(g, psi);
    if (integrator == 1) gridcalc::solve::diffuse(f, D, dt, n_steps, gridcalc::solve::RK4{});
    else gridcalc::solve::diffuse(f, D, dt, n_steps, gridcalc::solve::ExplicitEuler{});
    store(f, psi);
  });
}

// Heterogeneous-D FVM heat equation, solve/Diffusion.hpp:161-216.
int ref_diffuse_fvm(int nx, int ny, int nz, double hx, double hy, double hz, double* psi,
                    const double* D, double dt, int n_steps, int integrator) {
  return guarded([&] {
    const Grid g = makeGrid(nx, ny, nz, hx, hy, hz);
    Field<double> f = load(g, psi);
    const Field<double> d = load(g, D);
    if (integrator == 1) gridcalc::solve::diffuse(f, d, dt, n_steps, gridcalc::solve::RK4{});
    else gridcalc::solve::diffuse(f, d, dt, n_steps, gridcalc::solve::ExplicitEuler{});
    store(f, psi);
  });
}

}  // extern "C"
