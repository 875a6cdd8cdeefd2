// The C++ drop-in used the way the reference's own tests use gridcalc:
// the same headers, names and calls, restating known answers of
// test/fvm_cell_laplacian_test.cpp, test/integrate_test.cpp,
// test/laplacian_test.cpp, test/diffusion_test.cpp,
// test/stencil_axis_extent_test.cpp and test/cahn_hilliard_test.cpp.
// Prints "PASS <name>" per check and exits non-zero on the first failure.
#include <gridcalc/core/Field.hpp>
#include <gridcalc/core/Grid.hpp>
#include <gridcalc/diff/Gradient.hpp>
#include <gridcalc/diff/FourthOrder.hpp>
#include <gridcalc/diff/Laplacian.hpp>
#include <gridcalc/diff/MixedPartial.hpp>
#include <gridcalc/diff/ThirdOrder.hpp>
#include <gridcalc/func/Functional.hpp>
#include <gridcalc/spectral/Derivatives.hpp>
#include <gridcalc/func/Integrate.hpp>
#include <gridcalc/fvm/CellLaplacian.hpp>
#include <gridcalc/solve/Diffusion.hpp>
#include <gridcalc/solve/Integrator.hpp>

#include <common/vtk_writer.hpp>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>

using gridcalc::core::Field;
using gridcalc::core::Grid;
using gridcalc::core::Vec3d;

static void require(bool ok, const char* name) {
  if (!ok) {
    std::printf("FAIL %s\n", name);
    std::exit(1);
  }
  std::printf("PASS %s\n", name);
}

int main() {
  const double kPi = 3.14159265358979323846;
  {  // harmonic-mean face coefficient, +-1.6
    Grid g(4, 1, 1, Vec3d(1.0, 1.0, 1.0));
    Field<double> psi(g, 0.0), D(g, 0.0);
    psi(1, 0, 0) = 1.0;
    psi(2, 0, 0) = 1.0;
    D(0, 0, 0) = 1.0; D(1, 0, 0) = 4.0; D(2, 0, 0) = 4.0; D(3, 0, 0) = 1.0;
    auto rhs = gridcalc::fvm::cellLaplacian(psi, D);
    require(std::abs(rhs(0, 0, 0) - 1.6) < 1e-15 && std::abs(rhs(1, 0, 0) + 1.6) < 1e-15 &&
                std::abs(rhs(2, 0, 0) + 1.6) < 1e-15 && std::abs(rhs(3, 0, 0) - 1.6) < 1e-15,
            "fvm harmonic mean face coefficient");
  }
  {  // unit field integrates to the domain volume, both tags
    Grid g(8, 16, 4, Vec3d(0.25, 0.125, 0.5));
    Field<double> ones(g, 1.0);
    const double vol = (8 * 0.25) * (16 * 0.125) * (4 * 0.5);
    require(gridcalc::func::integrate(ones) == vol && gridcalc::func::integrate(ones, gridcalc::func::Kahan{}) == vol,
            "integrate unit field");
  }
  {  // laplacian eigenfunction, relative max error < 1.5e-2 at N = 32
    const int N = 32;
    const double h = 2 * kPi / N;
    Grid g(N, N, N, Vec3d(h, h, h));
    Field<double> f(g, [](double x, double y, double z) { return std::sin(x) * std::sin(y) * std::sin(z); });
    auto lap = gridcalc::diff::laplacian<2>(f);
    double err = 0, ref = 0;
    for (size_t i = 0; i < f.size(); ++i) {
      err = std::max(err, std::abs(lap.data()[i] + 3 * f.data()[i]));
      ref = std::max(ref, std::abs(3 * f.data()[i]));
    }
    require(err / ref < 1.5e-2, "laplacian eigenfunction");
    auto grad = gridcalc::diff::gradient<4>(f);
    require(std::abs(grad(3, 5, 7)(0) - std::cos(3 * h) * std::sin(5 * h) * std::sin(7 * h)) < 1e-4, "gradient order 4");
  }
  {  // axis-extent error names the axis
    Grid g(8, 3, 8, Vec3d(1, 1, 1));
    Field<double> f(g, 0.0);
    bool threw = false;
    try {
      gridcalc::diff::laplacian<4>(f);
    } catch (const std::invalid_argument& e) {
      threw = std::string(e.what()).find("axis y") != std::string::npos;
    }
    require(threw, "axis extent message");
  }
  {  // diffusion decays as exp(-3 D t); CFL violation throws with solve::diffuse
    const int N = 32;
    const double h = 2 * kPi / N;
    Grid g(N, N, N, Vec3d(h, h, h));
    Field<double> f(g, [](double x, double y, double z) { return std::sin(x) * std::sin(y) * std::sin(z); });
    const double m0 = f(8, 8, 8);
    gridcalc::solve::diffuse(f, 0.5, 0.01, 100, gridcalc::solve::RK4{});
    require(std::abs(f(8, 8, 8) / m0 - std::exp(-1.5)) < 5e-3, "diffusion decay");
    bool threw = false;
    try {
      gridcalc::solve::diffuse(f, 1.0, 1.0, 1, gridcalc::solve::RK4{});
    } catch (const std::invalid_argument& e) {
      threw = std::string(e.what()).find("solve::diffuse") != std::string::npos;
    }
    require(threw, "CFL message");
  }
  {  // Cahn-Hilliard: mass conserved, free energy decreases (cahn_hilliard_test.cpp)
    Grid g(64, 64, 1, Vec3d(1, 1, 1));
    std::srand(42);
    Field<double> psi(g, [](double, double, double) { return 0.1 * (2.0 * std::rand() / RAND_MAX - 1.0); });
    double mean = gridcalc::func::integrate(psi) / g.getSize();
    for (auto& v : psi) v -= mean;
    const double F0 = gridcalc::func::evaluate(psi, gridcalc::func::FreeEnergy{1.0});
    const double m0 = gridcalc::func::integrate(psi, gridcalc::func::Kahan{});
    gridcalc::solve::integrate(psi, gridcalc::solve::CahnHilliardRhs{1.0, 1.0, 2}, 0.01, 3000, gridcalc::solve::RK4{});
    const double F1 = gridcalc::func::evaluate(psi, gridcalc::func::FreeEnergy{1.0});
    const double m1 = gridcalc::func::integrate(psi, gridcalc::func::Kahan{});
    require(F1 < F0 && std::abs(m1 - m0) < 1e-10, "cahn-hilliard energy decay and mass");
  }
  {  // named partials on sin x sin y sin z (phase_8_test.cpp style): dxy, d3dxdydz, d4dx2dy2
    const int N = 32;
    const double h = 2 * kPi / N;
    Grid g(N, N, N, Vec3d(h, h, h));
    Field<double> f(g, [](double x, double y, double z) { return std::sin(x) * std::sin(y) * std::sin(z); });
    const auto fxy = gridcalc::diff::dxy<4>(f);
    const auto fxyz = gridcalc::diff::d3dxdydz<4>(f);
    const auto fxxyy = gridcalc::diff::d4dx2dy2<4>(f);
    double e2 = 0, e3 = 0, e4 = 0;
    for (int k = 0; k < N; ++k)
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) {
          const double x = i * h, y = j * h, z = k * h;
          e2 = std::max(e2, std::abs(fxy(i, j, k) - std::cos(x) * std::cos(y) * std::sin(z)));
          e3 = std::max(e3, std::abs(fxyz(i, j, k) - std::cos(x) * std::cos(y) * std::cos(z)));
          e4 = std::max(e4, std::abs(fxxyy(i, j, k) - std::sin(x) * std::sin(y) * std::sin(z)));
        }
    require(e2 < 2e-4 && e3 < 3e-4 && e4 < 1e-4, "named partials dxy, d3dxdydz, d4dx2dy2");
  }
  {  // rank-2 forms (vector_tensor_test.cpp): trace(grad v) == div v, div(grad v) ~ -2 v
    const int N = 32;
    const double h = 2 * kPi / N;
    Grid g(N, N, N, Vec3d(h, h, h));
    Field<Vec3d> v(g);
    for (int k = 0; k < N; ++k)
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) {
          const double x = i * h, y = j * h, z = k * h;
          v(i, j, k) = Vec3d(std::sin(x) * std::cos(y), std::sin(y) * std::cos(z), std::sin(z) * std::cos(x));
        }
    const Field<gridcalc::core::Mat3d> M = gridcalc::diff::gradient(v);
    const Field<double> div = gridcalc::diff::divergence(v);
    const Field<Vec3d> lap = gridcalc::diff::divergence(M);
    double dtr = 0, elap = 0;
    for (size_t i = 0; i < v.size(); ++i) {
      const auto& m = M.data()[i];
      dtr = std::max(dtr, std::abs((m(0, 0) + m(1, 1)) + m(2, 2) - div.data()[i]));
      for (int c = 0; c < 3; ++c) elap = std::max(elap, std::abs(lap.data()[i](c) + 2 * v.data()[i](c)));
    }
    require(dtr == 0.0 && elap < 3e-2, "rank-2 gradient and divergence");
  }
  {  // func::evaluate with generic callables: recorded free energy == the device functor,
     // trace(grad u) integrates to the integral of div u, bit for bit
    const int N = 24;
    const double h = 2 * kPi / N;
    Grid g(N, N, N, Vec3d(h, h, h));
    Field<double> psi(g, [](double x, double y, double z) { return 0.3 * std::sin(x) * std::cos(2 * y) + 0.1 * z; });
    const double fe = gridcalc::func::evaluate(
        psi, [](auto p, const auto& d) { return -0.5 * p * p + 0.25 * p * p * p * p + 0.5 * 1.0 * d.squaredNorm(); });
    const double fe_dev = gridcalc::func::evaluate(psi, gridcalc::func::FreeEnergy{1.0});
    const double b4 = gridcalc::func::evaluate(psi, [](auto p, const auto&, auto lap, auto bih) {
      return gridcalc::func::max(p, 0.0) + lap * bih / (1.0 + gridcalc::func::abs(p));
    });
    Field<Vec3d> u(g);
    for (int k = 0; k < N; ++k)
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i)
          u(i, j, k) = Vec3d(std::sin(i * h) * std::cos(j * h), std::sin(j * h) * std::cos(k * h), std::sin(k * h));
    const double tr = gridcalc::func::evaluate(u, [](const auto&, const auto& M) { return M.trace(); });
    const double dv = gridcalc::func::integrate(gridcalc::diff::divergence(u));
    require(fe == fe_dev && std::isfinite(b4) && tr == dv, "func::evaluate with recorded callables");
  }
  {  // examples/common/vtk_writer.hpp: header lines and 17-digit values
    Grid g(3, 2, 1, Vec3d(0.5, 0.25, 1.0));
    Field<double> f(g, [](double x, double y, double) { return x / 3.0 - y; });
    const std::string path = "dropin_snapshot.vtk";
    gridcalc::examples::writeVtkStructuredPoints(f, path, "psi");
    std::FILE* in = std::fopen(path.c_str(), "r");
    char line[128];
    int lines = 0;
    bool ok = in != nullptr;
    std::string eleventh, spacing;
    while (ok && std::fgets(line, sizeof line, in)) {
      ++lines;
      if (lines == 7) spacing = line;
      if (lines == 11) eleventh = line;
    }
    if (in) std::fclose(in);
    std::remove(path.c_str());
    char want[64];
    std::snprintf(want, sizeof want, "%.17g\n", f.data()[0]);
    bool threw = false;
    try {
      gridcalc::examples::writeVtkStructuredPoints(f, "no/such/dir/x.vtk", "psi");
    } catch (const std::runtime_error&) {
      threw = true;
    }
    require(ok && lines == 16 && spacing == "SPACING 0.5 0.25 1\n" && eleventh == want && threw, "vtk writer");
  }
  {  // spectral/Derivatives.hpp: exact on a band-limited field
    const int N = 16;
    const double h = 2 * kPi / N;
    Grid g(N, N, N, Vec3d(h, h, h));
    Field<double> f(g, [](double x, double y, double z) { return std::sin(x) * std::cos(2 * y) * std::sin(z); });
    const auto lap = gridcalc::spectral::laplacian(f);
    const auto fxy = gridcalc::spectral::partial<1, 1, 0>(f);
    const auto grad = gridcalc::spectral::gradient(f);
    double e1 = 0, e2 = 0, e3 = 0;
    for (int k = 0; k < N; ++k)
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) {
          const double x = i * h, y = j * h, z = k * h;
          e1 = std::max(e1, std::abs(lap(i, j, k) + 6 * f(i, j, k)));
          e2 = std::max(e2, std::abs(fxy(i, j, k) + 2 * std::cos(x) * std::sin(2 * y) * std::sin(z)));
          e3 = std::max(e3, std::abs(grad(i, j, k)(2) - std::sin(x) * std::cos(2 * y) * std::cos(z)));
        }
    require(e1 < 1e-12 && e2 < 1e-12 && e3 < 1e-12, "spectral derivatives");
  }
  std::printf("version %s\n", gridcalc::version());
  return 0;
}
