// Drop-in for the reference header of the same path: spectral::partial,
// laplacian, biharmonic and gradient (spectral/Derivatives.hpp) computed on
// the GPU (this library's own FFT kernels around its multiplier kernel).  The
// reference compiles these only with GRIDCALC_USE_FFT; here they are always
// available.
#pragma once

#include <gridcalc/b200.hpp>

namespace gridcalc::spectral {

template <int Nx, int Ny, int Nz>
inline core::Field<double> partial(const core::Field<double>& field) {
  return diff::detail::scalar_op(field, [](const gc_grid* g, const double* in, double* out) {
    return gc_spectral_partial(b200::context(), g, GC_F64, Nx, Ny, Nz, in, out);
  });
}

inline core::Field<double> laplacian(const core::Field<double>& field) {
  return diff::detail::scalar_op(field, [](const gc_grid* g, const double* in, double* out) {
    return gc_spectral_laplacian(b200::context(), g, GC_F64, in, out);
  });
}

inline core::Field<double> biharmonic(const core::Field<double>& field) {
  return diff::detail::scalar_op(field, [](const gc_grid* g, const double* in, double* out) {
    return gc_spectral_biharmonic(b200::context(), g, GC_F64, in, out);
  });
}

inline core::Field<core::Vec3d> gradient(const core::Field<double>& field) {
  const core::Grid& grid = field.getGrid();
  const size_t n = grid.getSize();
  core::DeviceField<double> in(field), out(grid, 3);
  const gc_grid g = grid.c();
  b200::check(gc_spectral_gradient(b200::context(), &g, GC_F64, in.data(), out.data()));
  std::vector<double> planes(3 * n);
  out.download(planes.data());
  core::Field<core::Vec3d> r(grid);
  for (size_t i = 0; i < n; ++i) r.data()[i] = core::Vec3d(planes[i], planes[n + i], planes[2 * n + i]);
  return r;
}

}  // namespace gridcalc::spectral
