// gridcalc drop-in over libgridcalc_b200 (header-only C++17 host side).
//
// Mirrors the reference gridcalc 0.15.1 hot-path API -- core::Grid,
// core::Field<T> (core/Grid.hpp, core/Field.hpp), diff::laplacian /
// gradient / divergence / biharmonic / d4 (diff/*.hpp), fvm::cellLaplacian
// (fvm/CellLaplacian.hpp), func::integrate / evaluate (func/*.hpp),
// solve::integrate with RK4 / ExplicitEuler and solve::diffuse
// (solve/*.hpp) -- with the same names, argument meaning and error
// behaviour (std::invalid_argument carrying the same message substrings),
// computed on the GPU through the C ABI in gridcalc_b200.h.
//
// Host fields (Field<double>) are copied to the device per call and back;
// DeviceField<T> keeps a field resident for device-side pipelines.  Where the
// reference accepts an arbitrary host callable (an RHS or an integrand) the
// drop-in takes a device functor type instead: solve::CahnHilliardRhs for
// solve::integrate (the diffusion right-hand sides are reached through
// solve::diffuse, as in the reference); func::FreeEnergy,
// func::GradientEnergy, func::Identity, func::Square for func::evaluate.  Vector fields are Field<Vec3d>
// (interleaved, as the reference) on the host and three planes on the device.
#pragma once

#include <gridcalc_b200.h>

#include <array>
#include <cstddef>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#if __has_include(<Eigen/Core>)
#include <Eigen/Core>
#define GRIDCALC_B200_HAVE_EIGEN 1
#endif

namespace gridcalc {

namespace b200 {

inline void check(gc_status s) {
  if (s != GC_OK) throw std::invalid_argument(gc_last_error());
}

// Thread-local context on device 0, created on first use.
inline gc_context* context() {
  struct Holder {
    gc_context* ctx = nullptr;
    Holder() { check(gc_context_create(&ctx, 0, nullptr)); }
    ~Holder() { gc_context_destroy(ctx); }
  };
  thread_local Holder holder;
  return holder.ctx;
}

// Owning device buffer.
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  explicit DeviceBuffer(size_t bytes) : bytes_(bytes) {
    if (bytes) check(gc_malloc(context(), bytes, &ptr_));
  }
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  DeviceBuffer(DeviceBuffer&& o) noexcept : ptr_(o.ptr_), bytes_(o.bytes_) { o.ptr_ = nullptr; o.bytes_ = 0; }
  DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
    std::swap(ptr_, o.ptr_);
    std::swap(bytes_, o.bytes_);
    return *this;
  }
  ~DeviceBuffer() {
    if (ptr_) gc_free(context(), ptr_);
  }
  void* get() const { return ptr_; }
  size_t bytes() const { return bytes_; }
  void upload(const void* host) { check(gc_memcpy_h2d(context(), ptr_, host, bytes_)); }
  void download(void* host) const { check(gc_memcpy_d2h(context(), host, ptr_, bytes_)); }

 private:
  void* ptr_ = nullptr;
  size_t bytes_ = 0;
};

template <class T>
constexpr gc_dtype dtype_of() {
  static_assert(std::is_same_v<T, double> || std::is_same_v<T, float>, "fields are double or float");
  return std::is_same_v<T, double> ? GC_F64 : GC_F32;
}

}  // namespace b200

namespace core {

#ifdef GRIDCALC_B200_HAVE_EIGEN
using Vec3d = Eigen::Vector3d;
using Mat3d = Eigen::Matrix3d;
#else
// Stand-in for Eigen::Vector3d when Eigen is not on the include path.
class Vec3d {
 public:
  Vec3d() : v_{0.0, 0.0, 0.0} {}
  Vec3d(double x, double y, double z) : v_{x, y, z} {}
  double& operator()(int i) { return v_[i]; }
  const double& operator()(int i) const { return v_[i]; }
  double squaredNorm() const { return v_[0] * v_[0] + v_[1] * v_[1] + v_[2] * v_[2]; }
 private:
  double v_[3];
};

// Stand-in for Eigen::Matrix3d: M(row, col), zero-initialised.
class Mat3d {
 public:
  Mat3d() : m_{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0} {}
  double& operator()(int r, int c) { return m_[3 * r + c]; }
  const double& operator()(int r, int c) const { return m_[3 * r + c]; }
  double trace() const { return m_[0] + m_[4] + m_[8]; }
 private:
  double m_[9];
};
#endif

// core::Grid (core/Grid.hpp:28-148).
class Grid {
 public:
  Grid(int Nx, int Ny, int Nz, const Vec3d& cell_size) : nx_(Nx), ny_(Ny), nz_(Nz), h_{cell_size(0), cell_size(1), cell_size(2)} {
    if (Nx <= 0 || Ny <= 0 || Nz <= 0)
      throw std::invalid_argument("Grid: extents (Nx, Ny, Nz) must be > 0; got (" + std::to_string(Nx) + ", " +
                                  std::to_string(Ny) + ", " + std::to_string(Nz) + ")");
    if (!(h_[0] > 0.0) || !(h_[1] > 0.0) || !(h_[2] > 0.0))
      throw std::invalid_argument("Grid: cell_size components must be > 0");
  }
  int getNx() const noexcept { return nx_; }
  int getNy() const noexcept { return ny_; }
  int getNz() const noexcept { return nz_; }
  Vec3d getCellSize() const { return Vec3d(h_[0], h_[1], h_[2]); }
  bool operator==(const Grid& o) const noexcept {
    return nx_ == o.nx_ && ny_ == o.ny_ && nz_ == o.nz_ && h_[0] == o.h_[0] && h_[1] == o.h_[1] && h_[2] == o.h_[2];
  }
  bool operator!=(const Grid& o) const noexcept { return !(*this == o); }
  double getCellVolume() const noexcept { return h_[0] * h_[1] * h_[2]; }
  std::size_t getSize() const noexcept { return static_cast<std::size_t>(nx_) * ny_ * nz_; }
  std::size_t size() const noexcept { return getSize(); }
  std::size_t getLinearIndex(int i, int j, int k) const noexcept {
    return static_cast<std::size_t>(i) + static_cast<std::size_t>(nx_) * (static_cast<std::size_t>(j) + static_cast<std::size_t>(ny_) * k);
  }
  gc_grid c() const { return gc_grid{nx_, ny_, nz_, h_[0], h_[1], h_[2]}; }

 private:
  int nx_, ny_, nz_;
  double h_[3];
};

namespace IndexPolicy {
struct Periodic {
  static constexpr int wrap(int i, int N) noexcept { return ((i % N) + N) % N; }
};
}  // namespace IndexPolicy

// core::Field<T, Policy> (core/Field.hpp:36-145): host storage.
template <class T, class Policy = IndexPolicy::Periodic>
class Field {
 public:
  using value_type = T;
  using policy_type = Policy;
  explicit Field(const Grid& grid) : grid_(grid), data_(grid.getSize()) {}
  Field(const Grid& grid, const T& value) : grid_(grid), data_(grid.getSize(), value) {}
  template <class F, std::enable_if_t<std::is_invocable_r_v<T, F&, double, double, double>, int> = 0>
  Field(const Grid& grid, F&& f) : grid_(grid), data_(grid.getSize()) {
    const auto h = grid_.getCellSize();
    for (int k = 0; k < grid_.getNz(); ++k)
      for (int j = 0; j < grid_.getNy(); ++j)
        for (int i = 0; i < grid_.getNx(); ++i)
          data_[grid_.getLinearIndex(i, j, k)] = static_cast<T>(f(i * h(0), j * h(1), k * h(2)));
  }
  T& operator()(int i, int j, int k) noexcept {
    return data_[grid_.getLinearIndex(Policy::wrap(i, grid_.getNx()), Policy::wrap(j, grid_.getNy()), Policy::wrap(k, grid_.getNz()))];
  }
  const T& operator()(int i, int j, int k) const noexcept {
    return data_[grid_.getLinearIndex(Policy::wrap(i, grid_.getNx()), Policy::wrap(j, grid_.getNy()), Policy::wrap(k, grid_.getNz()))];
  }
  const Grid& getGrid() const noexcept { return grid_; }
  std::size_t getSize() const noexcept { return data_.size(); }
  std::size_t size() const noexcept { return data_.size(); }
  T* data() noexcept { return data_.data(); }
  const T* data() const noexcept { return data_.data(); }
  T* begin() noexcept { return data_.data(); }
  const T* begin() const noexcept { return data_.data(); }
  T* end() noexcept { return data_.data() + data_.size(); }
  const T* end() const noexcept { return data_.data() + data_.size(); }

 private:
  Grid grid_;
  std::vector<T> data_;
};

// A field resident on the device (float or double), for device pipelines.
template <class T>
class DeviceField {
 public:
  explicit DeviceField(const Grid& grid, int components = 1)
      : grid_(grid), comps_(components), buf_(sizeof(T) * grid.getSize() * components) {}
  explicit DeviceField(const Field<T>& host) : DeviceField(host.getGrid()) { buf_.upload(host.data()); }
  const Grid& getGrid() const { return grid_; }
  T* data() { return static_cast<T*>(buf_.get()); }
  const T* data() const { return static_cast<const T*>(buf_.get()); }
  int components() const { return comps_; }
  void upload(const T* host) { buf_.upload(host); }
  void download(T* host) const { buf_.download(host); }
  Field<T> toHost() const {
    Field<T> f(grid_);
    buf_.download(f.data());
    return f;
  }

 private:
  Grid grid_;
  int comps_;
  b200::DeviceBuffer buf_;
};

}  // namespace core

namespace diff {

namespace detail {
template <class Call>
core::Field<double> scalar_op(const core::Field<double>& f, Call&& call) {
  core::DeviceField<double> in(f), out(f.getGrid());
  const gc_grid g = f.getGrid().c();
  b200::check(call(&g, in.data(), out.data()));
  return out.toHost();
}
}  // namespace detail

// diff::laplacian<Order> (diff/Laplacian.hpp:44-75); Order 2, 4 or 6.
template <int Order = 2>
inline core::Field<double> laplacian(const core::Field<double>& field) {
  return detail::scalar_op(field, [](const gc_grid* g, const double* in, double* out) {
    return gc_laplacian(b200::context(), g, GC_F64, Order, in, out);
  });
}
template <int Order = 2, class T>
inline void laplacian(const core::DeviceField<T>& in, core::DeviceField<T>& out) {
  const gc_grid g = in.getGrid().c();
  b200::check(gc_laplacian(b200::context(), &g, b200::dtype_of<T>(), Order, in.data(), out.data()));
}

// diff::detail::mixedDerivative<Nx, Ny, Nz, Order>
// (diff/detail/MultiIndexDerivative.hpp:96-137) and the 31 named partials
// that forward to it (diff/MixedPartial.hpp, ThirdOrder.hpp, FourthOrder.hpp).
namespace detail {
template <int Nx, int Ny, int Nz, int Order>
inline core::Field<double> mixedDerivative(const core::Field<double>& psi) {
  return scalar_op(psi, [](const gc_grid* g, const double* in, double* out) {
    return gc_partial(b200::context(), g, GC_F64, Order, Nx, Ny, Nz, in, out);
  });
}
template <int Nx, int Ny, int Nz, int Order, class T>
inline void mixedDerivative(const core::DeviceField<T>& in, core::DeviceField<T>& out) {
  const gc_grid g = in.getGrid().c();
  b200::check(gc_partial(b200::context(), &g, b200::dtype_of<T>(), Order, Nx, Ny, Nz, in.data(), out.data()));
}
}  // namespace detail

#define GRIDCALC_B200_PARTIAL(name, nx, ny, nz)                                         \
  template <int Order = 2>                                                              \
  inline core::Field<double> name(const core::Field<double>& psi) {                     \
    return detail::mixedDerivative<nx, ny, nz, Order>(psi);                             \
  }                                                                                     \
  template <int Order = 2, class T>                                                     \
  inline void name(const core::DeviceField<T>& in, core::DeviceField<T>& out) {         \
    detail::mixedDerivative<nx, ny, nz, Order>(in, out);                                \
  }
GRIDCALC_B200_PARTIAL(dxx, 2, 0, 0)
GRIDCALC_B200_PARTIAL(dyy, 0, 2, 0)
GRIDCALC_B200_PARTIAL(dzz, 0, 0, 2)
GRIDCALC_B200_PARTIAL(dxy, 1, 1, 0)
GRIDCALC_B200_PARTIAL(dxz, 1, 0, 1)
GRIDCALC_B200_PARTIAL(dyz, 0, 1, 1)
GRIDCALC_B200_PARTIAL(d3dx3, 3, 0, 0)
GRIDCALC_B200_PARTIAL(d3dy3, 0, 3, 0)
GRIDCALC_B200_PARTIAL(d3dz3, 0, 0, 3)
GRIDCALC_B200_PARTIAL(d3dx2dy, 2, 1, 0)
GRIDCALC_B200_PARTIAL(d3dxdy2, 1, 2, 0)
GRIDCALC_B200_PARTIAL(d3dx2dz, 2, 0, 1)
GRIDCALC_B200_PARTIAL(d3dxdz2, 1, 0, 2)
GRIDCALC_B200_PARTIAL(d3dy2dz, 0, 2, 1)
GRIDCALC_B200_PARTIAL(d3dydz2, 0, 1, 2)
GRIDCALC_B200_PARTIAL(d3dxdydz, 1, 1, 1)
GRIDCALC_B200_PARTIAL(d4dx4, 4, 0, 0)
GRIDCALC_B200_PARTIAL(d4dy4, 0, 4, 0)
GRIDCALC_B200_PARTIAL(d4dz4, 0, 0, 4)
GRIDCALC_B200_PARTIAL(d4dx3dy, 3, 1, 0)
GRIDCALC_B200_PARTIAL(d4dxdy3, 1, 3, 0)
GRIDCALC_B200_PARTIAL(d4dx3dz, 3, 0, 1)
GRIDCALC_B200_PARTIAL(d4dxdz3, 1, 0, 3)
GRIDCALC_B200_PARTIAL(d4dy3dz, 0, 3, 1)
GRIDCALC_B200_PARTIAL(d4dydz3, 0, 1, 3)
GRIDCALC_B200_PARTIAL(d4dx2dy2, 2, 2, 0)
GRIDCALC_B200_PARTIAL(d4dx2dz2, 2, 0, 2)
GRIDCALC_B200_PARTIAL(d4dy2dz2, 0, 2, 2)
GRIDCALC_B200_PARTIAL(d4dx2dydz, 2, 1, 1)
GRIDCALC_B200_PARTIAL(d4dxdy2dz, 1, 2, 1)
GRIDCALC_B200_PARTIAL(d4dxdydz2, 1, 1, 2)
#undef GRIDCALC_B200_PARTIAL

// diff::biharmonic<Order> / d4 (diff/Biharmonic.hpp:48-119).
template <int Order = 2>
inline core::Field<double> biharmonic(const core::Field<double>& field) {
  return detail::scalar_op(field, [](const gc_grid* g, const double* in, double* out) {
    return gc_biharmonic(b200::context(), g, GC_F64, Order, in, out);
  });
}
template <int Order = 2>
inline core::Field<double> d4(const core::Field<double>& field) { return biharmonic<Order>(field); }

// diff::gradient<Order>, scalar -> Vec3d (diff/Gradient.hpp:43-74).
template <int Order = 2>
inline core::Field<core::Vec3d> gradient(const core::Field<double>& field) {
  const core::Grid& grid = field.getGrid();
  const size_t n = grid.getSize();
  core::DeviceField<double> in(field), out(grid, 3);
  const gc_grid g = grid.c();
  b200::check(gc_gradient(b200::context(), &g, GC_F64, Order, in.data(), out.data()));
  std::vector<double> planes(3 * n);
  out.download(planes.data());
  core::Field<core::Vec3d> r(grid);
  for (size_t i = 0; i < n; ++i) r.data()[i] = core::Vec3d(planes[i], planes[n + i], planes[2 * n + i]);
  return r;
}

// diff::divergence<Order>, Vec3d -> scalar (diff/Divergence.hpp:43-74).
template <int Order = 2>
inline core::Field<double> divergence(const core::Field<core::Vec3d>& vfield) {
  const core::Grid& grid = vfield.getGrid();
  const size_t n = grid.getSize();
  std::vector<double> planes(3 * n);
  for (size_t i = 0; i < n; ++i) {
    planes[i] = vfield.data()[i](0);
    planes[n + i] = vfield.data()[i](1);
    planes[2 * n + i] = vfield.data()[i](2);
  }
  core::DeviceField<double> in(grid, 3), out(grid);
  in.upload(planes.data());
  const gc_grid g = grid.c();
  b200::check(gc_divergence(b200::context(), &g, GC_F64, Order, in.data(), out.data()));
  return out.toHost();
}

// diff::gradient<Order>, Vec3d -> Mat3d (diff/Gradient.hpp:100-137):
// M(row, col) = d_col v_row.
template <int Order = 2>
inline core::Field<core::Mat3d> gradient(const core::Field<core::Vec3d>& vfield) {
  const core::Grid& grid = vfield.getGrid();
  const size_t n = grid.getSize();
  std::vector<double> planes(3 * n);
  for (size_t i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) planes[c * n + i] = vfield.data()[i](c);
  core::DeviceField<double> in(grid, 3), out(grid, 9);
  in.upload(planes.data());
  const gc_grid g = grid.c();
  b200::check(gc_gradient_vec(b200::context(), &g, GC_F64, Order, in.data(), out.data()));
  std::vector<double> m(9 * n);
  out.download(m.data());
  core::Field<core::Mat3d> r(grid);
  for (size_t i = 0; i < n; ++i)
    for (int row = 0; row < 3; ++row)
      for (int col = 0; col < 3; ++col) r.data()[i](row, col) = m[(3 * row + col) * n + i];
  return r;
}

// diff::divergence<Order>, Mat3d -> Vec3d (diff/Divergence.hpp:100-135):
// (div M)_row = sum over col of d_col M(row, col).
template <int Order = 2>
inline core::Field<core::Vec3d> divergence(const core::Field<core::Mat3d>& mfield) {
  const core::Grid& grid = mfield.getGrid();
  const size_t n = grid.getSize();
  std::vector<double> m(9 * n);
  for (size_t i = 0; i < n; ++i)
    for (int row = 0; row < 3; ++row)
      for (int col = 0; col < 3; ++col) m[(3 * row + col) * n + i] = mfield.data()[i](row, col);
  core::DeviceField<double> in(grid, 9), out(grid, 3);
  in.upload(m.data());
  const gc_grid g = grid.c();
  b200::check(gc_divergence_mat(b200::context(), &g, GC_F64, Order, in.data(), out.data()));
  std::vector<double> planes(3 * n);
  out.download(planes.data());
  core::Field<core::Vec3d> r(grid);
  for (size_t i = 0; i < n; ++i) r.data()[i] = core::Vec3d(planes[i], planes[n + i], planes[2 * n + i]);
  return r;
}

}  // namespace diff

namespace fvm {

// fvm::cellLaplacian (fvm/CellLaplacian.hpp:91-143).
inline core::Field<double> cellLaplacian(const core::Field<double>& psi, const core::Field<double>& D) {
  if (psi.getGrid() != D.getGrid())
    throw std::invalid_argument("gridcalc: fvm::cellLaplacian: D produced a Field on a different Grid than expected.");
  core::DeviceField<double> p(psi), d(D), out(psi.getGrid());
  const gc_grid g = psi.getGrid().c();
  int64_t bad = -1;
  b200::check(gc_cell_laplacian(b200::context(), &g, GC_F64, p.data(), d.data(), out.data(), &bad));
  return out.toHost();
}

}  // namespace fvm

namespace func {

struct Pairwise {};
struct Kahan {};

// func::integrate(field, Pairwise|Kahan) (func/Integrate.hpp:116-135).
template <class Tag = Pairwise>
inline double integrate(const core::Field<double>& field, Tag = {}) {
  core::DeviceField<double> d(field);
  const gc_grid g = field.getGrid().c();
  double r = 0.0;
  b200::check(gc_integrate(b200::context(), &g, GC_F64, d.data(),
                           std::is_same_v<Tag, Kahan> ? GC_SUM_KAHAN : GC_SUM_PAIRWISE, &r));
  return r;
}
template <class T, class Tag = Pairwise>
inline double integrate(const core::DeviceField<T>& field, Tag = {}) {
  const gc_grid g = field.getGrid().c();
  double r = 0.0;
  b200::check(gc_integrate(b200::context(), &g, b200::dtype_of<T>(), field.data(),
                           std::is_same_v<Tag, Kahan> ? GC_SUM_KAHAN : GC_SUM_PAIRWISE, &r));
  return r;
}

// Device integrands for func::evaluate (func/Functional.hpp:88-148).
struct Identity { gc_integrand c() const { return {GC_INTEGRAND_PSI, 0.0}; } };
struct Square { gc_integrand c() const { return {GC_INTEGRAND_PSI_SQUARED, 0.0}; } };
struct GradientEnergy { gc_integrand c() const { return {GC_INTEGRAND_GRAD_SQUARED, 0.0}; } };
struct FreeEnergy {
  double kappa;
  gc_integrand c() const { return {GC_INTEGRAND_CH_FREE_ENERGY, kappa}; }
};

template <class F, class Tag = Pairwise, class = decltype(std::declval<F>().c())>
inline double evaluate(const core::Field<double>& psi, F f, Tag = {}) {
  core::DeviceField<double> d(psi);
  const gc_grid g = psi.getGrid().c();
  const gc_integrand in = f.c();
  double r = 0.0;
  b200::check(gc_evaluate(b200::context(), &g, GC_F64, d.data(), &in,
                          std::is_same_v<Tag, Kahan> ? GC_SUM_KAHAN : GC_SUM_PAIRWISE, &r));
  return r;
}

}  // namespace func

namespace solve {

// Integrator tags (solve/ExplicitEuler.hpp:37-41, solve/RK4.hpp:30-35).
struct ExplicitEuler { static constexpr double diffusionCFLLimit = 0.5; };
struct RK4 { static constexpr double diffusionCFLLimit = 0.6963; };

template <class Tag>
constexpr gc_integrator integrator_of() {
  static_assert(std::is_same_v<Tag, RK4> || std::is_same_v<Tag, ExplicitEuler>, "RK4 or ExplicitEuler");
  return std::is_same_v<Tag, RK4> ? GC_RK4 : GC_EXPLICIT_EULER;
}

// Device RHS functor: M lap(-psi + psi^3 - kappa lap psi)
// (examples/common/cahn_hilliard.hpp:38-59) at Laplacian order 2, 4 or 6.
struct CahnHilliardRhs {
  double mobility = 1.0;
  double kappa = 1.0;
  int order = 2;
  gc_ch_params c() const { return gc_ch_params{mobility, kappa, order}; }
};

// solve::integrate(psi, rhs, dt, n_steps, Tag) (solve/RK4.hpp:99-154,
// solve/ExplicitEuler.hpp:79-112) for the device Cahn-Hilliard RHS.
template <class Tag>
inline void integrate(core::Field<double>& psi, const CahnHilliardRhs& rhs, double dt, int n_steps, Tag) {
  core::DeviceField<double> d(psi);
  const gc_grid g = psi.getGrid().c();
  const gc_ch_params p = rhs.c();
  b200::check(gc_ch_integrate(b200::context(), &g, GC_F64, &p, d.data(), dt, n_steps, integrator_of<Tag>()));
  d.download(psi.data());
}
template <class T, class Tag>
inline void integrate(core::DeviceField<T>& psi, const CahnHilliardRhs& rhs, double dt, int n_steps, Tag) {
  const gc_grid g = psi.getGrid().c();
  const gc_ch_params p = rhs.c();
  b200::check(gc_ch_integrate(b200::context(), &g, b200::dtype_of<T>(), &p, psi.data(), dt, n_steps, integrator_of<Tag>()));
}

// solve::explicitEuler (solve/ExplicitEuler.hpp:129-135).
inline void explicitEuler(core::Field<double>& psi, const CahnHilliardRhs& rhs, double dt, int n_steps) {
  integrate(psi, rhs, dt, n_steps, ExplicitEuler{});
}

// solve::diffuse(psi, double D, dt, n_steps, Tag) (solve/Diffusion.hpp:89-112).
template <class Integrator = ExplicitEuler>
inline void diffuse(core::Field<double>& psi, double D, double dt, int n_steps, Integrator = {}) {
  core::DeviceField<double> d(psi);
  const gc_grid g = psi.getGrid().c();
  b200::check(gc_diffuse(b200::context(), &g, GC_F64, d.data(), D, dt, n_steps, integrator_of<Integrator>()));
  d.download(psi.data());
}

// solve::diffuse(psi, Field D, dt, n_steps, Tag) (solve/Diffusion.hpp:161-216).
template <class Integrator = ExplicitEuler>
inline void diffuse(core::Field<double>& psi, const core::Field<double>& D, double dt, int n_steps, Integrator = {}) {
  if (psi.getGrid() != D.getGrid())
    throw std::invalid_argument("gridcalc: solve::diffuse: D produced a Field on a different Grid than expected.");
  core::DeviceField<double> d(psi), dd(D);
  const gc_grid g = psi.getGrid().c();
  int64_t bad = -1;
  b200::check(gc_diffuse_fvm(b200::context(), &g, GC_F64, d.data(), dd.data(), dt, n_steps,
                             integrator_of<Integrator>(), &bad));
  d.download(psi.data());
}

}  // namespace solve

// gridcalc::version() (include/gridcalc/version.hpp.in:16-18).
inline const char* version() { return gc_version(); }

}  // namespace gridcalc
