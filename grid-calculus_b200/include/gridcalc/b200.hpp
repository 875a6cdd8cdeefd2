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

// Integrand programs.  The reference's func::evaluate calls a host callable
// per cell (func/Functional.hpp:88-148 scalar, :183-220 Vec3d).  Here a
// generic callable (auto parameters) is called once on symbolic arguments;
// the operations it performs are recorded in order and become a gc_program
// that the device runs for every cell with the same correctly rounded double
// arithmetic, so the integrand is the one the callable computes, bit for
// bit.  Supported: + - * / (and the compound forms) with doubles on either
// side, unary -, func::sqrt / abs / fabs / min / max (std::min / std::max
// semantics); Vec3 offers (i), [i], dot, squaredNorm, norm; Mat3 offers
// (row, col), trace, squaredNorm, doubleContract, with Eigen's summation
// order (components in order; matrices in column-major storage order from
// 0.0).  std:: math functions and comparisons cannot be recorded.
namespace program {

class Recorder {
 public:
  struct Node {
    int op, a, b;  // operand node ids; for GC_OPC_INPUT, a is the input number
    double value;
  };
  int add(int op, int a = -1, int b = -1, double value = 0.0) {
    nodes_.push_back(Node{op, a, b, value});
    return static_cast<int>(nodes_.size()) - 1;
  }
  int input(int k) {
    for (const auto& kv : inputs_)
      if (kv.first == k) return kv.second;
    const int id = add(GC_OPC_INPUT, k);
    inputs_.push_back({k, id});
    return id;
  }
  // Emits the nodes the result depends on, in recording order, on at most
  // GC_PROGRAM_REGS registers (a register is reused after its last read).
  gc_program compile(int components, int arity, int root) const {
    const int n = static_cast<int>(nodes_.size());
    std::vector<char> live(n, 0);
    std::vector<int> stack{root};
    while (!stack.empty()) {
      const int k = stack.back();
      stack.pop_back();
      if (live[k]) continue;
      live[k] = 1;
      if (nodes_[k].op != GC_OPC_INPUT && nodes_[k].op != GC_OPC_CONST) {
        if (nodes_[k].a >= 0) stack.push_back(nodes_[k].a);
        if (nodes_[k].b >= 0) stack.push_back(nodes_[k].b);
      }
    }
    std::vector<int> order;
    for (int k = 0; k < n; ++k)
      if (live[k]) order.push_back(k);
    if (order.size() > GC_PROGRAM_MAX_INSTR)
      throw std::invalid_argument("gridcalc: func::evaluate: integrand needs " + std::to_string(order.size()) +
                                  " instructions, at most " + std::to_string(GC_PROGRAM_MAX_INSTR));
    std::vector<int> last(n, -1);
    for (size_t pos = 0; pos < order.size(); ++pos) {
      const Node& nd = nodes_[order[pos]];
      if (nd.op == GC_OPC_INPUT || nd.op == GC_OPC_CONST) continue;
      if (nd.a >= 0) last[nd.a] = static_cast<int>(pos);
      if (nd.b >= 0) last[nd.b] = static_cast<int>(pos);
    }
    last[root] = static_cast<int>(order.size());
    gc_program p{};
    p.components = components;
    p.arity = arity;
    p.n_instr = static_cast<int32_t>(order.size());
    std::vector<int> reg(n, -1), free_regs;
    for (int r = GC_PROGRAM_REGS - 1; r >= 0; --r) free_regs.push_back(r);
    for (size_t pos = 0; pos < order.size(); ++pos) {
      const Node& nd = nodes_[order[pos]];
      const bool ops = nd.op != GC_OPC_INPUT && nd.op != GC_OPC_CONST;
      const int ra = ops && nd.a >= 0 ? reg[nd.a] : 0;
      const int rb = ops && nd.b >= 0 ? reg[nd.b] : 0;
      if (ops && nd.a >= 0 && last[nd.a] == static_cast<int>(pos)) free_regs.push_back(reg[nd.a]);
      if (ops && nd.b >= 0 && nd.b != nd.a && last[nd.b] == static_cast<int>(pos)) free_regs.push_back(reg[nd.b]);
      if (free_regs.empty())
        throw std::invalid_argument("gridcalc: func::evaluate: integrand keeps more than " +
                                    std::to_string(GC_PROGRAM_REGS) + " values live");
      const int dst = free_regs.back();
      free_regs.pop_back();
      reg[order[pos]] = dst;
      gc_instr& I = p.instr[pos];
      I.op = static_cast<int16_t>(nd.op);
      I.dst = static_cast<int16_t>(dst);
      I.a = static_cast<int16_t>(nd.op == GC_OPC_INPUT ? nd.a : ra);
      I.b = static_cast<int16_t>(rb);
      I.value = nd.op == GC_OPC_CONST ? nd.value : 0.0;
    }
    return p;
  }

 private:
  std::vector<Node> nodes_;
  std::vector<std::pair<int, int>> inputs_;
};

class Sym {
 public:
  Sym(Recorder* r, int id) : r_(r), id_(id) {}
  Recorder* rec() const { return r_; }
  int id() const { return id_; }

 private:
  Recorder* r_;
  int id_;
};

inline Sym constant(Recorder* r, double v) { return Sym(r, r->add(GC_OPC_CONST, -1, -1, v)); }
inline Sym op2(int op, const Sym& a, const Sym& b) { return Sym(a.rec(), a.rec()->add(op, a.id(), b.id())); }
inline Sym op1(int op, const Sym& a) { return Sym(a.rec(), a.rec()->add(op, a.id())); }

#define GRIDCALC_B200_SYM_BINARY(SYM, OPC)                                                               \
  inline Sym operator SYM(const Sym& a, const Sym& b) { return op2(OPC, a, b); }                        \
  inline Sym operator SYM(const Sym& a, double b) { return op2(OPC, a, constant(a.rec(), b)); }         \
  inline Sym operator SYM(double a, const Sym& b) { return op2(OPC, constant(b.rec(), a), b); }         \
  inline Sym& operator SYM##=(Sym& a, const Sym& b) { return a = a SYM b; }                              \
  inline Sym& operator SYM##=(Sym& a, double b) { return a = a SYM b; }
GRIDCALC_B200_SYM_BINARY(+, GC_OPC_ADD)
GRIDCALC_B200_SYM_BINARY(-, GC_OPC_SUB)
GRIDCALC_B200_SYM_BINARY(*, GC_OPC_MUL)
GRIDCALC_B200_SYM_BINARY(/, GC_OPC_DIV)
#undef GRIDCALC_B200_SYM_BINARY

inline Sym operator-(const Sym& a) { return op1(GC_OPC_NEG, a); }
inline Sym operator+(const Sym& a) { return a; }
inline Sym sqrt(const Sym& a) { return op1(GC_OPC_SQRT, a); }
inline Sym abs(const Sym& a) { return op1(GC_OPC_ABS, a); }
inline Sym fabs(const Sym& a) { return op1(GC_OPC_ABS, a); }
inline Sym min(const Sym& a, const Sym& b) { return op2(GC_OPC_MIN, a, b); }
inline Sym max(const Sym& a, const Sym& b) { return op2(GC_OPC_MAX, a, b); }
inline Sym min(const Sym& a, double b) { return op2(GC_OPC_MIN, a, constant(a.rec(), b)); }
inline Sym max(const Sym& a, double b) { return op2(GC_OPC_MAX, a, constant(a.rec(), b)); }
inline Sym min(double a, const Sym& b) { return op2(GC_OPC_MIN, constant(b.rec(), a), b); }
inline Sym max(double a, const Sym& b) { return op2(GC_OPC_MAX, constant(b.rec(), a), b); }

// Vec3d of one cell.
struct Vec3 {
  Sym v[3];
  Sym operator()(int i) const { return v[i]; }
  Sym operator[](int i) const { return v[i]; }
  Sym x() const { return v[0]; }
  Sym y() const { return v[1]; }
  Sym z() const { return v[2]; }
  Sym dot(const Vec3& o) const { return (v[0] * o.v[0] + v[1] * o.v[1]) + v[2] * o.v[2]; }
  Sym squaredNorm() const { return dot(*this); }
  Sym norm() const { return sqrt(squaredNorm()); }
};

// Mat3d of one cell, M(row, col).
struct Mat3 {
  Sym m[3][3];
  Sym operator()(int r, int c) const { return m[r][c]; }
  Sym trace() const { return (m[0][0] + m[1][1]) + m[2][2]; }
  Sym doubleContract(const Mat3& o) const {
    Sym acc = constant(m[0][0].rec(), 0.0);
    for (int c = 0; c < 3; ++c)
      for (int r = 0; r < 3; ++r) acc = acc + m[r][c] * o.m[r][c];
    return acc;
  }
  Sym squaredNorm() const { return doubleContract(*this); }
};

template <class F>
constexpr int scalar_arity() {
  if constexpr (std::is_invocable_v<F&, Sym, Vec3, Sym, Sym>) return 4;
  else if constexpr (std::is_invocable_v<F&, Sym, Vec3, Sym>) return 3;
  else if constexpr (std::is_invocable_v<F&, Sym, Vec3>) return 2;
  else if constexpr (std::is_invocable_v<F&, Sym>) return 1;
  else return 0;
}

template <class F>
constexpr int vector_arity() {
  if constexpr (std::is_invocable_v<F&, Vec3, Mat3>) return 2;
  else if constexpr (std::is_invocable_v<F&, Vec3>) return 1;
  else return 0;
}

// Lazy forms for overload selection: a generic callable is only probed with
// the symbols of the field kind it is called on (probing a vector callable
// with scalar symbols would instantiate its body and fail to compile).
template <class F>
struct scalar_callable : std::bool_constant<(scalar_arity<F>() > 0)> {};
template <class F>
struct vector_callable : std::bool_constant<(vector_arity<F>() > 0)> {};

inline int root_of(Recorder&, const Sym& s) { return s.id(); }
inline int root_of(Recorder& rec, double v) { return rec.add(GC_OPC_CONST, -1, -1, v); }

template <class F>
gc_program record_scalar(F& f) {
  constexpr int arity = scalar_arity<F>();
  Recorder rec;
  const Sym psi(&rec, rec.input(GC_IN_PSI));
  const Vec3 g{{Sym(&rec, rec.input(GC_IN_GRAD_X)), Sym(&rec, rec.input(GC_IN_GRAD_Y)),
                Sym(&rec, rec.input(GC_IN_GRAD_Z))}};
  const Sym lap(&rec, rec.input(GC_IN_LAP));
  const Sym bih(&rec, rec.input(GC_IN_BIH));
  int root;
  if constexpr (arity == 4) root = root_of(rec, f(psi, g, lap, bih));
  else if constexpr (arity == 3) root = root_of(rec, f(psi, g, lap));
  else if constexpr (arity == 2) root = root_of(rec, f(psi, g));
  else root = root_of(rec, f(psi));
  return rec.compile(1, arity, root);
}

template <class F>
gc_program record_vector(F& f) {
  constexpr int arity = vector_arity<F>();
  Recorder rec;
  Vec3 u{{Sym(&rec, rec.input(GC_IN_U_X)), Sym(&rec, rec.input(GC_IN_U_Y)), Sym(&rec, rec.input(GC_IN_U_Z))}};
  auto du = [&](int r, int c) { return Sym(&rec, rec.input(GC_IN_DU + 3 * r + c)); };
  const Mat3 M{{{du(0, 0), du(0, 1), du(0, 2)}, {du(1, 0), du(1, 1), du(1, 2)}, {du(2, 0), du(2, 1), du(2, 2)}}};
  int root;
  if constexpr (arity == 2) root = root_of(rec, f(u, M));
  else root = root_of(rec, f(u));
  return rec.compile(3, arity, root);
}

template <class Tag>
constexpr gc_sum sum_of() { return std::is_same_v<Tag, Kahan> ? GC_SUM_KAHAN : GC_SUM_PAIRWISE; }

}  // namespace program

using program::abs;
using program::fabs;
using program::max;
using program::min;
using program::sqrt;

// func::evaluate(psi, f, tag) for a generic callable of arity 1..4
// (func/Functional.hpp:88-148).
template <class FieldT, class F, class Tag = Pairwise,
          std::enable_if_t<std::conjunction_v<std::is_same<FieldT, core::Field<double>>, program::scalar_callable<F>>,
                           int> = 0>
inline double evaluate(const FieldT& psi, F f, Tag = {}) {
  const gc_program p = program::record_scalar(f);
  core::DeviceField<double> d(psi);
  const gc_grid g = psi.getGrid().c();
  double r = 0.0;
  b200::check(gc_evaluate_program(b200::context(), &g, GC_F64, d.data(), &p, program::sum_of<Tag>(), &r));
  return r;
}

// func::evaluate(u, f, tag) for a Vec3d field and a generic callable f(u) or
// f(u, grad u) (func/Functional.hpp:183-220).
template <class FieldT, class F, class Tag = Pairwise,
          std::enable_if_t<
              std::conjunction_v<std::is_same<FieldT, core::Field<core::Vec3d>>, program::vector_callable<F>>, int> = 0>
inline double evaluate(const FieldT& u, F f, Tag = {}) {
  const gc_program p = program::record_vector(f);
  const core::Grid& grid = u.getGrid();
  const size_t n = grid.getSize();
  std::vector<double> planes(3 * n);
  for (size_t i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) planes[c * n + i] = u.data()[i](c);
  core::DeviceField<double> d(grid, 3);
  d.upload(planes.data());
  const gc_grid g = grid.c();
  double r = 0.0;
  b200::check(gc_evaluate_program(b200::context(), &g, GC_F64, d.data(), &p, program::sum_of<Tag>(), &r));
  return r;
}

// The same on device-resident fields: a scalar field with f(psi[, grad[,
// lap[, bih]]]), and a vector field (three planes) with f(u[, grad_u]).
template <class T, class F, class Tag = Pairwise, std::enable_if_t<program::scalar_callable<F>::value, int> = 0>
inline double evaluate(const core::DeviceField<T>& psi, F f, Tag = {}) {
  if (psi.components() != 1)
    throw std::invalid_argument("gridcalc: func::evaluate: a scalar integrand needs a one-component field");
  const gc_program p = program::record_scalar(f);
  const gc_grid g = psi.getGrid().c();
  double r = 0.0;
  b200::check(gc_evaluate_program(b200::context(), &g, b200::dtype_of<T>(), psi.data(), &p, program::sum_of<Tag>(), &r));
  return r;
}
template <class T, class F, class Tag = Pairwise>
inline double evaluateVector(const core::DeviceField<T>& u, F f, Tag = {}) {
  static_assert(program::vector_callable<F>::value, "func::evaluateVector: f must be invocable as f(u) or f(u, grad_u)");
  if (u.components() != 3)
    throw std::invalid_argument("gridcalc: func::evaluateVector: a vector integrand needs a three-component field");
  const gc_program p = program::record_vector(f);
  const gc_grid g = u.getGrid().c();
  double r = 0.0;
  b200::check(gc_evaluate_program(b200::context(), &g, b200::dtype_of<T>(), u.data(), &p, program::sum_of<Tag>(), &r));
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
