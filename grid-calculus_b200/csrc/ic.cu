// Seeded initial condition of the Cahn-Hilliard examples (host code).
//
// makeRandomIc (examples/common/cahn_hilliard.hpp:85-103) draws one value per
// cell in flat-index order from std::uniform_real_distribution<double>(-a, a)
// over std::mt19937_64(seed), then subtracts the values' mean.  The engine is
// the 64-bit Mersenne Twister of Matsumoto and Nishimura with the parameters
// the C++ standard fixes for mt19937_64 ([rand.predef]); the distribution
// draws one engine output per value (53 mantissa bits need one 64-bit draw,
// [rand.util.canonical]) and scales it as libstdc++ does.  Both are restated
// here from those published definitions, so the product produces the same
// bytes as the reference build without linking a C++ standard library's
// generator into the device path.
#include <cmath>
#include <cstdint>
#include <vector>

#include "common.cuh"

namespace {

// mt19937_64 = mersenne_twister_engine<uint_fast64_t, 64, 312, 156, 31,
//   0xb5026f5aa96619e9, 29, 0x5555555555555555, 17, 0x71d67fffeda60000, 37,
//   0xfff7eee000000000, 43, 6364136223846793005> (C++ standard [rand.predef]).
class Mt64 {
 public:
  explicit Mt64(uint64_t seed) : state_(kN), next_(kN) {
    state_[0] = seed;
    for (int i = 1; i < kN; ++i) {
      const uint64_t p = state_[i - 1];
      state_[i] = kInitMul * (p ^ (p >> 62)) + static_cast<uint64_t>(i);
    }
  }

  uint64_t operator()() {
    if (next_ >= kN) refill();
    uint64_t z = state_[next_++];
    z ^= (z >> 29) & 0x5555555555555555ULL;
    z ^= (z << 17) & 0x71d67fffeda60000ULL;
    z ^= (z << 37) & 0xfff7eee000000000ULL;
    z ^= z >> 43;
    return z;
  }

 private:
  static constexpr int kN = 312;
  static constexpr int kM = 156;
  static constexpr uint64_t kInitMul = 6364136223846793005ULL;
  static constexpr uint64_t kA = 0xb5026f5aa96619e9ULL;
  static constexpr uint64_t kLow = (1ULL << 31) - 1;  // r = 31 low bits
  static constexpr uint64_t kHigh = ~kLow;

  // The recurrence x[k + n] = x[k + m] ^ twist((x[k] & upper) | (x[k+1] & lower)),
  // applied to the whole block of n words at once.
  void refill() {
    for (int k = 0; k < kN; ++k) {
      const uint64_t y = (state_[k] & kHigh) | (state_[(k + 1) % kN] & kLow);
      state_[k] = state_[(k + kM) % kN] ^ (y >> 1) ^ ((y & 1ULL) ? kA : 0ULL);
    }
    next_ = 0;
  }

  std::vector<uint64_t> state_;
  int next_;
};

// uniform_real_distribution<double>(lo, hi) over a 64-bit engine:
// canonical u = double(x) / 2^64 (one draw: ceil(53 / 64) = 1), pulled below
// 1 when the conversion rounds up to 2^64, then u * (hi - lo) + lo.
inline double uniform(Mt64& eng, double lo, double hi) {
  double u = static_cast<double>(eng()) / 18446744073709551616.0;
  if (u >= 1.0) u = std::nextafter(1.0, 0.0);
  const double scaled = u * (hi - lo);
  return scaled + lo;
}

}  // namespace

GC_API gc_status gc_random_ic(const gc_grid* g, uint64_t seed, double amplitude, int32_t subtract_mean,
                              double* out) {
  using namespace gcb;
  if (gc_status s = check_grid(g); s != GC_OK) return s;
  if (!out) return fail(GC_ERR_INVALID_ARG, "gc_random_ic: null output buffer");
  if (!(amplitude >= 0.0) || !std::isfinite(amplitude))
    return fail(GC_ERR_INVALID_ARG, "gc_random_ic: amplitude must be finite and >= 0");
  const size_t n = static_cast<size_t>(g->nx) * g->ny * g->nz;
  Mt64 eng(seed);
  double sum = 0.0;
  for (size_t i = 0; i < n; ++i) {
    const double v = uniform(eng, -amplitude, amplitude);
    out[i] = v;
    sum += v;
  }
  if (subtract_mean) {
    const double mean = sum / static_cast<double>(n);
    for (size_t i = 0; i < n; ++i) out[i] -= mean;
  }
  return GC_OK;
}
