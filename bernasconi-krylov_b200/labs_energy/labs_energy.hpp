#pragma once
// The LABS types the sampler interface is written against — SpinState and
// LabsEvaluator — with the reference's API (src/labs_energy/labs_energy.hpp of
// ssk1001/bernasconi-krylov), for builds of this repository without a
// reference checkout. In a reference checkout the reference's own header is used.
#include <cstddef>
#include <cstdint>
#include <vector>

struct SpinState {
  uint64_t bits = 0;
  constexpr SpinState() = default;
  constexpr explicit SpinState(uint64_t b) : bits(b) {}
  bool get_bit(size_t i) const { return (bits >> i) & 1ULL; }
  int get_spin(size_t i) const { return ((bits >> i) & 1ULL) ? -1 : 1; }  // bit 1 <-> spin -1
  void flip(size_t i) { bits ^= (1ULL << i); }
  SpinState flipped(size_t i) const { return SpinState{bits ^ (1ULL << i)}; }
  int hamming_distance(const SpinState& o) const { return __builtin_popcountll(bits ^ o.bits); }
  static uint64_t reverse_bits(uint64_t x, int n) {
    uint64_t r = 0;
    for (int i = 0; i < n; ++i) r |= ((x >> i) & 1ULL) << (n - 1 - i);
    return r;
  }
  // smallest member of the orbit {id, alternating flip, reversal, both} x {negation}
  SpinState canonical(int n) const {
    const uint64_t m = (n >= 64) ? ~0ULL : ((1ULL << n) - 1ULL);
    const uint64_t a = bits & m, b = a ^ (0x5555555555555555ULL & m);
    const uint64_t c[4] = {a, b, reverse_bits(a, n), reverse_bits(b, n)};
    uint64_t best = ~0ULL;
    for (uint64_t x : c) {
      if (x < best) best = x;
      if (((~x) & m) < best) best = (~x) & m;
    }
    return SpinState{best};
  }
  bool operator==(const SpinState& o) const { return bits == o.bits; }
  bool operator!=(const SpinState& o) const { return bits != o.bits; }
  bool operator<(const SpinState& o) const { return bits < o.bits; }
};

struct SpinStateHash {
  size_t operator()(const SpinState& s) const noexcept {
    uint64_t x = s.bits;  // splitmix64 finaliser
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ULL;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebULL;
    x ^= x >> 31;
    return (size_t)x;
  }
};

class LabsEvaluator {
 public:
  explicit LabsEvaluator(int n) : n_(n), mask_((n >= 64) ? ~0ULL : ((1ULL << n) - 1ULL)) {}
  int get_n() const { return n_; }
  int64_t calcEnergy(const SpinState& s) const {
    const std::vector<int64_t> c = calcCk(s);
    int64_t e = 0;
    for (int k = 1; k < n_; ++k) e += c[(size_t)k] * c[(size_t)k];
    return e;
  }
  int64_t energy(const SpinState& s) const { return calcEnergy(s); }
  std::vector<int64_t> calcCk(const SpinState& s) const {
    const uint64_t x = s.bits & mask_;
    std::vector<int64_t> c((size_t)n_, 0);
    for (int k = 1; k < n_; ++k)
      c[(size_t)k] = (int64_t)(n_ - k) - 2 * (int64_t)__builtin_popcountll((x ^ (x >> k)) & ((1ULL << (n_ - k)) - 1ULL));
    return c;
  }
  SpinState get_canonical(const SpinState& s) const { return s.canonical(n_); }
  static int64_t known_optimal_energy(int n) {
    static const int64_t t[33] = {-1, -1, -1, 1, 2, 2, 7, 3, 8, 12, 13, 5, 10, 6, 19, 15, 24,
                                  32, 25, 29, 26, 26, 39, 47, 36, 36, 45, 37, 50, 62, 59, 67, 64};
    return (n >= 0 && n <= 32) ? t[n] : -1;
  }
  // smallest Hamming distance to a state with E < target (n, or max_d + 1, if none)
  int compute_d_min(const SpinState& s0, int64_t target = -1, int max_d = -1) const {
    if (target < 0) target = calcEnergy(s0);
    const int none = (max_d > 0) ? (max_d + 1) : n_;
    const int64_t opt = known_optimal_energy(n_);
    if (opt >= 0 && target <= opt) return none;
    const uint64_t s = s0.bits & mask_;
    const int limit = (max_d > 0 && max_d <= n_) ? max_d : n_;
    for (int d = 1; d <= limit; ++d) {
      if (d == n_) return (calcEnergy(SpinState{s ^ mask_}) < target) ? n_ : none;
      for (uint64_t f = (1ULL << d) - 1ULL; f <= mask_ && f != 0;) {
        if (calcEnergy(SpinState{s ^ f}) < target) return d;
        const uint64_t low = f & (~f + 1ULL), ripple = f + low;
        f = ripple | (((f ^ ripple) >> 2) / low);
      }
    }
    return none;
  }

 private:
  int n_;
  uint64_t mask_;
};
