// ============================================================================
// ORACLE — test infrastructure only, never part of the product path.
//
// CPU restatement (C++17 + OpenMP, complex128) of the reference's
// transverse-field Trotter sampler and of the LABS energy core it depends on.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU legs (cpu_baseline and
// `--impl reference`) may load the shared library built from this file, and
// there only as the checker / timed CPU baseline.
//
// Parity pins (checked by tests/test_oracle_*.py against data read from the
// reference repository and committed under tests/golden/):
//   * E(s) against the reference's exhaustive tables data_raw/classical/exhaustive/{n}.csv
//   * E(s), d_min, canonical form, steepest descent against the reference's own
//     header-only C++ (labs_energy.hpp, classical.cuh) compiled into oracle/_ref/
//   * P_<(t), <d_H(t)> against data_processed/probability_dynamics_n{16,20}.csv
//
// Every function cites the reference file:line it restates. Paths are relative
// to the reference project root.
// ============================================================================
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <limits>
#include <random>
#include <unordered_set>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

inline uint64_t mask_of(int n) { return (n >= 64) ? ~0ULL : ((1ULL << n) - 1ULL); }

// src/labs_energy/labs_energy.hpp:121-132 — E(s) = sum_{k=1}^{n-1} C_k^2 with
// C_k = (n-k) - 2 popcount((x ^ (x >> k)) & (2^{n-k} - 1)); bit 1 <-> spin -1.
inline int64_t energy_of(int n, uint64_t x) {
  x &= mask_of(n);
  int64_t e = 0;
  for (int k = 1; k < n; ++k) {
    const uint64_t m = (1ULL << (n - k)) - 1ULL;
    const int64_t ck = (int64_t)(n - k) - 2 * (int64_t)__builtin_popcountll((x ^ (x >> k)) & m);
    e += ck * ck;
  }
  return e;
}

// src/labs_energy/labs_energy.hpp:40-48 (reverse the lowest n bits)
inline uint64_t reverse_low_bits(uint64_t x, int n) {
  uint64_t r = 0;
  for (int i = 0; i < n; ++i) r |= ((x >> i) & 1ULL) << (n - 1 - i);
  return r;
}

// src/labs_energy/labs_energy.hpp:156-168 — table of optimal LABS energies E*(n).
int64_t optimal_energy(int n) {
  static const int64_t table[33] = {-1, -1, -1, 1, 2, 2, 7, 3, 8, 12, 13, 5, 10, 6, 19, 15, 24,
                                    32, 25, 29, 26, 26, 39, 47, 36, 36, 45, 37, 50, 62, 59, 67, 64};
  return (n >= 0 && n <= 32) ? table[n] : -1;
}

}  // namespace

extern "C" {

int64_t orc_labs_energy(int n, uint64_t bits) { return energy_of(n, bits); }

// src/labs_energy/labs_energy.hpp:139-149 — autocorrelations C_1..C_{n-1} (out[0] = 0).
void orc_labs_ck(int n, uint64_t bits, int64_t* out) {
  const uint64_t x = bits & mask_of(n);
  out[0] = 0;
  for (int k = 1; k < n; ++k) {
    const uint64_t m = (1ULL << (n - k)) - 1ULL;
    out[k] = (int64_t)(n - k) - 2 * (int64_t)__builtin_popcountll((x ^ (x >> k)) & m);
  }
}

int64_t orc_known_optimal_energy(int n) { return optimal_energy(n); }

// src/labs_energy/labs_energy.hpp:51-78 — minimum over the order-8 symmetry orbit
// {identity, alternating flip, reversal, both} x {global negation}.
uint64_t orc_canonical(int n, uint64_t bits) {
  const uint64_t m = mask_of(n);
  const uint64_t alt = 0x5555555555555555ULL & m;
  const uint64_t a = bits & m, b = a ^ alt;
  const uint64_t cand[4] = {a, b, reverse_low_bits(a, n), reverse_low_bits(b, n)};
  uint64_t best = ~0ULL;
  for (uint64_t c : cand) {
    best = std::min(best, c);
    best = std::min(best, (~c) & m);
  }
  return best;
}

// src/labs_energy/labs_energy.hpp:175-207 — smallest Hamming distance d from s0
// to any state with E < target, scanning Hamming spheres d = 1, 2, ...; returns
// n (or max_d + 1) when none is found or when target <= E*(n).
int orc_d_min(int n, uint64_t bits, int64_t target, int max_d) {
  if (target < 0) target = energy_of(n, bits);
  const int64_t opt = optimal_energy(n);
  const int not_found = (max_d > 0) ? (max_d + 1) : n;
  if (opt >= 0 && target <= opt) return not_found;
  const uint64_t m = mask_of(n);
  const uint64_t s = bits & m;
  const int limit = (max_d > 0 && max_d <= n) ? max_d : n;
  for (int d = 1; d <= limit; ++d) {
    if (d == n) {  // the only weight-n flip mask is the full mask
      if (energy_of(n, s ^ m) < target) return n;
      break;
    }
    // enumerate all n-bit masks of weight d in increasing order (next permutation of bits)
    uint64_t f = (1ULL << d) - 1ULL;
    while (f <= m && f != 0) {
      if (energy_of(n, s ^ f) < target) return d;
      const uint64_t low = f & (~f + 1ULL);
      const uint64_t ripple = f + low;
      f = ripple | (((f ^ ripple) >> 2) / low);
    }
  }
  return not_found;
}

// All E(s), s in [0, 2^n), as uint16 (max E at n = 30 is 8555) — the reference
// caches the same values as double (src/sampling/sampler.cuh:54-70, 323-338).
void orc_energy_table_u16(int n, uint16_t* out) {
  const int64_t count = 1LL << n;
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < count; ++s) out[s] = (uint16_t)energy_of(n, (uint64_t)s);
}

// src/sampling/sampler.cuh:198-227, 383-399 — #{s : E(s) < e0}.
uint64_t orc_count_below(int n, int64_t e0) {
  const int64_t count = 1LL << n;
  uint64_t c = 0;
#pragma omp parallel for reduction(+ : c) schedule(static)
  for (int64_t s = 0; s < count; ++s) c += (energy_of(n, (uint64_t)s) < e0) ? 1 : 0;
  return c;
}

// src/classical/classical.cuh:557-604 — ClassicalOptimizer(n, seed): mt19937_64(seed),
// random_state() = rng() & mask, drawn in sequence.
void orc_random_states(int n, uint64_t seed, int64_t count, uint64_t* out) {
  std::mt19937_64 rng(seed);
  const uint64_t m = mask_of(n);
  for (int64_t i = 0; i < count; ++i) out[i] = rng() & m;
}

// src/classical/classical.cuh:625-712 — single-flip steepest descent: each sweep
// probes all n flips with incremental C_k updates and takes the first strictly
// best neighbour (lowest bit index wins ties); stops when no flip improves or
// when evals_used + n would exceed max_evals (0 = unlimited).
void orc_steepest_descent(int n, uint64_t start, uint64_t max_evals, uint64_t* final_state,
                          int64_t* final_energy, uint64_t* evals_used, int64_t* steps_taken) {
  const uint64_t budget = (max_evals == 0) ? std::numeric_limits<uint64_t>::max() : max_evals;
  uint64_t cur = start;
  int64_t C[64] = {0};
  orc_labs_ck(n, cur, C);
  int64_t e = 0;
  for (int k = 1; k < n; ++k) e += C[k] * C[k];
  uint64_t evals = 1;
  int64_t steps = 0;
  auto spin = [&](int i) { return ((cur >> i) & 1ULL) ? -1 : 1; };
  while (true) {
    if (evals + (uint64_t)n > budget) break;
    int64_t best_e = e;
    int best_p = -1;
    int64_t best_d[64] = {0}, d[64] = {0};
    for (int p = 0; p < n; ++p) {
      const int sp = spin(p);
      int64_t ne = 0;
      for (int k = 1; k < n; ++k) {
        int64_t dk = 0;
        if (p + k < n) dk -= 2 * sp * spin(p + k);
        if (p - k >= 0) dk -= 2 * spin(p - k) * sp;
        d[k] = dk;
        ne += (C[k] + dk) * (C[k] + dk);
      }
      if (ne < best_e) {
        best_e = ne;
        best_p = p;
        std::memcpy(best_d, d, sizeof(d));
      }
    }
    evals += (uint64_t)n;
    if (best_p < 0) break;
    cur ^= (1ULL << best_p);
    e = best_e;
    for (int k = 1; k < n; ++k) C[k] += best_d[k];
    ++steps;
  }
  *final_state = cur;
  *final_energy = e;
  *evals_used = evals;
  *steps_taken = steps;
}

// ---------------------------------------------------------------------------
// Complex128 statevector evolution, restating src/sampling/sampler.cuh:
//   * state init |s0> (:428-438),
//   * per step: diagonal phase exp(-i (dt/n) E(s)) (:73-91, :607-609), then the
//     2x2 matrix Rx(-2 g dt) = [[cos(g dt), i sin(g dt)], [i sin(g dt), cos(g dt)]]
//     applied to every qubit in turn (:451-457, :611-617),
//   * measurement BEFORE stepping at the flagged steps 0..n_steps (:509-557):
//     P_< = sum_{E(s) < e0} |psi_s|^2, <d_H> = sum |psi_s|^2 popcount(s ^ s0)
//     (:149-195), plus the norm.
// g_per_step has n_steps entries (a piecewise-constant schedule); diag_scale <= 0
// means the reference's dt/n.
// ---------------------------------------------------------------------------
int orc_trotter_evolve(int n, uint64_t s0, int64_t e0, const double* g_per_step, double dt,
                       double diag_scale, int n_steps, const uint8_t* measure, double* p_less,
                       double* d_h, double* norm, int n_threads, double* state_out,
                       double* step_seconds) {
  if (n < 1 || n > 30 || n_steps < 0) return 1;
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
  const int64_t A = 1LL << n;
  const uint64_t m = mask_of(n);
  s0 &= m;
  std::vector<std::complex<double>> psi((size_t)A, {0.0, 0.0});
  std::vector<uint16_t> E((size_t)A);
  orc_energy_table_u16(n, E.data());
  psi[(size_t)s0] = {1.0, 0.0};
  const double scale = (diag_scale > 0.0) ? (dt * diag_scale) : (dt / (double)n);

  int mi = 0;
  for (int step = 0; step <= n_steps; ++step) {
    // a step's wall time covers its measurement (if flagged) and the step itself
    const double t_step0 = (step_seconds && step < n_steps) ? omp_get_wtime() : 0.0;
    if (measure == nullptr || measure[step]) {
      // fixed-order blocked reduction (deterministic for a given thread count)
      const int64_t nblk = std::min<int64_t>(A, 4096);
      std::vector<double> bp((size_t)nblk), bd((size_t)nblk), bn((size_t)nblk);
#pragma omp parallel for schedule(static)
      for (int64_t b = 0; b < nblk; ++b) {
        const int64_t lo = A * b / nblk, hi = A * (b + 1) / nblk;
        double sp = 0, sd = 0, sn = 0;
        for (int64_t s = lo; s < hi; ++s) {
          const double w = std::norm(psi[(size_t)s]);
          sn += w;
          if ((int64_t)E[(size_t)s] < e0) sp += w;
          sd += w * (double)__builtin_popcountll((uint64_t)s ^ s0);
        }
        bp[(size_t)b] = sp;
        bd[(size_t)b] = sd;
        bn[(size_t)b] = sn;
      }
      double P = 0, D = 0, Nn = 0;
      for (int64_t b = 0; b < nblk; ++b) {
        P += bp[(size_t)b];
        D += bd[(size_t)b];
        Nn += bn[(size_t)b];
      }
      p_less[mi] = P;
      d_h[mi] = D;
      if (norm) norm[mi] = Nn;
      ++mi;
    }
    if (step == n_steps) break;
    // (i) diagonal phase; theta = -(dt/n) * E as in sampler.cuh:83
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < A; ++s) {
      const double th = -scale * (double)E[(size_t)s];
      psi[(size_t)s] *= std::complex<double>(std::cos(th), std::sin(th));
    }
    // (ii) Rx(-2 g dt) on every qubit; matrix entries as sampler.cuh:451-457
    const double rx = -2.0 * g_per_step[step] * dt;
    const double c = std::cos(rx / 2.0), sn = -std::sin(rx / 2.0);
    const std::complex<double> m00(c, 0.0), m01(0.0, sn);
    for (int q = 0; q < n; ++q) {
      const int64_t bit = 1LL << q;
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < A / 2; ++i) {
        const int64_t a = ((i >> q) << (q + 1)) | (i & (bit - 1));
        const int64_t b = a | bit;
        const std::complex<double> x = psi[(size_t)a], y = psi[(size_t)b];
        psi[(size_t)a] = m00 * x + m01 * y;
        psi[(size_t)b] = m01 * x + m00 * y;
      }
    }
    if (step_seconds) step_seconds[step] = omp_get_wtime() - t_step0;
  }
  if (state_out) std::memcpy(state_out, psi.data(), sizeof(double) * 2 * (size_t)A);
  return 0;
}

}  // extern "C"

namespace {

using cvec = std::vector<std::complex<double>>;

// One reference-order Trotter step psi <- M(g) D psi, exact gates as in
// orc_trotter_evolve (sampler.cuh:73-91 phase, :451-457 + :611-617 mixer).
void trotter_step(cvec& psi, const std::vector<uint16_t>& E, int n, double angle_unit, double g, double dt) {
  const int64_t A = (int64_t)psi.size();
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < A; ++s) {
    const double th = -angle_unit * (double)E[(size_t)s];
    psi[(size_t)s] *= std::complex<double>(std::cos(th), std::sin(th));
  }
  const double c = std::cos(g * dt), sn = std::sin(g * dt);
  const std::complex<double> m00(c, 0.0), m01(0.0, sn);
  for (int q = 0; q < n; ++q) {
    const int64_t bit = 1LL << q;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < A / 2; ++i) {
      const int64_t a = ((i >> q) << (q + 1)) | (i & (bit - 1));
      const int64_t b = a | bit;
      const std::complex<double> x = psi[(size_t)a], y = psi[(size_t)b];
      psi[(size_t)a] = m00 * x + m01 * y;
      psi[(size_t)b] = m01 * x + m00 * y;
    }
  }
}

// The adjoint step lambda <- (M(g) D)^dagger lambda = D^dagger M(-g) lambda.
void adjoint_step(cvec& lam, const std::vector<uint16_t>& E, int n, double angle_unit, double g, double dt) {
  const int64_t A = (int64_t)lam.size();
  const double c = std::cos(g * dt), sn = -std::sin(g * dt);
  const std::complex<double> m00(c, 0.0), m01(0.0, sn);
  for (int q = 0; q < n; ++q) {
    const int64_t bit = 1LL << q;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < A / 2; ++i) {
      const int64_t a = ((i >> q) << (q + 1)) | (i & (bit - 1));
      const int64_t b = a | bit;
      const std::complex<double> x = lam[(size_t)a], y = lam[(size_t)b];
      lam[(size_t)a] = m00 * x + m01 * y;
      lam[(size_t)b] = m01 * x + m00 * y;
    }
  }
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < A; ++s) {
    const double th = angle_unit * (double)E[(size_t)s];
    lam[(size_t)s] *= std::complex<double>(std::cos(th), std::sin(th));
  }
}

// Im <lam| G |psi> with G = sum_q X_q, summed in a fixed order.
double im_lam_g_psi(const cvec& lam, const cvec& psi, int n) {
  const int64_t A = (int64_t)psi.size();
  const int64_t nblk = std::min<int64_t>(A, 1024);
  std::vector<double> part((size_t)nblk, 0.0);
#pragma omp parallel for schedule(static)
  for (int64_t b = 0; b < nblk; ++b) {
    const int64_t lo = A * b / nblk, hi = A * (b + 1) / nblk;
    double acc = 0.0;
    for (int64_t s = lo; s < hi; ++s) {
      std::complex<double> gp(0.0, 0.0);
      for (int q = 0; q < n; ++q) gp += psi[(size_t)(s ^ (1LL << q))];
      acc += (std::conj(lam[(size_t)s]) * gp).imag();
    }
    part[(size_t)b] = acc;
  }
  double tot = 0.0;
  for (double v : part) tot += v;
  return tot;
}

}  // namespace

extern "C" {

// Gradient of a diagonal observable at the final time with respect to the
// per-step transverse field, by the adjoint method. The reference has no
// gradient; this restates the textbook derivation for its step
// psi_{k+1} = M(g_k) D psi_k (sampler.cuh:604-618) with
// M(g) = prod_q exp(+i g dt X_q), dM/dg = i dt G M, G = sum_q X_q:
//   O = <psi_T| W |psi_T>,  lambda_T = W psi_T,  lambda_k = (M(g_k) D)^dagger lambda_{k+1},
//   dO/dg_k = 2 Re <lambda_{k+1}| i dt G |psi_{k+1}> = -2 dt Im <lambda_{k+1}| G |psi_{k+1}>.
// W = [E(s) < e0] (objective 0, P_<) or popcount(s ^ s0) (objective 1, <d_H>).
// The forward states psi_{k+1} are recomputed from checkpoints every C ~ sqrt(T)
// steps (exact gates, no inverse steps), so this checker shares no numerical
// shortcut with the device adjoint. grad_out[k] = dO/dg_k for k < n_steps.
int orc_trotter_adjoint(int n, uint64_t s0, int64_t e0, const double* g_per_step, double dt, double diag_scale,
                        int n_steps, int objective, int n_threads, double* value_out, double* grad_out) {
  if (n < 1 || n > 26 || n_steps < 0 || (objective != 0 && objective != 1)) return 1;
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
  const int64_t A = 1LL << n;
  s0 &= mask_of(n);
  std::vector<uint16_t> E((size_t)A);
  orc_energy_table_u16(n, E.data());
  const double angle_unit = (diag_scale > 0.0) ? (dt * diag_scale) : (dt / (double)n);
  const int C = std::max(1, (int)std::ceil(std::sqrt((double)std::max(n_steps, 1))));
  // forward with checkpoints psi_{jC}
  std::vector<cvec> ckpt;
  cvec psi((size_t)A, {0.0, 0.0});
  psi[(size_t)s0] = {1.0, 0.0};
  for (int k = 0; k < n_steps; ++k) {
    if (k % C == 0) ckpt.push_back(psi);
    trotter_step(psi, E, n, angle_unit, g_per_step[k], dt);
  }
  // objective and lambda_T = W psi_T
  cvec lam((size_t)A);
  double value = 0.0;
  {
    const int64_t nblk = std::min<int64_t>(A, 1024);
    std::vector<double> part((size_t)nblk, 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < nblk; ++b) {
      const int64_t lo = A * b / nblk, hi = A * (b + 1) / nblk;
      double acc = 0.0;
      for (int64_t s = lo; s < hi; ++s) {
        const double w = (objective == 0) ? (((int64_t)E[(size_t)s] < e0) ? 1.0 : 0.0)
                                          : (double)__builtin_popcountll((uint64_t)s ^ s0);
        lam[(size_t)s] = w * psi[(size_t)s];
        acc += w * std::norm(psi[(size_t)s]);
      }
      part[(size_t)b] = acc;
    }
    for (double v : part) value += v;
  }
  if (value_out) *value_out = value;
  // reverse sweep window by window; psi_{k+1} recomputed forward inside the window
  for (int w = (int)ckpt.size() - 1; w >= 0; --w) {
    const int k0 = w * C, k1 = std::min(n_steps, k0 + C);
    std::vector<cvec> traj;  // psi_{k0+1} .. psi_{k1}
    cvec x = ckpt[(size_t)w];
    for (int k = k0; k < k1; ++k) {
      trotter_step(x, E, n, angle_unit, g_per_step[k], dt);
      traj.push_back(x);
    }
    for (int k = k1 - 1; k >= k0; --k) {
      // lam = lambda_{k+1}, traj[k - k0] = psi_{k+1}
      grad_out[k] = -2.0 * dt * im_lam_g_psi(lam, traj[(size_t)(k - k0)], n);
      adjoint_step(lam, E, n, angle_unit, g_per_step[k], dt);
    }
  }
  return 0;
}

}  // extern "C"

extern "C" {

// Projective sampling by inverse CDF over |psi|^2 (the reference delegates to the
// closed cuStateVec sampler, sampler.cuh:464-466, 564-573; output in random-number
// order): shot k returns the smallest index s with u_k * total < cdf(s), where
// cdf(s) = sum_{t <= s} |psi_t|^2 accumulated in index order in FP64.
void orc_sample_indices(int n, const double* state_ri, const double* randnums, int64_t shots,
                        uint64_t* out) {
  const int64_t A = 1LL << n;
  std::vector<double> cdf((size_t)A);
  double acc = 0.0;
  for (int64_t s = 0; s < A; ++s) {
    acc += state_ri[2 * s] * state_ri[2 * s] + state_ri[2 * s + 1] * state_ri[2 * s + 1];
    cdf[(size_t)s] = acc;
  }
  for (int64_t k = 0; k < shots; ++k) {
    const double target = randnums[k] * acc;
    int64_t idx = std::upper_bound(cdf.begin(), cdf.end(), target) - cdf.begin();
    if (idx >= A) idx = A - 1;
    out[k] = (uint64_t)idx;
  }
}

// mt19937_64(seed) + std::uniform_real_distribution<double>(0,1), as the
// reference draws shots (sampler.cuh:476-487, 568).
void orc_uniform_randoms(uint64_t seed, int64_t count, double* out) {
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> dist(0.0, 1.0);
  for (int64_t i = 0; i < count; ++i) out[i] = dist(rng);
}

// ---------------------------------------------------------------------------
// Full ISampler::sample() semantics (src/sampling/sampler.cuh:412-707) on the
// complex128 restatement above: measurement / sampling schedule (:496-602),
// per-shot host statistics (:575-596), post-processing (:621-683).
// Arrays are caller-allocated: times/p_less/d_h hold n_steps + 1 entries,
// seed arrays hold max(1, num_sampling_seeds) entries.
// ---------------------------------------------------------------------------
struct orc_sampler_config {
  int32_t n;
  int32_t num_sample_points;
  int32_t shots_per_point;
  int32_t num_sampling_seeds;
  int32_t track_p_less;
  int32_t record_trajectory;
  uint64_t seed;
  uint64_t seed_stride;
  double g, dt, t_max, t_start, dt_sample, dt_trajectory;
};

struct orc_sampling_result {
  int64_t n_points;
  double* time_points;
  double* p_less_history;
  double* dh_history;
  int64_t start_energy;
  int32_t d_min;
  double p_blind, peak_p_less, peak_time, window_avg_dh;
  double initial_rise_rate_avg, initial_rise_rate_max;
  uint64_t total_shots_collected, improved_shots, total_evals, unique_basis_size;
  double success_rate, per_eval_rate, mean_hamming_flips;
  int32_t n_seeds;
  uint64_t* seed_values;
  uint64_t* seed_total_shots;
  uint64_t* seed_improved_shots;
  double* seed_success_rate;
  double* seed_mean_hamming;
  int64_t* seed_best_energy;
};

int orc_sampler_run(const orc_sampler_config* cfg, uint64_t start_bits, orc_sampling_result* r) {
  const int n = cfg->n;
  if (n < 1 || n > 30) return 1;
  const uint64_t m = mask_of(n);
  const int64_t A = 1LL << n;
  r->start_energy = energy_of(n, start_bits);
  r->d_min = orc_d_min(n, start_bits, r->start_energy, -1);
  r->p_blind = (double)orc_count_below(n, r->start_energy) / (double)A;
  const uint64_t s0 = start_bits & m;

  std::vector<std::complex<double>> psi((size_t)A, {0.0, 0.0});
  std::vector<uint16_t> E((size_t)A);
  orc_energy_table_u16(n, E.data());
  psi[(size_t)s0] = {1.0, 0.0};

  const int shots = std::max(1, cfg->shots_per_point);
  const int n_seeds = std::max(1, cfg->num_sampling_seeds);
  std::vector<std::mt19937_64> rngs((size_t)n_seeds);
  r->n_seeds = n_seeds;
  for (int s = 0; s < n_seeds; ++s) {
    const uint64_t cs = cfg->seed + (uint64_t)s * cfg->seed_stride;
    rngs[(size_t)s].seed(cs);
    r->seed_values[s] = cs;
    r->seed_total_shots[s] = 0;
    r->seed_improved_shots[s] = 0;
    r->seed_mean_hamming[s] = 0.0;
    r->seed_best_energy[s] = r->start_energy;
  }
  std::uniform_real_distribution<double> dist(0.0, 1.0);
  std::unordered_set<uint64_t> uniq;
  uint64_t flips_primary = 0;
  r->total_shots_collected = 0;
  r->improved_shots = 0;
  r->peak_p_less = 0.0;
  r->peak_time = 0.0;
  r->n_points = 0;

  const int T = (int)std::round(cfg->t_max / cfg->dt);
  const double sample_interval = (cfg->dt_sample > 0.0)
      ? cfg->dt_sample : (cfg->t_max / std::max(1, cfg->num_sample_points));
  double next_sample = cfg->t_start;
  const double traj_interval = (cfg->dt_trajectory > 0.0) ? cfg->dt_trajectory : cfg->dt;
  double next_traj = 0.0;
  const double sample_end = (cfg->num_sample_points > 1 && cfg->dt_sample > 0.0)
      ? (cfg->t_start + (cfg->num_sample_points - 1) * cfg->dt_sample) : cfg->t_max;
  int taken = 0;
  const double rx = -2.0 * cfg->g * cfg->dt;
  const std::complex<double> m00(std::cos(rx / 2.0), 0.0), m01(0.0, -std::sin(rx / 2.0));
  const double scale = cfg->dt / (double)n;

  auto measure = [&](double t) {
    double P = 0, D = 0;
    for (int64_t s = 0; s < A; ++s) {
      const double w = std::norm(psi[(size_t)s]);
      if ((int64_t)E[(size_t)s] < r->start_energy) P += w;
      D += w * (double)__builtin_popcountll((uint64_t)s ^ s0);
    }
    r->time_points[r->n_points] = t;
    r->p_less_history[r->n_points] = P;
    r->dh_history[r->n_points] = D;
    r->n_points++;
    if (P > r->peak_p_less) { r->peak_p_less = P; r->peak_time = t; }
  };

  std::vector<double> rnd((size_t)shots);
  std::vector<uint64_t> idx((size_t)shots);
  std::vector<double> state_ri;
  for (int step = 0; step <= T; ++step) {
    const double t = step * cfg->dt;
    if (cfg->record_trajectory) {
      if (t >= next_traj - 1e-9 && next_traj <= cfg->t_max + 1e-9) {
        measure(t);
        next_traj += traj_interval;
      }
    } else if (cfg->track_p_less) {
      if (t >= next_sample - 1e-9 && next_sample <= cfg->t_max + 1e-9) measure(t);
    }
    if (cfg->shots_per_point > 0 && t >= cfg->t_start - 1e-9 && t >= next_sample - 1e-9 &&
        next_sample <= sample_end + 1e-9 &&
        (cfg->num_sample_points <= 0 || taken < cfg->num_sample_points)) {
      ++taken;
      state_ri.resize(2 * (size_t)A);
      std::memcpy(state_ri.data(), psi.data(), sizeof(double) * 2 * (size_t)A);
      for (int si = 0; si < n_seeds; ++si) {
        for (int i = 0; i < shots; ++i) rnd[(size_t)i] = dist(rngs[(size_t)si]);
        orc_sample_indices(n, state_ri.data(), rnd.data(), shots, idx.data());
        uint64_t flips = 0;
        for (int i = 0; i < shots; ++i) {
          const uint64_t b = idx[(size_t)i];
          uniq.insert(b);
          const int d = __builtin_popcountll(b ^ start_bits);
          flips += (uint64_t)d;
          if (si == 0) flips_primary += (uint64_t)d;
          const int64_t e = energy_of(n, b);
          if (e < r->seed_best_energy[si]) r->seed_best_energy[si] = e;
          if (e < r->start_energy) {
            r->seed_improved_shots[si]++;
            if (si == 0) r->improved_shots++;
          }
        }
        r->seed_total_shots[si] += (uint64_t)shots;
        r->seed_mean_hamming[si] += (double)flips;
      }
      r->total_shots_collected += (uint64_t)shots;
      next_sample += sample_interval;
    } else if (cfg->shots_per_point == 0 && !cfg->record_trajectory && cfg->track_p_less &&
               t >= next_sample - 1e-9 && next_sample <= cfg->t_max + 1e-9) {
      next_sample += sample_interval;
    }
    if (step < T) {
      for (int64_t s = 0; s < A; ++s) {
        const double th = -scale * (double)E[(size_t)s];
        psi[(size_t)s] *= std::complex<double>(std::cos(th), std::sin(th));
      }
      for (int q = 0; q < n; ++q) {
        const int64_t bit = 1LL << q;
        for (int64_t i = 0; i < A / 2; ++i) {
          const int64_t a = ((i >> q) << (q + 1)) | (i & (bit - 1));
          const int64_t b = a | bit;
          const std::complex<double> x = psi[(size_t)a], y = psi[(size_t)b];
          psi[(size_t)a] = m00 * x + m01 * y;
          psi[(size_t)b] = m01 * x + m00 * y;
        }
      }
    }
  }

  // post-processing, sampler.cuh:621-683
  r->unique_basis_size = uniq.size();
  r->total_evals = r->total_shots_collected;
  r->success_rate = 0.0;
  r->per_eval_rate = 0.0;
  r->mean_hamming_flips = 0.0;
  if (r->total_shots_collected > 0) {
    r->mean_hamming_flips = (double)flips_primary / (double)r->total_shots_collected;
    r->success_rate = (double)r->improved_shots / (double)r->total_shots_collected;
    r->per_eval_rate = (double)r->improved_shots / (double)r->total_evals;
  }
  for (int s = 0; s < n_seeds; ++s) {
    r->seed_success_rate[s] = 0.0;
    if (r->seed_total_shots[s] > 0) {
      r->seed_success_rate[s] = (double)r->seed_improved_shots[s] / (double)r->seed_total_shots[s];
      r->seed_mean_hamming[s] /= (double)r->seed_total_shots[s];
    }
  }
  r->initial_rise_rate_avg = 0.0;
  r->initial_rise_rate_max = 0.0;
  const int64_t np = r->n_points;
  if (np > 0) {
    int64_t first_drop = np - 1;
    for (int64_t i = 1; i < np; ++i)
      if (r->p_less_history[i] < r->p_less_history[i - 1]) { first_drop = i - 1; break; }
    const double tp = r->time_points[first_drop];
    r->initial_rise_rate_avg = (tp > 0.0) ? (r->p_less_history[first_drop] / tp) : 0.0;
    double mx = (r->time_points[0] > 1e-9) ? (r->p_less_history[0] / r->time_points[0]) : 0.0;
    for (int64_t i = 0; i < first_drop; ++i) {
      const double h = r->time_points[i + 1] - r->time_points[i];
      if (h > 1e-9) mx = std::max(mx, (r->p_less_history[i + 1] - r->p_less_history[i]) / h);
    }
    r->initial_rise_rate_max = mx;
  }
  const double a0 = cfg->t_start;
  const double a1 = (cfg->num_sample_points > 1 && cfg->dt_sample > 0.0)
      ? (cfg->t_start + (cfg->num_sample_points - 1) * cfg->dt_sample) : cfg->t_max;
  double sum = 0.0;
  int64_t cnt = 0;
  for (int64_t i = 0; i < np; ++i)
    if (r->time_points[i] >= a0 - 1e-9 && r->time_points[i] <= a1 + 1e-9) { sum += r->dh_history[i]; ++cnt; }
  r->window_avg_dh = (cnt > 0) ? sum / (double)cnt : (np > 0 ? r->dh_history[np - 1] : 0.0);
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Full-space Hamiltonian H = diag(scale E(s)) - g sum_j X_j and the plain
// Lanczos iteration over it (src/subspace/diagonalizer.cuh).
// ---------------------------------------------------------------------------
namespace {

// y = H x, each state in the reference's order: diag * x_i, then - g x[i ^ 2^j]
// for j = 0..n-1 (fullspace_matvec_kernel_d, diagonalizer.cuh:60-77; the
// diagonal scale * E(s), :388-392)
void fs_matvec(int n, double g, double scale, const double* x, double* y) {
  const int64_t dim = int64_t(1) << n;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < dim; ++i) {
    double yi = static_cast<double>(energy_of(n, static_cast<uint64_t>(i))) * scale * x[i];
    for (int j = 0; j < n; ++j) yi -= g * x[i ^ (int64_t(1) << j)];
    y[i] = yi;
  }
}

double dot(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0.0;
  for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
  return s;
}

}  // namespace

extern "C" {

int orc_fullspace_matvec(int n, double g, double scale, const double* x, double* y, int n_threads) {
  if (n < 1 || n > 26 || !x || !y) return 1;
  if (n_threads > 0) omp_set_num_threads(n_threads);
  fs_matvec(n, g, scale, x, y);
  return 0;
}

// The reference's run_gpu_lanczos_internal (diagonalizer.cuh:418-482) in FP64 on
// the CPU: start vector mt19937_64(42) / uniform(-0.5, 0.5) normalised; per step
// w = H v_j, w -= beta_{j-1} v_{j-1}, alpha_j = v_j . w, w -= alpha_j v_j, and
// (j < m - 1) beta_j = |w|, stop when beta_j < tol, v_{j+1} = w / beta_j.
// alphas[m_actual], betas[m_actual - 1]; *m_actual = steps taken.
int orc_fullspace_lanczos(int n, double g, double scale, int max_krylov_dim, double tol, double* alphas,
                          double* betas, int* m_actual, int n_threads) {
  if (n < 1 || n > 24 || max_krylov_dim < 1 || !alphas || !betas || !m_actual) return 1;
  if (n_threads > 0) omp_set_num_threads(n_threads);
  const int64_t N = int64_t(1) << n;
  const int m = static_cast<int>(std::min<int64_t>(N, max_krylov_dim));
  std::vector<double> v(N), vprev(N, 0.0), w(N);
  std::mt19937_64 rng(42);
  std::uniform_real_distribution<double> dist(-0.5, 0.5);
  for (int64_t i = 0; i < N; ++i) v[i] = dist(rng);
  const double inv0 = 1.0 / std::sqrt(dot(v, v));
  for (auto& a : v) a *= inv0;
  int mm = m;
  for (int j = 0; j < m; ++j) {
    fs_matvec(n, g, scale, v.data(), w.data());
    if (j > 0)
      for (int64_t i = 0; i < N; ++i) w[i] -= betas[j - 1] * vprev[i];
    alphas[j] = dot(v, w);
    for (int64_t i = 0; i < N; ++i) w[i] -= alphas[j] * v[i];
    if (j < m - 1) {
      betas[j] = std::sqrt(dot(w, w));
      if (std::fabs(betas[j]) < tol) {
        mm = j + 1;
        break;
      }
      const double inv = 1.0 / betas[j];
      vprev.swap(v);
      for (int64_t i = 0; i < N; ++i) v[i] = w[i] * inv;
    }
  }
  *m_actual = mm;
  return 0;
}

}  // extern "C"
