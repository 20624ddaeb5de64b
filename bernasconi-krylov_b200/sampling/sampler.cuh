#pragma once
// Drop-in replacement for the reference's src/sampling/sampler.cuh
// (ssk1001/bernasconi-krylov): same SamplerConfig / SeedSamplingStats /
// SamplingResult / ISampler / create_sampler, backed by the B200 engine's C ABI
// (include/bk_engine.h, library libbk_b200.so) instead of cuStateVec.
//
// Placed at src/sampling/sampler.cuh of a reference checkout (or found first on
// the include path), the reference's connector (src/connector/connector.cuh:646-680)
// and run_benchmark driver build unchanged: HAS_CUSTATEVEC is 1, so the connector
// takes its GPU branch, and create_sampler(n) returns the B200 sampler.
//
// Environment: BK_SAMPLER_DEVICE (default 0), BK_SAMPLER_PRECISION = c128 (default,
// the reference's precision) or c64.

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../labs_energy/labs_energy.hpp"
#include "bk_engine.h"

#ifndef HAS_CUSTATEVEC
#define HAS_CUSTATEVEC 1
#endif

// reference: src/sampling/sampler.cuh:235-260
struct SamplerConfig {
  int n = 16;
  double g = 0.5;
  double dt = 0.05;
  double t_max = 60.0;
  int num_sample_points = 20;
  int shots_per_point = 100;
  uint64_t seed = 42;
  int num_sampling_seeds = 3;
  uint64_t seed_stride = 10007;
  double t_start = 0.0;
  double dt_sample = 0.0;
  bool track_p_less = true;
  bool verbose = true;
  bool record_trajectory = false;
  double dt_trajectory = 0.0;
};

// reference: src/sampling/sampler.cuh:262-270
struct SeedSamplingStats {
  uint64_t seed = 0;
  size_t total_shots_collected = 0;
  size_t improved_shots = 0;
  double success_rate = 0.0;
  double per_eval_rate = 0.0;
  double mean_hamming_flips = 0.0;
  int64_t best_energy = std::numeric_limits<int64_t>::max();
};

// reference: src/sampling/sampler.cuh:272-297
struct SamplingResult {
  std::vector<SpinState> unique_basis;
  size_t total_shots_collected = 0;
  size_t improved_shots = 0;
  double success_rate = 0.0;
  double per_eval_rate = 0.0;
  size_t total_evals = 0;
  double mean_hamming_flips = 0.0;
  std::vector<SeedSamplingStats> seed_stats;
  std::vector<double> time_points;
  std::vector<double> p_less_history;
  std::vector<double> dh_history;
  double window_avg_dh = 0.0;
  double initial_rise_rate_avg = 0.0;
  double initial_rise_rate_max = 0.0;
  int d_min = 0;
  int64_t start_energy = 0;
  double p_blind = 0.0;
  double peak_p_less = 0.0;
  double peak_time = 0.0;
};

// reference: src/sampling/sampler.cuh:303-310
class ISampler {
 public:
  virtual ~ISampler() = default;
  virtual SamplingResult sample(const SpinState& start_state, const SamplerConfig& config) = 0;
};

// Statevector sampler on the B200 engine (n <= 30). Errors surface as
// std::runtime_error, as the reference's CHECK_CUDA / CHECK_CUSTATEVEC do.
class B200StateVecSampler : public ISampler {
 public:
  explicit B200StateVecSampler(int device = -1, int precision = -1, int method = BK_FUSED) : method_(method) {
    if (device < 0) device = env_int("BK_SAMPLER_DEVICE", 0);
    if (precision < 0) {
      const char* p = std::getenv("BK_SAMPLER_PRECISION");
      precision = (p && std::string(p) == "c64") ? BK_C64 : BK_C128;
    }
    precision_ = precision;
    const int st = bk_create(device, &ctx_);
    if (st != BK_OK) throw std::runtime_error(std::string("B200 engine unavailable: ") + bk_status_string(st));
  }
  ~B200StateVecSampler() override { bk_destroy(ctx_); }
  B200StateVecSampler(const B200StateVecSampler&) = delete;
  B200StateVecSampler& operator=(const B200StateVecSampler&) = delete;

  SamplingResult sample(const SpinState& start_state, const SamplerConfig& config) override {
    bk_sampler_config c;
    std::memset(&c, 0, sizeof(c));
    c.n = config.n;
    c.num_sample_points = config.num_sample_points;
    c.shots_per_point = config.shots_per_point;
    c.num_sampling_seeds = config.num_sampling_seeds;
    c.track_p_less = config.track_p_less ? 1 : 0;
    c.record_trajectory = config.record_trajectory ? 1 : 0;
    c.verbose = config.verbose ? 1 : 0;
    c.precision = precision_;
    c.method = method_;
    c.seed = config.seed;
    c.seed_stride = config.seed_stride;
    c.g = config.g;
    c.dt = config.dt;
    c.t_max = config.t_max;
    c.t_start = config.t_start;
    c.dt_sample = config.dt_sample;
    c.dt_trajectory = config.dt_trajectory;
    bk_sampling_result r;
    const int st = bk_sampler_run(ctx_, &c, start_state.bits, &r);
    if (st != BK_OK)
      throw std::runtime_error(std::string("bk_sampler_run: ") + bk_status_string(st) + ": " + bk_last_error(ctx_));
    SamplingResult out;
    out.unique_basis.reserve((size_t)r.unique_basis_size);
    for (int64_t i = 0; i < r.unique_basis_size; ++i) out.unique_basis.push_back(SpinState{r.unique_basis[i]});
    out.total_shots_collected = (size_t)r.total_shots_collected;
    out.improved_shots = (size_t)r.improved_shots;
    out.success_rate = r.success_rate;
    out.per_eval_rate = r.per_eval_rate;
    out.total_evals = (size_t)r.total_evals;
    out.mean_hamming_flips = r.mean_hamming_flips;
    for (int i = 0; i < r.n_seed_stats; ++i) {
      SeedSamplingStats s;
      s.seed = r.seed_stats[i].seed;
      s.total_shots_collected = (size_t)r.seed_stats[i].total_shots_collected;
      s.improved_shots = (size_t)r.seed_stats[i].improved_shots;
      s.success_rate = r.seed_stats[i].success_rate;
      s.per_eval_rate = r.seed_stats[i].per_eval_rate;
      s.mean_hamming_flips = r.seed_stats[i].mean_hamming_flips;
      s.best_energy = r.seed_stats[i].best_energy;
      out.seed_stats.push_back(s);
    }
    out.time_points.assign(r.time_points, r.time_points + r.n_points);
    out.p_less_history.assign(r.p_less_history, r.p_less_history + r.n_points);
    out.dh_history.assign(r.dh_history, r.dh_history + r.n_points);
    out.window_avg_dh = r.window_avg_dh;
    out.initial_rise_rate_avg = r.initial_rise_rate_avg;
    out.initial_rise_rate_max = r.initial_rise_rate_max;
    out.d_min = r.d_min;
    out.start_energy = r.start_energy;
    out.p_blind = r.p_blind;
    out.peak_p_less = r.peak_p_less;
    out.peak_time = r.peak_time;
    bk_sampling_result_release(&r);
    return out;
  }

 private:
  static int env_int(const char* k, int d) {
    const char* v = std::getenv(k);
    return v ? std::atoi(v) : d;
  }
  bk_ctx* ctx_ = nullptr;
  int precision_ = BK_C128;
  int method_ = BK_FUSED;
};

// The reference's class name, for code that constructs it directly.
using CuStateVecSampler = B200StateVecSampler;

// reference: src/sampling/sampler.cuh:726-731 (placeholder beyond n = 30)
class CuTensorNetSampler : public ISampler {
 public:
  SamplingResult sample(const SpinState&, const SamplerConfig&) override {
    throw std::runtime_error("cuTensorNet backend for N > 30 is under development.");
  }
};

// reference: src/sampling/sampler.cuh:737-743
inline std::unique_ptr<ISampler> create_sampler(int n) {
  if (n <= 30) return std::make_unique<B200StateVecSampler>();
  return std::make_unique<CuTensorNetSampler>();
}
