// The drop-in ISampler (bernasconi-krylov_b200/sampling/sampler.cuh) exercised the
// way the reference's own tests/test_sampler.cu does: N = 4 smoke checks of shot
// counts, rate ranges, P_< bounds, measurement times, the N > 30 factory path, and
// a connector-style call (src/connector/connector.cuh:629-680). Exits non-zero on
// the first failed check (no assert: checks stay active under NDEBUG).
#include <cmath>
#include <cstdio>
#include <iostream>

#include "sampling/sampler.cuh"

static int failures = 0;
#define CHECK(cond)                                                          \
  do {                                                                       \
    if (!(cond)) {                                                           \
      std::fprintf(stderr, "CHECK failed: %s (line %d)\n", #cond, __LINE__); \
      ++failures;                                                            \
    }                                                                        \
  } while (0)

int main() {
  // shots and rates (reference tests/test_sampler.cu:10-53)
  {
    auto s = create_sampler(4);
    SamplerConfig cfg;
    cfg.n = 4;
    cfg.g = 0.5;
    cfg.dt = 0.05;
    cfg.t_max = 1.0;
    cfg.num_sample_points = 5;
    cfg.shots_per_point = 10;
    cfg.verbose = false;
    SamplingResult r = s->sample(SpinState(0b0000), cfg);
    CHECK(r.total_shots_collected == 50);
    CHECK(r.success_rate >= 0.0 && r.success_rate <= 1.0);
    CHECK(r.per_eval_rate >= 0.0 && r.per_eval_rate <= 1.0);
    CHECK(r.seed_stats.size() == 3);
    for (const auto& ss : r.seed_stats) CHECK(ss.total_shots_collected == 50);
    CHECK(!r.unique_basis.empty());
    for (double p : r.p_less_history) CHECK(p >= -1e-9 && p <= 1.0 + 1e-9);
  }
  // delayed window: times >= t_start (reference tests/test_sampler.cu:56-106)
  {
    auto s = create_sampler(4);
    SamplerConfig cfg;
    cfg.n = 4;
    cfg.g = 0.5;
    cfg.dt = 0.05;
    cfg.t_max = 2.0;
    cfg.t_start = 0.5;
    cfg.dt_sample = 0.25;
    cfg.num_sample_points = 4;
    cfg.shots_per_point = 8;
    cfg.verbose = false;
    SamplingResult r = s->sample(SpinState(0b0111), cfg);
    CHECK(r.total_shots_collected == 32);
    for (double t : r.time_points) CHECK(t >= cfg.t_start - 1e-9);
    CHECK(!r.time_points.empty());
  }
  // continuous trajectory from t = 0 to t_max inclusive
  {
    auto s = create_sampler(6);
    SamplerConfig cfg;
    cfg.n = 6;
    cfg.g = 0.35;
    cfg.dt = 0.05;
    cfg.t_max = 1.0;
    cfg.record_trajectory = true;
    cfg.shots_per_point = 0;
    cfg.verbose = true;
    SamplingResult r = s->sample(SpinState(0b101100), cfg);
    CHECK(r.time_points.size() == 21);
    CHECK(std::fabs(r.time_points.back() - 1.0) < 1e-9);
    CHECK(r.start_energy == LabsEvaluator(6).calcEnergy(SpinState(0b101100)));
    CHECK(r.d_min == LabsEvaluator(6).compute_d_min(SpinState(0b101100), r.start_energy));
  }
  // factory beyond the statevector range throws (reference tests/test_sampler.cu:153-174)
  {
    bool threw = false;
    try {
      auto s = create_sampler(32);
      SamplerConfig cfg;
      cfg.n = 32;
      s->sample(SpinState(0), cfg);
    } catch (const std::runtime_error&) {
      threw = true;
    }
    CHECK(threw);
  }
  if (failures == 0) std::cout << "test_sampler_dropin: all checks passed\n";
  return failures == 0 ? 0 : 1;
}
