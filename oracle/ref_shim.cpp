// ============================================================================
// ORACLE — test infrastructure only. C-ABI shim that compiles the reference's
// OWN header-only C++ (src/labs_energy/labs_energy.hpp, the host part of
// src/classical/classical.cuh) from the reference tree, so the restatement in
// trotter_oracle.cpp and the product can be checked against the real code.
// Built by oracle/Makefile into oracle/_ref/libbk_ref.so (git-ignored) only when
// the reference tree is present; nothing on the GPU box needs it.
// ============================================================================
#include "labs_energy/labs_energy.hpp"
#include "classical/classical.cuh"

extern "C" {

int64_t ref_calc_energy(int n, uint64_t bits) { return LabsEvaluator(n).calcEnergy(SpinState{bits}); }

void ref_calc_ck(int n, uint64_t bits, int64_t* out) {
  std::vector<int64_t> c = LabsEvaluator(n).calcCk(SpinState{bits});
  for (int k = 0; k < n; ++k) out[k] = c[(size_t)k];
}

uint64_t ref_canonical(int n, uint64_t bits) { return SpinState{bits}.canonical(n).bits; }

int ref_d_min(int n, uint64_t bits, int64_t target, int max_d) {
  return LabsEvaluator(n).compute_d_min(SpinState{bits}, target, max_d);
}

int64_t ref_known_optimal_energy(int n) { return LabsEvaluator::known_optimal_energy(n); }

void ref_random_states(int n, uint64_t seed, int64_t count, uint64_t* out) {
  ClassicalOptimizer opt(n, seed);
  for (int64_t i = 0; i < count; ++i) out[i] = opt.random_state().bits;
}

void ref_steepest_descent(int n, uint64_t start, uint64_t max_evals, uint64_t* final_state,
                          int64_t* final_energy, uint64_t* evals_used, int64_t* steps_taken) {
  ClassicalOptimizer opt(n, 42);
  DescentResult r = opt.steepest_descent(SpinState{start},
                                         max_evals == 0 ? std::numeric_limits<size_t>::max()
                                                        : (size_t)max_evals);
  *final_state = r.final_state.bits;
  *final_energy = r.final_energy;
  *evals_used = (uint64_t)r.evals_used;
  *steps_taken = (int64_t)r.steps_taken;
}

}  // extern "C"
