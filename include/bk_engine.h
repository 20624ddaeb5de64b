/*
 * bk_engine.h — C ABI of the B200 statevector engine for the transverse-field
 * Trotter path of ssk1001/bernasconi-krylov.
 *
 * Plain C: no C++ or torch types cross this boundary. Every entry point returns
 * a bk_status; human-readable detail for the last failure on a context is
 * available from bk_last_error(). Citations name the reference interface each
 * entry point replaces (paths relative to the reference project root).
 */
#ifndef BK_ENGINE_H
#define BK_ENGINE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BK_ABI_VERSION 1

typedef enum bk_status {
  BK_OK = 0,
  BK_ERR_INVALID = 1,     /* bad argument (n out of range, NaN field, NULL pointer, ...) */
  BK_ERR_CUDA = 2,        /* CUDA runtime/driver error */
  BK_ERR_OOM = 3,         /* device allocation failed or size overflow */
  BK_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up (kernel returned early) */
  BK_ERR_NORM = 5,        /* |psi|^2 left the tolerance band at a measured step */
  BK_ERR_UNSUPPORTED = 6, /* configuration not provided by this build (e.g. n > 30) */
  BK_ERR_NO_DEVICE = 7,   /* no CUDA device / not an sm_100 device */
  BK_ERR_TOO_LARGE = 8    /* request beyond a fixed limit (bk_measure_noalloc: n <= 30) */
} bk_status;

typedef enum bk_precision { BK_C64 = 0, BK_C128 = 1 } bk_precision;

/* BK_FUSED: tiled passes (diagonal phase + mixer + reductions fused, 64 KB tiles).
 * BK_PLAIN: one diagonal-phase kernel then one 2x2 Rx kernel per qubit, the
 *           launch structure of the reference's cuStateVec loop (sampler.cuh:604-618). */
typedef enum bk_method { BK_FUSED = 0, BK_PLAIN = 1 } bk_method;

/* BK_ORDER_REFERENCE: psi_k = (M D)^k psi_0, the reference's step (sampler.cuh:604-618).
 * BK_ORDER_STRANG:    psi_k = (D^1/2 M D^1/2)^k psi_0. |psi|^2 — hence P_<, <d_H>,
 *                     norms and samples — equals the reference ordering; only the
 *                     exported amplitudes differ by the diagonal phase D^1/2. */
typedef enum bk_ordering { BK_ORDER_REFERENCE = 0, BK_ORDER_STRANG = 1 } bk_ordering;

typedef struct bk_ctx bk_ctx;

/* Context = one device + one stream + cached device buffers (E table per n,
 * statevector, reduction scratch). One context per host thread.
 * Replaces CuStateVecSampler construction / destruction (sampler.cuh:402-410). */
int bk_create(int device, bk_ctx** out);
int bk_destroy(bk_ctx* ctx);
const char* bk_last_error(const bk_ctx* ctx);
const char* bk_status_string(int status);
int bk_abi_version(void);

/* ---- LABS energy core (labs_energy.hpp:121-132, sampler.cuh:54-70, 198-227) ---- */

/* E(s) for `count` host states (exact integers). */
int bk_labs_energy(int n, const uint64_t* states, int64_t count, int64_t* energies_out);

/* Device E table for n (cached on ctx); optionally copied to host (2^n uint16). */
int bk_energy_table(bk_ctx* ctx, int n, uint16_t* host_out);

/* #{s : E(s) < e0} and p_blind = count / 2^n (sampler.cuh:383-399). */
int bk_p_blind(bk_ctx* ctx, int n, int64_t e0, uint64_t* count_out, double* p_blind_out);

/* ---- Trap generation (classical.cuh:557-604, 625-712) ---- */

/* ClassicalOptimizer(n, seed).random_state() drawn `count` times: mt19937_64(seed) & mask. */
int bk_random_states(int n, uint64_t seed, int64_t count, uint64_t* out);

/* Single-flip steepest descent from each start (first strictly best flip, lowest
 * bit wins ties); max_evals = 0 means unlimited. Bit-exact with the reference's
 * ClassicalOptimizer::steepest_descent. evals_out may be NULL. */
int bk_steepest_descent(int n, const uint64_t* starts, int64_t count, uint64_t max_evals,
                        uint64_t* final_states, int64_t* final_energies, uint64_t* evals_out);

/* Trap selection used by the benchmark configurations: n_descents seeded
 * descents (bk_random_states(n, seed) starts); among the local minima with
 * E > E*(n) (not global optima), the threshold is the energy at `quantile` of
 * their sorted energies, and the trap is the first minimum in generation order
 * at or below it. */
int bk_select_trap(int n, uint64_t seed, int32_t n_descents, double quantile, uint64_t* trap_bits,
                   int64_t* trap_energy);

/* Device form of bk_steepest_descent, bit-exact with it (replaces
 * ClassicalOptimizer::run_batch_gpu, classical.cuh:719-770, and its
 * batch_steepest_descent_kernel, :459-540): one warp per start. */
int bk_steepest_descent_gpu(bk_ctx* ctx, int n, const uint64_t* starts, int64_t count, uint64_t max_evals,
                            uint64_t* final_states, int64_t* final_energies, uint64_t* evals_out);

/* Distinct local-minimum families (replaces collect_distinct_minima_gpu,
 * classical.cuh:861-959): batches of batch_size starts from mt19937_64(seed) & mask
 * (one stream across batches), descended on the device (unlimited evaluations);
 * families keyed by the canonical orbit representative, first sample kept, visits
 * counted, evaluations until first find recorded; stops at target_families, at
 * max_starts, or after 4 batches without a new family (saturated). Output sorted
 * by energy, then visits (descending), then discovery order; ids 1..n_out.
 * At most `capacity` families are written; *n_out is the number found. */
typedef struct bk_minimum_family {
  uint64_t id;
  uint64_t canonical_state;
  uint64_t sample_state;
  int64_t energy;
  uint64_t times_visited;
  uint64_t evals_to_first_find;
} bk_minimum_family;

typedef struct bk_collect_stats {
  uint64_t total_starts;
  uint64_t total_evals;
  uint64_t batches;
  int32_t saturated;
  int32_t reserved;
} bk_collect_stats;

int bk_collect_minima(bk_ctx* ctx, int n, uint64_t seed, int64_t target_families, int64_t batch_size,
                      int64_t max_starts, bk_minimum_family* out, int64_t capacity, int64_t* n_out,
                      bk_collect_stats* stats);

/* ---- Evolution (sampler.cuh:428-438, 451-457, 509-619, 149-195) ---- */

typedef struct bk_evolve_params {
  int32_t n;           /* qubits, 1..30 */
  int32_t precision;   /* bk_precision */
  int32_t method;      /* bk_method */
  int32_t ordering;    /* bk_ordering */
  uint64_t s0;         /* trap bits (masked to n); psi_0 = |s0> */
  int64_t e0;          /* P_< threshold: E(s) < e0; < 0 means E(s0) */
  double dt;           /* Trotter step */
  double diag_scale;   /* phase exp(-i dt diag_scale E); <= 0 means 1/n (the reference's dt/n) */
  int32_t n_steps;     /* Trotter steps */
  int32_t reserved0;
  const double* g;     /* host, n_steps entries (piecewise-constant schedule), or NULL */
  double g_const;      /* field used when g == NULL */
  const uint8_t* measure; /* host, n_steps + 1 flags: measure BEFORE step k (k = n_steps: final) */
  double norm_tol;     /* > 0: fail with BK_ERR_NORM when | |psi|^2 - 1 | > norm_tol at a measured step */
  /* projective sampling inside the run (sampler.cuh:559-598): at every flagged
   * step k, `shots` basis states are drawn from |psi_k|^2 (inverse CDF, FP64
   * prefix sums) using the next `shots` host uniforms; results in random-number
   * order. sample == NULL disables sampling. */
  const uint8_t* sample;    /* host, n_steps + 1 flags */
  int32_t shots;            /* draws per flagged step */
  int32_t reserved1;
  const double* randnums;   /* host, (#flagged) * shots uniforms in [0, 1) */
  uint64_t* samples_out;    /* host, (#flagged) * shots basis states */
} bk_evolve_params;

/* Runs the whole schedule on the device and returns one row per flagged step:
 * p_less[m], d_h[m], norm[m] (host arrays of length sum(measure); norm may be NULL).
 * complex128 returns the reference's sums (sampler.cuh:149-195); complex64
 * returns them divided by the measured |psi|^2 (the expectation values of the
 * normalised state: FP32 rounding lets the norm wander ~1e-6 over thousands of
 * steps), and norm[m] is always the raw |psi|^2. */
int bk_evolve(bk_ctx* ctx, const bk_evolve_params* p, double* p_less, double* d_h, double* norm);

/* ---- Batched evolution: many statevectors in one persistent launch ----
 *
 * Every instance has its own n, trap and field; all share dt, the step count and
 * the measurement schedule. The tile tasks of all instances run in ONE
 * persistent kernel (launched through a captured CUDA graph when use_graph is
 * set), interleaved so that each statevector's A1 output is re-read from L2.
 * Outputs are row-major [instance][measurement], normalised like bk_evolve's. */
typedef struct bk_batch_instance {
  int32_t n;           /* qubits: 14..30 (complex64) or 13..30 (complex128) */
  int32_t reserved;
  uint64_t s0;         /* trap bits */
  int64_t e0;          /* P_< threshold; < 0 means E(s0) */
  double g_const;      /* field when g == NULL */
  const double* g;     /* n_steps entries, or NULL */
} bk_batch_instance;

typedef struct bk_batch_params {
  int32_t precision;   /* bk_precision */
  int32_t n_steps;
  double dt;
  double diag_scale;   /* <= 0: 1/n of each instance */
  const uint8_t* measure; /* n_steps + 1 flags, shared */
  int32_t use_graph;   /* 1: launch through a captured CUDA graph */
  int32_t lag;         /* task blocks between a slab's A1 and S2 tasks (<= 0: engine default) */
} bk_batch_params;

int bk_evolve_batch(bk_ctx* ctx, const bk_batch_params* p, const bk_batch_instance* inst, int32_t n_inst,
                    double* p_less, double* d_h, double* norm);

/* Copies the statevector left by the last bk_evolve to host as interleaved
 * (re, im) doubles, 2 * 2^n entries, in the requested ordering's convention. */
int bk_export_state(bk_ctx* ctx, double* host_state_ri);

/* Per-kernel device time of the last bk_evolve when timing is enabled
 * (CUDA events around every launch): name, launches, total milliseconds. */
int bk_set_kernel_timing(bk_ctx* ctx, int enabled);
int bk_kernel_timing(bk_ctx* ctx, int index, const char** name, int64_t* launches, double* total_ms);

/* The context's CUDA stream (a cudaStream_t) so callers can order their own
 * work and record CUDA events around the engine's launches. */
int bk_stream(bk_ctx* ctx, void** stream_out);

/* ---- The reference's ISampler::sample() (sampler.cuh:303-310, 412-707) ---- */

/* SamplerConfig (sampler.cuh:235-260) plus the engine's precision / method. */
typedef struct bk_sampler_config {
  int32_t n;
  int32_t num_sample_points;
  int32_t shots_per_point;
  int32_t num_sampling_seeds;
  int32_t track_p_less;
  int32_t record_trajectory;
  int32_t verbose;
  int32_t precision;        /* bk_precision (the reference computes in complex128) */
  int32_t method;           /* bk_method */
  int32_t reserved;
  uint64_t seed;
  uint64_t seed_stride;
  double g, dt, t_max, t_start, dt_sample, dt_trajectory;
} bk_sampler_config;

/* SeedSamplingStats (sampler.cuh:262-270). */
typedef struct bk_seed_stats {
  uint64_t seed;
  uint64_t total_shots_collected;
  uint64_t improved_shots;
  double success_rate;
  double per_eval_rate;
  double mean_hamming_flips;
  int64_t best_energy;
} bk_seed_stats;

/* SamplingResult (sampler.cuh:272-297). Arrays are allocated by the library and
 * freed by bk_sampling_result_release. */
typedef struct bk_sampling_result {
  uint64_t* unique_basis;
  int64_t unique_basis_size;
  uint64_t total_shots_collected;
  uint64_t improved_shots;
  double success_rate;
  double per_eval_rate;
  uint64_t total_evals;
  double mean_hamming_flips;
  bk_seed_stats* seed_stats;
  int32_t n_seed_stats;
  int32_t d_min;
  double* time_points;
  double* p_less_history;
  double* dh_history;
  int64_t n_points;
  double window_avg_dh;
  double initial_rise_rate_avg;
  double initial_rise_rate_max;
  int64_t start_energy;
  double p_blind;
  double peak_p_less;
  double peak_time;
} bk_sampling_result;

/* Full sample() semantics: E0 and d_min of the start state, p_blind, the
 * measurement / sampling schedule with the reference's time accumulators and
 * 1e-9 tolerances, shots drawn with mt19937_64(seed + s * seed_stride) and
 * uniform_real_distribution<double>(0, 1) in the reference's order, per-shot
 * statistics and the post-processing of rise rates and window averages.
 * n > 30 returns BK_ERR_UNSUPPORTED (the reference throws). */
int bk_sampler_run(bk_ctx* ctx, const bk_sampler_config* cfg, uint64_t start_bits, bk_sampling_result* out);
void bk_sampling_result_release(bk_sampling_result* r);

/* d_min: smallest Hamming distance from s to a state with E < target (target < 0:
 * E(s)); n (or max_d + 1) when none exists or target <= E*(n)
 * (labs_energy.hpp:175-207). Hamming spheres are enumerated on the device. */
int bk_d_min(bk_ctx* ctx, int n, uint64_t bits, int64_t target, int max_d, int* d_out);

/* Engine options (tuning knobs; the autotuner sets them from its cache):
 *   BK_OPT_ENGINE_MODE: 0 = persistent dataflow kernel (all steps in one launch,
 *       L2 hand-off between the A1 and S2 tasks), 1 = one grid launch per pass,
 *       2 = a grid launch for the A1 pass and ONE persistent launch for both
 *       strided passes (S3 re-reads each slab S2 wrote from L2, so the strided
 *       part of a step crosses HBM once; sizes with a single strided pass run
 *       as mode 1), 3 = mode 2 with the fused strided launch served by two
 *       compute groups that load their own tiles (no producer warp); results
 *       bit-identical to mode 2;
 *   BK_OPT_SLAB_LAG: persistent engine, slabs between A1 and S2 of a slab (>= 1);
 *   BK_OPT_SPLIT_W2: qubits of the S2 pass (1..9; the rest go to S3, at most 9),
 *       0 = the engine's default split; a width that does not fit a size is ignored;
 *   BK_OPT_E_SOURCE: where the diagonal phase and P_< get E(s): 0 = the cached
 *       uint16 table (read with the A1 tile), 1 = recomputed in the pass from the
 *       popcount form C_k = (n-k) - 2 popcount((x ^ (x >> k)) & (2^(n-k) - 1));
 *   BK_OPT_A1_WIDE: per-pass schedule (mode 1), the A1 kernel: 0 = 256 threads x
 *       16 elements over element bits 0-11, 1 = 512 threads x 8 elements (more
 *       warps per SM for the diagonal phase), 2 = warp-local: the A1 pass covers
 *       element bits 0-8, one warp per 512-element block with no CTA barrier,
 *       and the strided passes take bits 9 and up (sizes up to 27 element bits;
 *       larger sizes run value 0), 3 = the same warp-local A1 with 4-warp CTAs
 *       over half tiles (2048 elements, 32 KB; four CTAs per SM);
 *   BK_OPT_ADJ_A1: bk_adjoint's reverse sweep, 1 = the warp-local A1 layout for
 *       both statevectors (element bits 0-8, strided passes from bit 9; up to 27
 *       element bits), 0 (default) = the 12-bit A1 of the forward geometry;
 *   BK_OPT_WAIT_POLLS: persistent engine, polls of one dependency wait before
 *       it gives up with BK_ERR_TIMEOUT (1000 .. 2^24; 0 = the default 2^24);
 *   BK_OPT_TEST_HOLD_STEP: failure-path test hook, off (-1) by default: in the
 *       persistent engine (BK_OPT_ENGINE_MODE 0), the A1 tasks of this step of a
 *       launch wait for one completion more than can arrive, as if a producer
 *       were lost; the bounded wait runs out, every CTA leaves, and bk_evolve
 *       returns BK_ERR_TIMEOUT with the context still usable;
 *   BK_OPT_PHASE_TABLE: complex64, per-pass schedules (modes 1 and 2), every
 *       A1 kernel: 1 = the diagonal phase of every energy level from one
 *       table entry (E = floor(n/2) mod 4 for every LABS energy, so at most 2139
 *       levels, 17 KB) applied as two half-angle shear rotations; 0 (default) =
 *       a 16-entry level table and residual polynomials. bk_adjoint's complex64
 *       reverse A1 pass takes it too (D^dagger as the negated rotations); other
 *       kernels and complex128 ignore it. */
enum {
  BK_OPT_ENGINE_MODE = 0,
  BK_OPT_SLAB_LAG = 1,
  BK_OPT_SPLIT_W2 = 2,
  BK_OPT_E_SOURCE = 3,
  BK_OPT_A1_WIDE = 4,
  BK_OPT_ADJ_A1 = 5,
  BK_OPT_WAIT_POLLS = 6,
  BK_OPT_TEST_HOLD_STEP = 7,
  BK_OPT_PHASE_TABLE = 8
};
int bk_set_option(bk_ctx* ctx, int option, int64_t value);
int bk_get_option(const bk_ctx* ctx, int option, int64_t* value);

/* ---- Adjoint gradient of a piecewise-constant field schedule ----
 *
 * No counterpart in the reference (whose field is constant in time); the step
 * is the reference's psi_{k+1} = M(g_k) D psi_k (sampler.cuh:604-618) with the
 * field g_k = g[segment_of_step[k]]. Computes O(T) = <psi_T| W |psi_T> for a
 * diagonal W (BK_OBJ_P_LESS: [E(s) < e0], the reference's P_< of
 * sampler.cuh:149-195; BK_OBJ_D_H: popcount(s ^ s0), its <d_H>) and dO/dg_j for
 * every segment by one forward run and one reverse sweep of the adjoint state
 * lambda_k = (M D)^dagger lambda_{k+1} together with psi_k rebuilt by inverse
 * steps (no stored trajectory); psi is reset from a checkpoint every
 * checkpoint_every steps to bound the drift of the inverse steps. */
enum { BK_OBJ_P_LESS = 0, BK_OBJ_D_H = 1 };

typedef struct bk_adjoint_params {
  int32_t n;                      /* qubits: 14..30 (complex64) or 13..30 (complex128) */
  int32_t precision;              /* bk_precision */
  uint64_t s0;                    /* trap bits (initial state |s0>) */
  int64_t e0;                     /* P_< threshold; < 0 means E(s0) */
  double dt;
  double diag_scale;              /* <= 0: 1/n */
  int32_t n_steps;
  int32_t n_segments;
  const double* g;                /* [n_segments] field of each segment */
  const int32_t* segment_of_step; /* [n_steps] segment of each step, or NULL: equal consecutive
                                     segments (n_steps a multiple of n_segments) */
  int32_t checkpoint_every;       /* K; <= 0: 128, enlarged until the checkpoints fit in free memory */
  int32_t objective;              /* BK_OBJ_P_LESS or BK_OBJ_D_H */
} bk_adjoint_params;

typedef struct bk_adjoint_stats {
  double value;                   /* O(T) */
  double norm;                    /* |psi_T|^2 */
  int32_t checkpoint_every;       /* K used */
  int32_t n_checkpoints;
  double max_drift;               /* max over checkpoints of |psi_rebuilt - psi_k| (2-norm) */
  double forward_ms;              /* device time of the forward run (with checkpoint copies) */
  double reverse_ms;              /* device time of the reverse sweep */
} bk_adjoint_stats;

/* grad_out[n_segments] = dO/dg_j; grad_steps_out (NULL or [n_steps]) = dO/dg_k per
 * step; value_out and stats may be NULL. */
int bk_adjoint(bk_ctx* ctx, const bk_adjoint_params* p, double* value_out, double* grad_out,
               double* grad_steps_out, bk_adjoint_stats* stats);

/* ---- Projective sampling (sampler.cuh:459-487, 559-598) ---- */

/* Samples `shots` basis states from |psi|^2 of the state left by the last
 * bk_evolve: inverse CDF (FP64 prefix sums), results in random-number order. */
int bk_sample(bk_ctx* ctx, const double* randnums, int64_t shots, uint64_t* out_states);

/* ---- Measurement without device allocation ----
 *
 * No counterpart in the reference. For callers that cannot let a library
 * allocate device memory — a host framework that owns all GPU memory through
 * its own allocator or fixed arena, or a latency-critical loop that must not
 * synchronise on an allocation: measures a caller-owned statevector and writes
 * d_out[0] = P_< (sum of |psi_s|^2 over E(s) < e0; e0 < 0 means E(s0)),
 * d_out[1] = <d_H> (weights popcount(s ^ s0)), d_out[2] = |psi|^2, all FP64.
 *   d_state: device, 2^n amplitudes, interleaved (re, im), float (BK_C64) or
 *            double (BK_C128), natural index order; d_out: device, 3 doubles;
 *   stream:  a cudaStream_t (NULL = the legacy default stream); the call only
 *            enqueues work (read d_out after synchronising that stream).
 * Allocates nothing: its scratch is a fixed 24.25 KiB array inside the library
 * (1024 block partial sums and a ticket), which every GPU that loads the
 * library holds until the process exits. Limit: 1 <= n <= 30, else
 * BK_ERR_TOO_LARGE; d_state must be aligned to its amplitude type (8 bytes for
 * complex64, 16 for complex128) and d_out to 8 bytes, else BK_ERR_INVALID. The
 * first call on a device resolves the array's device address, and so does the
 * first call after the device's context was replaced (cudaDeviceReset); make
 * that first call before any stream capture. All calls share the array (it
 * keeps the last call's contents; the ticket is cleared at the start of every
 * call), so calls that overlap on the GPU race: serialise them. */
int bk_measure_noalloc(int n, int precision, const void* d_state, int64_t e0, uint64_t s0, double* d_out,
                       void* stream);

/* ---- full-space Hamiltonian (H = diag(scale E(s)) - g sum_j X_j, all 2^n states, FP64) ----
 *
 * bk_fullspace_matvec: y = H x for device vectors of 2^n doubles (replaces the
 * reference's fullspace_matvec_kernel_d, src/subspace/diagonalizer.cuh:60-77, with
 * diag = scale * E(s) as in :388-392). x and y are 16-byte aligned device pointers on
 * the context's device and must not alias; the call runs on the context's stream and returns
 * after it has finished (the caller's own work on x must be complete before).
 * method: BK_FUSED = tile passes over 64 KB shared-memory tiles (x read once per
 * pass), BK_PLAIN = the reference's one-thread-per-state form (comparison).
 *
 * bk_fullspace_lanczos: the reference's Diagonalizer::solve_fullspace_lanczos
 * (diagonalizer.cuh:377-416 with run_gpu_lanczos_internal :418-560): plain Lanczos
 * from the start vector mt19937_64(42) / uniform(-0.5, 0.5), m = min(2^n,
 * max_krylov_dim) steps, stopping when beta < tolerance; the lowest
 * num_eigenpairs Ritz values in energies (NaN beyond the Krylov dimension) and,
 * when vectors != NULL, their Ritz vectors ([num_eigenpairs][2^n] doubles, host;
 * rows beyond the Krylov dimension are left as the caller allocated them).
 * alphas / betas (optional, host, max_krylov_dim entries) receive the tridiagonal
 * matrix. Needs (m + 1) 2^n doubles of device memory (BK_ERR_UNSUPPORTED if not free). */
typedef struct bk_lanczos_params {
  int n;
  double g;
  int num_eigenpairs;  /* reference default 1 */
  int max_krylov_dim;  /* reference default 100 */
  double tolerance;    /* reference default 1e-12 */
  int normalize_by_n;  /* reference default 1: diagonal E / n */
  double* alphas;      /* optional out [max_krylov_dim] */
  double* betas;       /* optional out [max_krylov_dim] */
} bk_lanczos_params;
typedef struct bk_lanczos_stats {
  int krylov_dim;      /* steps taken (m_actual) */
  int matvecs;
  double seconds;      /* wall time of the run, start vector included */
} bk_lanczos_stats;
int bk_fullspace_matvec(bk_ctx* ctx, int n, double g, double scale, const double* d_x, double* d_y, int method);
int bk_fullspace_lanczos(bk_ctx* ctx, const bk_lanczos_params* params, double* energies, double* vectors,
                         bk_lanczos_stats* stats);

#ifdef __cplusplus
}
#endif
#endif /* BK_ENGINE_H */
