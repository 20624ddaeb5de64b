// Host side of the B200 statevector engine: the C ABI declared in
// include/bk_engine.h. One bk_ctx = one device, one stream and cached device
// buffers. Replaces the device part of CuStateVecSampler
// (src/sampling/sampler.cuh:318-707 of the reference).
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <utility>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <limits>
#include <map>
#include <random>
#include <string>
#include <unordered_set>
#include <unordered_map>
#include <vector>

#include "bk_adjoint.cuh"
#include "bk_aux.cuh"
#include "bk_engine.h"
#include "bk_fused.cuh"
#include "bk_lanczos.cuh"
#include "bk_persist.cuh"
#include "bk_s23.cuh"

using namespace bk;

namespace {

constexpr int kMaxN = 30;
constexpr int kMeasureGrid = 148 * 8;
// The omitted cos(g dt)^n factors are tracked as log2 on the host; once the
// computed amplitudes have grown by 2^kRescaleLog2 an exact 2^-kRescaleLog2 is
// folded into the next diagonal phase.
constexpr int kRescaleLog2 = 32;

struct TmaDesc {
  CUtensorMap map;
  int mid_dim = -1, hi_dim = -1;
  uint32_t mid_bits = 0;
};

struct TimingRec {
  std::string name;
  int64_t launches = 0;
  double total_ms = 0.0;
};

}  // namespace

struct bk_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string last_error;
  // E table cache (per n), like the reference's ensure_cached_energies
  int e_n = -1;
  uint16_t* d_E = nullptr;
  // statevector
  int st_n = -1, st_prec = -1;
  void* d_state = nullptr;
  size_t state_bytes = 0;
  // scratch
  double* d_partials = nullptr;
  size_t partials_cap = 0;  // doubles
  double* d_results = nullptr;
  size_t results_cap = 0;   // rows of 4 doubles
  unsigned int* d_ticket = nullptr;
  int* d_err = nullptr;
  unsigned long long* d_count = nullptr;
  void* d_phase = nullptr;  // hi table then lo table
  size_t phase_cap = 0;
  void* d_small = nullptr;  // per-step arrays of the whole-state kernel
  size_t small_cap = 0;
  double* d_chunks = nullptr;
  size_t chunks_cap = 0;
  void* d_io = nullptr;
  size_t io_cap = 0;
  double* d_rand = nullptr;  // in-run sampling: uniforms and drawn states
  size_t rand_cap = 0;
  unsigned long long* d_samples = nullptr;
  size_t samples_cap = 0;
  unsigned long long* d_binom = nullptr;
  int* d_found = nullptr;
  void* d_persist = nullptr;  // persistent engine: maps, descriptors, tasks, per-step arrays, counters
  size_t persist_cap = 0;
  int num_sms = 148;
  bool planar = false;        // complex64 state stored pair-planar (persistent engine)
  int slab_lag = 3;           // persistent engine: S2 queue lag behind A1, in slabs
  int engine_mode = 0;        // 0 persistent dataflow, 1 one launch per pass (tile grid)
  int force_w2 = 0;           // S2 width when > 0 and valid for the size (else the default split)
  int e_recompute = 0;        // tile engine: 1 = E(s) recomputed from popcounts in A1, 0 = uint16 table
  int a1_wide = 0;            // per-pass schedule A1: 1 = 512 threads x 8 elements, 2 = warp-local (bits 0-8)
  int phase_table = 0;        // complex64 per-pass A1 (kernels 1-3): 1 = the full per-energy phase table
  int adj_a1 = 0;             // adjoint reverse sweep A1: 0 = 12-bit, 1 = warp-local (element bits 0-8)
  uint32_t wait_polls = 0;    // persistent engine: polls of a dependency wait before it gives up (0 = default)
  uint64_t s23_checked = 0;   // fused strided pass geometry (np, a1, w2, lag) whose closed form was checked
  int64_t hold_step = -1;     // test hook: launch step whose dependency can never be met (-1 = off)
  std::map<int, uint16_t*> batch_E;  // E tables of batched runs, per n
  void* d_batch_state = nullptr;
  size_t batch_state_cap = 0;
  void* d_batch = nullptr;    // batched run: maps, descriptors, tasks, tables, counters, partials
  size_t batch_cap = 0;
  double* d_batch_results = nullptr;
  size_t batch_results_cap = 0;
  void* d_lam = nullptr;      // adjoint: lambda statevector
  size_t lam_cap = 0;
  void* d_ckpt = nullptr;     // adjoint: checkpoints of psi
  size_t ckpt_cap = 0;
  void* d_adj = nullptr;      // adjoint: maps, descriptor, per-step arrays, partials
  size_t adj_cap = 0;
  void* d_fsmap = nullptr;    // full-space strided pass: the tensor map of x (device memory, 64-byte aligned)
  size_t fsmap_cap = 0;
  void* d_descent = nullptr;  // batched steepest descent: starts, final states, energies, evaluations
  size_t descent_cap = 0;
  void* d_lz = nullptr;       // full-space Lanczos: Krylov basis, work vector, partial sums, alpha / beta
  size_t lz_cap = 0;
  // last evolution (for export / sampling)
  bool have_state = false;
  bool last_planar = false;
  int last_n = 0, last_prec = 0, last_ordering = 0;
  long double last_log2_scale = 0.0L;
  double last_angle_unit = 0.0;
  // kernel timing
  bool timing = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pool;
  size_t ev_used = 0;
  std::vector<std::pair<int, size_t>> ev_marks;  // (timing index, event pair)
  std::vector<TimingRec> timings;
  std::map<std::string, int> timing_index;
  std::map<const void*, int> smem_configured;  // kernel -> dynamic smem bytes set
};

namespace {

int fail(bk_ctx* c, int code, const char* fmt, ...) {
  if (c) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    c->last_error = buf;
  }
  return code;
}

#define BK_CUDA(ctx, call)                                                                          \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess)                                                                          \
      return fail((ctx), e_ == cudaErrorMemoryAllocation ? BK_ERR_OOM : BK_ERR_CUDA, "%s: %s (%s:%d)", \
                  #call, cudaGetErrorString(e_), __FILE__, __LINE__);                               \
  } while (0)

#define BK_TRY(expr)          \
  do {                        \
    int r_ = (expr);          \
    if (r_ != BK_OK) return r_; \
  } while (0)

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// Opt a kernel into more than 48 KB of dynamic shared memory (once per context).
int allow_smem(bk_ctx* c, const void* fn, int bytes) {
  auto it = c->smem_configured.find(fn);
  if (it != c->smem_configured.end() && it->second >= bytes) return BK_OK;
  BK_CUDA(c, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  c->smem_configured[fn] = bytes;
  return BK_OK;
}

int ensure_buffer(bk_ctx* c, void** ptr, size_t* cap, size_t bytes) {
  if (*cap >= bytes && *ptr) return BK_OK;
  if (*ptr) cudaFree(*ptr);
  *ptr = nullptr;
  *cap = 0;
  BK_CUDA(c, cudaMalloc(ptr, bytes));
  *cap = bytes;
  return BK_OK;
}

// ---- kernel timing ----
int timing_slot(bk_ctx* c, const std::string& name) {
  auto it = c->timing_index.find(name);
  if (it != c->timing_index.end()) return it->second;
  c->timings.push_back({name, 0, 0.0});
  c->timing_index[name] = (int)c->timings.size() - 1;
  return (int)c->timings.size() - 1;
}
int ev_begin(bk_ctx* c, const char* name, size_t* pair) {
  if (!c->timing) return BK_OK;
  if (c->ev_used == c->ev_pool.size()) {
    cudaEvent_t a, b;
    BK_CUDA(c, cudaEventCreate(&a));
    BK_CUDA(c, cudaEventCreate(&b));
    c->ev_pool.push_back({a, b});
  }
  *pair = c->ev_used++;
  c->ev_marks.push_back({timing_slot(c, name), *pair});
  BK_CUDA(c, cudaEventRecord(c->ev_pool[*pair].first, c->stream));
  return BK_OK;
}
int ev_end(bk_ctx* c, size_t pair) {
  if (!c->timing) return BK_OK;
  BK_CUDA(c, cudaEventRecord(c->ev_pool[pair].second, c->stream));
  return BK_OK;
}
int collect_timing(bk_ctx* c) {
  if (!c->timing) return BK_OK;
  for (auto& m : c->ev_marks) {
    float ms = 0;
    BK_CUDA(c, cudaEventElapsedTime(&ms, c->ev_pool[m.second].first, c->ev_pool[m.second].second));
    c->timings[(size_t)m.first].launches += 1;
    c->timings[(size_t)m.first].total_ms += ms;
  }
  c->ev_marks.clear();
  c->ev_used = 0;
  return BK_OK;
}

// ---- geometry ----
constexpr int tile_bits(int prec) { return prec == BK_C64 ? 13 : 12; }
constexpr size_t amp_bytes(int prec) { return prec == BK_C64 ? 8 : 16; }

// Tensor map over the statevector for tiles = amp bits [0, cp) u [h0, h0 + w),
// with 8-byte elements (complex128 amps are two elements).
int build_amp_map(bk_ctx* c, void* base, int n, int prec, int cp, int h0, int w, TmaDesc* out) {
  auto enc = encode_fn();
  if (!enc) return fail(c, BK_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable from the driver");
  const uint64_t epa = amp_bytes(prec) / 8;
  const uint64_t S = amp_bytes(prec);
  std::vector<uint64_t> dims, strides, boxes;  // strides in bytes (dims[0] stride implicit)
  auto push = [&](uint64_t size, uint64_t stride, uint64_t box) {
    dims.push_back(size);
    strides.push_back(stride);
    boxes.push_back(box);
  };
  // contiguous low part, in elements
  const uint64_t in_el = (1ull << cp) * epa;
  if (in_el <= 256) {
    push(in_el, 8, in_el);
  } else {
    push(256, 8, 256);
    push(in_el / 256, 256 * 8, in_el / 256);
  }
  out->mid_dim = -1;
  out->hi_dim = -1;
  out->mid_bits = (uint32_t)(h0 - cp);
  if (w > 0 && h0 > cp) {
    out->mid_dim = (int)dims.size();
    push(1ull << (h0 - cp), (1ull << cp) * S, 1);
  }
  if (w > 0) {
    const uint64_t act = 1ull << w;
    if (act <= 256) {
      push(act, (1ull << h0) * S, act);
    } else {
      push(256, (1ull << h0) * S, 256);
      push(act / 256, (1ull << (h0 + 8)) * S, act / 256);
    }
  }
  const int top = (w > 0) ? h0 + w : cp;
  if (n > top) {
    out->hi_dim = (int)dims.size();
    push(1ull << (n - top), (1ull << top) * S, 1);
  }
  if (dims.size() > 5) return fail(c, BK_ERR_UNSUPPORTED, "tile geometry needs %zu TMA dims", dims.size());
  const uint64_t total_bytes = (1ull << n) * S;
  while (dims.size() < 5) push(1, total_bytes, 1);
  cuuint64_t gdim[5], gstride[4];
  cuuint32_t box[5], estr[5];
  for (int i = 0; i < 5; ++i) {
    gdim[i] = dims[(size_t)i];
    box[i] = (cuuint32_t)boxes[(size_t)i];
    estr[i] = 1;
    if (i > 0) gstride[i - 1] = strides[(size_t)i];
  }
  CUresult r = enc(&out->map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 5, base, gdim, gstride, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(c, BK_ERR_CUDA, "cuTensorMapEncodeTiled(amp) failed: %d", (int)r);
  return BK_OK;
}

// A1 tiles (4096 16-byte elements, element bits [0, 12)) as 128-byte rows with the
// 128-byte TMA swizzle, for the warp-local A1: dims (16, 256, 2, tiles) of
// 8-byte units, box (16, 256, 2, 1); the tile index is coordinate 3. half: box
// (16, 256, 1, 1), one 2048-element half tile per load (coordinates 2 and 3).
int build_a1_swizzled_map(bk_ctx* c, void* base, int np, TmaDesc* out, bool half = false) {
  auto enc = encode_fn();
  if (!enc) return fail(c, BK_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable from the driver");
  const uint64_t total = (1ull << np) * 16;
  cuuint64_t gdim[5] = {16, 256, 2, 1ull << (np - kElemBits), 1};
  cuuint64_t gstride[4] = {128, 32768, 65536, total};
  cuuint32_t box[5] = {16, 256, half ? 1u : 2u, 1, 1};
  cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  CUresult r = enc(&out->map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 5, base, gdim, gstride, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(c, BK_ERR_CUDA, "cuTensorMapEncodeTiled(A1, swizzled) failed: %d", (int)r);
  out->mid_dim = -1;
  out->hi_dim = 3;
  out->mid_bits = 0;
  return BK_OK;
}

int build_e_map(bk_ctx* c, const uint16_t* E, int n, int T, TmaDesc* out) {
  auto enc = encode_fn();
  if (!enc) return fail(c, BK_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable from the driver");
  cuuint64_t gdim[5] = {256, 1ull << (T - 8), 1ull << (n - T), 1, 1};
  const uint64_t total = (1ull << n) * 2;
  cuuint64_t gstride[4] = {512, (1ull << T) * 2, total, total};
  cuuint32_t box[5] = {256, (cuuint32_t)(1u << (T - 8)), 1, 1, 1};
  cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  CUresult r = enc(&out->map, CU_TENSOR_MAP_DATA_TYPE_UINT16, 5, const_cast<uint16_t*>(E), gdim, gstride, box,
                   estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(c, BK_ERR_CUDA, "cuTensorMapEncodeTiled(E) failed: %d", (int)r);
  return BK_OK;
}

int ensure_energy(bk_ctx* c, int n) {
  if (c->e_n == n && c->d_E) return BK_OK;
  if (c->d_E) cudaFree(c->d_E);
  c->d_E = nullptr;
  c->e_n = -1;
  const size_t count = 1ull << n;
  BK_CUDA(c, cudaMalloc(&c->d_E, std::max<size_t>(count, 8) * sizeof(uint16_t)));
  const uint32_t threads = 256, per = (uint32_t)((count + 7) / 8);
  energy_table_kernel<<<(per + threads - 1) / threads, threads, 0, c->stream>>>(c->d_E, n, (uint32_t)count);
  BK_CUDA(c, cudaGetLastError());
  c->e_n = n;
  return BK_OK;
}

int ensure_state(bk_ctx* c, int n, int prec) {
  const size_t bytes = (1ull << n) * amp_bytes(prec);
  if (c->d_state && c->state_bytes >= bytes && c->st_n == n && c->st_prec == prec) return BK_OK;
  if (c->d_state) cudaFree(c->d_state);
  c->d_state = nullptr;
  c->state_bytes = 0;
  BK_CUDA(c, cudaMalloc(&c->d_state, bytes));
  c->state_bytes = bytes;
  c->st_n = n;
  c->st_prec = prec;
  return BK_OK;
}

// Host side of the diagonal phase exp(-i angle_unit E).
// complex64: E = h K + l; n_h table entries (the fewest in 16, 32, ..., 256 with
// angle_unit (K - 1) <= 1/2 so the residual polynomials stay accurate);
// h = umulhi(E, M) checked exact for every E <= Emax.
int build_phase(bk_ctx* c, int n, double angle_unit, Phase32* P) {
  const int emax = (n - 1) * n * (2 * n - 1) / 6;
  int n_h = 16;
  uint32_t K = 0;
  for (;; n_h *= 2) {
    if (n_h > kPhaseH)
      return fail(c, BK_ERR_UNSUPPORTED, "phase angle per unit energy %g too large for the table", angle_unit);
    K = std::max<uint32_t>(2u, (uint32_t)((emax + n_h) / n_h));  // ceil((emax + 1) / n_h), >= 2 so M fits 32 bits
    if (std::fabs(angle_unit) * (double)(K - 1) <= 0.5) break;
  }
  const uint32_t M = (uint32_t)((((uint64_t)1 << 32) + K - 1) / K);
  for (uint64_t e = 0; e <= (uint64_t)emax; ++e)
    if (((e * M) >> 32) != e / K) return fail(c, BK_ERR_UNSUPPORTED, "no exact level split for n = %d", n);
  std::vector<float2> hab((size_t)n_h);
  std::vector<int> hq((size_t)n_h);
  const double half_pi = 1.5707963267948966;
  for (int h = 0; h < n_h; ++h) {
    const double th = -angle_unit * (double)h * (double)K;
    const double q = std::nearbyint(th / half_pi);
    const double r = th - q * half_pi;  // |r| <= pi/4
    hab[(size_t)h] = make_float2((float)(-std::tan(0.5 * r)), (float)std::sin(r));
    hq[(size_t)h] = (int)(((long long)std::fmod(q, 4.0) + 4) % 4);
  }
  const size_t b1 = hab.size() * sizeof(float2), b2 = hq.size() * sizeof(int);
  BK_TRY(ensure_buffer(c, &c->d_phase, &c->phase_cap, b1 + b2));
  BK_CUDA(c, cudaMemcpyAsync(c->d_phase, hab.data(), b1, cudaMemcpyHostToDevice, c->stream));
  BK_CUDA(c, cudaMemcpyAsync(static_cast<char*>(c->d_phase) + b1, hq.data(), b2, cudaMemcpyHostToDevice, c->stream));
  BK_CUDA(c, cudaStreamSynchronize(c->stream));  // host vectors die at return
  P->hab = reinterpret_cast<const float2*>(c->d_phase);
  P->hq = reinterpret_cast<const int*>(static_cast<char*>(c->d_phase) + b1);
  P->K = K;
  P->M = M;
  P->theta = (float)(-angle_unit);
  P->theta_lo = (float)(-angle_unit - (double)P->theta);
  P->n_h = n_h;
  return BK_OK;
}
// complex128: E = 128 h + l, FP64 (cos, sin) tables.
int build_phase(bk_ctx* c, int n, double angle_unit, Phase64* P) {
  const int emax = (n - 1) * n * (2 * n - 1) / 6;
  const int n_hi = (emax >> kPhaseLoBits) + 1;
  if (n_hi > kPhaseHi64) return fail(c, BK_ERR_UNSUPPORTED, "n = %d exceeds the phase table", n);
  std::vector<double2> t((size_t)n_hi + kPhaseLo);
  for (int h = 0; h < n_hi; ++h) {
    const double th = -angle_unit * (double)(h << kPhaseLoBits);
    t[(size_t)h] = make_double2(std::cos(th), std::sin(th));
  }
  for (int l = 0; l < kPhaseLo; ++l) {
    const double th = -angle_unit * (double)l;
    t[(size_t)n_hi + l] = make_double2(std::cos(th), std::sin(th));
  }
  BK_TRY(ensure_buffer(c, &c->d_phase, &c->phase_cap, t.size() * sizeof(double2)));
  BK_CUDA(c, cudaMemcpyAsync(c->d_phase, t.data(), t.size() * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
  BK_CUDA(c, cudaStreamSynchronize(c->stream));
  P->hi = reinterpret_cast<const double2*>(c->d_phase);
  P->lo = P->hi + n_hi;
  P->n_hi = n_hi;
  return BK_OK;
}

bool is_finite(double x) { return std::isfinite(x); }

// ---- trap generation (host) ----
static int64_t host_energy(int n, uint64_t x) {
  int64_t e = 0;
  for (int k = 1; k < n; ++k) {
    const int64_t ck = (int64_t)(n - k) - 2 * (int64_t)__builtin_popcountll((x ^ (x >> k)) & ((1ull << (n - k)) - 1ull));
    e += ck * ck;
  }
  return e;
}

// Canonical representative of the LABS symmetry orbit of s (reference:
// SpinState::canonical, labs_energy.hpp:40-106): the smallest of s, its
// alternating-sign image, their bit reversals, and the complements of all four.
static uint64_t host_canonical(int n, uint64_t s) {
  const uint64_t m = (1ull << n) - 1ull;
  const uint64_t alt = 0x5555555555555555ull & m;
  auto rev = [n](uint64_t x) {
    uint64_t r = 0;
    for (int i = 0; i < n; ++i) r |= ((x >> i) & 1ull) << (n - 1 - i);
    return r;
  };
  const uint64_t a = s & m, b = a ^ alt;
  const uint64_t cand[4] = {a, b, rev(a), rev(b)};
  uint64_t best = ~0ull;
  for (uint64_t c : cand) best = std::min(best, std::min(c, (~c) & m));
  return best;
}

// Optimal LABS energies E*(n) for n <= 32 (reference: labs_energy.hpp:156-168).
static int64_t optimal_energy(int n) {
  static const int64_t t[33] = {-1, -1, -1, 1, 2, 2, 7, 3, 8, 12, 13, 5, 10, 6, 19, 15, 24,
                                32, 25, 29, 26, 26, 39, 47, 36, 36, 45, 37, 50, 62, 59, 67, 64};
  return (n >= 0 && n <= 32) ? t[n] : -1;
}

// One descent with incremental C_k (reference: classical.cuh:625-712). Each
// sweep costs n evaluations; a flip is taken only when strictly better, the
// lowest bit index winning ties.
static void descend(int n, uint64_t start, uint64_t max_evals, uint64_t* fs, int64_t* fe, uint64_t* ev) {
  const uint64_t budget = max_evals == 0 ? ~0ull : max_evals;
  uint64_t x = start;
  int64_t C[64];
  int64_t e = 0;
  for (int k = 1; k < n; ++k) {
    C[k] = (int64_t)(n - k) - 2 * (int64_t)__builtin_popcountll((x ^ (x >> k)) & ((1ull << (n - k)) - 1ull));
    e += C[k] * C[k];
  }
  uint64_t evals = 1;
  while (evals + (uint64_t)n <= budget) {
    int best = -1;
    int64_t best_e = e;
    for (int p = 0; p < n; ++p) {
      const int sp = ((x >> p) & 1ull) ? -1 : 1;
      int64_t ne = 0;
      for (int k = 1; k < n; ++k) {
        int64_t d = 0;
        if (p + k < n) d -= 2 * sp * (((x >> (p + k)) & 1ull) ? -1 : 1);
        if (p - k >= 0) d -= 2 * sp * (((x >> (p - k)) & 1ull) ? -1 : 1);
        ne += (C[k] + d) * (C[k] + d);
      }
      if (ne < best_e) {
        best_e = ne;
        best = p;
      }
    }
    evals += (uint64_t)n;
    if (best < 0) break;
    const int sp = ((x >> best) & 1ull) ? -1 : 1;
    for (int k = 1; k < n; ++k) {
      if (best + k < n) C[k] -= 2 * sp * (((x >> (best + k)) & 1ull) ? -1 : 1);
      if (best - k >= 0) C[k] -= 2 * sp * (((x >> (best - k)) & 1ull) ? -1 : 1);
    }
    x ^= 1ull << best;
    e = best_e;
  }
  *fs = x;
  *fe = e;
  if (ev) *ev = evals;
}

struct Schedule {
  std::vector<double> g;        // per step
  std::vector<int> slot;        // per step (n_steps + 1): measurement row or -1
  int n_meas = 0;
  std::vector<int> sample_pt;   // per step (n_steps + 1): sampling point index or -1
  int n_pts = 0;
  int shots = 0;
};

// Projective sampling of the current state at sampling point `pt`: chunk sums
// of |psi|^2, exclusive scan, one warp per draw.
template <class A>
int launch_sampling_t(bk_ctx* c, const A* psi, int n, int pt, int shots) {
  const uint32_t count = 1u << n;
  const uint32_t m = (count + (1u << kSampleChunkBits) - 1) >> kSampleChunkBits;
  BK_TRY(ensure_buffer(c, reinterpret_cast<void**>(&c->d_chunks), &c->chunks_cap, (m + 1) * sizeof(double)));
  size_t ev = 0;
  BK_TRY(ev_begin(c, "sample", &ev));
  chunk_sums_kernel<A><<<m, 256, 0, c->stream>>>(psi, count, c->d_chunks);
  scan_chunks_kernel<<<1, 1024, 0, c->stream>>>(c->d_chunks, m);
  const unsigned blocks = (unsigned)(((size_t)shots * 32 + 255) / 256);
  sample_kernel<A><<<blocks, 256, 0, c->stream>>>(psi, count, c->d_chunks, m, c->d_rand + (size_t)pt * shots,
                                                  shots, c->d_samples + (size_t)pt * shots);
  BK_CUDA(c, cudaGetLastError());
  return ev_end(c, ev);
}
template <class A>
int launch_sampling(bk_ctx* c, const A* psi, int n, int pt, int shots) {
  if (c->planar) return launch_sampling_t(c, reinterpret_cast<const Planar64*>(psi), n, pt, shots);
  return launch_sampling_t(c, psi, n, pt, shots);
}

// ---------------------------------------------------------------------------
// persistent dataflow engine (csrc/bk_persist.cuh)
// ---------------------------------------------------------------------------
// complex64 level table for the vectorised phase: hab[h] = {-tan(th/4), sin(th/2)}
// for th = -angle_unit h K reduced to (-pi, pi], applied twice.
int build_phase_v(bk_ctx* c, int n, double angle_unit, PhaseV32* P, std::vector<float2>* hab) {
  const int emax = (n - 1) * n * (2 * n - 1) / 6;
  int n_h = 16;
  uint32_t K = 0;
  for (;; n_h *= 2) {
    if (n_h > kPhaseH)
      return fail(c, BK_ERR_UNSUPPORTED, "phase angle per unit energy %g too large for the table", angle_unit);
    K = std::max<uint32_t>(2u, (uint32_t)((emax + n_h) / n_h));
    if (std::fabs(angle_unit) * (double)(K - 1) <= 0.5) break;
  }
  const uint32_t M = (uint32_t)((((uint64_t)1 << 32) + K - 1) / K);
  for (uint64_t e = 0; e <= (uint64_t)emax; ++e)
    if (((e * M) >> 32) != e / K) return fail(c, BK_ERR_UNSUPPORTED, "no exact level split for n = %d", n);
  hab->resize((size_t)n_h);
  const double two_pi = 6.283185307179586;
  for (int h = 0; h < n_h; ++h) {
    double th = std::remainder(-angle_unit * (double)h * (double)K, two_pi);  // [-pi, pi]
    (*hab)[(size_t)h] = make_float2((float)(-std::tan(0.25 * th)), (float)std::sin(0.5 * th));
  }
  P->K = K;
  P->M = M;
  P->theta = (float)(-angle_unit);
  P->theta_lo = (float)(-angle_unit - (double)P->theta);
  P->n_h = n_h;
  return BK_OK;
}

// complex64 full phase table of the looping A1: every LABS energy is
// E = c0 + 4 j with c0 = floor(n/2) mod 4 (C_k has the parity of n - k, and an
// odd square is 1 mod 8, an even one 0 mod 4), so j < (Emax - c0) / 4 + 1 indexes
// every level; tab[j] = {-tan(r/4), sin(r/2)} for r = -angle_unit E reduced to
// (-pi, pi], applied as two half-angle shear rotations.
int build_phase_table(bk_ctx* c, int n, double angle_unit, PhaseV32* P, std::vector<float2>* tab) {
  const int emax = (n - 1) * n * (2 * n - 1) / 6;
  const int c0 = (n / 2) & 3;
  const int n_j = (emax - c0) / 4 + 1;
  if (n_j > kPhaseTabMax) return fail(c, BK_ERR_UNSUPPORTED, "phase table of %d entries for n = %d", n_j, n);
  tab->assign((size_t)((n_j + 1) & ~1), make_float2(0.f, 0.f));  // even count: the copy is a 16-byte multiple
  const double two_pi = 6.283185307179586;
  for (int j = 0; j < n_j; ++j) {
    const double r = std::remainder(-angle_unit * (double)(c0 + 4 * j), two_pi);  // [-pi, pi]
    (*tab)[(size_t)j] = make_float2((float)(-std::tan(0.25 * r)), (float)std::sin(0.5 * r));
  }
  P->c0 = c0;
  P->n_j = n_j;
  return BK_OK;
}

// bump allocator over the context's persistent-engine buffer (256-byte aligned pieces)
struct Bump {
  size_t off = 0;
  size_t take(size_t bytes) {
    const size_t o = off;
    off += (bytes + 255) & ~(size_t)255;
    return o;
  }
};

// A prepared persistent-engine run over c->d_state: device buffers laid out,
// tasks and per-step arrays uploaded; persist_launch runs any range of steps.
template <class R>
struct PersistRun {
  char* base = nullptr;
  size_t o_desc = 0, o_tasks = 0, o_final = 0, o_tan = 0, o_scale = 0, o_slot = 0;
  InstDesc<R> D{};
  unsigned int* ctr = nullptr;
  uint32_t slabs = 0;
  size_t n_tasks = 0, n_final = 0;
  unsigned int* next = nullptr;
  int* err = nullptr;
  int* abort_w = nullptr;
  uint32_t n_a1 = 0, n_s2 = 0, n_s3 = 0;
  typename PhaseV<R>::params phase{};  // device tables of the diagonal phase
  // fused strided pass (engine mode 2): S2 / S3 tasks in slab order, counters
  size_t n_tasks23 = 0;
  uint32_t slabs23 = 0;
  S23Program prog23{};            // the task order's closed form (counters set at launch)
  unsigned int* ctr23 = nullptr;  // [slab_done: slabs23][next][ctas_done][abort]
  bool a1_table = false;          // the A1 pass takes its phase from the full table (complex64)
};

// Slab of a strided tile for the fused S2 + S3 pass: the element bits
// [cpm, a1) (cpm = max(12 - w2, 12 - w3)) that neither tile covers. S2 tile ids
// are mid | hi << (a1 - cp2) with mid = bits [cp2, a1); S3 tile ids are bits
// [cp3, a1 + w2) (S3 reaches the top bit).
struct SlabMap {
  int cp2, cp3, cpm, bits;
  uint32_t of_s2(uint32_t t, int mb2) const {
    return ((t & ((1u << mb2) - 1u)) >> (cpm - cp2)) & ((1u << bits) - 1u);
  }
  uint32_t of_s3(uint32_t t) const { return (t >> (cpm - cp3)) & ((1u << bits) - 1u); }
};

// Width of the S2 pass for `rest` element bits above the A1 tile: the engine's
// default (everything in S2 up to 9 bits, else an even split), or the forced
// width when it leaves at most 9 bits for S3.
int split_w2(const bk_ctx* c, int rest) {
  const int w = c->force_w2;
  if (w >= 1 && w <= 9 && w <= rest && rest - w <= 9) return w;
  return (rest <= 9) ? rest : (rest + 1) / 2;
}

// complex64 per-pass A1 kernels with the full phase table (complex128 has none)
template <class R>
int allow_table_a1(bk_ctx* c) {
  if constexpr (sizeof(R) == 4) {
    BK_TRY(allow_smem(c, reinterpret_cast<const void*>(tile_a1_wide_kernel<R, true>), A1Smem<true>::kBytes));
    BK_TRY(allow_smem(c, reinterpret_cast<const void*>(tile_a1_tab_kernel<R>), A1Smem<true>::kBytes));
    BK_TRY(allow_smem(c, reinterpret_cast<const void*>(tile_a1_warp_kernel<R, 8, true>), WarpA1Smem<8, true>::kBytes));
    BK_TRY(allow_smem(c, reinterpret_cast<const void*>(tile_a1_warp_kernel<R, 4, true>), WarpA1Smem<4, true>::kBytes));
  }
  return BK_OK;
}
template <class R>
void launch_table_a1(const InstDesc<R>& D, int a1_wide, uint32_t n_a1, cudaStream_t st, uint32_t step, int* err) {
  if constexpr (sizeof(R) == 4) {
    if (D.a1_bits == kA1WarpBits && a1_wide == 3)
      tile_a1_warp_kernel<R, 4, true><<<2 * n_a1, 128, WarpA1Smem<4, true>::kBytes, st>>>(D, step, err);
    else if (D.a1_bits == kA1WarpBits)
      tile_a1_warp_kernel<R, 8, true><<<n_a1, kComputeThreads, WarpA1Smem<8, true>::kBytes, st>>>(D, step, err);
    else if (a1_wide == 1)
      tile_a1_wide_kernel<R, true><<<n_a1, kA1WideThreads, A1Smem<true>::kBytes, st>>>(D, step, err);
    else
      tile_a1_tab_kernel<R><<<n_a1, kComputeThreads, A1Smem<true>::kBytes, st>>>(D, step, err);
  }
}

template <class R>
int persist_prepare(bk_ctx* c, const bk_evolve_params* p, const Schedule& S, double angle_unit,
                    const std::vector<R>& tans, const std::vector<R>& scales, PersistRun<R>* run,
                    bool grid_mode = false) {
  const int n = p->n;
  const bool c64 = sizeof(R) == 4;
  const int np = c64 ? n - 1 : n;  // element bits
  if (np - kElemBits < 1)
    return fail(c, BK_ERR_UNSUPPORTED, "persistent engine needs n > %d", kElemBits + (c64 ? 1 : 0));
  // the warp-local A1 (per-pass schedule) covers element bits 0-8; the strided
  // passes then take the remaining np - 9 <= 18 bits, the S2 width at least 3
  // (its tile keeps 12 - w2 <= 9 contiguous bits)
  const bool a1_warp = grid_mode && (c->a1_wide == 2 || c->a1_wide == 3) && np - kA1WarpBits <= 18;
  const bool a1_half = a1_warp && c->a1_wide == 3;  // 4-warp CTAs over half tiles
  const int a1_bits = a1_warp ? kA1WarpBits : kElemBits;
  const int rest = np - a1_bits;
  int w2 = split_w2(c, rest);
  if (a1_warp && w2 < 3) w2 = (rest <= 9) ? rest : (rest + 1) / 2;
  const int w3 = rest - w2;
  if (w2 > 9 || w3 > 9) return fail(c, BK_ERR_UNSUPPORTED, "n = %d needs more than two strided passes", n);
  const int e_tile_bits = c64 ? 13 : 12;

  // tensor maps in element space (16-byte elements = two 8-byte TMA elements)
  TmaDesc a1m, em, m2, m3, a1s, eh;
  BK_TRY(build_amp_map(c, c->d_state, np, BK_C128, kElemBits, kElemBits, 0, &a1m));
  BK_TRY(build_e_map(c, c->d_E, n, e_tile_bits, &em));
  BK_TRY(build_amp_map(c, c->d_state, np, BK_C128, kElemBits - w2, a1_bits, w2, &m2));
  if (w3 > 0) BK_TRY(build_amp_map(c, c->d_state, np, BK_C128, kElemBits - w3, a1_bits + w2, w3, &m3));
  if (a1_warp) BK_TRY(build_a1_swizzled_map(c, c->d_state, np, &a1s, a1_half));
  if (a1_half) BK_TRY(build_e_map(c, c->d_E, n, e_tile_bits - 1, &eh));

  // phase
  typename PhaseV<R>::params ph{};
  std::vector<float2> hab;
  std::vector<double2> t64;
  std::vector<float2> ptab;
  if constexpr (sizeof(R) == 4) {
    BK_TRY(build_phase_v(c, n, angle_unit, &ph, &hab));
    // the full phase table for the per-pass A1 kernels
    if (grid_mode && c->phase_table)
      BK_TRY(build_phase_table(c, n, angle_unit, &ph, &ptab));
  } else {
    Phase64 p64{};
    BK_TRY(build_phase(c, n, angle_unit, &p64));  // uploads to d_phase
    ph.hi = p64.hi;
    ph.lo = p64.lo;
    ph.n_hi = p64.n_hi;
  }

  // tasks of one step: A1 of slab h+1 is queued ahead of S2 of slab h (L2 hand-off)
  const uint32_t n_a1 = 1u << (np - kElemBits), n_s2 = n_a1, n_s3 = w3 > 0 ? n_a1 : 0u;
  const uint32_t slabs = 1u << std::max(0, np - kElemBits - w2);
  const uint32_t per_slab = 1u << w2;
  std::vector<unsigned long long> tasks;
  tasks.reserve(n_a1 + n_s2 + n_s3);
  auto task = [](int kind, int inst, uint32_t tile) {
    return ((unsigned long long)kind << 56) | ((unsigned long long)inst << 32) | tile;
  };
  // S2 of slab h is queued `lag` slabs after A1 of slab h: far enough behind the
  // ~2 tasks per CTA in flight that the slab is finished, close enough that its
  // data is still in L2 (lag x slab bytes of dirty lines)
  const uint32_t lag = std::max<uint32_t>(1u, std::min<uint32_t>(slabs, (uint32_t)c->slab_lag));
  for (uint32_t h = 0; !a1_warp && h < slabs + lag; ++h) {
    if (h < slabs)
      for (uint32_t j = 0; j < per_slab; ++j) tasks.push_back(task(TASK_A1, 0, h * per_slab + j));
    if (h >= lag)
      for (uint32_t j = 0; j < per_slab; ++j) tasks.push_back(task(TASK_S2, 0, (h - lag) * per_slab + j));
  }
  for (uint32_t j = 0; !a1_warp && j < n_s3; ++j) tasks.push_back(task(TASK_S3, 0, j));
  std::vector<unsigned long long> final_tasks;
  if (S.slot[(size_t)p->n_steps] >= 0)
    for (uint32_t j = 0; j < n_a1; ++j) final_tasks.push_back(task(TASK_M, 0, j));

  // device buffer layout
  Bump b;
  const size_t o_maps = b.take(6 * sizeof(CUtensorMap));
  const size_t o_desc = b.take(sizeof(InstDesc<R>));
  const size_t o_tasks = b.take(tasks.size() * 8);
  const size_t o_final = b.take(std::max<size_t>(final_tasks.size(), 1) * 8);
  const size_t o_tan = b.take(std::max<size_t>(tans.size(), 1) * sizeof(R));
  const size_t o_scale = b.take(std::max<size_t>(scales.size(), 1) * sizeof(R));
  const size_t o_slot = b.take(S.slot.size() * sizeof(int));
  const size_t o_hab = b.take(std::max<size_t>(hab.size(), 1) * sizeof(float2));
  const size_t o_ptab = b.take(std::max<size_t>(ptab.size(), 1) * sizeof(float2));
  const size_t o_ctr = b.take((slabs + 8) * sizeof(unsigned int));
  const size_t o_part = b.take(3 * (size_t)n_a1 * (a1_half ? 2 : 1) * sizeof(double));
  // fused strided pass: tasks in slab order (S2 of slab h after S3 of slab h + lag)
  std::vector<unsigned long long> tasks23;
  uint32_t slabs23 = 0, per_slab23 = 0;
  S23Program prog23{};
  if (grid_mode && (c->engine_mode == 2 || c->engine_mode == 3) && w3 > 0) {
    SlabMap sm{kElemBits - w2, kElemBits - w3, 0, 0};
    sm.cpm = std::max(sm.cp2, sm.cp3);
    sm.bits = std::max(0, a1_bits - sm.cpm);
    slabs23 = 1u << sm.bits;
    per_slab23 = n_s2 / slabs23;
    const uint32_t lag23 = std::max<uint32_t>(1u, std::min<uint32_t>(slabs23, (uint32_t)c->slab_lag));
    const uint64_t key = ((uint64_t)np << 48) | ((uint64_t)a1_bits << 40) | ((uint64_t)w2 << 32) | lag23;
    int lb = 0;
    while ((1u << lb) < per_slab23) ++lb;
    prog23.slabs = slabs23;
    prog23.lag = lag23;
    prog23.lb = (uint32_t)lb;
    prog23.x = (uint32_t)(sm.cpm - sm.cp2);
    prog23.y = (uint32_t)(sm.cpm - sm.cp3);
    prog23.mb2 = (uint32_t)(a1_bits - sm.cp2);
    prog23.bits = (uint32_t)sm.bits;
    prog23.n_tasks = 2u * n_s2;
    if ((1u << lb) != per_slab23 || n_s3 != n_s2)
      return fail(c, BK_ERR_UNSUPPORTED, "fused strided pass: slab size not a power of two for n = %d", n);
    // the kernel decodes its task order in closed form; the first run of a
    // geometry checks it against the order built here tile by tile
    if (c->s23_checked != key) {
      std::vector<std::vector<uint32_t>> s2_of(slabs23), s3_of(slabs23);
      for (uint32_t t = 0; t < n_s2; ++t) s2_of[sm.of_s2(t, a1_bits - sm.cp2)].push_back(t);
      for (uint32_t t = 0; t < n_s3; ++t) s3_of[sm.of_s3(t)].push_back(t);
      for (uint32_t v = 0; v < slabs23; ++v)
        if (s2_of[v].size() != per_slab23 || s3_of[v].size() != n_s3 / slabs23)
          return fail(c, BK_ERR_UNSUPPORTED, "fused strided pass: uneven slabs for n = %d", n);
      auto w23 = [](uint32_t kind, uint32_t slab, uint32_t tile) {
        return ((unsigned long long)kind << 56) | ((unsigned long long)slab << 32) | tile;
      };
      for (uint32_t h = 0; h < slabs23 + lag23; ++h) {  // S3 of a slab first, its S2 lag slabs later
        if (h < slabs23)
          for (uint32_t t : s3_of[h]) tasks23.push_back(w23(S23_S3, h, t));
        if (h >= lag23)
          for (uint32_t t : s2_of[h - lag23]) tasks23.push_back(w23(S23_S2, h - lag23, t));
      }
      if (tasks23.size() != prog23.n_tasks)
        return fail(c, BK_ERR_UNSUPPORTED, "fused strided pass: %zu tasks for n = %d", tasks23.size(), n);
      for (uint32_t g = 0; g < prog23.n_tasks; ++g) {
        const S23Task t = s23_decode(prog23, g);
        if (w23(t.kind, t.slab, t.tile) != tasks23[g])
          return fail(c, BK_ERR_UNSUPPORTED, "fused strided pass: task order mismatch at %u (n = %d)", g, n);
      }
      c->s23_checked = key;
    }
  }
  const size_t o_ctr23 = b.take((slabs23 + 4) * sizeof(unsigned int));
  BK_TRY(ensure_buffer(c, &c->d_persist, &c->persist_cap, b.off));
  char* base = static_cast<char*>(c->d_persist);
  CUtensorMap* d_maps = reinterpret_cast<CUtensorMap*>(base + o_maps);
  unsigned int* ctr = reinterpret_cast<unsigned int*>(base + o_ctr);
  // counter block: [a1_done: slabs][s2_done][s3_done][ticket][next][err][abort]
  unsigned int* a1_done = ctr;
  unsigned int* s2_done = ctr + slabs;
  unsigned int* s3_done = ctr + slabs + 1;
  unsigned int* ticket = ctr + slabs + 2;
  unsigned int* next = ctr + slabs + 3;
  int* err = reinterpret_cast<int*>(ctr + slabs + 4);
  int* abort_w = reinterpret_cast<int*>(ctr + slabs + 5);

  CUtensorMap maps[6] = {a1m.map, em.map, m2.map, w3 > 0 ? m3.map : m2.map, a1_warp ? a1s.map : a1m.map,
                         a1_half ? eh.map : em.map};
  InstDesc<R> D{};
  D.state = static_cast<unsigned char*>(c->d_state);
  D.map_a1 = d_maps + 0;
  D.map_e = d_maps + 1;
  D.map_s2 = d_maps + 2;
  D.map_s3 = d_maps + 3;
  D.np = np;
  D.n = n;
  D.w2 = w2;
  D.w3 = w3;
  D.a1_hi_dim = a1m.hi_dim;
  D.s2_mid_dim = m2.mid_dim;
  D.s2_hi_dim = m2.hi_dim;
  D.s2_mid_bits = (int)m2.mid_bits;
  D.s3_mid_dim = w3 > 0 ? m3.mid_dim : -1;
  D.s3_hi_dim = w3 > 0 ? m3.hi_dim : -1;
  D.s3_mid_bits = w3 > 0 ? (int)m3.mid_bits : 0;
  D.e0 = (int)p->e0;
  D.s0 = (uint32_t)(p->s0 & ((1ull << n) - 1ull));
  if constexpr (sizeof(R) == 4) {
    ph.hab = reinterpret_cast<const float2*>(base + o_hab);
    if (!ptab.empty()) ph.tab = reinterpret_cast<const float2*>(base + o_ptab);
  }
  D.phase = ph;
  D.tan = reinterpret_cast<const R*>(base + o_tan);
  D.scale = reinterpret_cast<const R*>(base + o_scale);
  D.slot = reinterpret_cast<const int*>(base + o_slot);
  D.a1_done = a1_done;
  D.s2_done = s2_done;
  D.s3_done = s3_done;
  D.ticket = ticket;
  D.partials = reinterpret_cast<double*>(base + o_part);
  D.results = c->d_results;
  D.n_a1 = n_a1;
  D.n_s2 = n_s2;
  D.n_s3 = n_s3;
  D.e_recompute = c->e_recompute;
  D.a1_bits = a1_bits;
  D.map_a1s = d_maps + 4;
  D.a1_evict_first = (grid_mode && (c->engine_mode == 2 || c->engine_mode == 3)) ? 1 : 0;
  D.map_e_half = d_maps + 5;

  cudaStream_t st = c->stream;
  BK_CUDA(c, cudaMemcpyAsync(d_maps, maps, sizeof(maps), cudaMemcpyHostToDevice, st));
  BK_CUDA(c, cudaMemcpyAsync(base + o_tasks, tasks.data(), tasks.size() * 8, cudaMemcpyHostToDevice, st));
  if (!final_tasks.empty())
    BK_CUDA(c, cudaMemcpyAsync(base + o_final, final_tasks.data(), final_tasks.size() * 8, cudaMemcpyHostToDevice, st));
  if (!tans.empty()) {
    BK_CUDA(c, cudaMemcpyAsync(base + o_tan, tans.data(), tans.size() * sizeof(R), cudaMemcpyHostToDevice, st));
    BK_CUDA(c, cudaMemcpyAsync(base + o_scale, scales.data(), scales.size() * sizeof(R), cudaMemcpyHostToDevice, st));
  }
  BK_CUDA(c, cudaMemcpyAsync(base + o_slot, S.slot.data(), S.slot.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  if (!hab.empty())
    BK_CUDA(c, cudaMemcpyAsync(base + o_hab, hab.data(), hab.size() * sizeof(float2), cudaMemcpyHostToDevice, st));
  if (!ptab.empty())
    BK_CUDA(c, cudaMemcpyAsync(base + o_ptab, ptab.data(), ptab.size() * sizeof(float2), cudaMemcpyHostToDevice, st));
  if (prog23.n_tasks > 0) BK_CUDA(c, cudaMemsetAsync(base + o_ctr23, 0, (slabs23 + 4) * sizeof(unsigned int), st));
  BK_TRY(allow_smem(c, reinterpret_cast<const void*>(persist_kernel<R, true>), PersistSmem::kBytes));
  run->base = base;
  run->o_desc = o_desc;
  run->o_tasks = o_tasks;
  run->o_final = o_final;
  run->o_tan = o_tan;
  run->o_scale = o_scale;
  run->o_slot = o_slot;
  run->D = D;
  run->ctr = ctr;
  run->slabs = slabs;
  run->n_tasks = tasks.size();
  run->n_final = final_tasks.size();
  run->next = next;
  run->err = err;
  run->abort_w = abort_w;
  run->n_a1 = n_a1;
  run->n_s2 = n_s2;
  run->n_s3 = n_s3;
  run->phase = D.phase;
  run->n_tasks23 = prog23.n_tasks;
  run->slabs23 = slabs23;
  run->prog23 = prog23;
  run->ctr23 = reinterpret_cast<unsigned int*>(base + o_ctr23);
  run->a1_table = !ptab.empty();
  return BK_OK;
}

// Wait bounds and the test hook of a persistent launch, from the context's options.
void program_limits(const bk_ctx* c, Program* P) {
  P->poll_limit = c->wait_polls > 0 ? c->wait_polls : kWaitPolls * 4u;
  P->hold_step = c->hold_step >= 0 ? (uint32_t)c->hold_step : 0xFFFFFFFFu;
}

// Steps [k0, k0 + n_steps) in one persistent launch, then `n_final`
// measurement-only tasks (0 or all of them) for step k0 + n_steps; waits for the
// launch and reports a bounded device wait that gave up.
template <class R>
int persist_launch(bk_ctx* c, PersistRun<R>& r, int k0, int n_steps, size_t n_final, bool wait = true) {
  cudaStream_t st = c->stream;
  InstDesc<R> D = r.D;
  D.tan = reinterpret_cast<const R*>(r.base + r.o_tan) + k0;
  D.scale = reinterpret_cast<const R*>(r.base + r.o_scale) + k0;
  D.slot = reinterpret_cast<const int*>(r.base + r.o_slot) + k0;
  BK_CUDA(c, cudaMemcpyAsync(r.base + r.o_desc, &D, sizeof(D), cudaMemcpyHostToDevice, st));
  BK_CUDA(c, cudaMemsetAsync(r.ctr, 0, (r.slabs + 8) * sizeof(unsigned int), st));
  Program P{};
  P.tasks = reinterpret_cast<const unsigned long long*>(r.base + r.o_tasks);
  P.per_step = (uint32_t)r.n_tasks;
  P.n_steps = (uint32_t)n_steps;
  P.final_tasks = reinterpret_cast<const unsigned long long*>(r.base + r.o_final);
  P.n_final = (uint32_t)n_final;
  P.step0 = (uint32_t)k0;
  P.next = r.next;
  P.err = r.err;
  P.abort = r.abort_w;
  program_limits(c, &P);
  if (P.n_steps == 0 && P.n_final == 0) return BK_OK;
  size_t ev = 0;
  BK_TRY(ev_begin(c, "persist", &ev));
  persist_kernel<R, true><<<2 * c->num_sms, kPersistThreads, PersistSmem::kBytes, st>>>(
      reinterpret_cast<const InstDesc<R>*>(r.base + r.o_desc), P);
  BK_CUDA(c, cudaGetLastError());
  BK_TRY(ev_end(c, ev));
  if (!wait) return BK_OK;  // the caller reads r.err after its own synchronisation
  int e = 0;
  BK_CUDA(c, cudaMemcpyAsync(&e, r.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  BK_CUDA(c, cudaStreamSynchronize(st));
  if (e != 0) return fail(c, BK_ERR_TIMEOUT, "persistent engine: a bounded device wait gave up (%d)", e);
  return BK_OK;
}

template <class R>
int evolve_persist(bk_ctx* c, const bk_evolve_params* p, const Schedule& S, double angle_unit,
                   const std::vector<R>& tans, const std::vector<R>& scales) {
  PersistRun<R> run;
  BK_TRY(persist_prepare<R>(c, p, S, angle_unit, tans, scales, &run, c->engine_mode != 0));
  const int n = p->n;
  cudaStream_t st = c->stream;
  unsigned int* ctr = run.ctr;
  const uint32_t slabs = run.slabs;
  int* err = run.err;
  const uint32_t n_a1 = run.n_a1, n_s2 = run.n_s2, n_s3 = run.n_s3;
  const InstDesc<R> D = run.D;

  if (c->engine_mode == 1 || c->engine_mode == 2 || c->engine_mode == 3) {
    // one grid launch per pass: A1, S2, S3 per step, measurement tiles at the end;
    // mode 2 runs S2 + S3 as one fused launch (S3 reads S2's slabs from L2)
    const bool fused23 = run.n_tasks23 > 0;
    S23Program P23 = run.prog23;
    const bool self_served = c->engine_mode == 3;  // the fused strided pass without a producer warp
    if (fused23) {
      BK_TRY(allow_smem(c, reinterpret_cast<const void*>(s23_kernel<R>), kS23Smem));
      BK_TRY(allow_smem(c, reinterpret_cast<const void*>(s23g_kernel<R>), kS23gSmem));
      P23.slab_done = run.ctr23;
      P23.next = run.ctr23 + run.slabs23;
      P23.ctas_done = run.ctr23 + run.slabs23 + 1;
      P23.err = err;
      P23.abort = reinterpret_cast<int*>(run.ctr23 + run.slabs23 + 2);
      P23.poll_limit = c->wait_polls > 0 ? c->wait_polls : kWaitPolls * 4u;
    }
    BK_TRY(allow_smem(c, reinterpret_cast<const void*>(tile_pass_kernel<R>), PersistSmem::kBytes));
    BK_TRY(allow_smem(c, reinterpret_cast<const void*>(tile_a1_wide_kernel<R, false>), A1Smem<false>::kBytes));
    BK_TRY(allow_smem(c, reinterpret_cast<const void*>(tile_a1_warp_kernel<R, 8, false>),
                      WarpA1Smem<8, false>::kBytes));
    BK_TRY(allow_smem(c, reinterpret_cast<const void*>(tile_a1_warp_kernel<R, 4, false>),
                      WarpA1Smem<4, false>::kBytes));
    // the full phase table (complex64 A1 kernels 1-3)
    const bool a1_table = run.a1_table;
    if (a1_table) BK_TRY(allow_table_a1<R>(c));
    using SampT = typename std::conditional<sizeof(R) == 4, Planar64, double2>::type;
    BK_CUDA(c, cudaMemsetAsync(ctr, 0, (slabs + 8) * sizeof(unsigned int), st));
    for (int k = 0; k <= p->n_steps; ++k) {
      if (S.sample_pt[(size_t)k] >= 0)
        BK_TRY(launch_sampling_t(c, reinterpret_cast<const SampT*>(c->d_state), n, S.sample_pt[(size_t)k], S.shots));
      size_t ev = 0;
      if (k == p->n_steps) {
        if (S.slot[(size_t)k] >= 0) {
          BK_TRY(ev_begin(c, "tile_m", &ev));
          tile_pass_kernel<R><<<n_a1, kComputeThreads, PersistSmem::kBytes, st>>>(D, TASK_M, (uint32_t)k, err);
          BK_CUDA(c, cudaGetLastError());
          BK_TRY(ev_end(c, ev));
        }
        break;
      }
      BK_TRY(ev_begin(c, "tile_a1", &ev));
      if (a1_table)
        launch_table_a1(D, c->a1_wide, n_a1, st, (uint32_t)k, err);
      else if (D.a1_bits == kA1WarpBits && c->a1_wide == 3)
        tile_a1_warp_kernel<R, 4, false><<<2 * n_a1, 128, WarpA1Smem<4, false>::kBytes, st>>>(D, (uint32_t)k, err);
      else if (D.a1_bits == kA1WarpBits)
        tile_a1_warp_kernel<R, 8, false><<<n_a1, kComputeThreads, WarpA1Smem<8, false>::kBytes, st>>>(D, (uint32_t)k,
                                                                                                     err);
      else if (c->a1_wide == 1)
        tile_a1_wide_kernel<R, false><<<n_a1, kA1WideThreads, A1Smem<false>::kBytes, st>>>(D, (uint32_t)k, err);
      else
        tile_pass_kernel<R><<<n_a1, kComputeThreads, PersistSmem::kBytes, st>>>(D, TASK_A1, (uint32_t)k, err);
      BK_CUDA(c, cudaGetLastError());
      BK_TRY(ev_end(c, ev));
      if (fused23) {
        BK_TRY(ev_begin(c, "tile_s23", &ev));
        P23.step = (uint32_t)k;
        if (self_served)
          s23g_kernel<R><<<c->num_sms, kS23gThreads, kS23gSmem, st>>>(D, P23);
        else
          s23_kernel<R><<<c->num_sms, kS23Threads, kS23Smem, st>>>(D, P23);
        BK_CUDA(c, cudaGetLastError());
        BK_TRY(ev_end(c, ev));
        continue;
      }
      BK_TRY(ev_begin(c, "tile_s2", &ev));
      tile_pass_kernel<R><<<n_s2, kComputeThreads, PersistSmem::kBytes, st>>>(D, TASK_S2, (uint32_t)k, err);
      BK_CUDA(c, cudaGetLastError());
      BK_TRY(ev_end(c, ev));
      if (n_s3 > 0) {
        BK_TRY(ev_begin(c, "tile_s3", &ev));
        tile_pass_kernel<R><<<n_s3, kComputeThreads, PersistSmem::kBytes, st>>>(D, TASK_S3, (uint32_t)k, err);
        BK_CUDA(c, cudaGetLastError());
        BK_TRY(ev_end(c, ev));
      }
    }
    int e = 0;
    BK_CUDA(c, cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    BK_CUDA(c, cudaStreamSynchronize(st));
    if (e != 0) return fail(c, BK_ERR_TIMEOUT, "tile pass: a bounded device wait gave up (%d)", e);
    return BK_OK;
  }

  // one launch per segment between sampling points (sampling reads psi_k before step k)
  using Samp = typename std::conditional<sizeof(R) == 4, Planar64, double2>::type;
  int k0 = 0, search = 0;
  for (;;) {
    int k1 = search;
    while (k1 < p->n_steps && S.sample_pt[(size_t)k1] < 0) ++k1;
    // launch steps [k0, k1) (+ the final measurement when k1 == n_steps)
    const bool last = (k1 == p->n_steps);
    const bool sample_final = last && S.sample_pt[(size_t)k1] >= 0;
    BK_TRY(persist_launch<R>(c, run, k0, k1 - k0, (last && !sample_final) ? run.n_final : 0));
    if (k1 >= p->n_steps && !sample_final) break;
    // sampling point k1 (state psi_k1 is in place)
    BK_TRY(launch_sampling_t(c, reinterpret_cast<const Samp*>(c->d_state), n, S.sample_pt[(size_t)k1], S.shots));
    if (sample_final) {
      // final measurement after sampling
      BK_TRY(persist_launch<R>(c, run, k1, 0, run.n_final));
      break;
    }
    k0 = k1;
    search = k1 + 1;
    // the next segment starts at k1; its first A1 measures step k1 if flagged
  }
  return BK_OK;
}

// ---------------------------------------------------------------------------
// batched evolution (persistent engine over many statevectors)
// ---------------------------------------------------------------------------
int batch_energy(bk_ctx* c, int n, uint16_t** out) {
  auto it = c->batch_E.find(n);
  if (it != c->batch_E.end()) {
    *out = it->second;
    return BK_OK;
  }
  uint16_t* d = nullptr;
  const size_t count = 1ull << n;
  BK_CUDA(c, cudaMalloc(&d, std::max<size_t>(count, 8) * sizeof(uint16_t)));
  const uint32_t per = (uint32_t)((count + 7) / 8);
  energy_table_kernel<<<(per + 255) / 256, 256, 0, c->stream>>>(d, n, (uint32_t)count);
  BK_CUDA(c, cudaGetLastError());
  c->batch_E[n] = d;
  *out = d;
  return BK_OK;
}

__global__ void set_basis_many_kernel(unsigned char* base, const unsigned long long* offsets,
                                      const unsigned int* idx, int planar, int n_inst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_inst) return;
  unsigned char* st = base + offsets[i];
  const uint32_t s = idx[i];
  if (planar)
    reinterpret_cast<float*>(st)[4u * (s >> 1) + (s & 1u)] = 1.0f;
  else
    reinterpret_cast<double2*>(st)[s] = make_double2(1.0, 0.0);
}

template <class R>
int evolve_batch_t(bk_ctx* c, const bk_batch_params* bp, const bk_batch_instance* inst, int n_inst,
                   double* p_less, double* d_h, double* norm_out) {
  const bool c64 = sizeof(R) == 4;
  const int T = bp->n_steps;
  std::vector<int> slot((size_t)T + 1, -1);
  int n_meas = 0;
  for (int k = 0; k <= T; ++k)
    if (bp->measure == nullptr || bp->measure[k]) slot[(size_t)k] = n_meas++;
  if (n_meas > 0 && (!p_less || !d_h)) return fail(c, BK_ERR_INVALID, "output arrays are NULL");

  struct Geo {
    int n, np, w2, w3, e0;
    uint32_t n_a1, slabs, s0;
    size_t state_off;
    double angle_unit;
  };
  std::vector<Geo> geo((size_t)n_inst);
  size_t state_bytes = 0;
  for (int i = 0; i < n_inst; ++i) {
    const bk_batch_instance& b = inst[i];
    Geo g{};
    g.n = b.n;
    g.np = c64 ? b.n - 1 : b.n;
    if (g.np <= kElemBits || b.n > kMaxN)
      return fail(c, BK_ERR_UNSUPPORTED, "batched instance %d: n = %d outside [%d, %d]", i, b.n,
                  kElemBits + (c64 ? 2 : 1), kMaxN);
    const int rest = g.np - kElemBits;
    g.w2 = split_w2(c, rest);
    g.w3 = rest - g.w2;
    if (g.w2 > 9 || g.w3 > 9) return fail(c, BK_ERR_UNSUPPORTED, "n = %d needs more than two strided passes", b.n);
    g.n_a1 = 1u << (g.np - kElemBits);
    g.slabs = 1u << (g.np - kElemBits - g.w2);
    g.s0 = (uint32_t)(b.s0 & ((1ull << b.n) - 1ull));
    int64_t e0 = b.e0;
    if (e0 < 0) e0 = host_energy(b.n, g.s0);
    g.e0 = (int)e0;
    g.angle_unit = (bp->diag_scale > 0.0) ? bp->dt * bp->diag_scale : bp->dt / (double)b.n;
    g.state_off = state_bytes;
    state_bytes += (1ull << b.n) * (c64 ? 8 : 16);
    geo[(size_t)i] = g;
    if (b.g == nullptr && !is_finite(b.g_const)) return fail(c, BK_ERR_INVALID, "instance %d: g not finite", i);
  }
  BK_TRY(ensure_buffer(c, &c->d_batch_state, &c->batch_state_cap, state_bytes));
  BK_TRY(ensure_buffer(c, reinterpret_cast<void**>(&c->d_batch_results), &c->batch_results_cap,
                       std::max<size_t>((size_t)n_inst * n_meas * 4, 1) * sizeof(double)));
  unsigned char* state = static_cast<unsigned char*>(c->d_batch_state);

  // per-instance schedules of tangents, exact rescales and the log2 of the omitted factors
  std::vector<R> tans((size_t)n_inst * std::max(T, 1)), scales((size_t)n_inst * std::max(T, 1));
  std::vector<long double> row_log2((size_t)n_inst * std::max(n_meas, 1), 0.0L);
  for (int i = 0; i < n_inst; ++i) {
    long double lg = 0.0L;
    for (int k = 0; k <= T; ++k) {
      if (slot[(size_t)k] >= 0) row_log2[(size_t)i * n_meas + slot[(size_t)k]] = lg;
      if (k == T) break;
      const double gk = inst[i].g ? inst[i].g[k] : inst[i].g_const;
      if (!is_finite(gk)) return fail(c, BK_ERR_INVALID, "instance %d: g[%d] not finite", i, k);
      const R tf = (R)std::tan(gk * bp->dt);
      R sc = (R)1;
      if (lg >= (long double)kRescaleLog2) {
        sc = (R)std::ldexp(1.0, -kRescaleLog2);
        lg -= (long double)kRescaleLog2;
      }
      tans[(size_t)i * T + k] = tf;
      scales[(size_t)i * T + k] = sc;
      lg += 0.5L * (long double)geo[(size_t)i].n * std::log2(1.0L + (long double)tf * (long double)tf);
    }
  }

  // phase tables per distinct n
  std::map<int, std::vector<unsigned char>> tables;
  std::map<int, typename PhaseV<R>::params> phase_of;
  for (const Geo& g : geo) {
    if (tables.count(g.n)) continue;
    typename PhaseV<R>::params ph{};
    std::vector<unsigned char> bytes;
    if constexpr (sizeof(R) == 4) {
      std::vector<float2> hab;
      BK_TRY(build_phase_v(c, g.n, g.angle_unit, &ph, &hab));
      bytes.resize(hab.size() * sizeof(float2));
      std::memcpy(bytes.data(), hab.data(), bytes.size());
    } else {
      const int emax = (g.n - 1) * g.n * (2 * g.n - 1) / 6;
      const int n_hi = (emax >> kPhaseLoBits) + 1;
      std::vector<double2> t((size_t)n_hi + kPhaseLo);
      for (int h = 0; h < n_hi; ++h) {
        const double th = -g.angle_unit * (double)(h << kPhaseLoBits);
        t[(size_t)h] = make_double2(std::cos(th), std::sin(th));
      }
      for (int l = 0; l < kPhaseLo; ++l) {
        const double th = -g.angle_unit * (double)l;
        t[(size_t)n_hi + l] = make_double2(std::cos(th), std::sin(th));
      }
      ph.n_hi = n_hi;
      bytes.resize(t.size() * sizeof(double2));
      std::memcpy(bytes.data(), t.data(), bytes.size());
    }
    tables[g.n] = std::move(bytes);
    phase_of[g.n] = ph;
  }

  // tasks of one step: A1 blocks in order, each slab's S2 block `lag` blocks later, then S3
  auto task = [](int kind, int in, uint32_t tile) {
    return ((unsigned long long)kind << 56) | ((unsigned long long)in << 32) | tile;
  };
  std::vector<std::pair<int, uint32_t>> blocks;  // (instance, slab)
  for (int i = 0; i < n_inst; ++i)
    for (uint32_t h = 0; h < geo[(size_t)i].slabs; ++h) blocks.push_back({i, h});
  const size_t lag = (size_t)std::max(1, bp->lag > 0 ? bp->lag : c->slab_lag);
  std::vector<unsigned long long> tasks, final_tasks;
  for (size_t j = 0; j < blocks.size() + lag; ++j) {
    if (j < blocks.size()) {
      const auto [i, h] = blocks[j];
      const uint32_t per = 1u << geo[(size_t)i].w2;
      for (uint32_t t = 0; t < per; ++t) tasks.push_back(task(TASK_A1, i, h * per + t));
    }
    if (j >= lag && j - lag < blocks.size()) {
      const auto [i, h] = blocks[j - lag];
      const uint32_t per = 1u << geo[(size_t)i].w2;
      for (uint32_t t = 0; t < per; ++t) tasks.push_back(task(TASK_S2, i, h * per + t));
    }
  }
  for (int i = 0; i < n_inst; ++i)
    if (geo[(size_t)i].w3 > 0)
      for (uint32_t t = 0; t < geo[(size_t)i].n_a1; ++t) tasks.push_back(task(TASK_S3, i, t));
  if (slot[(size_t)T] >= 0)
    for (int i = 0; i < n_inst; ++i)
      for (uint32_t t = 0; t < geo[(size_t)i].n_a1; ++t) final_tasks.push_back(task(TASK_M, i, t));

  // device buffer
  Bump b;
  const size_t o_maps = b.take((size_t)n_inst * 4 * sizeof(CUtensorMap));
  const size_t o_desc = b.take((size_t)n_inst * sizeof(InstDesc<R>));
  const size_t o_tasks = b.take(tasks.size() * 8);
  const size_t o_final = b.take(std::max<size_t>(final_tasks.size(), 1) * 8);
  const size_t o_tan = b.take(tans.size() * sizeof(R));
  const size_t o_scale = b.take(scales.size() * sizeof(R));
  const size_t o_slot = b.take(slot.size() * sizeof(int));
  std::map<int, size_t> o_tab;
  for (auto& kv : tables) o_tab[kv.first] = b.take(kv.second.size());
  std::vector<size_t> o_ctr((size_t)n_inst), o_part((size_t)n_inst);
  for (int i = 0; i < n_inst; ++i) {
    o_ctr[(size_t)i] = b.take((geo[(size_t)i].slabs + 4) * sizeof(unsigned int));
    o_part[(size_t)i] = b.take(3 * (size_t)geo[(size_t)i].n_a1 * sizeof(double));
  }
  const size_t o_glob = b.take(8 * sizeof(unsigned int));  // next, err, abort
  const size_t o_offs = b.take((size_t)n_inst * sizeof(unsigned long long));
  const size_t o_idx = b.take((size_t)n_inst * sizeof(unsigned int));
  const size_t ctr_begin = o_ctr.empty() ? o_glob : o_ctr[0];
  BK_TRY(ensure_buffer(c, &c->d_batch, &c->batch_cap, b.off));
  char* base = static_cast<char*>(c->d_batch);
  CUtensorMap* d_maps = reinterpret_cast<CUtensorMap*>(base + o_maps);

  std::vector<CUtensorMap> maps((size_t)n_inst * 4);
  std::vector<InstDesc<R>> descs((size_t)n_inst);
  std::vector<unsigned long long> offs((size_t)n_inst);
  std::vector<unsigned int> idx((size_t)n_inst);
  for (int i = 0; i < n_inst; ++i) {
    const Geo& g = geo[(size_t)i];
    uint16_t* dE = nullptr;
    BK_TRY(batch_energy(c, g.n, &dE));
    void* st = state + g.state_off;
    TmaDesc a1m, em, m2, m3;
    BK_TRY(build_amp_map(c, st, g.np, BK_C128, kElemBits, kElemBits, 0, &a1m));
    BK_TRY(build_e_map(c, dE, g.n, c64 ? 13 : 12, &em));
    BK_TRY(build_amp_map(c, st, g.np, BK_C128, kElemBits - g.w2, kElemBits, g.w2, &m2));
    if (g.w3 > 0) BK_TRY(build_amp_map(c, st, g.np, BK_C128, kElemBits - g.w3, kElemBits + g.w2, g.w3, &m3));
    maps[(size_t)i * 4 + 0] = a1m.map;
    maps[(size_t)i * 4 + 1] = em.map;
    maps[(size_t)i * 4 + 2] = m2.map;
    maps[(size_t)i * 4 + 3] = g.w3 > 0 ? m3.map : m2.map;
    InstDesc<R> D{};
    D.state = static_cast<unsigned char*>(st);
    D.map_a1 = d_maps + (size_t)i * 4 + 0;
    D.map_e = d_maps + (size_t)i * 4 + 1;
    D.map_s2 = d_maps + (size_t)i * 4 + 2;
    D.map_s3 = d_maps + (size_t)i * 4 + 3;
    D.np = g.np;
    D.n = g.n;
    D.w2 = g.w2;
    D.w3 = g.w3;
    D.a1_hi_dim = a1m.hi_dim;
    D.s2_mid_dim = m2.mid_dim;
    D.s2_hi_dim = m2.hi_dim;
    D.s2_mid_bits = (int)m2.mid_bits;
    D.s3_mid_dim = g.w3 > 0 ? m3.mid_dim : -1;
    D.s3_hi_dim = g.w3 > 0 ? m3.hi_dim : -1;
    D.s3_mid_bits = g.w3 > 0 ? (int)m3.mid_bits : 0;
    D.e0 = g.e0;
    D.s0 = g.s0;
    typename PhaseV<R>::params ph = phase_of[g.n];
    if constexpr (sizeof(R) == 4) {
      ph.hab = reinterpret_cast<const float2*>(base + o_tab[g.n]);
    } else {
      ph.hi = reinterpret_cast<const double2*>(base + o_tab[g.n]);
      ph.lo = ph.hi + ph.n_hi;
    }
    D.phase = ph;
    D.tan = reinterpret_cast<const R*>(base + o_tan) + (size_t)i * T;
    D.scale = reinterpret_cast<const R*>(base + o_scale) + (size_t)i * T;
    D.slot = reinterpret_cast<const int*>(base + o_slot);
    unsigned int* ctr = reinterpret_cast<unsigned int*>(base + o_ctr[(size_t)i]);
    D.a1_done = ctr;
    D.s2_done = ctr + g.slabs;
    D.s3_done = ctr + g.slabs + 1;
    D.ticket = ctr + g.slabs + 2;
    D.partials = reinterpret_cast<double*>(base + o_part[(size_t)i]);
    D.results = c->d_batch_results + (size_t)i * n_meas * 4;
    D.n_a1 = g.n_a1;
    D.n_s2 = g.n_a1;
    D.n_s3 = g.w3 > 0 ? g.n_a1 : 0u;
    D.e_recompute = c->e_recompute;
    descs[(size_t)i] = D;
    offs[(size_t)i] = g.state_off;
    idx[(size_t)i] = g.s0;
  }
  cudaStream_t st = c->stream;
  BK_CUDA(c, cudaMemcpyAsync(d_maps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice, st));
  BK_CUDA(c, cudaMemcpyAsync(base + o_desc, descs.data(), descs.size() * sizeof(InstDesc<R>), cudaMemcpyHostToDevice, st));
  BK_CUDA(c, cudaMemcpyAsync(base + o_tasks, tasks.data(), tasks.size() * 8, cudaMemcpyHostToDevice, st));
  if (!final_tasks.empty())
    BK_CUDA(c, cudaMemcpyAsync(base + o_final, final_tasks.data(), final_tasks.size() * 8, cudaMemcpyHostToDevice, st));
  if (T > 0) {
    BK_CUDA(c, cudaMemcpyAsync(base + o_tan, tans.data(), tans.size() * sizeof(R), cudaMemcpyHostToDevice, st));
    BK_CUDA(c, cudaMemcpyAsync(base + o_scale, scales.data(), scales.size() * sizeof(R), cudaMemcpyHostToDevice, st));
  }
  BK_CUDA(c, cudaMemcpyAsync(base + o_slot, slot.data(), slot.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  for (auto& kv : tables)
    BK_CUDA(c, cudaMemcpyAsync(base + o_tab[kv.first], kv.second.data(), kv.second.size(), cudaMemcpyHostToDevice, st));
  BK_CUDA(c, cudaMemcpyAsync(base + o_offs, offs.data(), offs.size() * 8, cudaMemcpyHostToDevice, st));
  BK_CUDA(c, cudaMemcpyAsync(base + o_idx, idx.data(), idx.size() * 4, cudaMemcpyHostToDevice, st));
  BK_TRY(allow_smem(c, reinterpret_cast<const void*>(persist_kernel<R, false>), PersistSmem::kBytes));

  Program P{};
  P.tasks = reinterpret_cast<const unsigned long long*>(base + o_tasks);
  P.per_step = (uint32_t)tasks.size();
  P.n_steps = (uint32_t)T;
  P.final_tasks = reinterpret_cast<const unsigned long long*>(base + o_final);
  P.n_final = (uint32_t)final_tasks.size();
  P.step0 = 0;
  unsigned int* glob = reinterpret_cast<unsigned int*>(base + o_glob);
  P.next = glob;
  P.err = reinterpret_cast<int*>(glob + 1);
  P.abort = reinterpret_cast<int*>(glob + 2);
  program_limits(c, &P);
  const InstDesc<R>* dd = reinterpret_cast<const InstDesc<R>*>(base + o_desc);

  // the whole run: zero the states and counters, set the basis states, one persistent launch
  auto enqueue = [&]() -> int {
    BK_CUDA(c, cudaMemsetAsync(state, 0, state_bytes, st));
    BK_CUDA(c, cudaMemsetAsync(base + ctr_begin, 0, o_glob + 8 * sizeof(unsigned int) - ctr_begin, st));
    set_basis_many_kernel<<<(n_inst + 127) / 128, 128, 0, st>>>(state, reinterpret_cast<unsigned long long*>(base + o_offs),
                                                                reinterpret_cast<unsigned int*>(base + o_idx),
                                                                c64 ? 1 : 0, n_inst);
    BK_CUDA(c, cudaGetLastError());
    persist_kernel<R, false><<<2 * c->num_sms, kPersistThreads, PersistSmem::kBytes, st>>>(dd, P);
    BK_CUDA(c, cudaGetLastError());
    return BK_OK;
  };
  size_t ev = 0;
  BK_TRY(ev_begin(c, "batch", &ev));
  if (bp->use_graph) {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    BK_CUDA(c, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const int r = enqueue();
    cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (r != BK_OK) {
      if (graph) cudaGraphDestroy(graph);
      return r;
    }
    BK_CUDA(c, ce);
    ce = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    BK_CUDA(c, ce);
    ce = cudaGraphLaunch(exec, st);
    cudaGraphExecDestroy(exec);  // destruction is deferred until the launch completes
    BK_CUDA(c, ce);
  } else {
    BK_TRY(enqueue());
  }
  BK_TRY(ev_end(c, ev));
  std::vector<double> rows((size_t)n_inst * n_meas * 4);
  int e = 0;
  BK_CUDA(c, cudaMemcpyAsync(&e, P.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  if (!rows.empty())
    BK_CUDA(c, cudaMemcpyAsync(rows.data(), c->d_batch_results, rows.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  BK_CUDA(c, cudaStreamSynchronize(st));
  BK_TRY(collect_timing(c));
  if (e != 0) return fail(c, BK_ERR_TIMEOUT, "batched persistent engine: a bounded device wait gave up (%d)", e);
  for (int i = 0; i < n_inst; ++i)
    for (int m = 0; m < n_meas; ++m) {
      const size_t r = (size_t)i * n_meas + m;
      const long double f = std::exp2(-2.0L * row_log2[r]);
      // complex64: expectation values of the normalised state (see bk_evolve)
      const long double nrm = (sizeof(R) == 4 && rows[4 * r + 2] > 0.0) ? (long double)rows[4 * r + 2] * f : 1.0L;
      p_less[r] = (double)((long double)rows[4 * r + 0] * f / nrm);
      d_h[r] = (double)((long double)rows[4 * r + 1] * f / nrm);
      if (norm_out) norm_out[r] = (double)((long double)rows[4 * r + 2] * f);
    }
  return BK_OK;
}

// Fused / whole-state evolution in precision R. Fills results rows on device
// and returns the per-row log2 scale of the computed state (host side).
template <class R>
int evolve_fused(bk_ctx* c, const bk_evolve_params* p, const Schedule& S, double angle_unit,
                 std::vector<long double>* row_log2, long double* final_log2) {
  using amp = typename AmpTraits<R>::amp;
  constexpr int T = AmpTraits<R>::kTileBits;
  const int n = p->n;
  const double dt = p->dt;
  typename PhaseOf<R>::params phase{};
  BK_TRY(build_phase(c, n, angle_unit, &phase));
  const int e0 = (int)p->e0;
  const uint32_t s0 = (uint32_t)(p->s0 & ((1ull << n) - 1ull));

  // host schedule of the omitted cos^n factors and power-of-two rescales
  std::vector<R> tans((size_t)p->n_steps), scales((size_t)p->n_steps);
  row_log2->assign((size_t)S.n_meas, 0.0L);
  long double lg = 0.0L;
  for (int k = 0; k <= p->n_steps; ++k) {
    if (S.slot[(size_t)k] >= 0) (*row_log2)[(size_t)S.slot[(size_t)k]] = lg;
    if (k == p->n_steps) break;
    const double gd = S.g[(size_t)k] * dt;
    tans[(size_t)k] = (R)std::tan(gd);
    R sc = (R)1;
    if (lg >= (long double)kRescaleLog2) {
      sc = (R)std::ldexp(1.0, -kRescaleLog2);
      lg -= (long double)kRescaleLog2;
    }
    scales[(size_t)k] = sc;
    // each butterfly multiplies the norm^2 of its pair by 1 + t^2, t the value the kernel uses
    const long double tf = (long double)tans[(size_t)k];
    lg += 0.5L * (long double)n * std::log2(1.0L + tf * tf);
  }
  *final_log2 = lg;

  if (n <= T) {
    // whole state in one CTA's shared memory; all steps between two sampling
    // points in one launch
    const size_t smem = PhaseOf<R>::kSmemBytes + (1ull << n) * (sizeof(amp) + 2);
    const size_t bytes = tans.size() * sizeof(R) * 2 + S.slot.size() * sizeof(int) + 64;
    BK_TRY(ensure_buffer(c, &c->d_small, &c->small_cap, bytes));
    char* base = reinterpret_cast<char*>(c->d_small);
    R* d_t = reinterpret_cast<R*>(base);
    R* d_sc = d_t + tans.size();
    int* d_slot = reinterpret_cast<int*>(base + tans.size() * sizeof(R) * 2);
    if (!tans.empty()) {
      BK_CUDA(c, cudaMemcpyAsync(d_t, tans.data(), tans.size() * sizeof(R), cudaMemcpyHostToDevice, c->stream));
      BK_CUDA(c, cudaMemcpyAsync(d_sc, scales.data(), scales.size() * sizeof(R), cudaMemcpyHostToDevice, c->stream));
    }
    BK_CUDA(c, cudaMemcpyAsync(d_slot, S.slot.data(), S.slot.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    BK_TRY(allow_smem(c, reinterpret_cast<const void*>(small_state_kernel<R>),
                      (int)(PhaseOf<R>::kSmemBytes + (1ull << T) * (sizeof(amp) + 2))));
    // Segments end at sampling points: sampling reads psi_k before step k, so a
    // segment runs steps [k0, k1) and leaves the measurement of step k1 to the
    // next segment (measure_last = 0); the last segment measures its end.
    int k0 = 0, search = 0;
    while (true) {
      int k1 = search;
      while (k1 <= p->n_steps && S.sample_pt[(size_t)k1] < 0) ++k1;
      const bool sample_here = (k1 <= p->n_steps);
      SmallParams<R> sp;
      sp.state = reinterpret_cast<amp*>(c->d_state);
      sp.n = n;
      sp.n_steps = (sample_here ? k1 : p->n_steps) - k0;
      sp.t = d_t + k0;
      sp.amp_scale = d_sc + k0;
      sp.slot = d_slot + k0;
      sp.phase = phase;
      sp.e0 = e0;
      sp.s0 = s0;
      sp.results = c->d_results;
      sp.inverse = 0;
      sp.measure_last = sample_here ? 0 : 1;
      if (sp.n_steps > 0 || sp.measure_last) {
        size_t ev = 0;
        BK_TRY(ev_begin(c, "small_state", &ev));
        small_state_kernel<R><<<1, kThreads, smem, c->stream>>>(sp);
        BK_CUDA(c, cudaGetLastError());
        BK_TRY(ev_end(c, ev));
      }
      if (!sample_here) break;
      BK_TRY(launch_sampling<amp>(c, reinterpret_cast<amp*>(c->d_state), n, S.sample_pt[(size_t)k1], S.shots));
      k0 = k1;
      search = k1 + 1;
      if (k1 == p->n_steps) {
        // sampling at the final step; its measurement follows in a zero-step launch
        SmallParams<R> fp = sp;
        fp.n_steps = 0;
        fp.t = d_t;
        fp.amp_scale = d_sc;
        fp.slot = d_slot + k1;
        fp.measure_last = 1;
        size_t ev = 0;
        BK_TRY(ev_begin(c, "small_state", &ev));
        small_state_kernel<R><<<1, kThreads, smem, c->stream>>>(fp);
        BK_CUDA(c, cudaGetLastError());
        BK_TRY(ev_end(c, ev));
        break;
      }
    }
    return BK_OK;
  }

  return evolve_persist<R>(c, p, S, angle_unit, tans, scales);
}

// Plain path (reference launch structure), exact gates: no scale tracking.
template <class R>
int evolve_plain(bk_ctx* c, const bk_evolve_params* p, const Schedule& S, double angle_unit) {
  using amp = typename AmpTraits<R>::amp;
  const int n = p->n;
  const uint32_t count = 1u << n;
  const uint32_t s0 = (uint32_t)(p->s0 & ((1ull << n) - 1ull));
  amp* psi = reinterpret_cast<amp*>(c->d_state);
  const unsigned th = 256;
  for (int k = 0; k <= p->n_steps; ++k) {
    const int slot = S.slot[(size_t)k];
    if (S.sample_pt[(size_t)k] >= 0) BK_TRY(launch_sampling<amp>(c, psi, n, S.sample_pt[(size_t)k], S.shots));
    if (slot >= 0) {
      size_t ev = 0;
      BK_TRY(ev_begin(c, "measure", &ev));
      measure_kernel<amp><<<kMeasureGrid, kThreads, 0, c->stream>>>(psi, c->d_E, count, (int)p->e0, s0,
                                                                     c->d_partials, c->d_ticket, c->d_results,
                                                                     slot);
      BK_CUDA(c, cudaGetLastError());
      BK_TRY(ev_end(c, ev));
    }
    if (k == p->n_steps) break;
    size_t ev = 0;
    BK_TRY(ev_begin(c, "plain_phase", &ev));
    plain_phase_kernel<amp><<<(count + th - 1) / th, th, 0, c->stream>>>(psi, c->d_E, count, angle_unit);
    BK_CUDA(c, cudaGetLastError());
    BK_TRY(ev_end(c, ev));
    // Rx(-2 g dt): entries as the reference builds them (sampler.cuh:451-457)
    const double rx = -2.0 * S.g[(size_t)k] * p->dt;
    const double cs = std::cos(rx / 2.0), sn = -std::sin(rx / 2.0);
    for (int q = 0; q < n; ++q) {
      BK_TRY(ev_begin(c, "plain_rx", &ev));
      plain_rx_kernel<amp><<<(count / 2 + th - 1) / th, th, 0, c->stream>>>(psi, count / 2, q, cs, sn);
      BK_CUDA(c, cudaGetLastError());
      BK_TRY(ev_end(c, ev));
    }
  }
  return BK_OK;
}

// ---------------------------------------------------------------------------
// adjoint gradient (csrc/bk_adjoint.cuh)
// ---------------------------------------------------------------------------
constexpr int kResetGrid = 148 * 4;

// A launch that may start while the previous kernel on the stream finishes
// (programmatic dependent launch): the kernel itself waits (griddepcontrol.wait)
// before it touches anything that kernel writes.
template <class... P, class... A>
cudaError_t launch_dependent(void (*kern)(P...), unsigned grid, unsigned block, int smem, cudaStream_t st,
                             A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = (size_t)smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

// the reverse-pass kernel for a pass kind: width 0 = the A1 pass, 1..9 = a strided pass
template <class R>
using AdjKernel = void (*)(AdjDesc<R>, int, uint32_t, int, int, int*);
template <class R, bool kWarpA1, int... W>
AdjKernel<R> adj_kernel_of(int w, std::integer_sequence<int, W...>) {
  static const AdjKernel<R> table[] = {adj_pass_kernel<R, kWarpA1, W>...};
  return table[w];
}
template <class R>
AdjKernel<R> adj_kernel(bool warp_a1, int w) {
  using Ws = std::make_integer_sequence<int, 10>;
  return warp_a1 ? adj_kernel_of<R, true>(w, Ws{}) : adj_kernel_of<R, false>(w, Ws{});
}
// the reverse A1 pass with the full complex64 phase table (complex128 has none)
template <class R>
AdjKernel<R> adj_table_kernel(bool warp_a1) {
  if constexpr (sizeof(R) == 4)
    return warp_a1 ? adj_pass_kernel<R, true, 0, true> : adj_pass_kernel<R, false, 0, true>;
  else
    return adj_kernel<R>(warp_a1, 0);
}

// Forward run with checkpoints every K steps (persistent engine), lambda_T = W
// psi_T, then the reverse sweep: per reverse step one dual A1 / S2 / S3 launch
// each, a checkpoint put back every K steps. grad_step[k] = dO/dg_k.
template <class R>
int adjoint_t(bk_ctx* c, const bk_adjoint_params* p, const std::vector<double>& g_step, int64_t e0,
              double angle_unit, int K, int n_ckpt, double* value_out, std::vector<double>* grad_step,
              bk_adjoint_stats* stats) {
  const int n = p->n, T = p->n_steps;
  constexpr bool kC64 = sizeof(R) == 4;
  const int np = kC64 ? n - 1 : n;
  const size_t n_el = 1ull << np;
  const size_t sbytes = n_el * 16;
  cudaStream_t st = c->stream;
  const uint32_t s0 = (uint32_t)(p->s0 & ((1ull << n) - 1ull));

  // forward schedule (measurement at T only) and the host scale bookkeeping
  Schedule S;
  S.g = g_step;
  S.slot.assign((size_t)T + 1, -1);
  S.slot[(size_t)T] = 0;
  S.n_meas = 1;
  S.sample_pt.assign((size_t)T + 1, -1);
  std::vector<R> tans((size_t)T), scales((size_t)T);
  std::vector<long double> lgf((size_t)T + 1, 0.0L);
  long double lg = 0.0L;
  for (int k = 0; k <= T; ++k) {
    lgf[(size_t)k] = lg;
    if (k == T) break;
    tans[(size_t)k] = (R)std::tan(g_step[(size_t)k] * p->dt);
    R sc = (R)1;
    if (lg >= (long double)kRescaleLog2) {
      sc = (R)std::ldexp(1.0, -kRescaleLog2);
      lg -= (long double)kRescaleLog2;
    }
    scales[(size_t)k] = sc;
    const long double tf = (long double)tans[(size_t)k];
    lg += 0.5L * (long double)n * std::log2(1.0L + tf * tf);
  }
  bk_evolve_params q{};
  q.n = n;
  q.precision = p->precision;
  q.method = BK_FUSED;
  q.s0 = p->s0;
  q.e0 = e0;
  q.dt = p->dt;
  q.diag_scale = p->diag_scale;
  q.n_steps = T;

  BK_CUDA(c, cudaMemsetAsync(c->d_state, 0, sbytes, st));
  if constexpr (kC64)
    set_basis_planar_kernel<<<1, 1, 0, st>>>(reinterpret_cast<float*>(c->d_state), s0);
  else
    set_basis_kernel<double2><<<1, 1, 0, st>>>(reinterpret_cast<double2*>(c->d_state), s0);
  BK_CUDA(c, cudaGetLastError());
  c->planar = kC64;
  c->have_state = false;

  cudaEvent_t ev[4];
  for (auto& e : ev) BK_CUDA(c, cudaEventCreate(&e));
  struct EvGuard {
    cudaEvent_t* e;
    ~EvGuard() {
      for (int i = 0; i < 4; ++i) cudaEventDestroy(e[i]);
    }
  } guard{ev};

  PersistRun<R> run;
  BK_TRY(persist_prepare<R>(c, &q, S, angle_unit, tans, scales, &run));
  unsigned char* ckpt = static_cast<unsigned char*>(c->d_ckpt);
  grad_step->assign((size_t)T, 0.0);
  // forward: one persistent launch per window of K steps, psi copied to a
  // checkpoint between windows; enqueued without host synchronisation
  auto enqueue_forward = [&]() -> int {
    BK_CUDA(c, cudaEventRecord(ev[0], st));
    for (int w = 0; w <= n_ckpt; ++w) {
      const int k0 = w * K, k1 = (w == n_ckpt) ? T : (w + 1) * K;
      if (w > 0)
        BK_CUDA(c, cudaMemcpyAsync(ckpt + (size_t)(w - 1) * sbytes, c->d_state, sbytes, cudaMemcpyDeviceToDevice, st));
      BK_TRY(persist_launch<R>(c, run, k0, k1 - k0, (w == n_ckpt) ? run.n_final : 0, false));
    }
    BK_CUDA(c, cudaEventRecord(ev[1], st));
    return BK_OK;
  };
  double row[4] = {0, 0, 0, 0};
  int e_fwd = 0;
  auto finish_forward = [&]() -> int {
    if (e_fwd != 0) return fail(c, BK_ERR_TIMEOUT, "persistent engine: a bounded device wait gave up (%d)", e_fwd);
    const long double f = std::exp2(-2.0L * lgf[(size_t)T]);
    const double value = (double)((long double)row[p->objective == BK_OBJ_P_LESS ? 0 : 1] * f);
    if (value_out) *value_out = value;
    float fw_ms = 0.f;
    BK_CUDA(c, cudaEventElapsedTime(&fw_ms, ev[0], ev[1]));
    if (stats) {
      stats->value = value;
      stats->norm = (double)((long double)row[2] * f);
      stats->checkpoint_every = K;
      stats->n_checkpoints = n_ckpt;
      stats->max_drift = 0.0;
      stats->forward_ms = fw_ms;
      stats->reverse_ms = 0.0;
    }
    return BK_OK;
  };
  if (T == 0) {
    BK_TRY(enqueue_forward());
    BK_CUDA(c, cudaMemcpyAsync(row, c->d_results, sizeof(row), cudaMemcpyDeviceToHost, st));
    BK_CUDA(c, cudaMemcpyAsync(&e_fwd, run.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    BK_CUDA(c, cudaStreamSynchronize(st));
    return finish_forward();
  }

  // reverse-sweep bookkeeping on the host: tangents, rescales, round-weight
  // logs, the log2 scale of both vectors at each step's cross terms, resets
  const InstDesc<R>& FD = run.D;
  // reverse pass geometry: the warp-local A1 (element bits 0-8) when chosen and
  // the strided passes can take the remaining np - 9 <= 18 bits, else the
  // forward's 12-bit A1 split
  const bool adj_warp = c->adj_a1 == 1 && np - kA1WarpBits <= 18;
  const int a1r = adj_warp ? kA1WarpBits : kElemBits;
  const int rest_r = np - a1r;
  const int w2 = adj_warp ? ((rest_r <= 9) ? rest_r : (rest_r + 1) / 2) : FD.w2;
  const int w3 = adj_warp ? rest_r - w2 : FD.w3;
  std::vector<R> t_rev((size_t)T), sc_rev((size_t)T);
  std::vector<double> lg_rev((size_t)T);
  std::vector<long double> wlog2((size_t)T);
  struct Reset {
    int after_j, ck;
    double a, b;
  };
  std::vector<Reset> resets;
  long double lp = lgf[(size_t)T], ll = lgf[(size_t)T];
  for (int j = 0; j < T; ++j) {
    const int k = T - 1 - j;
    R sc = (R)1;
    if (std::max(lp, ll) >= (long double)kRescaleLog2) {
      sc = (R)std::ldexp(1.0, -kRescaleLog2);
      lp -= (long double)kRescaleLog2;
      ll -= (long double)kRescaleLog2;
    }
    sc_rev[(size_t)j] = sc;
    t_rev[(size_t)j] = -tans[(size_t)k];
    const long double tf = (long double)tans[(size_t)k];
    const long double l2 = std::log2(1.0L + tf * tf);
    lg_rev[(size_t)j] = (double)l2;
    wlog2[(size_t)j] = lp + ll;
    lp += 0.5L * (long double)n * l2;
    ll += 0.5L * (long double)n * l2;
    if (k > 0 && k % K == 0) {
      const int m = k / K;  // checkpoint m - 1 holds psi_k
      resets.push_back(Reset{j, m - 1, (double)std::exp2(-lp), (double)std::exp2(-lgf[(size_t)k])});
      lp = lgf[(size_t)k];
    }
  }

  // device layout
  const uint32_t n_a1 = FD.n_a1, n_s2 = FD.n_s2, n_s3 = w3 > 0 ? n_a1 : 0u;
  Bump b;
  const size_t o_maps = b.take(9 * sizeof(CUtensorMap));
  const size_t o_tan = b.take((size_t)T * sizeof(R));
  const size_t o_sc = b.take((size_t)T * sizeof(R));
  const size_t o_lg = b.take((size_t)T * sizeof(double));
  const size_t o_part = b.take((size_t)(n_a1 + n_s2 + n_s3) * sizeof(double));
  const size_t o_ctr = b.take(64);
  const size_t o_cross = b.take((size_t)T * sizeof(double));
  const size_t o_dev = b.take(std::max<size_t>(resets.size(), 1) * kResetGrid * sizeof(double));
  // complex64 reverse A1 with the full phase table (BK_OPT_PHASE_TABLE)
  std::vector<float2> ptab;
  typename PhaseV<R>::params aph = run.phase;
  if constexpr (kC64)
    if (c->phase_table) BK_TRY(build_phase_table(c, n, angle_unit, &aph, &ptab));
  const size_t o_ptab = b.take(std::max<size_t>(ptab.size(), 1) * sizeof(float2));
  BK_TRY(ensure_buffer(c, &c->d_adj, &c->adj_cap, b.off));
  char* base = static_cast<char*>(c->d_adj);
  CUtensorMap* d_maps = reinterpret_cast<CUtensorMap*>(base + o_maps);
  unsigned int* ticket = reinterpret_cast<unsigned int*>(base + o_ctr);
  int* err = reinterpret_cast<int*>(base + o_ctr + 16);
  double* d_cross = reinterpret_cast<double*>(base + o_cross);
  double* d_dev = reinterpret_cast<double*>(base + o_dev);

  TmaDesc a1p, a1l, em, s2p, s2l, s3p, s3l, a1sp, a1sl;
  BK_TRY(build_amp_map(c, c->d_state, np, BK_C128, kElemBits, kElemBits, 0, &a1p));
  BK_TRY(build_amp_map(c, c->d_lam, np, BK_C128, kElemBits, kElemBits, 0, &a1l));
  BK_TRY(build_e_map(c, c->d_E, n, kC64 ? 13 : 12, &em));
  BK_TRY(build_amp_map(c, c->d_state, np, BK_C128, kElemBits - w2, a1r, w2, &s2p));
  BK_TRY(build_amp_map(c, c->d_lam, np, BK_C128, kElemBits - w2, a1r, w2, &s2l));
  if (w3 > 0) {
    BK_TRY(build_amp_map(c, c->d_state, np, BK_C128, kElemBits - w3, a1r + w2, w3, &s3p));
    BK_TRY(build_amp_map(c, c->d_lam, np, BK_C128, kElemBits - w3, a1r + w2, w3, &s3l));
  } else {
    s3p = s2p;
    s3l = s2l;
  }
  if (adj_warp) {
    BK_TRY(build_a1_swizzled_map(c, c->d_state, np, &a1sp));
    BK_TRY(build_a1_swizzled_map(c, c->d_lam, np, &a1sl));
  } else {
    a1sp = a1p;
    a1sl = a1l;
  }
  CUtensorMap maps[9] = {a1p.map, a1l.map, em.map, s2p.map, s2l.map, s3p.map, s3l.map, a1sp.map, a1sl.map};
  AdjDesc<R> A{};
  A.psi = static_cast<unsigned char*>(c->d_state);
  A.lam = static_cast<unsigned char*>(c->d_lam);
  A.map_a1 = d_maps + 0;
  A.map_e = d_maps + 2;
  A.map_s2 = d_maps + 3;
  A.map_s3 = d_maps + 5;
  A.np = np;
  A.n = n;
  A.w2 = w2;
  A.w3 = w3;
  A.a1_hi_dim = a1p.hi_dim;
  A.s2_mid_dim = s2p.mid_dim;
  A.s2_hi_dim = s2p.hi_dim;
  A.s2_mid_bits = (int)s2p.mid_bits;
  A.s3_mid_dim = w3 > 0 ? s3p.mid_dim : -1;
  A.s3_hi_dim = w3 > 0 ? s3p.hi_dim : -1;
  A.s3_mid_bits = w3 > 0 ? (int)s3p.mid_bits : 0;
  if constexpr (kC64)
    if (!ptab.empty()) aph.tab = reinterpret_cast<const float2*>(base + o_ptab);
  A.phase = aph;
  A.tan = reinterpret_cast<const R*>(base + o_tan);
  A.scale = reinterpret_cast<const R*>(base + o_sc);
  A.lg1t2 = reinterpret_cast<const double*>(base + o_lg);
  A.partials = reinterpret_cast<double*>(base + o_part);
  A.ticket = ticket;
  A.cross = d_cross;
  A.n_a1 = n_a1;
  A.n_s2 = n_s2;
  A.n_s3 = n_s3;
  A.map_a1s = d_maps + 7;
  BK_CUDA(c, cudaMemcpyAsync(d_maps, maps, sizeof(maps), cudaMemcpyHostToDevice, st));
  BK_CUDA(c, cudaMemcpyAsync(base + o_tan, t_rev.data(), (size_t)T * sizeof(R), cudaMemcpyHostToDevice, st));
  BK_CUDA(c, cudaMemcpyAsync(base + o_sc, sc_rev.data(), (size_t)T * sizeof(R), cudaMemcpyHostToDevice, st));
  BK_CUDA(c, cudaMemcpyAsync(base + o_lg, lg_rev.data(), (size_t)T * sizeof(double), cudaMemcpyHostToDevice, st));
  BK_CUDA(c, cudaMemsetAsync(base + o_ctr, 0, 64, st));
  // one kernel per pass kind: the A1 pass and a strided pass of each width used
  if (!ptab.empty())
    BK_CUDA(c, cudaMemcpyAsync(base + o_ptab, ptab.data(), ptab.size() * sizeof(float2), cudaMemcpyHostToDevice, st));
  const bool a_tab = !ptab.empty();
  const int a1_smem = a_tab ? AdjSmem::kAllocTab : AdjSmem::kAlloc;
  const AdjKernel<R> k_a1 = a_tab ? adj_table_kernel<R>(adj_warp) : adj_kernel<R>(adj_warp, 0),
                     k_s2 = adj_kernel<R>(adj_warp, w2),
                     k_s3 = adj_kernel<R>(adj_warp, w3 > 0 ? w3 : w2);
  for (AdjKernel<R> k : {k_a1, k_s2, k_s3})
    BK_TRY(allow_smem(c, reinterpret_cast<const void*>(k), k == k_a1 ? a1_smem : AdjSmem::kAlloc));
  const int ns = c->num_sms;
  const unsigned g1 = std::min<unsigned>(n_a1, (unsigned)ns), g2 = std::min<unsigned>(n_s2, (unsigned)ns),
                 g3 = std::min<unsigned>(std::max<unsigned>(n_s3, 1u), (unsigned)ns);

  // the whole gradient goes to the device back to back: forward, then the sweep
  BK_TRY(enqueue_forward());
  BK_CUDA(c, cudaEventRecord(ev[2], st));
  {
    const unsigned grid = (unsigned)std::min<size_t>((n_el + 255) / 256, (size_t)kResetGrid);
    adj_lambda_init_kernel<R><<<grid, 256, 0, st>>>(static_cast<const unsigned char*>(c->d_state),
                                                    static_cast<unsigned char*>(c->d_lam), c->d_E, (uint32_t)n_el,
                                                    p->objective, (int)e0, s0);
    BK_CUDA(c, cudaGetLastError());
  }
  size_t ri = 0;
  for (int j = 0; j < T; ++j) {
    size_t e = 0;
    BK_TRY(ev_begin(c, "adj_a1", &e));
    BK_CUDA(c, launch_dependent(k_a1, g1, kComputeThreads, a1_smem, st, A, (int)TASK_A1, (uint32_t)j, j > 0 ? 1 : 0,
                                0, err));
    BK_TRY(ev_end(c, e));
    BK_TRY(ev_begin(c, "adj_s2", &e));
    BK_CUDA(c, launch_dependent(k_s2, g2, kComputeThreads, AdjSmem::kAlloc, st, A, (int)TASK_S2, (uint32_t)j, 0,
                                w3 > 0 ? 0 : 1, err));
    BK_TRY(ev_end(c, e));
    if (w3 > 0) {
      BK_TRY(ev_begin(c, "adj_s3", &e));
      BK_CUDA(c, launch_dependent(k_s3, g3, kComputeThreads, AdjSmem::kAlloc, st, A, (int)TASK_S3, (uint32_t)j, 0,
                                  1, err));
      BK_TRY(ev_end(c, e));
    }
    if (ri < resets.size() && resets[ri].after_j == j) {
      const Reset& r = resets[ri];
      BK_TRY(ev_begin(c, "adj_reset", &e));
      adj_reset_kernel<R><<<kResetGrid, kComputeThreads, 0, st>>>(
          static_cast<unsigned char*>(c->d_state), ckpt + (size_t)r.ck * sbytes, c->d_E, (uint32_t)n_el, run.phase,
          r.a, r.b, d_dev + ri * kResetGrid);
      BK_CUDA(c, cudaGetLastError());
      BK_TRY(ev_end(c, e));
      ++ri;
    }
  }
  BK_CUDA(c, cudaEventRecord(ev[3], st));
  std::vector<double> cross((size_t)T), dev(std::max<size_t>(resets.size(), 1) * kResetGrid, 0.0);
  int e_dev = 0;
  BK_CUDA(c, cudaMemcpyAsync(cross.data(), d_cross, (size_t)T * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (!resets.empty())
    BK_CUDA(c, cudaMemcpyAsync(dev.data(), d_dev, resets.size() * kResetGrid * sizeof(double),
                               cudaMemcpyDeviceToHost, st));
  BK_CUDA(c, cudaMemcpyAsync(&e_dev, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  // the forward's result row is untouched by the sweep: read it with the rest
  BK_CUDA(c, cudaMemcpyAsync(row, c->d_results, sizeof(row), cudaMemcpyDeviceToHost, st));
  BK_CUDA(c, cudaMemcpyAsync(&e_fwd, run.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  BK_CUDA(c, cudaStreamSynchronize(st));
  BK_TRY(finish_forward());
  if (e_dev != 0) return fail(c, BK_ERR_TIMEOUT, "adjoint sweep: a bounded device wait gave up (%d)", e_dev);
  BK_TRY(collect_timing(c));
  for (int j = 0; j < T; ++j) {
    const int k = T - 1 - j;
    (*grad_step)[(size_t)k] =
        (double)(-2.0L * (long double)p->dt * (long double)cross[(size_t)j] * std::exp2(-wlog2[(size_t)j]));
  }
  if (stats) {
    float rv_ms = 0.f;
    BK_CUDA(c, cudaEventElapsedTime(&rv_ms, ev[2], ev[3]));
    stats->reverse_ms = rv_ms;
    double mx = 0.0;
    for (size_t r = 0; r < resets.size(); ++r) {
      double sacc = 0.0;
      for (int i = 0; i < kResetGrid; ++i) sacc += dev[r * kResetGrid + (size_t)i];
      mx = std::max(mx, std::sqrt(sacc));
    }
    stats->max_drift = mx;
  }
  return BK_OK;
}

int check_device_error(bk_ctx* c) {
  int e = 0;
  BK_CUDA(c, cudaMemcpyAsync(&e, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  BK_CUDA(c, cudaStreamSynchronize(c->stream));
  if (e == DEV_TIMEOUT) {
    cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream);
    cudaMemsetAsync(c->d_ticket, 0, sizeof(unsigned int), c->stream);
    cudaStreamSynchronize(c->stream);
    return fail(c, BK_ERR_TIMEOUT, "a kernel's bounded wait for its tile load gave up");
  }
  if (e != 0) return fail(c, BK_ERR_CUDA, "device error word %d", e);
  return BK_OK;
}

}  // namespace

// ============================================================================
// C ABI
// ============================================================================
extern "C" {

int bk_abi_version(void) { return BK_ABI_VERSION; }

const char* bk_status_string(int s) {
  switch (s) {
    case BK_OK: return "ok";
    case BK_ERR_INVALID: return "invalid argument";
    case BK_ERR_CUDA: return "CUDA error";
    case BK_ERR_OOM: return "out of device memory";
    case BK_ERR_TIMEOUT: return "device-side wait timed out";
    case BK_ERR_NORM: return "norm outside tolerance";
    case BK_ERR_UNSUPPORTED: return "unsupported configuration";
    case BK_ERR_NO_DEVICE: return "no usable CUDA device";
    case BK_ERR_TOO_LARGE: return "request beyond a fixed limit (bk_measure_noalloc: n <= 30)";
    default: return "unknown status";
  }
}

const char* bk_last_error(const bk_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

int bk_create(int device, bk_ctx** out) {
  if (!out) return BK_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return BK_ERR_NO_DEVICE;
  if (device < 0 || device >= ndev) return BK_ERR_INVALID;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return BK_ERR_NO_DEVICE;
  if (prop.major != 10) return BK_ERR_NO_DEVICE;  // kernels are built for sm_100a only
  if (cudaSetDevice(device) != cudaSuccess) return BK_ERR_CUDA;
  bk_ctx* c = new bk_ctx();
  c->device = device;
  c->num_sms = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&c->d_ticket, sizeof(unsigned int)) != cudaSuccess ||
      cudaMalloc(&c->d_err, sizeof(int)) != cudaSuccess ||
      cudaMalloc(&c->d_count, sizeof(unsigned long long)) != cudaSuccess) {
    bk_destroy(c);
    return BK_ERR_CUDA;
  }
  cudaMemset(c->d_ticket, 0, sizeof(unsigned int));
  cudaMemset(c->d_err, 0, sizeof(int));
  *out = c;
  return BK_OK;
}

int bk_destroy(bk_ctx* c) {
  if (!c) return BK_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (void* p : {(void*)c->d_E, c->d_state, (void*)c->d_partials, (void*)c->d_results, (void*)c->d_ticket,
                  (void*)c->d_err, (void*)c->d_count, c->d_phase, c->d_small, (void*)c->d_chunks, c->d_io,
                  (void*)c->d_rand, (void*)c->d_samples, (void*)c->d_binom, (void*)c->d_found})
    if (p) cudaFree(p);
  for (auto& kv : c->batch_E) cudaFree(kv.second);
  for (void* p : {c->d_batch_state, c->d_batch, (void*)c->d_batch_results, c->d_persist, c->d_lam, c->d_ckpt,
                  c->d_adj, c->d_descent, c->d_lz, c->d_fsmap})
    if (p) cudaFree(p);
  for (auto& e : c->ev_pool) {
    cudaEventDestroy(e.first);
    cudaEventDestroy(e.second);
  }
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return BK_OK;
}

int bk_labs_energy(int n, const uint64_t* states, int64_t count, int64_t* out) {
  if (n < 1 || n > 63 || count < 0 || (count > 0 && (!states || !out))) return BK_ERR_INVALID;
  const uint64_t m = (1ull << n) - 1ull;
  for (int64_t i = 0; i < count; ++i) out[i] = host_energy(n, states[i] & m);
  return BK_OK;
}

int bk_random_states(int n, uint64_t seed, int64_t count, uint64_t* out) {
  if (n < 1 || n > 63 || count < 0 || (count > 0 && !out)) return BK_ERR_INVALID;
  std::mt19937_64 rng(seed);
  const uint64_t m = (1ull << n) - 1ull;
  for (int64_t i = 0; i < count; ++i) out[i] = rng() & m;
  return BK_OK;
}

int bk_steepest_descent(int n, const uint64_t* starts, int64_t count, uint64_t max_evals, uint64_t* fs,
                        int64_t* fe, uint64_t* ev) {
  if (n < 2 || n > 63 || count < 0 || (count > 0 && (!starts || !fs || !fe))) return BK_ERR_INVALID;
  const uint64_t m = (1ull << n) - 1ull;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t i = 0; i < count; ++i) descend(n, starts[i] & m, max_evals, &fs[i], &fe[i], ev ? &ev[i] : nullptr);
  return BK_OK;
}

int bk_steepest_descent_gpu(bk_ctx* c, int n, const uint64_t* starts, int64_t count, uint64_t max_evals,
                            uint64_t* fs, int64_t* fe, uint64_t* ev) {
  if (!c) return BK_ERR_INVALID;
  if (n < 2 || n > 63 || count < 0 || (count > 0 && (!starts || !fs || !fe)))
    return fail(c, BK_ERR_INVALID, "steepest descent: n = %d, count = %lld", n, (long long)count);
  if (count == 0) return BK_OK;
  BK_CUDA(c, cudaSetDevice(c->device));
  const size_t cnt = (size_t)count;
  BK_TRY(ensure_buffer(c, &c->d_descent, &c->descent_cap, cnt * 32));
  uint64_t* d_start = static_cast<uint64_t*>(c->d_descent);
  uint64_t* d_fs = d_start + cnt;
  long long* d_fe = reinterpret_cast<long long*>(d_fs + cnt);
  unsigned long long* d_ev = reinterpret_cast<unsigned long long*>(d_fe + cnt);
  cudaStream_t st = c->stream;
  BK_CUDA(c, cudaMemcpyAsync(d_start, starts, cnt * 8, cudaMemcpyHostToDevice, st));
  size_t e = 0;
  BK_TRY(ev_begin(c, "descent", &e));
  const unsigned grid = (unsigned)((cnt + kDescentWarps - 1) / kDescentWarps);
  descent_kernel<<<grid, 32 * kDescentWarps, 0, st>>>(n, d_start, (long long)count,
                                                      max_evals == 0 ? ~0ull : (unsigned long long)max_evals, d_fs,
                                                      d_fe, d_ev);
  BK_CUDA(c, cudaGetLastError());
  BK_TRY(ev_end(c, e));
  BK_CUDA(c, cudaMemcpyAsync(fs, d_fs, cnt * 8, cudaMemcpyDeviceToHost, st));
  BK_CUDA(c, cudaMemcpyAsync(fe, d_fe, cnt * 8, cudaMemcpyDeviceToHost, st));
  if (ev) BK_CUDA(c, cudaMemcpyAsync(ev, d_ev, cnt * 8, cudaMemcpyDeviceToHost, st));
  BK_CUDA(c, cudaStreamSynchronize(st));
  BK_TRY(collect_timing(c));
  return BK_OK;
}

int bk_collect_minima(bk_ctx* c, int n, uint64_t seed, int64_t target_families, int64_t batch_size,
                      int64_t max_starts, bk_minimum_family* out, int64_t capacity, int64_t* n_out,
                      bk_collect_stats* stats) {
  if (!c || !n_out) return BK_ERR_INVALID;
  if (n < 3 || n > 63 || target_families < 1 || batch_size < 1 || max_starts < 1 || capacity < 0 ||
      (capacity > 0 && !out))
    return fail(c, BK_ERR_INVALID, "collect_minima: bad arguments");
  std::mt19937_64 rng(seed);
  const uint64_t m = (1ull << n) - 1ull;
  struct Fam {
    bk_minimum_family f;
    size_t order;
  };
  std::unordered_map<uint64_t, size_t> index;  // canonical state -> position in fams
  std::vector<Fam> fams;
  std::vector<uint64_t> st((size_t)batch_size), fs((size_t)batch_size), ev((size_t)batch_size);
  std::vector<int64_t> fe((size_t)batch_size);
  uint64_t total_evals = 0, total_starts = 0, batches = 0;
  int stagnant = 0;
  bool saturated = false;
  while ((int64_t)fams.size() < target_families && total_starts < (uint64_t)max_starts) {
    ++batches;
    for (auto& x : st) x = rng() & m;
    BK_TRY(bk_steepest_descent_gpu(c, n, st.data(), batch_size, 0, fs.data(), fe.data(), ev.data()));
    total_starts += (uint64_t)batch_size;
    size_t fresh = 0;
    for (size_t i = 0; i < (size_t)batch_size; ++i) {
      total_evals += ev[i];
      const uint64_t canon = host_canonical(n, fs[i]);
      auto it = index.find(canon);
      if (it == index.end()) {
        Fam f{};
        f.f.id = fams.size() + 1;
        f.f.canonical_state = canon;
        f.f.sample_state = fs[i];
        f.f.energy = fe[i];
        f.f.times_visited = 1;
        f.f.evals_to_first_find = total_evals;
        f.order = fams.size();
        index.emplace(canon, fams.size());
        fams.push_back(f);
        ++fresh;
        if ((int64_t)fams.size() >= target_families) break;
      } else {
        fams[it->second].f.times_visited++;
      }
    }
    if (fresh == 0) {
      if (++stagnant >= 4) {
        saturated = true;
        break;
      }
    } else {
      stagnant = 0;
    }
  }
  // deepest traps first, then the most visited; discovery order breaks the remaining ties
  std::stable_sort(fams.begin(), fams.end(), [](const Fam& a, const Fam& b) {
    if (a.f.energy != b.f.energy) return a.f.energy < b.f.energy;
    return a.f.times_visited > b.f.times_visited;
  });
  *n_out = (int64_t)fams.size();
  for (size_t i = 0; i < fams.size() && (int64_t)i < capacity; ++i) {
    out[i] = fams[i].f;
    out[i].id = i + 1;
  }
  if (stats) {
    stats->total_starts = total_starts;
    stats->total_evals = total_evals;
    stats->batches = batches;
    stats->saturated = saturated ? 1 : 0;
  }
  return BK_OK;
}

int bk_select_trap(int n, uint64_t seed, int32_t n_descents, double quantile, uint64_t* bits, int64_t* e0) {
  if (n < 3 || n > 63 || n_descents <= 0 || !(quantile >= 0.0 && quantile <= 1.0) || !bits || !e0)
    return BK_ERR_INVALID;
  std::vector<uint64_t> st((size_t)n_descents), fs((size_t)n_descents);
  std::vector<int64_t> fe((size_t)n_descents);
  BK_TRY(bk_random_states(n, seed, n_descents, st.data()));
  BK_TRY(bk_steepest_descent(n, st.data(), n_descents, 0, fs.data(), fe.data(), nullptr));
  const int64_t opt = optimal_energy(n);
  std::vector<int64_t> kept;
  for (int64_t e : fe)
    if (opt < 0 || e > opt) kept.push_back(e);
  if (kept.empty()) return BK_ERR_UNSUPPORTED;  // every descent reached a global optimum
  std::sort(kept.begin(), kept.end());
  const int64_t thr = kept[(size_t)std::floor(quantile * (double)(kept.size() - 1))];
  for (int i = 0; i < n_descents; ++i) {
    if ((opt < 0 || fe[(size_t)i] > opt) && fe[(size_t)i] <= thr) {
      *bits = fs[(size_t)i];
      *e0 = fe[(size_t)i];
      return BK_OK;
    }
  }
  return BK_ERR_UNSUPPORTED;
}

int bk_energy_table(bk_ctx* c, int n, uint16_t* host_out) {
  if (!c) return BK_ERR_INVALID;
  if (n < 1 || n > kMaxN) return fail(c, BK_ERR_UNSUPPORTED, "n = %d outside [1, %d]", n, kMaxN);
  BK_CUDA(c, cudaSetDevice(c->device));
  BK_TRY(ensure_energy(c, n));
  if (host_out)
    BK_CUDA(c, cudaMemcpyAsync(host_out, c->d_E, (1ull << n) * 2, cudaMemcpyDeviceToHost, c->stream));
  BK_CUDA(c, cudaStreamSynchronize(c->stream));
  return BK_OK;
}

int bk_p_blind(bk_ctx* c, int n, int64_t e0, uint64_t* count_out, double* p_out) {
  if (!c) return BK_ERR_INVALID;
  if (n < 1 || n > kMaxN) return fail(c, BK_ERR_UNSUPPORTED, "n = %d outside [1, %d]", n, kMaxN);
  BK_CUDA(c, cudaSetDevice(c->device));
  BK_TRY(ensure_energy(c, n));
  const uint32_t count = 1u << n;
  BK_CUDA(c, cudaMemsetAsync(c->d_count, 0, sizeof(unsigned long long), c->stream));
  const int e = (int)std::min<int64_t>(std::max<int64_t>(e0, -1), 1 << 20);
  count_below_kernel<<<kMeasureGrid, 256, 0, c->stream>>>(c->d_E, count, e, c->d_count);
  BK_CUDA(c, cudaGetLastError());
  unsigned long long h = 0;
  BK_CUDA(c, cudaMemcpyAsync(&h, c->d_count, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  BK_CUDA(c, cudaStreamSynchronize(c->stream));
  if (count_out) *count_out = h;
  if (p_out) *p_out = (double)h / (double)count;
  return BK_OK;
}

int bk_set_option(bk_ctx* c, int option, int64_t value) {
  if (!c) return BK_ERR_INVALID;
  switch (option) {
    case BK_OPT_ENGINE_MODE:
      if (value < 0 || value > 3) return fail(c, BK_ERR_INVALID, "engine mode %lld", (long long)value);
      c->engine_mode = (int)value;
      return BK_OK;
    case BK_OPT_SLAB_LAG:
      if (value < 1 || value > 64) return fail(c, BK_ERR_INVALID, "slab lag %lld", (long long)value);
      c->slab_lag = (int)value;
      return BK_OK;
    case BK_OPT_SPLIT_W2:
      if (value < 0 || value > 9) return fail(c, BK_ERR_INVALID, "S2 width %lld", (long long)value);
      c->force_w2 = (int)value;
      return BK_OK;
    case BK_OPT_E_SOURCE:
      if (value != 0 && value != 1) return fail(c, BK_ERR_INVALID, "E source %lld", (long long)value);
      c->e_recompute = (int)value;
      return BK_OK;
    case BK_OPT_A1_WIDE:
      if (value < 0 || value > 3) return fail(c, BK_ERR_INVALID, "A1 kernel %lld", (long long)value);
      c->a1_wide = (int)value;
      return BK_OK;
    case BK_OPT_ADJ_A1:
      if (value != 0 && value != 1) return fail(c, BK_ERR_INVALID, "adjoint A1 %lld", (long long)value);
      c->adj_a1 = (int)value;
      return BK_OK;
    case BK_OPT_WAIT_POLLS:
      if (value != 0 && (value < 1000 || value > (int64_t)kWaitPolls * 4))
        return fail(c, BK_ERR_INVALID, "wait polls %lld", (long long)value);
      c->wait_polls = (uint32_t)value;
      return BK_OK;
    case BK_OPT_PHASE_TABLE:
      if (value != 0 && value != 1) return fail(c, BK_ERR_INVALID, "phase table %lld", (long long)value);
      c->phase_table = (int)value;
      return BK_OK;
    case BK_OPT_TEST_HOLD_STEP:
      if (value < -1 || value > (int64_t)1 << 30) return fail(c, BK_ERR_INVALID, "hold step %lld", (long long)value);
      c->hold_step = value;
      return BK_OK;
    default:
      return fail(c, BK_ERR_INVALID, "unknown option %d", option);
  }
}

int bk_get_option(const bk_ctx* c, int option, int64_t* value) {
  if (!c || !value) return BK_ERR_INVALID;
  switch (option) {
    case BK_OPT_ENGINE_MODE: *value = c->engine_mode; return BK_OK;
    case BK_OPT_SLAB_LAG: *value = c->slab_lag; return BK_OK;
    case BK_OPT_SPLIT_W2: *value = c->force_w2; return BK_OK;
    case BK_OPT_E_SOURCE: *value = c->e_recompute; return BK_OK;
    case BK_OPT_A1_WIDE: *value = c->a1_wide; return BK_OK;
    case BK_OPT_ADJ_A1: *value = c->adj_a1; return BK_OK;
    case BK_OPT_WAIT_POLLS: *value = c->wait_polls; return BK_OK;
    case BK_OPT_TEST_HOLD_STEP: *value = c->hold_step; return BK_OK;
    case BK_OPT_PHASE_TABLE: *value = c->phase_table; return BK_OK;
    default: return BK_ERR_INVALID;
  }
}

int bk_stream(bk_ctx* c, void** out) {
  if (!c || !out) return BK_ERR_INVALID;
  *out = reinterpret_cast<void*>(c->stream);
  return BK_OK;
}

int bk_set_kernel_timing(bk_ctx* c, int enabled) {
  if (!c) return BK_ERR_INVALID;
  c->timing = enabled != 0;
  c->timings.clear();
  c->timing_index.clear();
  c->ev_marks.clear();
  c->ev_used = 0;
  return BK_OK;
}

int bk_kernel_timing(bk_ctx* c, int index, const char** name, int64_t* launches, double* total_ms) {
  if (!c) return BK_ERR_INVALID;
  if (index < 0 || index >= (int)c->timings.size()) return BK_ERR_INVALID;
  if (name) *name = c->timings[(size_t)index].name.c_str();
  if (launches) *launches = c->timings[(size_t)index].launches;
  if (total_ms) *total_ms = c->timings[(size_t)index].total_ms;
  return BK_OK;
}

int bk_evolve(bk_ctx* c, const bk_evolve_params* p, double* p_less, double* d_h, double* norm) {
  if (!c || !p) return BK_ERR_INVALID;
  if (p->n < 1 || p->n > kMaxN) return fail(c, BK_ERR_UNSUPPORTED, "n = %d outside [1, %d]", p->n, kMaxN);
  if (p->precision != BK_C64 && p->precision != BK_C128) return fail(c, BK_ERR_INVALID, "precision %d", p->precision);
  if (p->method != BK_FUSED && p->method != BK_PLAIN) return fail(c, BK_ERR_INVALID, "method %d", p->method);
  if (p->ordering != BK_ORDER_REFERENCE && p->ordering != BK_ORDER_STRANG)
    return fail(c, BK_ERR_INVALID, "ordering %d", p->ordering);
  if (p->n_steps < 0) return fail(c, BK_ERR_INVALID, "n_steps %d", p->n_steps);
  if (!is_finite(p->dt) || !is_finite(p->diag_scale)) return fail(c, BK_ERR_INVALID, "dt / diag_scale not finite");
  if (p->g == nullptr && !is_finite(p->g_const)) return fail(c, BK_ERR_INVALID, "g_const not finite");
  const int n = p->n;
  Schedule S;
  S.g.resize((size_t)p->n_steps);
  for (int k = 0; k < p->n_steps; ++k) {
    S.g[(size_t)k] = p->g ? p->g[k] : p->g_const;
    if (!is_finite(S.g[(size_t)k])) return fail(c, BK_ERR_INVALID, "g[%d] not finite", k);
    if (std::cos(S.g[(size_t)k] * p->dt) == 0.0) return fail(c, BK_ERR_INVALID, "cos(g dt) = 0 at step %d", k);
  }
  S.slot.assign((size_t)p->n_steps + 1, -1);
  for (int k = 0; k <= p->n_steps; ++k)
    if (p->measure == nullptr || p->measure[k]) S.slot[(size_t)k] = S.n_meas++;
  if (S.n_meas > 0 && (!p_less || !d_h)) return fail(c, BK_ERR_INVALID, "output arrays are NULL");
  S.sample_pt.assign((size_t)p->n_steps + 1, -1);
  if (p->sample != nullptr) {
    if (p->shots <= 0 || !p->randnums || !p->samples_out)
      return fail(c, BK_ERR_INVALID, "sampling needs shots > 0, randnums and samples_out");
    for (int k = 0; k <= p->n_steps; ++k)
      if (p->sample[k]) S.sample_pt[(size_t)k] = S.n_pts++;
    S.shots = p->shots;
  }

  int64_t e0 = p->e0;
  if (e0 < 0) BK_TRY(bk_labs_energy(n, &p->s0, 1, &e0));
  bk_evolve_params q = *p;
  q.e0 = e0;
  const double angle_unit = (p->diag_scale > 0.0) ? p->dt * p->diag_scale : p->dt / (double)n;

  BK_CUDA(c, cudaSetDevice(c->device));
  BK_TRY(ensure_energy(c, n));
  BK_TRY(ensure_state(c, n, p->precision));
  const int T = tile_bits(p->precision);
  const size_t grid = (n > T) ? (1ull << (n - T)) : 1;
  BK_TRY(ensure_buffer(c, reinterpret_cast<void**>(&c->d_partials), &c->partials_cap,
                       3 * std::max<size_t>(grid, kMeasureGrid) * sizeof(double)));
  BK_TRY(ensure_buffer(c, reinterpret_cast<void**>(&c->d_results), &c->results_cap,
                       4 * std::max<size_t>((size_t)S.n_meas, 1) * sizeof(double)));
  if (S.n_pts > 0) {
    const size_t draws = (size_t)S.n_pts * (size_t)S.shots;
    BK_TRY(ensure_buffer(c, reinterpret_cast<void**>(&c->d_rand), &c->rand_cap, draws * sizeof(double)));
    BK_TRY(ensure_buffer(c, reinterpret_cast<void**>(&c->d_samples), &c->samples_cap, draws * sizeof(uint64_t)));
    BK_CUDA(c, cudaMemcpyAsync(c->d_rand, p->randnums, draws * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  }
  BK_CUDA(c, cudaMemsetAsync(c->d_ticket, 0, sizeof(unsigned int), c->stream));
  BK_CUDA(c, cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
  BK_CUDA(c, cudaMemsetAsync(c->d_state, 0, (1ull << n) * amp_bytes(p->precision), c->stream));
  const uint32_t s0 = (uint32_t)(p->s0 & ((1ull << n) - 1ull));
  c->planar = (p->precision == BK_C64 && p->method == BK_FUSED && n > 13);
  if (c->planar)
    set_basis_planar_kernel<<<1, 1, 0, c->stream>>>(reinterpret_cast<float*>(c->d_state), s0);
  else if (p->precision == BK_C64)
    set_basis_kernel<float2><<<1, 1, 0, c->stream>>>(reinterpret_cast<float2*>(c->d_state), s0);
  else
    set_basis_kernel<double2><<<1, 1, 0, c->stream>>>(reinterpret_cast<double2*>(c->d_state), s0);
  BK_CUDA(c, cudaGetLastError());

  std::vector<long double> row_log2((size_t)S.n_meas, 0.0L);
  long double final_log2 = 0.0L;
  c->have_state = false;
  if (p->method == BK_PLAIN) {
    if (p->precision == BK_C64)
      BK_TRY(evolve_plain<float>(c, &q, S, angle_unit));
    else
      BK_TRY(evolve_plain<double>(c, &q, S, angle_unit));
  } else {
    if (p->precision == BK_C64)
      BK_TRY(evolve_fused<float>(c, &q, S, angle_unit, &row_log2, &final_log2));
    else
      BK_TRY(evolve_fused<double>(c, &q, S, angle_unit, &row_log2, &final_log2));
  }
  std::vector<double> rows(4 * (size_t)S.n_meas);
  if (S.n_meas > 0)
    BK_CUDA(c, cudaMemcpyAsync(rows.data(), c->d_results, rows.size() * sizeof(double), cudaMemcpyDeviceToHost,
                               c->stream));
  if (S.n_pts > 0)
    BK_CUDA(c, cudaMemcpyAsync(p->samples_out, c->d_samples, (size_t)S.n_pts * S.shots * sizeof(uint64_t),
                               cudaMemcpyDeviceToHost, c->stream));
  BK_TRY(check_device_error(c));
  BK_TRY(collect_timing(c));
  c->have_state = true;
  c->last_planar = c->planar;
  c->last_n = n;
  c->last_prec = p->precision;
  c->last_ordering = p->ordering;
  c->last_log2_scale = final_log2;
  c->last_angle_unit = angle_unit;
  int status = BK_OK;
  for (int m = 0; m < S.n_meas; ++m) {
    const long double f = std::exp2(-2.0L * row_log2[(size_t)m]);
    // complex64 results are the expectation values of the normalised state,
    // sum |psi_s|^2 w_s / sum |psi_s|^2: FP32 rounding of the amplitudes makes
    // |psi|^2 random-walk away from 1 (~1e-6 over 2000 steps at N = 28), which
    // would otherwise scale <d_H> (~15) by the same factor. complex128 keeps its
    // norm to ~1e-14 and returns the reference's unnormalised sums.
    const long double nrm = (p->precision == BK_C64 && rows[4 * (size_t)m + 2] > 0.0)
                                ? (long double)rows[4 * (size_t)m + 2] * f : 1.0L;
    p_less[m] = (double)((long double)rows[4 * (size_t)m + 0] * f / nrm);
    d_h[m] = (double)((long double)rows[4 * (size_t)m + 1] * f / nrm);
    const double nn = (double)((long double)rows[4 * (size_t)m + 2] * f);
    if (norm) norm[m] = nn;
    if (p->norm_tol > 0.0 && !(std::fabs(nn - 1.0) <= p->norm_tol)) status = BK_ERR_NORM;
  }
  if (status == BK_ERR_NORM) return fail(c, BK_ERR_NORM, "norm left the tolerance band %g", p->norm_tol);
  return BK_OK;
}

int bk_adjoint(bk_ctx* c, const bk_adjoint_params* p, double* value_out, double* grad_out,
               double* grad_steps_out, bk_adjoint_stats* stats) {
  if (!c || !p) return BK_ERR_INVALID;
  if (p->precision != BK_C64 && p->precision != BK_C128) return fail(c, BK_ERR_INVALID, "precision %d", p->precision);
  const int nmin = p->precision == BK_C64 ? 14 : 13;
  if (p->n < nmin || p->n > kMaxN)
    return fail(c, BK_ERR_UNSUPPORTED, "adjoint: n = %d outside [%d, %d] for this precision", p->n, nmin, kMaxN);
  if (p->n_steps < 0 || p->n_segments < 1) return fail(c, BK_ERR_INVALID, "n_steps / n_segments");
  if (p->objective != BK_OBJ_P_LESS && p->objective != BK_OBJ_D_H)
    return fail(c, BK_ERR_INVALID, "objective %d", p->objective);
  if (!p->g || !grad_out) return fail(c, BK_ERR_INVALID, "g and grad_out must not be NULL");
  if (!is_finite(p->dt) || !is_finite(p->diag_scale)) return fail(c, BK_ERR_INVALID, "dt / diag_scale not finite");
  if (!p->segment_of_step && p->n_steps % p->n_segments != 0)
    return fail(c, BK_ERR_INVALID, "n_steps %d is not a multiple of n_segments %d", p->n_steps, p->n_segments);
  const int n = p->n, T = p->n_steps;
  std::vector<int> seg((size_t)T);
  std::vector<double> g_step((size_t)T);
  for (int k = 0; k < T; ++k) {
    seg[(size_t)k] = p->segment_of_step ? p->segment_of_step[k] : k / (T / p->n_segments);
    if (seg[(size_t)k] < 0 || seg[(size_t)k] >= p->n_segments)
      return fail(c, BK_ERR_INVALID, "segment_of_step[%d] = %d", k, seg[(size_t)k]);
    g_step[(size_t)k] = p->g[seg[(size_t)k]];
    if (!is_finite(g_step[(size_t)k])) return fail(c, BK_ERR_INVALID, "g of segment %d not finite", seg[(size_t)k]);
    if (std::cos(g_step[(size_t)k] * p->dt) == 0.0) return fail(c, BK_ERR_INVALID, "cos(g dt) = 0 at step %d", k);
  }
  int64_t e0 = p->e0;
  if (e0 < 0) BK_TRY(bk_labs_energy(n, &p->s0, 1, &e0));
  const double angle_unit = (p->diag_scale > 0.0) ? p->dt * p->diag_scale : p->dt / (double)n;
  BK_CUDA(c, cudaSetDevice(c->device));
  BK_TRY(ensure_energy(c, n));
  BK_TRY(ensure_state(c, n, p->precision));
  BK_TRY(ensure_buffer(c, reinterpret_cast<void**>(&c->d_results), &c->results_cap, 4 * sizeof(double)));
  BK_CUDA(c, cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
  const size_t sbytes = (1ull << n) * amp_bytes(p->precision);
  // checkpoints: every K steps strictly inside (0, T); K enlarged until they fit
  size_t free_b = 0, total_b = 0;
  BK_CUDA(c, cudaMemGetInfo(&free_b, &total_b));
  const size_t reserve = (size_t)1 << 30;
  const size_t avail = free_b + c->lam_cap + c->ckpt_cap;
  if (avail < sbytes + reserve) return fail(c, BK_ERR_OOM, "adjoint: no room for the adjoint statevector");
  int K = p->checkpoint_every;
  const bool auto_k = K <= 0;
  if (auto_k) K = 128;
  auto n_ck = [&](int k) { return T > 0 ? (T - 1) / k : 0; };
  while (sbytes * (size_t)(1 + n_ck(K)) + reserve > avail) {
    if (!auto_k) return fail(c, BK_ERR_OOM, "adjoint: %d checkpoints of %zu bytes do not fit", n_ck(K), sbytes);
    K *= 2;
  }
  const int n_ckpt = n_ck(K);
  BK_TRY(ensure_buffer(c, &c->d_lam, &c->lam_cap, sbytes));
  if (n_ckpt > 0) BK_TRY(ensure_buffer(c, &c->d_ckpt, &c->ckpt_cap, sbytes * (size_t)n_ckpt));
  std::vector<double> gs;
  if (p->precision == BK_C64)
    BK_TRY(adjoint_t<float>(c, p, g_step, e0, angle_unit, K, n_ckpt, value_out, &gs, stats));
  else
    BK_TRY(adjoint_t<double>(c, p, g_step, e0, angle_unit, K, n_ckpt, value_out, &gs, stats));
  for (int j = 0; j < p->n_segments; ++j) grad_out[j] = 0.0;
  for (int k = 0; k < T; ++k) grad_out[seg[(size_t)k]] += gs[(size_t)k];
  if (grad_steps_out)
    for (int k = 0; k < T; ++k) grad_steps_out[k] = gs[(size_t)k];
  return check_device_error(c);
}

int bk_d_min(bk_ctx* c, int n, uint64_t bits, int64_t target, int max_d, int* d_out) {
  if (!c || !d_out) return BK_ERR_INVALID;
  if (n < 1 || n > kMaxN) return fail(c, BK_ERR_UNSUPPORTED, "n = %d outside [1, %d]", n, kMaxN);
  const uint64_t m = (1ull << n) - 1ull;
  const uint64_t sb = bits & m;
  if (target < 0) target = host_energy(n, sb);
  const int not_found = (max_d > 0) ? (max_d + 1) : n;
  const int64_t opt = optimal_energy(n);
  if (opt >= 0 && target <= opt) {
    *d_out = not_found;
    return BK_OK;
  }
  BK_CUDA(c, cudaSetDevice(c->device));
  if (!c->d_binom) {
    std::vector<unsigned long long> b(32 * 32, 0ull);
    for (int i = 0; i < 32; ++i) {
      b[(size_t)i * 32] = 1;
      for (int k = 1; k <= i; ++k) b[(size_t)i * 32 + k] = b[(size_t)(i - 1) * 32 + k - 1] + (k < i ? b[(size_t)(i - 1) * 32 + k] : 0);
    }
    BK_CUDA(c, cudaMalloc(&c->d_binom, b.size() * sizeof(unsigned long long)));
    BK_CUDA(c, cudaMalloc(&c->d_found, sizeof(int)));
    BK_CUDA(c, cudaMemcpy(c->d_binom, b.data(), b.size() * sizeof(unsigned long long), cudaMemcpyHostToDevice));
  }
  const int limit = (max_d > 0 && max_d <= n) ? max_d : n;
  for (int d = 1; d <= limit; ++d) {
    if (d == n) {  // the full flip is the only weight-n mask
      *d_out = (host_energy(n, sb ^ m) < target) ? n : not_found;
      return BK_OK;
    }
    unsigned long long count = 1;
    for (int k = 1; k <= d; ++k) count = count * (unsigned long long)(n - d + k) / (unsigned long long)k;
    BK_CUDA(c, cudaMemsetAsync(c->d_found, 0, sizeof(int), c->stream));
    const unsigned long long blocks = std::min<unsigned long long>((count + 255) / 256, 148ull * 16);
    dmin_sphere_kernel<<<(unsigned)blocks, 256, 0, c->stream>>>(n, (uint32_t)sb, (int)target, d, count,
                                                                 c->d_binom, c->d_found);
    BK_CUDA(c, cudaGetLastError());
    int found = 0;
    BK_CUDA(c, cudaMemcpyAsync(&found, c->d_found, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    BK_CUDA(c, cudaStreamSynchronize(c->stream));
    if (found) {
      *d_out = d;
      return BK_OK;
    }
  }
  *d_out = not_found;
  return BK_OK;
}

void bk_sampling_result_release(bk_sampling_result* r) {
  if (!r) return;
  free(r->unique_basis);
  free(r->seed_stats);
  free(r->time_points);
  free(r->p_less_history);
  free(r->dh_history);
  std::memset(r, 0, sizeof(*r));
}

int bk_sampler_run(bk_ctx* c, const bk_sampler_config* cfg, uint64_t start_bits, bk_sampling_result* out) {
  if (!c || !cfg || !out) return BK_ERR_INVALID;
  std::memset(out, 0, sizeof(*out));
  const int n = cfg->n;
  // reference: sampler.cuh:416-418 (n > 30 is out of the statevector backend's range)
  if (n > 30) return fail(c, BK_ERR_UNSUPPORTED, "statevector backend supports n <= 30 (got %d)", n);
  if (n < 1) return fail(c, BK_ERR_INVALID, "n = %d", n);
  if (!(cfg->dt > 0.0) || !is_finite(cfg->dt) || !is_finite(cfg->t_max) || !is_finite(cfg->g) ||
      !is_finite(cfg->t_start) || !is_finite(cfg->dt_sample) || !is_finite(cfg->dt_trajectory))
    return fail(c, BK_ERR_INVALID, "non-finite or non-positive time parameters");
  const uint64_t m = (1ull << n) - 1ull;
  const int64_t E0 = host_energy(n, start_bits & m);
  out->start_energy = E0;
  int dmin = 0;
  BK_TRY(bk_d_min(c, n, start_bits, E0, -1, &dmin));
  out->d_min = dmin;
  uint64_t below = 0;
  BK_TRY(bk_p_blind(c, n, E0, &below, &out->p_blind));

  // ---- schedule (sampler.cuh:496-602): measurement and sampling flags per step
  const int T = (int)std::round(cfg->t_max / cfg->dt);
  if (T < 0 || T > 100000000) return fail(c, BK_ERR_INVALID, "t_max / dt gives %d steps", T);
  const double sample_interval = (cfg->dt_sample > 0.0) ? cfg->dt_sample
                                                        : (cfg->t_max / std::max(1, cfg->num_sample_points));
  double next_sample = cfg->t_start;
  const double traj_interval = (cfg->dt_trajectory > 0.0) ? cfg->dt_trajectory : cfg->dt;
  double next_traj = 0.0;
  const double sample_end = (cfg->num_sample_points > 1 && cfg->dt_sample > 0.0)
                                ? (cfg->t_start + (cfg->num_sample_points - 1) * cfg->dt_sample)
                                : cfg->t_max;
  int taken = 0;
  std::vector<uint8_t> meas((size_t)T + 1, 0), samp((size_t)T + 1, 0);
  std::vector<double> times;
  std::vector<int> sample_steps;
  for (int step = 0; step <= T; ++step) {
    const double t = step * cfg->dt;
    if (cfg->record_trajectory) {
      if (t >= next_traj - 1e-9 && next_traj <= cfg->t_max + 1e-9) {
        meas[(size_t)step] = 1;
        times.push_back(t);
        next_traj += traj_interval;
      }
    } else if (cfg->track_p_less) {
      if (t >= next_sample - 1e-9 && next_sample <= cfg->t_max + 1e-9) {
        meas[(size_t)step] = 1;
        times.push_back(t);
      }
    }
    if (cfg->shots_per_point > 0 && t >= cfg->t_start - 1e-9 && t >= next_sample - 1e-9 &&
        next_sample <= sample_end + 1e-9 && (cfg->num_sample_points <= 0 || taken < cfg->num_sample_points)) {
      ++taken;
      samp[(size_t)step] = 1;
      sample_steps.push_back(step);
      next_sample += sample_interval;
    } else if (cfg->shots_per_point == 0 && !cfg->record_trajectory && cfg->track_p_less &&
               t >= next_sample - 1e-9 && next_sample <= cfg->t_max + 1e-9) {
      next_sample += sample_interval;
    }
  }

  // ---- random numbers in the reference's order (sampler.cuh:476-487, 567-568)
  const int shots = std::max(1, cfg->shots_per_point);
  const int n_seeds = std::max(1, cfg->num_sampling_seeds);
  std::vector<std::mt19937_64> rngs((size_t)n_seeds);
  for (int s = 0; s < n_seeds; ++s) rngs[(size_t)s].seed(cfg->seed + (uint64_t)s * cfg->seed_stride);
  std::uniform_real_distribution<double> dist(0.0, 1.0);
  const size_t per_point = (size_t)n_seeds * (size_t)shots;
  std::vector<double> rnd(sample_steps.size() * per_point);
  for (size_t pt = 0; pt < sample_steps.size(); ++pt)
    for (int s = 0; s < n_seeds; ++s)
      for (int i = 0; i < shots; ++i) rnd[pt * per_point + (size_t)s * shots + (size_t)i] = dist(rngs[(size_t)s]);
  std::vector<uint64_t> drawn(rnd.size());

  bk_evolve_params ep;
  std::memset(&ep, 0, sizeof(ep));
  ep.n = n;
  ep.precision = cfg->precision;
  ep.method = cfg->method;
  ep.ordering = BK_ORDER_REFERENCE;
  ep.s0 = start_bits & m;
  ep.e0 = E0;
  ep.dt = cfg->dt;
  ep.diag_scale = 0.0;
  ep.n_steps = T;
  ep.g = nullptr;
  ep.g_const = cfg->g;
  ep.measure = meas.data();
  if (!sample_steps.empty()) {
    ep.sample = samp.data();
    ep.shots = (int32_t)per_point;
    ep.randnums = rnd.data();
    ep.samples_out = drawn.data();
  }
  std::vector<double> pl(times.size()), dh(times.size());
  BK_TRY(bk_evolve(c, &ep, pl.data(), dh.data(), nullptr));

  // ---- per-shot energy and Hamming distance on the device (the drawn states are
  // still there), statistics on the host (sampler.cuh:575-597)
  const size_t n_draws = drawn.size();
  std::vector<int> shot_e(n_draws), shot_d(n_draws);
  if (n_draws > 0) {
    void* scratch = nullptr;
    BK_CUDA(c, cudaMallocAsync(&scratch, n_draws * 2 * sizeof(int), c->stream));
    int* d_e = static_cast<int*>(scratch);
    int* d_f = d_e + n_draws;
    shot_stats_kernel<<<(unsigned)((n_draws + 255) / 256), 256, 0, c->stream>>>(
        c->d_samples, (long long)n_draws, n, (unsigned long long)(start_bits & ((1ull << n) - 1ull)), d_e, d_f);
    const cudaError_t le = cudaGetLastError();
    cudaError_t ce = cudaMemcpyAsync(shot_e.data(), d_e, n_draws * sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(shot_d.data(), d_f, n_draws * sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    cudaFreeAsync(scratch, c->stream);
    BK_CUDA(c, le);
    BK_CUDA(c, ce);
    BK_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  std::vector<bk_seed_stats> ss((size_t)n_seeds);
  for (int s = 0; s < n_seeds; ++s) {
    std::memset(&ss[(size_t)s], 0, sizeof(bk_seed_stats));
    ss[(size_t)s].seed = cfg->seed + (uint64_t)s * cfg->seed_stride;
    ss[(size_t)s].best_energy = E0;
  }
  std::unordered_set<uint64_t> uniq;
  uint64_t flips_primary = 0;
  for (size_t pt = 0; pt < sample_steps.size(); ++pt) {
    for (int s = 0; s < n_seeds; ++s) {
      uint64_t flips = 0;
      for (int i = 0; i < shots; ++i) {
        const size_t k = pt * per_point + (size_t)s * shots + (size_t)i;
        const uint64_t b = drawn[k];
        uniq.insert(b);
        const int d = shot_d[k];
        flips += (uint64_t)d;
        if (s == 0) flips_primary += (uint64_t)d;
        const int64_t e = shot_e[k];
        if (e < ss[(size_t)s].best_energy) ss[(size_t)s].best_energy = e;
        if (e < E0) {
          ss[(size_t)s].improved_shots++;
          if (s == 0) out->improved_shots++;
        }
      }
      ss[(size_t)s].total_shots_collected += (uint64_t)shots;
      ss[(size_t)s].mean_hamming_flips += (double)flips;
    }
    out->total_shots_collected += (uint64_t)shots;
  }

  // ---- post-processing (sampler.cuh:621-683)
  out->total_evals = out->total_shots_collected;
  if (out->total_shots_collected > 0) {
    out->mean_hamming_flips = (double)flips_primary / (double)out->total_shots_collected;
    out->success_rate = (double)out->improved_shots / (double)out->total_shots_collected;
    out->per_eval_rate = out->total_evals > 0 ? (double)out->improved_shots / (double)out->total_evals : 0.0;
  }
  for (auto& x : ss) {
    if (x.total_shots_collected > 0) {
      x.success_rate = (double)x.improved_shots / (double)x.total_shots_collected;
      x.per_eval_rate = x.success_rate;
      x.mean_hamming_flips /= (double)x.total_shots_collected;
    }
  }
  const size_t np = times.size();
  for (size_t i = 0; i < np; ++i)
    if (pl[i] > out->peak_p_less) {
      out->peak_p_less = pl[i];
      out->peak_time = times[i];
    }
  if (np > 0) {
    size_t first_drop = np - 1;
    for (size_t i = 1; i < np; ++i)
      if (pl[i] < pl[i - 1]) {
        first_drop = i - 1;
        break;
      }
    const double tp = times[first_drop];
    out->initial_rise_rate_avg = (tp > 0.0) ? pl[first_drop] / tp : 0.0;
    double mx = (times[0] > 1e-9) ? pl[0] / times[0] : 0.0;
    for (size_t i = 0; i < first_drop; ++i) {
      const double h = times[i + 1] - times[i];
      if (h > 1e-9) mx = std::max(mx, (pl[i + 1] - pl[i]) / h);
    }
    out->initial_rise_rate_max = mx;
  }
  {
    const double a0 = cfg->t_start;
    const double a1 = (cfg->num_sample_points > 1 && cfg->dt_sample > 0.0)
                          ? (cfg->t_start + (cfg->num_sample_points - 1) * cfg->dt_sample)
                          : cfg->t_max;
    double sum = 0.0;
    size_t cnt = 0;
    for (size_t i = 0; i < np; ++i)
      if (times[i] >= a0 - 1e-9 && times[i] <= a1 + 1e-9) {
        sum += dh[i];
        ++cnt;
      }
    out->window_avg_dh = cnt > 0 ? sum / (double)cnt : (np > 0 ? dh[np - 1] : 0.0);
  }

  // ---- hand the arrays over (library-owned until bk_sampling_result_release)
  std::vector<uint64_t> ub(uniq.begin(), uniq.end());
  std::sort(ub.begin(), ub.end());
  out->unique_basis_size = (int64_t)ub.size();
  out->n_points = (int64_t)np;
  out->n_seed_stats = n_seeds;
  out->unique_basis = static_cast<uint64_t*>(malloc(std::max<size_t>(ub.size(), 1) * sizeof(uint64_t)));
  out->seed_stats = static_cast<bk_seed_stats*>(malloc(ss.size() * sizeof(bk_seed_stats)));
  out->time_points = static_cast<double*>(malloc(std::max<size_t>(np, 1) * sizeof(double)));
  out->p_less_history = static_cast<double*>(malloc(std::max<size_t>(np, 1) * sizeof(double)));
  out->dh_history = static_cast<double*>(malloc(std::max<size_t>(np, 1) * sizeof(double)));
  if (!out->unique_basis || !out->seed_stats || !out->time_points || !out->p_less_history || !out->dh_history) {
    bk_sampling_result_release(out);
    return fail(c, BK_ERR_OOM, "host allocation of the sampling result failed");
  }
  std::copy(ub.begin(), ub.end(), out->unique_basis);
  std::copy(ss.begin(), ss.end(), out->seed_stats);
  std::copy(times.begin(), times.end(), out->time_points);
  std::copy(pl.begin(), pl.end(), out->p_less_history);
  std::copy(dh.begin(), dh.end(), out->dh_history);

  if (cfg->verbose) {
    // the reference's console report (sampler.cuh:529-539, 686-696), replayed from the recorded series
    if (cfg->record_trajectory) {
      double peak = 0.0, peak_t = 0.0;
      for (size_t i = 0; i < np; ++i) {
        if (pl[i] > peak) {
          peak = pl[i];
          peak_t = times[i];
        }
        const int step = (int)std::llround(times[i] / cfg->dt);
        if (step % 200 == 0 || step == T) {
          const double pct = (T > 0) ? (100.0 * step / T) : 100.0;
          std::cout << "    [Progress " << std::setw(3) << (int)pct << "%] Step " << std::setw(4) << step << "/" << T
                    << " (t = " << std::fixed << std::setprecision(1) << times[i] << "s)"
                    << " | P_<(t) = " << std::scientific << std::setprecision(3) << pl[i]
                    << " | <dH> = " << std::fixed << std::setprecision(2) << dh[i] << " | Peak = " << peak
                    << " (at t=" << std::fixed << std::setprecision(1) << peak_t << "s)" << std::defaultfloat
                    << std::endl;
        }
      }
    }
    std::cout << "[Quantum Sampler] Successes / Trials: " << out->improved_shots << " / "
              << out->total_shots_collected << " (" << std::fixed << std::setprecision(2)
              << (out->success_rate * 100.0) << "%)" << " | E < E_og (E_og = " << E0 << ")"
              << " | Window <dH>: " << std::fixed << std::setprecision(2) << out->window_avg_dh
              << " | Rise Rate (avg): " << std::scientific << std::setprecision(3) << out->initial_rise_rate_avg
              << " | Evals: " << out->total_evals << " | Per-Eval Rate: " << std::scientific
              << std::setprecision(4) << out->per_eval_rate << std::defaultfloat << "\n";
  }
  return BK_OK;
}

int bk_evolve_batch(bk_ctx* c, const bk_batch_params* p, const bk_batch_instance* inst, int32_t n_inst,
                    double* p_less, double* d_h, double* norm) {
  if (!c || !p || (n_inst > 0 && !inst) || n_inst < 0) return BK_ERR_INVALID;
  if (n_inst == 0) return BK_OK;
  if (n_inst > (1 << 16)) return fail(c, BK_ERR_UNSUPPORTED, "at most 65536 instances per batch");
  if (p->n_steps < 0 || !is_finite(p->dt) || !is_finite(p->diag_scale))
    return fail(c, BK_ERR_INVALID, "invalid batch parameters");
  if (p->precision != BK_C64 && p->precision != BK_C128) return fail(c, BK_ERR_INVALID, "precision %d", p->precision);
  BK_CUDA(c, cudaSetDevice(c->device));
  if (p->precision == BK_C64) return evolve_batch_t<float>(c, p, inst, n_inst, p_less, d_h, norm);
  return evolve_batch_t<double>(c, p, inst, n_inst, p_less, d_h, norm);
}

int bk_export_state(bk_ctx* c, double* host) {
  if (!c || !host) return BK_ERR_INVALID;
  if (!c->have_state) return fail(c, BK_ERR_INVALID, "no evolved state to export");
  BK_CUDA(c, cudaSetDevice(c->device));
  const int n = c->last_n;
  const uint32_t count = 1u << n;
  BK_TRY(ensure_buffer(c, &c->d_io, &c->io_cap, (size_t)count * 16));
  const double scale = (double)std::exp2(-c->last_log2_scale);
  const double ang = (c->last_ordering == BK_ORDER_STRANG) ? 0.5 * c->last_angle_unit : 0.0;
  const unsigned th = 256;
  if (c->last_planar)
    export_kernel<Planar64><<<(count + th - 1) / th, th, 0, c->stream>>>(
        reinterpret_cast<const Planar64*>(c->d_state), c->d_E, count, ang, scale, reinterpret_cast<double2*>(c->d_io));
  else if (c->last_prec == BK_C64)
    export_kernel<float2><<<(count + th - 1) / th, th, 0, c->stream>>>(
        reinterpret_cast<const float2*>(c->d_state), c->d_E, count, ang, scale, reinterpret_cast<double2*>(c->d_io));
  else
    export_kernel<double2><<<(count + th - 1) / th, th, 0, c->stream>>>(
        reinterpret_cast<const double2*>(c->d_state), c->d_E, count, ang, scale, reinterpret_cast<double2*>(c->d_io));
  BK_CUDA(c, cudaGetLastError());
  BK_CUDA(c, cudaMemcpyAsync(host, c->d_io, (size_t)count * 16, cudaMemcpyDeviceToHost, c->stream));
  BK_CUDA(c, cudaStreamSynchronize(c->stream));
  return BK_OK;
}

int bk_sample(bk_ctx* c, const double* randnums, int64_t shots, uint64_t* out) {
  if (!c || shots < 0 || (shots > 0 && (!randnums || !out))) return BK_ERR_INVALID;
  if (!c->have_state) return fail(c, BK_ERR_INVALID, "no evolved state to sample");
  if (shots == 0) return BK_OK;
  BK_CUDA(c, cudaSetDevice(c->device));
  const int n = c->last_n;
  const uint32_t count = 1u << n;
  const uint32_t m = (count + (1u << kSampleChunkBits) - 1) >> kSampleChunkBits;
  BK_TRY(ensure_buffer(c, reinterpret_cast<void**>(&c->d_chunks), &c->chunks_cap, (m + 1) * sizeof(double)));
  BK_TRY(ensure_buffer(c, &c->d_io, &c->io_cap, (size_t)shots * 16));
  double* d_rand = reinterpret_cast<double*>(c->d_io);
  unsigned long long* d_out = reinterpret_cast<unsigned long long*>(d_rand + shots);
  BK_CUDA(c, cudaMemcpyAsync(d_rand, randnums, (size_t)shots * 8, cudaMemcpyHostToDevice, c->stream));
  const unsigned th = 256;
  const unsigned sblocks = (unsigned)(((size_t)shots * 32 + th - 1) / th);
  if (c->last_planar) {
    auto psi = reinterpret_cast<const Planar64*>(c->d_state);
    chunk_sums_kernel<Planar64><<<m, th, 0, c->stream>>>(psi, count, c->d_chunks);
    scan_chunks_kernel<<<1, 1024, 0, c->stream>>>(c->d_chunks, m);
    sample_kernel<Planar64><<<sblocks, th, 0, c->stream>>>(psi, count, c->d_chunks, m, d_rand, shots, d_out);
  } else if (c->last_prec == BK_C64) {
    auto psi = reinterpret_cast<const float2*>(c->d_state);
    chunk_sums_kernel<float2><<<m, th, 0, c->stream>>>(psi, count, c->d_chunks);
    scan_chunks_kernel<<<1, 1024, 0, c->stream>>>(c->d_chunks, m);
    sample_kernel<float2><<<sblocks, th, 0, c->stream>>>(psi, count, c->d_chunks, m, d_rand, shots, d_out);
  } else {
    auto psi = reinterpret_cast<const double2*>(c->d_state);
    chunk_sums_kernel<double2><<<m, th, 0, c->stream>>>(psi, count, c->d_chunks);
    scan_chunks_kernel<<<1, 1024, 0, c->stream>>>(c->d_chunks, m);
    sample_kernel<double2><<<sblocks, th, 0, c->stream>>>(psi, count, c->d_chunks, m, d_rand, shots, d_out);
  }
  BK_CUDA(c, cudaGetLastError());
  BK_CUDA(c, cudaMemcpyAsync(out, d_out, (size_t)shots * 8, cudaMemcpyDeviceToHost, c->stream));
  BK_CUDA(c, cudaStreamSynchronize(c->stream));
  return BK_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Full-space Hamiltonian matvec and Lanczos (reference: src/subspace/diagonalizer.cuh
// fullspace_matvec_kernel_d :60-77, solve_fullspace_lanczos :377-416,
// run_gpu_lanczos_internal :418-560)
// ---------------------------------------------------------------------------
namespace {

// n < 13: one CTA over the whole vector; else the block pass over index bits
// [0, min(n, 23)) and, for n > 23, one strided tile pass over bits [23, n)
// (w = n - 23 <= 7 bits, runs of 2^(13 - w) >= 64 doubles)
int fs_matvec(bk_ctx* c, int n, double g, double scale, const double* x, double* y) {
  BK_TRY(ensure_energy(c, n));
  const int tile_bytes = (1 << kFsTileBits) * (int)sizeof(double);
  size_t ev = 0;
  BK_TRY(ev_begin(c, n < kFsTileBits ? "fs_pass" : "fs_block", &ev));
  if (n < kFsTileBits) {
    BK_TRY(allow_smem(c, reinterpret_cast<const void*>(fs_pass_kernel), tile_bytes));
    fs_pass_kernel<<<1, kFsThreads, (size_t)(1u << n) * sizeof(double), c->stream>>>(x, y, c->d_E, scale, g, n, n, n,
                                                                                      0, 1, 0);
    BK_CUDA(c, cudaGetLastError());
    BK_TRY(ev_end(c, ev));
    return BK_OK;
  }
  BK_TRY(allow_smem(c, reinterpret_cast<const void*>(fs_block_kernel), tile_bytes));
  BK_TRY(allow_smem(c, reinterpret_cast<const void*>(fs_tile_kernel), kFsTileSmem));
  const uint32_t tiles = 1u << (n - kFsTileBits);
  fs_block_kernel<<<tiles, kFsThreads, tile_bytes, c->stream>>>(x, y, c->d_E, scale, g, std::min(n, kFsGatherBits),
                                                                c->d_err);
  BK_CUDA(c, cudaGetLastError());
  BK_TRY(ev_end(c, ev));
  if (n > kFsGatherBits) {
    const int w = n - kFsGatherBits, cp = kFsTileBits - w, h0 = kFsGatherBits;
    // x as 2^n doubles (8-byte TMA elements): runs of 2^cp, 2^w of them 2^h0 apart, tiles over bits [cp, h0)
    TmaDesc xm;
    BK_TRY(build_amp_map(c, const_cast<double*>(x), n, BK_C64, cp, h0, w, &xm));
    if (xm.hi_dim >= 0 || (int)xm.mid_bits != h0 - cp)
      return fail(c, BK_ERR_UNSUPPORTED, "full-space strided pass: tile geometry for n = %d", n);
    BK_TRY(ensure_buffer(c, &c->d_fsmap, &c->fsmap_cap, sizeof(CUtensorMap)));
    BK_CUDA(c, cudaMemcpyAsync(c->d_fsmap, &xm.map, sizeof(CUtensorMap), cudaMemcpyHostToDevice, c->stream));
    BK_TRY(ev_begin(c, "fs_tile", &ev));
    fs_tile_kernel<<<tiles, kFsThreads, kFsTileSmem, c->stream>>>(static_cast<const CUtensorMap*>(c->d_fsmap), y,
                                                                   c->d_E, scale, g, cp, h0, h0 - cp,
                                                                  xm.mid_dim, xm.hi_dim, 0, cp, c->d_err);
    BK_CUDA(c, cudaGetLastError());
    BK_TRY(ev_end(c, ev));
  }
  return BK_OK;
}

// the bounded waits' error word, cleared before and read after a full-space call
int fs_err_clear(bk_ctx* c) {
  BK_CUDA(c, cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
  return BK_OK;
}
int fs_err_check(bk_ctx* c) {
  int e = 0;
  BK_CUDA(c, cudaMemcpyAsync(&e, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  BK_CUDA(c, cudaStreamSynchronize(c->stream));
  if (e == DEV_TIMEOUT) return fail(c, BK_ERR_TIMEOUT, "fullspace matvec: a bounded device wait gave up");
  if (e != 0) return fail(c, BK_ERR_CUDA, "fullspace matvec: a kernel refused its launch geometry (%d)", e);
  return BK_OK;
}

// Eigenvalues (ascending) and eigenvectors of the symmetric tridiagonal matrix
// with diagonal d[0..m) and off-diagonal e[0..m-1): the implicit QL algorithm
// with Wilkinson shifts (Bowdler, Martin, Reinsch and Wilkinson, "The QR and QL
// algorithms for symmetric matrices", Numer. Math. 11 (1968); EISPACK tql2).
// z: m x m, column k = eigenvector k (row-major z[i * m + k]).
bool tridiag_eigen(std::vector<double>& d, std::vector<double> e, std::vector<double>& z, int m) {
  z.assign((size_t)m * m, 0.0);
  for (int i = 0; i < m; ++i) z[(size_t)i * m + i] = 1.0;
  e.resize((size_t)m, 0.0);
  e[(size_t)m - 1] = 0.0;
  const double eps = std::numeric_limits<double>::epsilon();
  for (int l = 0; l < m; ++l) {
    int iter = 0;
    for (;;) {
      int k = l;
      for (; k < m - 1; ++k) {
        const double dd = std::fabs(d[k]) + std::fabs(d[k + 1]);
        if (std::fabs(e[k]) <= eps * dd) break;
      }
      if (k == l) break;
      if (++iter > 60) return false;
      // shift from the leading 2 x 2 block
      double gq = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = std::hypot(gq, 1.0);
      gq = d[k] - d[l] + e[l] / (gq + std::copysign(r, gq));
      double sn = 1.0, cs = 1.0, pp = 0.0;
      int i = k - 1;
      bool deflated = false;
      for (; i >= l; --i) {
        const double f = sn * e[i], b = cs * e[i];
        r = std::hypot(f, gq);
        e[i + 1] = r;
        if (r == 0.0) {
          d[i + 1] -= pp;
          e[k] = 0.0;
          deflated = true;
          break;
        }
        sn = f / r;
        cs = gq / r;
        gq = d[i + 1] - pp;
        r = (d[i] - gq) * sn + 2.0 * cs * b;
        pp = sn * r;
        d[i + 1] = gq + pp;
        gq = cs * r - b;
        for (int row = 0; row < m; ++row) {
          const double fz = z[(size_t)row * m + i + 1];
          z[(size_t)row * m + i + 1] = sn * z[(size_t)row * m + i] + cs * fz;
          z[(size_t)row * m + i] = cs * z[(size_t)row * m + i] - sn * fz;
        }
      }
      if (deflated) continue;
      d[l] -= pp;
      e[l] = gq;
      e[k] = 0.0;
    }
  }
  // sort ascending with the vectors
  std::vector<int> idx((size_t)m);
  for (int i = 0; i < m; ++i) idx[(size_t)i] = i;
  std::sort(idx.begin(), idx.end(), [&](int a, int b) { return d[(size_t)a] < d[(size_t)b]; });
  std::vector<double> d2((size_t)m), z2((size_t)m * m);
  for (int k = 0; k < m; ++k) {
    d2[(size_t)k] = d[(size_t)idx[(size_t)k]];
    for (int row = 0; row < m; ++row) z2[(size_t)row * m + k] = z[(size_t)row * m + idx[(size_t)k]];
  }
  d.swap(d2);
  z.swap(z2);
  return true;
}

}  // namespace

extern "C" {

int bk_fullspace_matvec(bk_ctx* c, int n, double g, double scale, const double* d_x, double* d_y, int method) {
  if (!c || !d_x || !d_y) return BK_ERR_INVALID;
  if (method != BK_FUSED && method != BK_PLAIN) return fail(c, BK_ERR_INVALID, "fullspace matvec: method %d", method);
  if (n < 1 || n > kMaxN) return fail(c, BK_ERR_UNSUPPORTED, "n = %d outside [1, %d]", n, kMaxN);
  if (d_x == d_y) return fail(c, BK_ERR_INVALID, "fullspace matvec: x and y must not alias");
  if ((reinterpret_cast<uintptr_t>(d_x) | reinterpret_cast<uintptr_t>(d_y)) & 15u)
    return fail(c, BK_ERR_INVALID, "fullspace matvec: x and y must be 16-byte aligned (bulk copies)");
  BK_CUDA(c, cudaSetDevice(c->device));
  BK_TRY(fs_err_clear(c));
  if (method == BK_PLAIN) {
    BK_TRY(ensure_energy(c, n));
    const uint64_t N = 1ull << n;
    size_t ev = 0;
    BK_TRY(ev_begin(c, "fs_plain", &ev));
    fs_plain_kernel<<<(unsigned)((N + 255) / 256), 256, 0, c->stream>>>(d_x, d_y, c->d_E, scale, g, n, N);
    BK_CUDA(c, cudaGetLastError());
    BK_TRY(ev_end(c, ev));
  } else {
    BK_TRY(fs_matvec(c, n, g, scale, d_x, d_y));
  }
  BK_TRY(fs_err_check(c));
  BK_TRY(collect_timing(c));
  return BK_OK;
}

int bk_fullspace_lanczos(bk_ctx* c, const bk_lanczos_params* p, double* energies, double* vectors,
                         bk_lanczos_stats* stats) {
  if (!c || !p || !energies) return BK_ERR_INVALID;
  const int n = p->n;
  if (n < 1 || n > kMaxN) return fail(c, BK_ERR_UNSUPPORTED, "n = %d outside [1, %d]", n, kMaxN);
  if (p->num_eigenpairs < 1 || p->max_krylov_dim < 1)
    return fail(c, BK_ERR_INVALID, "lanczos: num_eigenpairs and max_krylov_dim must be >= 1");
  BK_CUDA(c, cudaSetDevice(c->device));
  cudaStream_t st = c->stream;
  const uint64_t N = 1ull << n;
  const int m = (int)std::min<uint64_t>(N, (uint64_t)p->max_krylov_dim);
  const double scale = p->normalize_by_n ? (1.0 / static_cast<double>(n)) : 1.0;
  // Krylov basis V[m][N], work vector w, partial sums, alpha[m], beta[m], norm
  const size_t need = ((size_t)m + 1) * N * sizeof(double) + (kLzBlocks + 2 * (size_t)m + 8) * sizeof(double);
  if (c->lz_cap < need) {
    // the old buffer is released before the new one is taken; keep 256 MB of headroom
    size_t free_b = 0, total_b = 0;
    BK_CUDA(c, cudaMemGetInfo(&free_b, &total_b));
    if (need + (256ull << 20) > free_b + c->lz_cap)
      return fail(c, BK_ERR_UNSUPPORTED, "lanczos: %d Krylov vectors of 2^%d doubles need %.1f GB (%.1f GB free)",
                  m + 1, n, need / 1e9, (free_b + c->lz_cap) / 1e9);
  }
  BK_TRY(ensure_buffer(c, &c->d_lz, &c->lz_cap, need));
  double* V = static_cast<double*>(c->d_lz);
  double* w = V + (size_t)m * N;
  double* partials = w + N;
  double* d_alpha = partials + kLzBlocks;
  double* d_beta = d_alpha + m;
  double* d_norm = d_beta + m;
  BK_TRY(ensure_energy(c, n));
  BK_TRY(fs_err_clear(c));
  auto t0 = std::chrono::steady_clock::now();
  // start vector: the reference's mt19937_64(42), uniform on (-0.5, 0.5) (diagonalizer.cuh:433-437)
  {
    std::mt19937_64 rng(42);
    std::uniform_real_distribution<double> dist(-0.5, 0.5);
    std::vector<double> v0(N);
    for (uint64_t i = 0; i < N; ++i) v0[i] = dist(rng);
    BK_CUDA(c, cudaMemcpyAsync(V, v0.data(), N * sizeof(double), cudaMemcpyHostToDevice, st));
    BK_CUDA(c, cudaStreamSynchronize(st));
  }
  const unsigned eg = kLzBlocks;
  lz_axpy_nrm_kernel<<<eg, 256, 0, st>>>(V, V, d_alpha, -1, N, partials);
  lz_reduce_kernel<<<1, 256, 0, st>>>(partials, (int)eg, d_norm, 0, 1);
  lz_scale_kernel<<<eg, 256, 0, st>>>(V, V, d_norm, 0, N);
  BK_CUDA(c, cudaGetLastError());
  int m_actual = m, matvecs = 0;
  std::vector<double> h_alpha((size_t)m, 0.0), h_beta((size_t)m, 0.0);
  for (int j = 0; j < m; ++j) {
    double* vj = V + (size_t)j * N;
    BK_TRY(fs_matvec(c, n, p->g, scale, vj, w));
    ++matvecs;
    lz_orth_dot_kernel<<<eg, 256, 0, st>>>(w, j > 0 ? vj - N : vj, vj, d_beta, j - 1, N, partials);
    lz_reduce_kernel<<<1, 256, 0, st>>>(partials, (int)eg, d_alpha, j, 0);
    if (j < m - 1) {
      lz_axpy_nrm_kernel<<<eg, 256, 0, st>>>(w, vj, d_alpha, j, N, partials);
      lz_reduce_kernel<<<1, 256, 0, st>>>(partials, (int)eg, d_beta, j, 1);
      BK_CUDA(c, cudaGetLastError());
      BK_CUDA(c, cudaMemcpyAsync(&h_beta[(size_t)j], d_beta + j, sizeof(double), cudaMemcpyDeviceToHost, st));
      BK_CUDA(c, cudaStreamSynchronize(st));
      if (std::fabs(h_beta[(size_t)j]) < p->tolerance) {  // breakdown (diagonalizer.cuh:463-466)
        m_actual = j + 1;
        break;
      }
      lz_scale_kernel<<<eg, 256, 0, st>>>(vj + N, w, d_beta, j, N);
    }
    BK_CUDA(c, cudaGetLastError());
  }
  BK_CUDA(c, cudaMemcpyAsync(h_alpha.data(), d_alpha, (size_t)m_actual * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (m_actual > 1)
    BK_CUDA(c, cudaMemcpyAsync(h_beta.data(), d_beta, (size_t)(m_actual - 1) * sizeof(double),
                               cudaMemcpyDeviceToHost, st));
  BK_CUDA(c, cudaStreamSynchronize(st));
  BK_TRY(fs_err_check(c));
  BK_TRY(collect_timing(c));
  std::vector<double> dvals(h_alpha.begin(), h_alpha.begin() + m_actual);
  std::vector<double> evals(h_beta.begin(), h_beta.begin() + std::max(m_actual - 1, 0));
  std::vector<double> z;
  if (!tridiag_eigen(dvals, evals, z, m_actual))
    return fail(c, BK_ERR_CUDA, "lanczos: the tridiagonal eigensolver did not converge");
  const int k_pairs = std::min(p->num_eigenpairs, m_actual);
  for (int k = 0; k < p->num_eigenpairs; ++k) energies[k] = k < k_pairs ? dvals[(size_t)k] : std::nan("");
  if (vectors) {
    // Ritz vectors x_k = V y_k (diagonalizer.cuh:526-538)
    std::vector<double> coef((size_t)m_actual);
    for (int k = 0; k < k_pairs; ++k) {
      for (int j = 0; j < m_actual; ++j) coef[(size_t)j] = z[(size_t)j * m_actual + k];
      BK_CUDA(c, cudaMemcpyAsync(partials, coef.data(), (size_t)m_actual * sizeof(double), cudaMemcpyHostToDevice, st));
      lz_combine_kernel<<<eg, 256, 0, st>>>(V, partials, m_actual, N, w);
      BK_CUDA(c, cudaGetLastError());
      BK_CUDA(c, cudaMemcpyAsync(vectors + (size_t)k * N, w, N * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    BK_CUDA(c, cudaStreamSynchronize(st));
  }
  if (p->alphas) std::copy(h_alpha.begin(), h_alpha.begin() + m_actual, p->alphas);
  if (p->betas) std::copy(h_beta.begin(), h_beta.begin() + std::max(m_actual - 1, 0), p->betas);
  if (stats) {
    stats->krylov_dim = m_actual;
    stats->matvecs = matvecs;
    stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  return BK_OK;
}

}  // extern "C"

