// Host side of the B200 statevector engine: the C ABI declared in
// include/bk_engine.h. One bk_ctx = one device, one stream and cached device
// buffers. Replaces the device part of CuStateVecSampler
// (src/sampling/sampler.cuh:318-707 of the reference).
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <random>
#include <string>
#include <vector>

#include "bk_aux.cuh"
#include "bk_engine.h"
#include "bk_fused.cuh"

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
  // tensor maps, keyed by (state ptr, n, precision, pass)
  std::map<std::string, TmaDesc> tma;
  // last evolution (for export / sampling)
  bool have_state = false;
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

int get_map(bk_ctx* c, const std::string& kind, int n, int prec, int cp, int h0, int w, const TmaDesc** out) {
  char key[160];
  snprintf(key, sizeof(key), "%s/%p/%p/%d/%d/%d/%d/%d", kind.c_str(), c->d_state, (void*)c->d_E, n, prec, cp,
           h0, w);
  auto it = c->tma.find(key);
  if (it == c->tma.end()) {
    TmaDesc d;
    if (kind == "E")
      BK_TRY(build_e_map(c, c->d_E, n, tile_bits(prec), &d));
    else
      BK_TRY(build_amp_map(c, c->d_state, n, prec, cp, h0, w, &d));
    it = c->tma.emplace(key, d).first;
  }
  *out = &it->second;
  return BK_OK;
}

int ensure_energy(bk_ctx* c, int n) {
  if (c->e_n == n && c->d_E) return BK_OK;
  if (c->d_E) cudaFree(c->d_E);
  c->d_E = nullptr;
  c->e_n = -1;
  c->tma.clear();
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
  c->tma.clear();
  BK_CUDA(c, cudaMalloc(&c->d_state, bytes));
  c->state_bytes = bytes;
  c->st_n = n;
  c->st_prec = prec;
  return BK_OK;
}

template <class R>
int upload_phase_tables(bk_ctx* c, int n, double angle_unit, int* n_hi_out) {
  using amp = typename AmpTraits<R>::amp;
  const int emax = (n - 1) * n * (2 * n - 1) / 6;
  const int n_hi = (emax >> kPhaseLoBits) + 1;
  std::vector<amp> h((size_t)n_hi + kPhaseLo);
  for (int i = 0; i < n_hi; ++i) {
    const double th = -angle_unit * (double)(i << kPhaseLoBits);
    h[(size_t)i].x = (R)std::cos(th);
    h[(size_t)i].y = (R)std::sin(th);
  }
  for (int i = 0; i < kPhaseLo; ++i) {
    const double th = -angle_unit * (double)i;
    h[(size_t)n_hi + i].x = (R)std::cos(th);
    h[(size_t)n_hi + i].y = (R)std::sin(th);
  }
  BK_TRY(ensure_buffer(c, &c->d_phase, &c->phase_cap, h.size() * sizeof(amp)));
  BK_CUDA(c, cudaMemcpyAsync(c->d_phase, h.data(), h.size() * sizeof(amp), cudaMemcpyHostToDevice, c->stream));
  *n_hi_out = n_hi;
  return BK_OK;
}

bool is_finite(double x) { return std::isfinite(x); }

struct Schedule {
  std::vector<double> g;        // per step
  std::vector<int> slot;        // per step (n_steps + 1): measurement row or -1
  int n_meas = 0;
};

template <class R>
int launch_a1(bk_ctx* c, int kind, const PassParams<R>& pp, const TmaDesc* am, const TmaDesc* em, int n) {
  constexpr int T = AmpTraits<R>::kTileBits;
  const unsigned grid = 1u << (n - T);
  const int smem = SmemLayout<R>::kA1Bytes;
  size_t ev = 0;
  if (kind == 0) {
    BK_TRY(allow_smem(c, reinterpret_cast<const void*>(a1_kernel<R, 0>), smem));
    BK_TRY(ev_begin(c, pp.measure ? "a1_step_measure" : "a1_step", &ev));
    a1_kernel<R, 0><<<grid, kThreads, smem, c->stream>>>(am->map, em->map, pp);
  } else {
    BK_TRY(allow_smem(c, reinterpret_cast<const void*>(a1_kernel<R, 1>), smem));
    BK_TRY(ev_begin(c, "a1_measure", &ev));
    a1_kernel<R, 1><<<grid, kThreads, smem, c->stream>>>(am->map, em->map, pp);
  }
  BK_CUDA(c, cudaGetLastError());
  return ev_end(c, ev);
}

template <class R, int W>
int launch_strided_w(bk_ctx* c, const PassParams<R>& pp, const TmaDesc* am, int n) {
  constexpr int T = AmpTraits<R>::kTileBits;
  const unsigned grid = 1u << (n - T);
  const int smem = SmemLayout<R>::kStridedBytes;
  BK_TRY(allow_smem(c, reinterpret_cast<const void*>(strided_kernel<R, W>), smem));
  size_t ev = 0;
  char name[32];
  snprintf(name, sizeof(name), "strided_w%d", W);
  BK_TRY(ev_begin(c, name, &ev));
  strided_kernel<R, W><<<grid, kThreads, smem, c->stream>>>(am->map, pp);
  BK_CUDA(c, cudaGetLastError());
  return ev_end(c, ev);
}

template <class R>
int launch_strided(bk_ctx* c, int w, const PassParams<R>& pp, const TmaDesc* am, int n) {
  switch (w) {
    case 1: return launch_strided_w<R, 1>(c, pp, am, n);
    case 2: return launch_strided_w<R, 2>(c, pp, am, n);
    case 3: return launch_strided_w<R, 3>(c, pp, am, n);
    case 4: return launch_strided_w<R, 4>(c, pp, am, n);
    case 5: return launch_strided_w<R, 5>(c, pp, am, n);
    case 6: return launch_strided_w<R, 6>(c, pp, am, n);
    case 7: return launch_strided_w<R, 7>(c, pp, am, n);
    case 8: return launch_strided_w<R, 8>(c, pp, am, n);
    case 9: return launch_strided_w<R, 9>(c, pp, am, n);
    default: return fail(c, BK_ERR_UNSUPPORTED, "strided pass width %d", w);
  }
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
  int n_hi = 0;
  BK_TRY(upload_phase_tables<R>(c, n, angle_unit, &n_hi));
  const amp* ph_hi = reinterpret_cast<const amp*>(c->d_phase);
  const amp* ph_lo = ph_hi + n_hi;
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
    lg += -(long double)n * std::log2(std::fabs((long double)std::cos((long double)gd)));
  }
  *final_log2 = lg;

  if (n <= T) {
    // whole state in one CTA's shared memory; all steps in one launch
    const size_t smem = (1ull << n) * (sizeof(amp) + 2);
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
    SmallParams<R> sp;
    sp.state = reinterpret_cast<amp*>(c->d_state);
    sp.n = n;
    sp.n_steps = p->n_steps;
    sp.t = d_t;
    sp.amp_scale = d_sc;
    sp.slot = d_slot;
    sp.phase_hi = ph_hi;
    sp.phase_lo = ph_lo;
    sp.n_hi = n_hi;
    sp.e0 = e0;
    sp.s0 = s0;
    sp.results = c->d_results;
    sp.inverse = 0;
    BK_TRY(allow_smem(c, reinterpret_cast<const void*>(small_state_kernel<R>),
                      (int)((1ull << T) * (sizeof(amp) + 2))));
    size_t ev = 0;
    BK_TRY(ev_begin(c, "small_state", &ev));
    small_state_kernel<R><<<1, kThreads, smem, c->stream>>>(sp);
    BK_CUDA(c, cudaGetLastError());
    return ev_end(c, ev);
  }

  // tiled passes
  const int rest = n - T;
  const int w2 = (rest <= 9) ? rest : (rest + 1) / 2;
  const int w3 = rest - w2;
  if (w2 > 9 || w3 > 9) return fail(c, BK_ERR_UNSUPPORTED, "n = %d needs more than two strided passes", n);
  const TmaDesc *a1m = nullptr, *em = nullptr, *m2 = nullptr, *m3 = nullptr;
  BK_TRY(get_map(c, "A1", n, p->precision, T, T, 0, &a1m));
  BK_TRY(get_map(c, "E", n, p->precision, 0, 0, 0, &em));
  BK_TRY(get_map(c, "S", n, p->precision, T - w2, T, w2, &m2));
  if (w3 > 0) BK_TRY(get_map(c, "S", n, p->precision, T - w3, T + w2, w3, &m3));

  PassParams<R> base{};
  base.state = reinterpret_cast<amp*>(c->d_state);
  base.n = (uint32_t)n;
  base.phase_hi = ph_hi;
  base.phase_lo = ph_lo;
  base.n_hi = n_hi;
  base.e0 = e0;
  base.s0 = s0;
  base.partials = c->d_partials;
  base.ticket = c->d_ticket;
  base.results = c->d_results;
  base.err = c->d_err;
  base.hi_dim = a1m->hi_dim;
  base.mid_dim = -1;

  for (int k = 0; k <= p->n_steps; ++k) {
    const int slot = S.slot[(size_t)k];
    if (k == p->n_steps) {
      if (slot >= 0) {
        PassParams<R> pp = base;
        pp.slot = slot;
        pp.measure = 1;
        BK_TRY(launch_a1<R>(c, 1, pp, a1m, em, n));
      }
      break;
    }
    PassParams<R> pp = base;
    pp.t = tans[(size_t)k];
    pp.amp_scale = scales[(size_t)k];
    pp.measure = slot >= 0 ? 1 : 0;
    pp.slot = slot >= 0 ? slot : 0;
    BK_TRY(launch_a1<R>(c, 0, pp, a1m, em, n));
    PassParams<R> q2 = base;
    q2.t = tans[(size_t)k];
    q2.cprime = (uint32_t)(T - w2);
    q2.h0 = (uint32_t)T;
    q2.mid_bits = m2->mid_bits;
    q2.mid_dim = m2->mid_dim;
    q2.hi_dim = m2->hi_dim;
    BK_TRY(launch_strided<R>(c, w2, q2, m2, n));
    if (w3 > 0) {
      PassParams<R> q3 = base;
      q3.t = tans[(size_t)k];
      q3.cprime = (uint32_t)(T - w3);
      q3.h0 = (uint32_t)(T + w2);
      q3.mid_bits = m3->mid_bits;
      q3.mid_dim = m3->mid_dim;
      q3.hi_dim = m3->hi_dim;
      BK_TRY(launch_strided<R>(c, w3, q3, m3, n));
    }
  }
  return BK_OK;
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

// ---- trap generation (host) ----
static int64_t host_energy(int n, uint64_t x) {
  int64_t e = 0;
  for (int k = 1; k < n; ++k) {
    const int64_t ck = (int64_t)(n - k) - 2 * (int64_t)__builtin_popcountll((x ^ (x >> k)) & ((1ull << (n - k)) - 1ull));
    e += ck * ck;
  }
  return e;
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
                  (void*)c->d_err, (void*)c->d_count, c->d_phase, c->d_small, (void*)c->d_chunks, c->d_io})
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
  BK_CUDA(c, cudaMemsetAsync(c->d_ticket, 0, sizeof(unsigned int), c->stream));
  BK_CUDA(c, cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
  BK_CUDA(c, cudaMemsetAsync(c->d_state, 0, (1ull << n) * amp_bytes(p->precision), c->stream));
  const uint32_t s0 = (uint32_t)(p->s0 & ((1ull << n) - 1ull));
  if (p->precision == BK_C64)
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
  BK_TRY(check_device_error(c));
  BK_TRY(collect_timing(c));
  c->have_state = true;
  c->last_n = n;
  c->last_prec = p->precision;
  c->last_ordering = p->ordering;
  c->last_log2_scale = final_log2;
  c->last_angle_unit = angle_unit;
  int status = BK_OK;
  for (int m = 0; m < S.n_meas; ++m) {
    const long double f = std::exp2(-2.0L * row_log2[(size_t)m]);
    p_less[m] = (double)((long double)rows[4 * (size_t)m + 0] * f);
    d_h[m] = (double)((long double)rows[4 * (size_t)m + 1] * f);
    const double nn = (double)((long double)rows[4 * (size_t)m + 2] * f);
    if (norm) norm[m] = nn;
    if (p->norm_tol > 0.0 && !(std::fabs(nn - 1.0) <= p->norm_tol)) status = BK_ERR_NORM;
  }
  if (status == BK_ERR_NORM) return fail(c, BK_ERR_NORM, "norm left the tolerance band %g", p->norm_tol);
  return BK_OK;
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
  if (c->last_prec == BK_C64)
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
  if (c->last_prec == BK_C64) {
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
