// Device-side building blocks shared by the engine's kernels: amplitude traits,
// TMA / mbarrier wrappers with bounded waits, the LABS energy in integers, the
// Rx butterfly in tangent form, and deterministic FP64 block reductions.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace bk {

// Error codes a kernel can leave in the context's device error word.
enum DeviceError : int { DEV_OK = 0, DEV_TIMEOUT = 1, DEV_BAD_LAUNCH = 2 };

// Bounded spin: each mbarrier.try_wait may suspend for a hardware-chosen slice,
// so 1 << 22 polls is seconds at most; past that the kernel records
// DEV_TIMEOUT and returns instead of hanging the device.
constexpr uint32_t kWaitPolls = 1u << 22;

template <class R>
struct AmpTraits;
template <>
struct AmpTraits<float> {
  using amp = float2;
  static constexpr int kTileBits = 13;  // 2^13 amps x 8 B = 64 KB tile
  static constexpr int kRegBits = 5;    // 32 amps per thread, 256 threads
};
template <>
struct AmpTraits<double> {
  using amp = double2;
  static constexpr int kTileBits = 12;  // 2^12 amps x 16 B = 64 KB tile
  static constexpr int kRegBits = 4;    // 16 amps per thread, 256 threads
};

constexpr int kThreads = 256;

__host__ __device__ constexpr uint32_t pdep(uint32_t v, uint32_t mask) {
  uint32_t r = 0;
  uint32_t b = 1;
  while (mask) {
    const uint32_t low = mask & (~mask + 1u);
    if (v & b) r |= low;
    mask &= mask - 1u;
    b <<= 1;
  }
  return r;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// 1-D bulk copy global -> this CTA's shared memory (16-byte aligned, size a multiple of 16), completion on `bar`
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
// Programmatic dependent launch: wait until the grids this launch depends on
// have completed and their memory is visible (a no-op for a normal launch), and
// let the dependent launch be scheduled once every CTA has signalled or exited.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dependents_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Returns false (and records DEV_TIMEOUT) when the phase did not complete in time.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, int* err) {
  for (uint32_t i = 0; i < kWaitPolls; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  atomicExch(err, DEV_TIMEOUT);
  return false;
}

// 5-D tiled TMA load (global -> this CTA's shared memory), completion counted on `bar`.
__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            int c3, int c4, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(bar)
      : "memory");
}

// Same load with an L2 cache-policy hint (createpolicy): streaming tiles are
// loaded evict-first so they do not displace data that is about to be re-read.
__device__ __forceinline__ void tma_load_5d_hint(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2,
                                                 int c3, int c4, uint32_t bar, uint64_t policy) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7], %8;" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(bar), "l"(policy)
      : "memory");
}
__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
// 16-byte global stores with an L2 cache-policy hint
__device__ __forceinline__ void st_global_hint(void* p, float4 v, uint64_t policy) {
  asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(p), "f"(v.x), "f"(v.y), "f"(v.z),
               "f"(v.w), "l"(policy)
               : "memory");
}
__device__ __forceinline__ void st_global_hint(void* p, double2 v, uint64_t policy) {
  asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(p), "d"(v.x), "d"(v.y), "l"(policy)
               : "memory");
}

// LABS energy (reference: src/labs_energy/labs_energy.hpp:121-132, and the device
// form src/sampling/sampler.cuh:54-70), exact in integers.
__device__ __forceinline__ int labs_energy(uint32_t x, int n) {
  int e = 0;
  for (int k = 1; k < n; ++k) {
    const uint32_t m = (1u << (n - k)) - 1u;
    const int ck = (n - k) - 2 * __popc((x ^ (x >> k)) & m);
    e += ck * ck;
  }
  return e;
}

// Rx(-2 g dt) = cos(g dt) (I + i tan(g dt) X) on the pair (a = bit 0, b = bit 1):
// a' = a + i t b, b' = b + i t a. The cos(g dt) factor is not applied; the host
// tracks the product of the omitted factors exactly.
__device__ __forceinline__ void bfly(float2& a, float2& b, float t) {
  const float2 x = a, y = b;
  a.x = fmaf(-t, y.y, x.x);
  a.y = fmaf(t, y.x, x.y);
  b.x = fmaf(-t, x.y, y.x);
  b.y = fmaf(t, x.x, y.y);
}
__device__ __forceinline__ void bfly(double2& a, double2& b, double t) {
  const double2 x = a, y = b;
  a.x = fma(-t, y.y, x.x);
  a.y = fma(t, y.x, x.y);
  b.x = fma(-t, x.y, y.x);
  b.y = fma(t, x.x, y.y);
}
// Same butterfly when the partner lives in another lane (symmetric form).
__device__ __forceinline__ void bfly_partner(float2& a, const float2 b, float t) {
  const float2 x = a;
  a.x = fmaf(-t, b.y, x.x);
  a.y = fmaf(t, b.x, x.y);
}
__device__ __forceinline__ void bfly_partner(double2& a, const double2 b, double t) {
  const double2 x = a;
  a.x = fma(-t, b.y, x.x);
  a.y = fma(t, b.x, x.y);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// ---- diagonal phase exp(i theta E), theta = -dt * diag_scale ----
// complex64: E = h K + l. The rotation by theta*l (|theta| (K-1) <= 1/2) takes
// its shear coefficients from Maclaurin polynomials; the rotation by theta*h K
// comes from a table of at most kPhaseH entries {a, b} (a bank row or two of
// shared memory, so the data-dependent lookups do not conflict) plus an exact
// quarter turn i^q. A rotation by r is applied as three shears (x += a y;
// y += b x; x += a y with a = -tan(r/2), b = sin r): a shear has determinant
// exactly 1 whatever the rounding of a and b, so no energy level gains or loses
// norm systematically from step to step (a rounded (cos, sin) pair would).
constexpr int kPhaseH = 256;  // table capacity (entries used: host choice, 16 typically)

struct Phase32 {
  const float2* hab;   // [n_h] {-tan(r_h / 2), sin r_h}
  const int* hq;       // [n_h] quarter turns of level h
  uint32_t K, M;       // h = umulhi(E, M) (exact for E <= Emax, checked on the host)
  float theta, theta_lo;  // angle per unit of E (negative) as a float pair
  int n_h;
};

__device__ __forceinline__ void shear_rotate(float& x, float& y, float a, float b) {
  x = fmaf(a, y, x);
  y = fmaf(b, x, y);
  x = fmaf(a, y, x);
}
__device__ __forceinline__ void shear_unrotate(float& x, float& y, float a, float b) {
  x = fmaf(-a, y, x);
  y = fmaf(-b, x, y);
  x = fmaf(-a, y, x);
}
// multiply by i^q (exact)
__device__ __forceinline__ void quarter_turns(float& x, float& y, int q) {
  const float x0 = x, y0 = y;
  const bool odd = q & 1, neg = q & 2;
  x = odd ? -y0 : x0;
  y = odd ? x0 : y0;
  if (neg) {
    x = -x;
    y = -y;
  }
}
// Shear coefficients of a rotation by r, |r| <= 1/2: a = -tan(r/2), b = sin r
// (Maclaurin series of tan to x^9 and sin to r^9; truncation < 2e-9 there).
__device__ __forceinline__ void small_rotation(float r, float& a, float& b) {
  const float x = 0.5f * r, x2 = x * x;
  float t = fmaf(x2, 62.0f / 2835.0f, 17.0f / 315.0f);
  t = fmaf(x2, t, 2.0f / 15.0f);
  t = fmaf(x2, t, 1.0f / 3.0f);
  t = fmaf(x2, t, 1.0f);
  a = -x * t;
  const float r2 = r * r;
  float u = fmaf(r2, 1.0f / 362880.0f, -1.0f / 5040.0f);
  u = fmaf(r2, u, 1.0f / 120.0f);
  u = fmaf(r2, u, -1.0f / 6.0f);
  u = fmaf(r2, u, 1.0f);
  b = r * u;
}
// level split of E and the residual angle
__device__ __forceinline__ float residual_angle(int e, const Phase32& P, uint32_t& h) {
  h = __umulhi((uint32_t)e, P.M);
  const uint32_t l = (uint32_t)e - h * P.K;
  const float lf = __int_as_float(0x4B000000 | l) - 8388608.0f;  // exact for l < 2^23
  return fmaf(lf, P.theta, lf * P.theta_lo);
}
__device__ __forceinline__ float2 apply_phase(float2 v, int e, const Phase32& P, const float2* hab, const int* hq) {
  uint32_t h;
  const float r = residual_angle(e, P, h);
  float a, b;
  small_rotation(r, a, b);
  shear_rotate(v.x, v.y, a, b);
  const float2 H = hab[h];
  shear_rotate(v.x, v.y, H.x, H.y);
  quarter_turns(v.x, v.y, hq[h]);
  return v;
}
__device__ __forceinline__ float2 apply_phase_inverse(float2 v, int e, const Phase32& P, const float2* hab,
                                                      const int* hq) {
  uint32_t h;
  const float r = residual_angle(e, P, h);
  float a, b;
  small_rotation(r, a, b);
  quarter_turns(v.x, v.y, (4 - hq[h]) & 3);
  const float2 H = hab[h];
  shear_unrotate(v.x, v.y, H.x, H.y);
  shear_unrotate(v.x, v.y, a, b);
  return v;
}

// complex128: rounded FP64 (cos, sin) tables, E = 128 h + l, hi[h] * lo[l]
// (gain per level ~1e-16 per step).
constexpr int kPhaseLoBits = 7;
constexpr int kPhaseLo = 1 << kPhaseLoBits;
constexpr int kPhaseHi64 = 72;  // > (8555 >> 7) + 1 entries at n = 30
struct Phase64 {
  const double2* hi;  // [n_hi] (cos, sin) of theta * 128 h
  const double2* lo;  // [128]  (cos, sin) of theta * l
  int n_hi;
};
__device__ __forceinline__ double2 apply_phase(double2 v, int e, const Phase64&, const double2* hi,
                                               const double2* lo) {
  const double2 h = hi[e >> kPhaseLoBits], l = lo[e & (kPhaseLo - 1)];
  const double c = fma(h.x, l.x, -h.y * l.y), s = fma(h.x, l.y, h.y * l.x);
  return make_double2(fma(v.x, c, -v.y * s), fma(v.x, s, v.y * c));
}
__device__ __forceinline__ double2 apply_phase_inverse(double2 v, int e, const Phase64&, const double2* hi,
                                                       const double2* lo) {
  const double2 h = hi[e >> kPhaseLoBits], l = lo[e & (kPhaseLo - 1)];
  const double c = fma(h.x, l.x, -h.y * l.y), s = fma(h.x, l.y, h.y * l.x);
  return make_double2(fma(v.x, c, v.y * s), fma(-v.x, s, v.y * c));
}

// Per-precision phase parameters and their shared-memory staging.
template <class R>
struct PhaseOf;
template <>
struct PhaseOf<float> {
  using params = Phase32;
  static constexpr int kSmemBytes = kPhaseH * (int)(sizeof(float2) + sizeof(int));
  struct Smem {
    const float2* a;
    const int* b;
  };
  __device__ static Smem stage(const Phase32& P, unsigned char* s) {
    float2* hab = reinterpret_cast<float2*>(s);
    int* hq = reinterpret_cast<int*>(hab + kPhaseH);
    for (int i = threadIdx.x; i < P.n_h; i += blockDim.x) {
      hab[i] = P.hab[i];
      hq[i] = P.hq[i];
    }
    return Smem{hab, hq};
  }
  __device__ static float2 apply(float2 v, int e, const Phase32& P, const Smem& t) {
    return apply_phase(v, e, P, t.a, t.b);
  }
  __device__ static float2 apply_inverse(float2 v, int e, const Phase32& P, const Smem& t) {
    return apply_phase_inverse(v, e, P, t.a, t.b);
  }
};
template <>
struct PhaseOf<double> {
  using params = Phase64;
  static constexpr int kSmemBytes = (kPhaseHi64 + kPhaseLo) * (int)sizeof(double2);
  struct Smem {
    const double2* a;
    const double2* b;
  };
  __device__ static Smem stage(const Phase64& P, unsigned char* s) {
    double2* hi = reinterpret_cast<double2*>(s);
    double2* lo = hi + kPhaseHi64;
    for (int i = threadIdx.x; i < P.n_hi; i += blockDim.x) hi[i] = P.hi[i];
    for (int i = threadIdx.x; i < kPhaseLo; i += blockDim.x) lo[i] = P.lo[i];
    return Smem{hi, lo};
  }
  __device__ static double2 apply(double2 v, int e, const Phase64& P, const Smem& t) {
    return apply_phase(v, e, P, t.a, t.b);
  }
  __device__ static double2 apply_inverse(double2 v, int e, const Phase64& P, const Smem& t) {
    return apply_phase_inverse(v, e, P, t.a, t.b);
  }
};

__device__ __forceinline__ double norm2d(float2 a) { return (double)fmaf(a.x, a.x, a.y * a.y); }
__device__ __forceinline__ double norm2d(double2 a) { return fma(a.x, a.x, a.y * a.y); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Measurement accumulators: |psi|^2 summed over all s, over E(s) < e0, and
// weighted by popcount(s ^ s0) — FP64 (reference: sampler.cuh:149-195).
struct MeasureAcc {
  double norm = 0.0, p_less = 0.0, d_h = 0.0;
  __device__ __forceinline__ void add(double w, bool below, int flips) {
    norm += w;
    if (below) p_less += w;
    d_h += w * (double)flips;
  }
};

// Deterministic two-level reduction: each block writes its triple to
// partials[blockIdx.x]; the last block to finish (ticket) sums all partials in
// index order and writes results[slot] = {p_less, d_h, norm}. The ticket
// resets itself so the next launch starts from zero.
__device__ __forceinline__ void block_reduce_and_finalize(MeasureAcc acc, double* partials,
                                                          unsigned int* ticket, double* results,
                                                          int slot, int nblocks) {
  __shared__ double red[3][kThreads / 32];
  __shared__ bool is_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double a = warp_sum(acc.norm), b = warp_sum(acc.p_less), c = warp_sum(acc.d_h);
  if (lane == 0) {
    red[0][warp] = a;
    red[1][warp] = b;
    red[2][warp] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0, s1 = 0, s2 = 0;
    for (int w = 0; w < kThreads / 32; ++w) {
      s0 += red[0][w];
      s1 += red[1][w];
      s2 += red[2][w];
    }
    partials[3 * (size_t)blockIdx.x + 0] = s0;
    partials[3 * (size_t)blockIdx.x + 1] = s1;
    partials[3 * (size_t)blockIdx.x + 2] = s2;
    __threadfence();
    const unsigned int t = atomicAdd(ticket, 1u);
    is_last = (t == (unsigned int)nblocks - 1u);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  double s0 = 0, s1 = 0, s2 = 0;
  for (int i = threadIdx.x; i < nblocks; i += kThreads) {
    s0 += __ldcg(&partials[3 * (size_t)i + 0]);
    s1 += __ldcg(&partials[3 * (size_t)i + 1]);
    s2 += __ldcg(&partials[3 * (size_t)i + 2]);
  }
  s0 = warp_sum(s0);
  s1 = warp_sum(s1);
  s2 = warp_sum(s2);
  __syncthreads();
  if (lane == 0) {
    red[0][warp] = s0;
    red[1][warp] = s1;
    red[2][warp] = s2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double n = 0, p = 0, d = 0;
    for (int w = 0; w < kThreads / 32; ++w) {
      n += red[0][w];
      p += red[1][w];
      d += red[2][w];
    }
    results[4 * (size_t)slot + 0] = p;
    results[4 * (size_t)slot + 1] = d;
    results[4 * (size_t)slot + 2] = n;
    *ticket = 0u;
  }
}

}  // namespace bk
