// Persistent dataflow engine (sm_100a): every Trotter step of one or many
// statevectors in ONE launch, scheduled as tile tasks with dependency counters.
//
// Elements. The tile machinery works on 16-byte elements: a complex128
// amplitude, or a PAIR of complex64 amplitudes stored pair-planar as
// (re[2k], re[2k+1], im[2k], im[2k+1]) so that packed f32x2 FMAs act on
// (re, re) and (im, im) register pairs. A tile is 4096 elements (64 KB); element
// bit b is amplitude bit b (complex128) or b + 1 (complex64, whose amplitude
// bit 0 lives inside the element).
//
// Tasks of one step (per statevector):
//   A1  elements bits [0, 12): measurement (optional), diagonal phase D, Rx on
//       the 12 element bits (+ amplitude bit 0 for complex64);
//   S2  bits [0, 12 - W2) u [12, 12 + W2): Rx on W2 high element bits;
//   S3  bits [0, 12 - W3) u [12 + W2, n'): Rx on the remaining W3 bits;
//   M   measurement only (after the last step).
// Dependencies (cumulative counters, never reset inside a launch):
//   S2 tile of slab h  <- all 2^W2 A1 tiles of slab h of the same step;
//   S3 tile            <- all S2 tiles of the statevector and step;
//   A1 of step k + 1   <- all S3 (or, without S3, all S2) tiles of step k.
// The task order interleaves A1 of slab h + 1 before S2 of slab h, so a slab
// written by A1 is re-read by S2 while it is still in L2: A1 + S2 together cost
// one HBM round trip.
//
// Two CTAs per SM (256 threads, one 80 KB stage each), so one CTA's stores and
// completion fence overlap the other's arithmetic. Thread 0 claims tasks from a
// global counter in order (every dependency points to an earlier task held by a
// running CTA, and a CTA signals its finished task before it waits on the next
// one's dependency: no deadlock), waits (bounded) for the dependency and issues
// the TMA; when the next task's dependency is already met its load is issued
// while the current task's stores drain. All waits are bounded and a global
// abort word stops every CTA after the first failure.
#pragma once
#include "bk_device.cuh"
#include "bk_fused.cuh"

namespace bk {

constexpr int kElemBits = 12;          // 4096 elements per tile
constexpr int kStageTileBytes = 65536;
constexpr int kStageEBytes = 16384;    // A1: uint16 E of 8192 (c64) / 4096 (c128) amplitudes
constexpr int kComputeThreads = 256;
constexpr int kPersistThreads = kComputeThreads;

enum TaskKind : int { TASK_A1 = 0, TASK_S2 = 1, TASK_S3 = 2, TASK_M = 3, TASK_END = 7 };

// ---------------------------------------------------------------------------
// element types
// ---------------------------------------------------------------------------
template <class R>
struct El;

template <>
struct El<float> {
  struct T {
    float2 re, im;  // amplitudes 2k (x) and 2k + 1 (y)
  };
  static constexpr int kAmps = 2;
  __device__ static T ld(const void* p) {
    const float4 q = *reinterpret_cast<const float4*>(p);
    return T{make_float2(q.x, q.y), make_float2(q.z, q.w)};
  }
  __device__ static void st(void* p, const T& v) {
    *reinterpret_cast<float4*>(p) = make_float4(v.re.x, v.re.y, v.im.x, v.im.y);
  }
  __device__ static void stg(void* p, const T& v, uint64_t pol) {
    st_global_hint(p, make_float4(v.re.x, v.re.y, v.im.x, v.im.y), pol);
  }
  // a' = a + i t b, b' = b + i t a on both amplitudes of the elements at once
  __device__ static void bfly(T& a, T& b, float t) {
    const float2 pt = make_float2(t, t), nt = make_float2(-t, -t);
    const T x = a, y = b;
    a.re = __ffma2_rn(nt, y.im, x.re);
    a.im = __ffma2_rn(pt, y.re, x.im);
    b.re = __ffma2_rn(nt, x.im, y.re);
    b.im = __ffma2_rn(pt, x.re, y.im);
  }
  // the butterfly between the two amplitudes inside the element (amplitude bit 0)
  __device__ static void bfly_inner(T& a, float t) {
    const T x = a;
    a.re.x = fmaf(-t, x.im.y, x.re.x);
    a.im.x = fmaf(t, x.re.y, x.im.x);
    a.re.y = fmaf(-t, x.im.x, x.re.y);
    a.im.y = fmaf(t, x.re.x, x.im.y);
  }
  __device__ static T shfl_xor(const T& v, int m) {
    T r;
    r.re.x = __shfl_xor_sync(0xffffffffu, v.re.x, m);
    r.re.y = __shfl_xor_sync(0xffffffffu, v.re.y, m);
    r.im.x = __shfl_xor_sync(0xffffffffu, v.im.x, m);
    r.im.y = __shfl_xor_sync(0xffffffffu, v.im.y, m);
    return r;
  }
  __device__ static void bfly_partner(T& a, const T& b, float t) {
    const float2 pt = make_float2(t, t), nt = make_float2(-t, -t);
    const T x = a;
    a.re = __ffma2_rn(nt, b.im, x.re);
    a.im = __ffma2_rn(pt, b.re, x.im);
  }
  __device__ static void scale(T& a, float s) {
    const float2 ss = make_float2(s, s);
    a.re = __fmul2_rn(a.re, ss);
    a.im = __fmul2_rn(a.im, ss);
  }
};

template <>
struct El<double> {
  struct T {
    double2 v;
  };
  static constexpr int kAmps = 1;
  __device__ static T ld(const void* p) { return T{*reinterpret_cast<const double2*>(p)}; }
  __device__ static void st(void* p, const T& v) { *reinterpret_cast<double2*>(p) = v.v; }
  __device__ static void stg(void* p, const T& v, uint64_t pol) { st_global_hint(p, v.v, pol); }
  __device__ static void bfly(T& a, T& b, double t) { bk::bfly(a.v, b.v, t); }
  __device__ static void bfly_inner(T&, double) {}
  __device__ static T shfl_xor(const T& v, int m) {
    T r;
    r.v.x = __shfl_xor_sync(0xffffffffu, v.v.x, m);
    r.v.y = __shfl_xor_sync(0xffffffffu, v.v.y, m);
    return r;
  }
  __device__ static void bfly_partner(T& a, const T& b, double t) { bk::bfly_partner(a.v, b.v, t); }
  __device__ static void scale(T& a, double s) {
    a.v.x *= s;
    a.v.y *= s;
  }
};

// ---------------------------------------------------------------------------
// diagonal phase on an element. complex64: E = h K + l per amplitude, residual
// rotation by polynomials and the level rotation hab[h] = {-tan(th_h/4),
// sin(th_h/2)} applied twice (th_h reduced to (-pi, pi]); every rotation as
// shears (determinant exactly 1), vectorised over the element's two amplitudes.
// ---------------------------------------------------------------------------
struct PhaseV32 {
  const float2* hab;  // [n_h]
  uint32_t K, M;      // h = umulhi(E, M)
  float theta, theta_lo;
  int n_h;
  // full table (BK_OPT_PHASE_TABLE): tab[j] = {-tan(r_j/4), sin(r_j/2)} for
  // E = c0 + 4 j (every LABS energy is floor(n/2) mod 4), padded to an even count
  const float2* tab;  // [n_j rounded up to even]
  int c0, n_j;
};
struct PhaseV64 {
  const double2* hi;  // [n_hi] (cos, sin)(theta 128 h)
  const double2* lo;  // [128]  (cos, sin)(theta l)
  int n_hi;
};
template <class R>
struct PhaseV;
template <>
struct PhaseV<float> {
  using params = PhaseV32;
  static constexpr int kSmemBytes = kPhaseH * (int)sizeof(float2);
  __device__ static void stage(const PhaseV32& P, unsigned char* s, int tid, int nthr) {
    float2* hab = reinterpret_cast<float2*>(s);
    for (int i = tid; i < P.n_h; i += nthr) hab[i] = P.hab[i];
  }
  __device__ static void shear2(float2& x, float2& y, float2 a, float2 b) {
    x = __ffma2_rn(a, y, x);
    y = __ffma2_rn(b, x, y);
    x = __ffma2_rn(a, y, x);
  }
  // the rotation coefficients of an element (two amplitudes); inverse: negated
  struct Coef {
    float2 a, b, A, B;
  };
  __device__ static Coef coef(uint32_t e2, const PhaseV32& P, const unsigned char* s, bool inverse) {
    const float2* hab = reinterpret_cast<const float2*>(s);
    const uint32_t e0 = e2 & 0xFFFFu, e1 = e2 >> 16;
    const uint32_t h0 = __umulhi(e0, P.M), h1 = __umulhi(e1, P.M);
    const uint32_t l0 = e0 - h0 * P.K, l1 = e1 - h1 * P.K;
    const float2 lf = __fadd2_rn(make_float2(__int_as_float(0x4B000000 | l0), __int_as_float(0x4B000000 | l1)),
                                 make_float2(-8388608.0f, -8388608.0f));
    const float2 r = __ffma2_rn(lf, make_float2(P.theta, P.theta), __fmul2_rn(lf, make_float2(P.theta_lo, P.theta_lo)));
    // a = -tan(r/2), b = sin r (Maclaurin to degree 9; |r| <= 1/2)
    const float2 x = __fmul2_rn(r, make_float2(0.5f, 0.5f));
    const float2 x2 = __fmul2_rn(x, x);
    float2 tt = __ffma2_rn(x2, make_float2(62.0f / 2835.0f, 62.0f / 2835.0f), make_float2(17.0f / 315.0f, 17.0f / 315.0f));
    tt = __ffma2_rn(x2, tt, make_float2(2.0f / 15.0f, 2.0f / 15.0f));
    tt = __ffma2_rn(x2, tt, make_float2(1.0f / 3.0f, 1.0f / 3.0f));
    tt = __ffma2_rn(x2, tt, make_float2(1.0f, 1.0f));
    Coef c;
    c.a = __fmul2_rn(make_float2(-x.x, -x.y), tt);
    const float2 r2 = __fmul2_rn(r, r);
    float2 u = __ffma2_rn(r2, make_float2(1.0f / 362880.0f, 1.0f / 362880.0f), make_float2(-1.0f / 5040.0f, -1.0f / 5040.0f));
    u = __ffma2_rn(r2, u, make_float2(1.0f / 120.0f, 1.0f / 120.0f));
    u = __ffma2_rn(r2, u, make_float2(-1.0f / 6.0f, -1.0f / 6.0f));
    u = __ffma2_rn(r2, u, make_float2(1.0f, 1.0f));
    c.b = __fmul2_rn(r, u);
    const float2 H0 = hab[h0], H1 = hab[h1];
    c.A = make_float2(H0.x, H1.x);
    c.B = make_float2(H0.y, H1.y);
    if (inverse) {
      c.A = make_float2(-c.A.x, -c.A.y);
      c.B = make_float2(-c.B.x, -c.B.y);
      c.a = make_float2(-c.a.x, -c.a.y);
      c.b = make_float2(-c.b.x, -c.b.y);
    }
    return c;
  }
  // forward: residual shear then the level shear twice; inverse: the negated
  // shears in reverse order
  __device__ static void rotate(El<float>::T& v, const Coef& c, bool inverse) {
    if (!inverse) {
      shear2(v.re, v.im, c.a, c.b);
      shear2(v.re, v.im, c.A, c.B);
      shear2(v.re, v.im, c.A, c.B);
    } else {
      shear2(v.re, v.im, c.A, c.B);
      shear2(v.re, v.im, c.A, c.B);
      shear2(v.re, v.im, c.a, c.b);
    }
  }
  __device__ static void apply(El<float>::T& v, uint32_t e2, const PhaseV32& P, const unsigned char* s,
                               bool inverse) {
    rotate(v, coef(e2, P, s, inverse), inverse);
  }
};
template <>
struct PhaseV<double> {
  using params = PhaseV64;
  static constexpr int kSmemBytes = (kPhaseHi64 + kPhaseLo) * (int)sizeof(double2);
  __device__ static void stage(const PhaseV64& P, unsigned char* s, int tid, int nthr) {
    double2* hi = reinterpret_cast<double2*>(s);
    double2* lo = hi + kPhaseHi64;
    for (int i = tid; i < P.n_hi; i += nthr) hi[i] = P.hi[i];
    for (int i = tid; i < kPhaseLo; i += nthr) lo[i] = P.lo[i];
  }
  using Coef = double2;  // (cos, sin) of the rotation
  __device__ static Coef coef(uint32_t e, const PhaseV64&, const unsigned char* s, bool inverse) {
    const double2* hi = reinterpret_cast<const double2*>(s);
    const double2* lo = hi + kPhaseHi64;
    const double2 h = hi[e >> kPhaseLoBits], l = lo[e & (kPhaseLo - 1)];
    const double c = fma(h.x, l.x, -h.y * l.y);
    const double sn = inverse ? -fma(h.x, l.y, h.y * l.x) : fma(h.x, l.y, h.y * l.x);
    return make_double2(c, sn);
  }
  __device__ static void rotate(El<double>::T& v, const Coef& cs, bool) {
    v.v = make_double2(fma(v.v.x, cs.x, -v.v.y * cs.y), fma(v.v.x, cs.y, v.v.y * cs.x));
  }
  __device__ static void apply(El<double>::T& v, uint32_t e, const PhaseV64& P, const unsigned char* s,
                               bool inverse) {
    rotate(v, coef(e, P, s, inverse), inverse);
  }
};

// ---------------------------------------------------------------------------
// per-statevector descriptor (device memory) and the launch's task program
// ---------------------------------------------------------------------------
template <class R>
struct InstDesc {
  unsigned char* state;          // 16-byte elements
  const CUtensorMap* map_a1;     // A1 / M tiles
  const CUtensorMap* map_e;      // E tile of an A1 task
  const CUtensorMap* map_s2;
  const CUtensorMap* map_s3;
  int np;                        // element bits (n for c128, n - 1 for c64)
  int n;                         // qubits
  int w2, w3;                    // widths of S2 / S3 (w3 = 0: no S3)
  int a1_hi_dim;
  int s2_mid_dim, s2_hi_dim, s2_mid_bits;
  int s3_mid_dim, s3_hi_dim, s3_mid_bits;
  int e0;
  uint32_t s0;
  typename PhaseV<R>::params phase;
  const R* tan;                  // [n_steps]
  const R* scale;                // [n_steps]: exact power of two applied with D
  const int* slot;               // [n_steps + 1]: measurement row or -1
  unsigned int* a1_done;         // [2^(np - 12 - w2)] per slab
  unsigned int* s2_done;
  unsigned int* s3_done;
  unsigned int* ticket;
  double* partials;              // [A1 tiles][3]
  double* results;               // [rows][4]
  uint32_t n_a1, n_s2, n_s3;     // tiles per step
  int e_recompute;               // 1: A1 / M recompute E(s) from popcounts instead of reading the E tile
  int a1_bits;                   // element bits the A1 pass butterflies (12; 9 for the warp-local A1)
  const CUtensorMap* map_a1s;    // warp-local A1: the A1 tile with the 128-byte TMA swizzle
  int a1_evict_first;            // per-pass A1 stores: 1 = evict-first (its output is not re-read soon)
  const CUtensorMap* map_e_half; // E of a half A1 tile (2^12 amplitude E values per box, complex64)
};

struct Program {
  const unsigned long long* tasks;  // one step's tasks: kind << 56 | inst << 32 | tile
  uint32_t per_step;
  uint32_t n_steps;
  const unsigned long long* final_tasks;  // measurement-only tasks after the last step
  uint32_t n_final;
  uint32_t step0;                   // global step index of this launch's first step
  unsigned int* next;               // work counter
  int* err;
  int* abort;
  uint32_t poll_limit;              // bound on the polls of one dependency wait
  // Test hook (0xFFFFFFFF = off): A1 / M tasks of this launch step wait for one
  // completion more than can ever arrive, so their bounded wait runs out and
  // the launch ends with DEV_TIMEOUT, as a lost producer would make it.
  uint32_t hold_step;
};

__device__ __forceinline__ uint32_t ld_acquire(const unsigned int* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void compute_sync() { __syncthreads(); }
// Barriers between the rounds of a tile: a round's layout change only moves
// data inside a warp (round 1 -> 2 of A1, the swizzled store after an
// unswizzled read) or inside a warp pair (512-thread A1, round 2 -> 3); a store
// back into the slots the same thread has just read needs no barrier.
__device__ __forceinline__ void warp_sync() { __syncwarp(); }
// warps 2m and 2m + 1 (named barrier 1 + m, 64 threads; at most 16 warps)
__device__ __forceinline__ void pair_sync() {
  asm volatile("bar.sync %0, 64;" ::"r"(1u + (threadIdx.x >> 6)) : "memory");
}
__device__ __forceinline__ bool aborted(const int* abort) {
  return *reinterpret_cast<const volatile int*>(abort) != 0;
}
__device__ __forceinline__ void raise_error(const Program& P, int code) {
  atomicCAS(P.err, 0, code);
  atomicExch(P.abort, 1);
}
// bounded wait on an mbarrier phase that also gives up on a global abort
__device__ __forceinline__ bool mbar_wait_or_abort(uint32_t bar, uint32_t parity, const Program& P) {
  for (uint32_t i = 0; i < kWaitPolls; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255u) == 255u && aborted(P.abort)) return false;
  }
  raise_error(P, DEV_TIMEOUT);
  return false;
}

struct StageMeta {
  int kind, inst;
  uint32_t tile, step;
};

// ---------------------------------------------------------------------------
// tile processing (compute warps; tid in [0, 256))
// ---------------------------------------------------------------------------
template <class R, uint32_t REG, bool SWZ>
__device__ __forceinline__ void el_load(const unsigned char* s, typename El<R>::T (&v)[16], uint32_t base) {
  const uint32_t sb = SWZ ? swz<double>(base) : base;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const uint32_t o = SWZ ? swz<double>(pdep((uint32_t)j, REG)) : pdep((uint32_t)j, REG);
    v[j] = El<R>::ld(s + 16u * (sb ^ o));
  }
}
template <class R, uint32_t REG>
__device__ __forceinline__ void el_store_swz(unsigned char* s, const typename El<R>::T (&v)[16], uint32_t base) {
  const uint32_t sb = swz<double>(base);
#pragma unroll
  for (int j = 0; j < 16; ++j) El<R>::st(s + 16u * (sb ^ swz<double>(pdep((uint32_t)j, REG))), v[j]);
}
template <class R, uint32_t REG, uint32_t ACT>
__device__ __forceinline__ void el_bflys(typename El<R>::T (&v)[16], R t) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if ((ACT & pdep(1u << k, REG)) != 0u) {
#pragma unroll
      for (int j = 0; j < 16; ++j)
        if (!(j & (1 << k))) El<R>::bfly(v[j], v[j | (1 << k)], t);
    }
  }
}
template <class R, uint32_t REG, int CP>
__device__ __forceinline__ void el_gstore(unsigned char* g, const typename El<R>::T (&v)[16], uint32_t tile_base,
                                          uint32_t base, uint32_t h0, uint64_t pol) {
  const uint32_t gb = tile_base | tile_to_global<CP>(base, h0);
#pragma unroll
  for (int j = 0; j < 16; ++j)
    El<R>::stg(g + 16ull * (gb | tile_to_global<CP>(pdep((uint32_t)j, REG), h0)), v[j], pol);
}

// measurement helpers on an element with E (c64: two uint16 packed)
__device__ __forceinline__ void measure_el(MeasureAcc& acc, const El<float>::T& v, uint32_t e2, uint32_t elem_g,
                                           int e0, uint32_t s0) {
  const uint32_t a0 = elem_g << 1;
  acc.add((double)fmaf(v.re.x, v.re.x, v.im.x * v.im.x), (int)(e2 & 0xFFFFu) < e0, __popc(a0 ^ s0));
  acc.add((double)fmaf(v.re.y, v.re.y, v.im.y * v.im.y), (int)(e2 >> 16) < e0, __popc((a0 | 1u) ^ s0));
}
__device__ __forceinline__ void measure_el(MeasureAcc& acc, const El<double>::T& v, uint32_t e, uint32_t elem_g,
                                           int e0, uint32_t s0) {
  acc.add(fma(v.v.x, v.v.x, v.v.y * v.v.y), (int)e < e0, __popc(elem_g ^ s0));
}
// E of a 16-byte element recomputed in integers (complex64: both amplitudes
// packed like the table's uint32 pair)
template <class R>
__device__ __forceinline__ uint32_t recompute_e(uint32_t elem_g, int n) {
  if constexpr (sizeof(R) == 4) {
    const uint32_t a0 = elem_g << 1;
    return (uint32_t)labs_energy(a0, n) | ((uint32_t)labs_energy(a0 | 1u, n) << 16);
  } else {
    return (uint32_t)labs_energy(elem_g, n);
  }
}
template <class R>
__device__ __forceinline__ uint32_t load_e(const unsigned char* etile, uint32_t elem) {
  if constexpr (sizeof(R) == 4)
    return reinterpret_cast<const uint32_t*>(etile)[elem];
  else
    return reinterpret_cast<const uint16_t*>(etile)[elem];
}

// consumer-side block reduction: per-tile partials, last tile of the step
// reduces all of them in index order into results[slot]; NW warps per CTA
template <int NW = kComputeThreads / 32>
__device__ __forceinline__ void compute_reduce(MeasureAcc acc, double* partials, unsigned int* ticket,
                                               double* results, int slot, uint32_t tile, uint32_t ntiles,
                                               double* red /* smem [3][NW] */, int* last_flag) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double a = warp_sum(acc.norm), b = warp_sum(acc.p_less), c = warp_sum(acc.d_h);
  if (lane == 0) {
    red[0 * NW + warp] = a;
    red[1 * NW + warp] = b;
    red[2 * NW + warp] = c;
  }
  __syncthreads();
  if (tid == 0) {
    double s0 = 0, s1 = 0, s2 = 0;
    for (int w = 0; w < NW; ++w) {
      s0 += red[w];
      s1 += red[NW + w];
      s2 += red[2 * NW + w];
    }
    partials[3 * (size_t)tile + 0] = s0;
    partials[3 * (size_t)tile + 1] = s1;
    partials[3 * (size_t)tile + 2] = s2;
    __threadfence();
    *last_flag = (atomicAdd(ticket, 1u) == ntiles - 1u);
  }
  __syncthreads();
  if (!*last_flag) return;
  __threadfence();
  double s0 = 0, s1 = 0, s2 = 0;
  for (uint32_t i = tid; i < ntiles; i += 32u * NW) {
    s0 += __ldcg(&partials[3 * (size_t)i + 0]);
    s1 += __ldcg(&partials[3 * (size_t)i + 1]);
    s2 += __ldcg(&partials[3 * (size_t)i + 2]);
  }
  s0 = warp_sum(s0);
  s1 = warp_sum(s1);
  s2 = warp_sum(s2);
  __syncthreads();
  if (lane == 0) {
    red[warp] = s0;
    red[NW + warp] = s1;
    red[2 * NW + warp] = s2;
  }
  __syncthreads();
  if (tid == 0) {
    double nn = 0, p = 0, d = 0;
    for (int w = 0; w < NW; ++w) {
      nn += red[w];
      p += red[NW + w];
      d += red[2 * NW + w];
    }
    results[4 * (size_t)slot + 0] = p;
    results[4 * (size_t)slot + 1] = d;
    results[4 * (size_t)slot + 2] = nn;
    *ticket = 0u;
  }
}

// ---------------------------------------------------------------------------
// Full phase table (BK_OPT_PHASE_TABLE, complex64 per-pass A1 kernels): every
// LABS energy is E = c0 + 4 j with c0 = floor(n/2) mod 4, so one table entry
// {-tan(r/4), sin(r/2)} per level j (r = theta E reduced to (-pi, pi]) gives the
// rotation as two half-angle shear rotations: no level split and no residual
// polynomial, a third of the phase's FMA work. The table (at most 2139 entries,
// 17 KB at n = 30) arrives by one bulk copy on the tile's own barrier.
// ---------------------------------------------------------------------------
constexpr int kPhaseTabMax = 2144;  // >= (8555 - 3) / 4 + 1 entries at n = 30, even
constexpr int kPhaseTabBytes = kPhaseTabMax * (int)sizeof(float2);
static_assert(kPhaseTabBytes >= 3328, "the table room also holds the level tables");

// bytes of the table copy (the count rounded up to an even number of entries: 16-byte multiple)
__device__ __forceinline__ uint32_t phase_tab_bytes(const PhaseV32& P) {
  return (uint32_t)((P.n_j + 1) & ~1) * (uint32_t)sizeof(float2);
}

// the full-table rotation of a complex64 element (two amplitudes, energies packed in e2)
__device__ __forceinline__ void phase_table_apply(El<float>::T& v, uint32_t e2, const unsigned char* s,
                                                  uint32_t c0) {
  const float2* tab = reinterpret_cast<const float2*>(s);
  const uint32_t j0 = ((e2 & 0xFFFFu) - c0) >> 2, j1 = ((e2 >> 16) - c0) >> 2;
  const float2 H0 = tab[j0], H1 = tab[j1];
  const float2 A = make_float2(H0.x, H1.x), B = make_float2(H0.y, H1.y);
  PhaseV<float>::shear2(v.re, v.im, A, B);
  PhaseV<float>::shear2(v.re, v.im, A, B);
}

// the A1 kernels' phase: the full table (kTab, complex64) or the level table with residual polynomials
template <class R, bool kTab>
__device__ __forceinline__ void a1_phase(typename El<R>::T& v, uint32_t e, const InstDesc<R>& D,
                                         const unsigned char* phase_smem) {
  if constexpr (kTab)
    phase_table_apply(v, e, phase_smem, (uint32_t)D.phase.c0);
  else
    PhaseV<R>::apply(v, e, D.phase, phase_smem, false);
}

// A1 (and measurement-only M) on a staged tile
// `stage_free()` runs (in every thread, after a barrier) as soon as the last
// shared-memory read of the staged tile is done, so the next tile's load can be
// issued while this tile's last round computes and its stores drain.
template <class R, bool MEASURE_ONLY, bool kTab = false, class F>
__device__ __forceinline__ void process_a1(unsigned char* tile, const unsigned char* etile, const InstDesc<R>& D,
                                           uint32_t t_idx, uint32_t step, const unsigned char* phase_smem,
                                           double* red, int* last_flag, F&& stage_free) {
  using PL = Plan<double>;
  using E = El<R>;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t tile_base = t_idx << kElemBits;
  typename E::T v[16];
  const uint32_t b1 = pdep(lane, PL::A1_R1_LANE) | pdep(warp, PL::A1_R1_WARP);
  el_load<R, PL::A1_R1_REG, false>(tile, v, b1);
  const int slot = D.slot[step];
  MeasureAcc acc;
  const R t = MEASURE_ONLY ? (R)0 : D.tan[step];
  if (MEASURE_ONLY) {
    // measurement only: read the E values first, then release the stage
    uint32_t ev[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const uint32_t i = b1 | pdep((uint32_t)j, PL::A1_R1_REG);
      ev[j] = D.e_recompute ? recompute_e<R>(tile_base | i, D.n) : load_e<R>(etile, i);
    }
    __syncthreads();
    stage_free();
#pragma unroll
    for (int j = 0; j < 16; ++j) measure_el(acc, v[j], ev[j], tile_base | (b1 | pdep((uint32_t)j, PL::A1_R1_REG)), D.e0, D.s0);
  }
#pragma unroll
  for (int j = 0; j < 16 && !MEASURE_ONLY; ++j) {
    const uint32_t i = b1 | pdep((uint32_t)j, PL::A1_R1_REG);
    const uint32_t e = D.e_recompute ? recompute_e<R>(tile_base | i, D.n) : load_e<R>(etile, i);
    if (slot >= 0) measure_el(acc, v[j], e, tile_base | i, D.e0, D.s0);
    if (!MEASURE_ONLY) {
      a1_phase<R, kTab>(v[j], e, D, phase_smem);
      E::bfly_inner(v[j], t);
    }
  }
  if (!MEASURE_ONLY) {
    const R sc = D.scale[step];
    if (sc != (R)1) {
#pragma unroll
      for (int j = 0; j < 16; ++j) E::scale(v[j], sc);
    }
    el_bflys<R, PL::A1_R1_REG, PL::A1_R1_REG>(v, t);
    warp_sync();  // round-1 reads vs swizzled stores: same warp (warp bits 9-11)
    el_store_swz<R, PL::A1_R1_REG>(tile, v, b1);
    warp_sync();  // rounds 1 and 2 share the warp bits
    const uint32_t b2 = pdep(lane, PL::A1_R2_LANE) | pdep(warp, PL::A1_R2_WARP);
    el_load<R, PL::A1_R2_REG, true>(tile, v, b2);
    el_bflys<R, PL::A1_R2_REG, PL::A1_R2_REG>(v, t);
    el_store_swz<R, PL::A1_R2_REG>(tile, v, b2);  // in place
    compute_sync();
    const uint32_t b3 = pdep(lane, PL::A1_R3_LANE) | pdep(warp, PL::A1_R3_WARP);
    el_load<R, PL::A1_R3_REG, true>(tile, v, b3);
    __syncthreads();
    stage_free();
    el_bflys<R, PL::A1_R3_REG, PL::A1_R3_ACT>(v, t);
    el_gstore<R, PL::A1_R3_REG, kElemBits>(D.state, v, tile_base, b3, 0,
                                            D.a1_evict_first ? policy_evict_first() : policy_evict_last());
  }
  if (MEASURE_ONLY || slot >= 0)
    compute_reduce(acc, D.partials, D.ticket, D.results, MEASURE_ONLY ? D.slot[step] : slot, t_idx, D.n_a1, red,
                   last_flag);
}

// Barrier over the threads that process one tile: the whole CTA (grid and
// persistent kernels), or one 256-thread compute group of the fused strided
// pass (named barrier `id`).
struct CtaSync {
  __device__ void sync() const { __syncthreads(); }
};
struct GroupSync {
  uint32_t id;
  __device__ void sync() const { asm volatile("bar.sync %0, 256;" ::"r"(id) : "memory"); }
};

// strided pass of width W on a staged tile (element bits [0, 12 - W) u [h0, h0 + W));
// tid in [0, 256) is the thread's index in the tile's group, `sy` its barrier
template <class R, int W, class Sync, class F>
__device__ __forceinline__ void process_s(unsigned char* tile, unsigned char* state, uint32_t tile_base,
                                          uint32_t h0, R t, F&& stage_free, uint32_t tid, const Sync& sy,
                                          uint64_t store_pol) {
  using PL = Plan<double>;
  using E = El<R>;
  constexpr int CP = kElemBits - W;
  const uint32_t lane = tid & 31u, warp = tid >> 5;
  typename E::T v[16];
  constexpr uint32_t ACT_ALL = ((1u << W) - 1u) << CP;
  const uint32_t b1 = pdep(lane, PL::S_R1_LANE) | pdep(warp, PL::S_R1_WARP);
  el_load<R, PL::S_R1_REG, false>(tile, v, b1);
  if constexpr (W <= 4) {
    sy.sync();
    stage_free();
  }
  el_bflys<R, PL::S_R1_REG, ACT_ALL>(v, t);
  if constexpr (W <= 4) {
    el_gstore<R, PL::S_R1_REG, CP>(state, v, tile_base, b1, h0, store_pol);
  } else {
    using R2 = StridedR2<double, W>;
    warp_sync();  // round-1 reads vs swizzled stores: same warp
    el_store_swz<R, PL::S_R1_REG>(tile, v, b1);
    sy.sync();
    const uint32_t b2 = pdep(lane, R2::LANE) | pdep(warp, R2::WARP);
    el_load<R, R2::REG, true>(tile, v, b2);
    sy.sync();
    stage_free();
    el_bflys<R, R2::REG, R2::ACT>(v, t);
    if constexpr (R2::kShuffleLaneBit >= 0) {
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const typename E::T q = E::shfl_xor(v[j], 1 << R2::kShuffleLaneBit);
        E::bfly_partner(v[j], q, t);
      }
    }
    el_gstore<R, R2::REG, CP>(state, v, tile_base, b2, h0, store_pol);
  }
}

template <class R, class Sync, class F>
__device__ __forceinline__ void process_s_dispatch(int w, unsigned char* tile, unsigned char* state,
                                                   uint32_t tile_base, uint32_t h0, R t, F&& f, uint32_t tid,
                                                   const Sync& sy, uint64_t pol) {
  switch (w) {
    case 1: process_s<R, 1>(tile, state, tile_base, h0, t, f, tid, sy, pol); break;
    case 2: process_s<R, 2>(tile, state, tile_base, h0, t, f, tid, sy, pol); break;
    case 3: process_s<R, 3>(tile, state, tile_base, h0, t, f, tid, sy, pol); break;
    case 4: process_s<R, 4>(tile, state, tile_base, h0, t, f, tid, sy, pol); break;
    case 5: process_s<R, 5>(tile, state, tile_base, h0, t, f, tid, sy, pol); break;
    case 6: process_s<R, 6>(tile, state, tile_base, h0, t, f, tid, sy, pol); break;
    case 7: process_s<R, 7>(tile, state, tile_base, h0, t, f, tid, sy, pol); break;
    case 8: process_s<R, 8>(tile, state, tile_base, h0, t, f, tid, sy, pol); break;
    default: process_s<R, 9>(tile, state, tile_base, h0, t, f, tid, sy, pol); break;
  }
}
template <class R, class F>
__device__ __forceinline__ void process_s_dispatch(int w, unsigned char* tile, unsigned char* state,
                                                   uint32_t tile_base, uint32_t h0, R t, F&& f) {
  process_s_dispatch<R>(w, tile, state, tile_base, h0, t, f, threadIdx.x, CtaSync{}, policy_evict_first());
}

// ---------------------------------------------------------------------------
// the persistent kernel: 2 CTAs per SM, one stage each; thread 0 claims tasks,
// waits (bounded) for their dependencies and issues the TMA; the next task's
// load is issued early, while this task's stores drain, whenever its
// dependency is already met (never blocking before this task has signalled).
// ---------------------------------------------------------------------------
struct PersistSmem {
  static constexpr int kStageBytes = kStageTileBytes + kStageEBytes;
  static constexpr int kPhaseOff = kStageBytes;
  static constexpr int kRedOff = kPhaseOff + 3328;  // >= both phase table footprints
  static constexpr int kBytes = kRedOff + 512;  // reduction scratch: [3][16] doubles
};

template <class R>
__device__ __forceinline__ bool decode_task(const Program& P, uint32_t g, StageMeta& m) {
  if (g >= P.per_step * P.n_steps + P.n_final) return false;
  unsigned long long task;
  uint32_t k;
  if (g < P.per_step * P.n_steps) {
    k = g / P.per_step;
    task = P.tasks[g - k * P.per_step];
  } else {
    k = P.n_steps;
    task = P.final_tasks[g - P.per_step * P.n_steps];
  }
  m.kind = (int)(task >> 56);
  m.inst = (int)((task >> 32) & 0xFFFFFFu);
  m.tile = (uint32_t)task;
  m.step = k;
  return true;
}

// dependency of a task: counter and target (ctr == nullptr: none)
template <class R>
__device__ __forceinline__ const unsigned int* task_dep(const InstDesc<R>& D, const StageMeta& m, uint32_t& target,
                                                        const Program& P) {
  if (m.kind == TASK_A1 || m.kind == TASK_M) {
    if (m.step == 0) return nullptr;
    target = (D.w3 > 0 ? D.n_s3 : D.n_s2) * m.step + (m.step == P.hold_step ? 1u : 0u);
    return D.w3 > 0 ? D.s3_done : D.s2_done;
  }
  if (m.kind == TASK_S2) {
    target = (1u << D.w2) * (m.step + 1u);
    return D.a1_done + (m.tile >> D.w2);
  }
  target = D.n_s2 * (m.step + 1u);
  return D.s2_done;
}

template <class R>
__device__ __forceinline__ void issue_task_load(const InstDesc<R>& D, const StageMeta& m, unsigned char* stage,
                                                uint32_t fb, uint32_t extra_tx = 0u) {
  if (m.kind == TASK_A1 || m.kind == TASK_M) {
    const bool e_tile = !D.e_recompute;
    mbar_arrive_expect_tx(fb, (uint32_t)kStageTileBytes + (e_tile ? 4096u * 2u * (uint32_t)El<R>::kAmps : 0u) +
                                  extra_tx);
    const int hd = D.a1_hi_dim;
    const uint64_t pol = policy_evict_first();
    tma_load_5d_hint(smem_addr(stage), D.map_a1, 0, 0, hd == 2 ? (int)m.tile : 0, hd == 3 ? (int)m.tile : 0, 0, fb,
                     pol);
    if (e_tile) tma_load_5d_hint(smem_addr(stage + kStageTileBytes), D.map_e, 0, 0, (int)m.tile, 0, 0, fb, pol);
  } else {
    const bool s2 = (m.kind == TASK_S2);
    const int mb = s2 ? D.s2_mid_bits : D.s3_mid_bits;
    const int md = s2 ? D.s2_mid_dim : D.s3_mid_dim;
    const int hd = s2 ? D.s2_hi_dim : D.s3_hi_dim;
    const int mid = (int)(m.tile & ((1u << mb) - 1u)), hi = (int)(m.tile >> mb);
    mbar_arrive_expect_tx(fb, (uint32_t)kStageTileBytes);
    tma_load_5d_hint(smem_addr(stage), s2 ? D.map_s2 : D.map_s3, tile_coord(0, md, mid, hd, hi),
                     tile_coord(1, md, mid, hd, hi), tile_coord(2, md, mid, hd, hi), tile_coord(3, md, mid, hd, hi),
                     tile_coord(4, md, mid, hd, hi), fb, policy_evict_first());
  }
}

// bounded wait for a dependency counter (thread 0); false on timeout / abort
__device__ __forceinline__ bool wait_counter(const unsigned int* ctr, uint32_t target, const Program& P) {
  uint32_t polls = 0;
  while (ld_acquire(ctr) < target) {
    if (++polls > P.poll_limit) {
      raise_error(P, DEV_TIMEOUT);
      return false;
    }
    if ((polls & 63u) == 0u && aborted(P.abort)) return false;
    __nanosleep(32);
  }
  fence_proxy_async_global();  // the TMA (async proxy) must see the data the counter released
  return true;
}

template <class R>
__device__ __forceinline__ bool dep_met(const unsigned int* ctr, uint32_t target, uint32_t seen) {
  return ctr == nullptr || seen >= target;
}

// kCacheDesc: keep the running statevector's descriptor in shared memory (a
// launch over one statevector); batched launches, whose consecutive tasks mostly
// belong to different statevectors, read it from global memory instead.
template <class R, bool kCacheDesc>
__global__ void __launch_bounds__(kComputeThreads, 2)
    persist_kernel(const InstDesc<R>* __restrict__ insts, const Program P) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t full_bar;
  __shared__ int last_flag;
  __shared__ int cur_phase_inst;
  __shared__ StageMeta cur, nxt;
  __shared__ uint32_t g_after;
  __shared__ int inflight;  // a tile load is issued and not yet consumed
  __shared__ int early;     // the current task's stage_free() issued the next load
  __shared__ StageMeta after;  // the task after next, decoded while the current one computes
  __shared__ __align__(16) InstDesc<R> sdesc;  // descriptor of the running task's statevector
  __shared__ int sdesc_inst;
  unsigned char* stage = smem;
  unsigned char* phase_smem = smem + PersistSmem::kPhaseOff;
  double* red = reinterpret_cast<double*>(smem + PersistSmem::kRedOff);
  const int tid = threadIdx.x;
  const uint32_t fb = smem_addr(&full_bar);
  // thread 0 keeps the next task decoded (nxt) and the one after that claimed
  // (g_after), so the claim's atomic and the dependency load are in flight while
  // the tile computes
  if (tid == 0) {
    mbar_init(fb, 1);
    fence_barrier_init();
    cur_phase_inst = -1;
    sdesc_inst = -1;
    inflight = 0;
    const uint32_t g0 = atomicAdd(P.next, 1u);
    const uint32_t g1 = atomicAdd(P.next, 1u);
    if (!decode_task<R>(P, g0, cur)) {
      cur.kind = TASK_END;
    } else {
      const InstDesc<R>& D = insts[cur.inst];
      uint32_t target = 0;
      const unsigned int* ctr = task_dep(D, cur, target, P);
      if (ctr && !wait_counter(ctr, target, P)) cur.kind = TASK_END;
      if (cur.kind != TASK_END) {
        issue_task_load(D, cur, stage, fb);
        inflight = 1;
      }
    }
    if (!decode_task<R>(P, g1, nxt)) nxt.kind = TASK_END;
    g_after = 0xFFFFFFFFu;
  }
  __syncthreads();
  uint32_t phase = 0;
  for (;;) {
    const StageMeta m = cur;
    if (m.kind == TASK_END) break;
    // thread 0: claim the task after next, read the next task's dependency early
    const unsigned int* nctr = nullptr;
    uint32_t ntarget = 0, nseen = 0;
    if (tid == 0) {
      g_after = aborted(P.abort) ? 0xFFFFFFFFu : atomicAdd(P.next, 1u);
      if (nxt.kind != TASK_END) {
        nctr = task_dep(insts[nxt.inst], nxt, ntarget, P);
        if (nctr) nseen = ld_acquire(nctr);
      }
    }
    if (!mbar_wait_or_abort(fb, phase, P)) break;
    phase ^= 1u;
    if (tid == 0) inflight = 0;
    if (kCacheDesc && m.inst != sdesc_inst) {
      // the statevector changed: cache its descriptor in shared memory
      const uint32_t* src = reinterpret_cast<const uint32_t*>(insts + m.inst);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&sdesc);
      for (int w = tid; w < (int)(sizeof(InstDesc<R>) / 4); w += kComputeThreads) dst[w] = src[w];
      __syncthreads();
      if (tid == 0) sdesc_inst = m.inst;
    }
    const InstDesc<R>& D = kCacheDesc ? sdesc : insts[m.inst];
    // the counter this task completes, read now: the next task may replace the
    // cached descriptor while warp 1 still signals this one
    unsigned int* done_ctr = m.kind == TASK_A1 ? D.a1_done + (m.tile >> D.w2)
                             : m.kind == TASK_S2 ? D.s2_done
                             : m.kind == TASK_S3 ? D.s3_done
                                                 : nullptr;
    // stage free: issue the next task's load now if its dependency is met, and
    // decode the task after next (its claim was issued at the top of the loop)
    auto stage_free = [&]() {
      if (tid == 0) {
        early = 0;
        // a dependency not met at the top of the loop may be met by now
        if (nxt.kind != TASK_END && nctr != nullptr && nseen < ntarget) nseen = ld_acquire(nctr);
        if (nxt.kind != TASK_END && dep_met<R>(nctr, ntarget, nseen)) {
          if (nctr) fence_proxy_async_global();
          issue_task_load(insts[nxt.inst], nxt, stage, fb);
          inflight = 1;
          early = 1;
        }
        if (!decode_task<R>(P, g_after, after)) after.kind = TASK_END;
      }
    };
    if (m.kind == TASK_A1) {
      if (cur_phase_inst != m.inst) {
        PhaseV<R>::stage(D.phase, phase_smem, tid, kComputeThreads);
        __syncthreads();
        if (tid == 0) cur_phase_inst = m.inst;
      }
      process_a1<R, false>(stage, stage + kStageTileBytes, D, m.tile, m.step, phase_smem, red, &last_flag,
                           stage_free);
    } else if (m.kind == TASK_M) {
      process_a1<R, true>(stage, stage + kStageTileBytes, D, m.tile, m.step, phase_smem, red, &last_flag,
                          stage_free);
    } else {
      const bool s2 = (m.kind == TASK_S2);
      const int w = s2 ? D.w2 : D.w3;
      const int mb = s2 ? D.s2_mid_bits : D.s3_mid_bits;
      const uint32_t h0 = s2 ? (uint32_t)kElemBits : (uint32_t)(kElemBits + D.w2);
      const uint32_t cp = (uint32_t)(kElemBits - w);
      const uint32_t mid = m.tile & ((1u << mb) - 1u), hi = m.tile >> mb;
      const uint32_t tile_base = (mid << cp) | (hi << (h0 + (uint32_t)w));
      process_s_dispatch<R>(w, stage, D.state, tile_base, h0, D.tan[m.step], stage_free);
    }
    __syncthreads();  // every store of this task is issued
    bool pending = false;
    if (tid == 0) {
      pending = (nxt.kind != TASK_END) && !early;
      cur = nxt;
      nxt = after;
    }
    __syncthreads();  // publish cur
    if (tid == 32) {
      // completion of task m: the stores of every thread precede the barrier
      // above; this gpu-scope fence releases them together with the counter
      __threadfence();
      if (done_ctr) atomicAdd(done_ctr, 1u);
    }
    if (tid == 0 && pending) {
      const InstDesc<R>& D2 = insts[cur.inst];
      uint32_t target = 0;
      const unsigned int* ctr = task_dep(D2, cur, target, P);
      if (wait_counter(ctr, target, P)) {
        issue_task_load(D2, cur, stage, fb);
        inflight = 1;
      } else {
        // the failure is recorded; the others see the abort while waiting for the tile
      }
    }
  }
  // a load still in flight (issued early for a task that will not run) lands before exit
  if (tid == 0 && inflight) mbar_wait_bounded(fb, phase, P.err);
}

// shared memory of a 64 KB-tile A1 kernel: the stage, the phase room, reduction scratch
template <bool kTab>
struct A1Smem {
  static constexpr int kPhaseOff = PersistSmem::kStageBytes;
  static constexpr int kRedOff = kPhaseOff + (kTab ? kPhaseTabBytes : 3328);
  static constexpr int kBytes = kRedOff + 512;
};

// ---------------------------------------------------------------------------
// Wide A1 for the per-pass schedule: 512 threads x 8 elements per tile, so 32
// warps share an SM (two CTAs) instead of 16 — more latency hiding for the
// diagonal phase, the pass's dominant cost. Four rounds of 3 register bits
// (tile bits 3-5 in the TMA layout, then 0-2, 6-8, 9-11 through the swizzled
// shared tile; every 16-byte access conflict free, the last round's stores
// 512 contiguous bytes per warp). Same arithmetic per element as process_a1.
// ---------------------------------------------------------------------------
struct PlanA1Wide {
  static constexpr uint32_t R1_REG = 0x038, R1_LANE = 0x0C7, R1_WARP = 0xF00;
  static constexpr uint32_t R2_REG = 0x007, R2_LANE = 0x0F8, R2_WARP = 0xF00;
  static constexpr uint32_t R3_REG = 0x1C0, R3_LANE = 0x01F, R3_WARP = 0xE20;
  static constexpr uint32_t R4_REG = 0xE00, R4_LANE = 0x01F, R4_WARP = 0x1E0;
};
constexpr int kA1WideThreads = 512;

template <class R, uint32_t REG, bool SWZ>
__device__ __forceinline__ void el8_load(const unsigned char* s, typename El<R>::T (&v)[8], uint32_t base) {
  const uint32_t sb = SWZ ? swz<double>(base) : base;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const uint32_t o = SWZ ? swz<double>(pdep((uint32_t)j, REG)) : pdep((uint32_t)j, REG);
    v[j] = El<R>::ld(s + 16u * (sb ^ o));
  }
}
template <class R, uint32_t REG>
__device__ __forceinline__ void el8_store_swz(unsigned char* s, const typename El<R>::T (&v)[8], uint32_t base) {
  const uint32_t sb = swz<double>(base);
#pragma unroll
  for (int j = 0; j < 8; ++j) El<R>::st(s + 16u * (sb ^ swz<double>(pdep((uint32_t)j, REG))), v[j]);
}
template <class R>
__device__ __forceinline__ void el8_bflys(typename El<R>::T (&v)[8], R t) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (!(j & (1 << k))) El<R>::bfly(v[j], v[j | (1 << k)], t);
  }
}

template <class R, bool kTab>
__global__ void __launch_bounds__(kA1WideThreads, 2)
    tile_a1_wide_kernel(const __grid_constant__ InstDesc<R> D, uint32_t step, int* err) {
  static_assert(!kTab || sizeof(R) == 4, "the full phase table is complex64 only");
  using PL = PlanA1Wide;
  using E = El<R>;
  using SM = A1Smem<kTab>;
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t full_bar;
  __shared__ int last_flag;
  unsigned char* tile = smem;
  const unsigned char* etile = smem + kStageTileBytes;
  unsigned char* phase_smem = smem + SM::kPhaseOff;
  double* red = reinterpret_cast<double*>(smem + SM::kRedOff);
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t fb = smem_addr(&full_bar);
  const uint32_t t_idx = blockIdx.x;
  const uint32_t tile_base = t_idx << kElemBits;
  StageMeta m;
  m.kind = TASK_A1;
  m.inst = 0;
  m.tile = t_idx;
  m.step = step;
  if (tid == 0) {
    mbar_init(fb, 1);
    fence_barrier_init();
    if constexpr (kTab) {
      const uint32_t tb = phase_tab_bytes(D.phase);
      issue_task_load(D, m, tile, fb, tb);
      bulk_load(smem_addr(phase_smem), D.phase.tab, tb, fb);
    } else {
      issue_task_load(D, m, tile, fb);
    }
  }
  if constexpr (!kTab) PhaseV<R>::stage(D.phase, phase_smem, (int)tid, kA1WideThreads);
  __syncthreads();
  const bool ok = mbar_wait_bounded(fb, 0, err);
  if (__syncthreads_or(!ok)) return;
  typename E::T v[8];
  const R t = D.tan[step];
  const int slot = D.slot[step];
  MeasureAcc acc;
  const uint32_t b1 = pdep(lane, PL::R1_LANE) | pdep(warp, PL::R1_WARP);
  el8_load<R, PL::R1_REG, false>(tile, v, b1);
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const uint32_t i = b1 | pdep((uint32_t)j, PL::R1_REG);
    const uint32_t e = D.e_recompute ? recompute_e<R>(tile_base | i, D.n) : load_e<R>(etile, i);
    if (slot >= 0) measure_el(acc, v[j], e, tile_base | i, D.e0, D.s0);
    a1_phase<R, kTab>(v[j], e, D, phase_smem);
    E::bfly_inner(v[j], t);
  }
  const R sc = D.scale[step];
  if (sc != (R)1) {
#pragma unroll
    for (int j = 0; j < 8; ++j) E::scale(v[j], sc);
  }
  el8_bflys<R>(v, t);
  warp_sync();  // round-1 reads vs swizzled stores: same warp
  el8_store_swz<R, PL::R1_REG>(tile, v, b1);
  warp_sync();  // rounds 1 and 2 share the warp bits (8-11)
  const uint32_t b2 = pdep(lane, PL::R2_LANE) | pdep(warp, PL::R2_WARP);
  el8_load<R, PL::R2_REG, true>(tile, v, b2);
  el8_bflys<R>(v, t);
  el8_store_swz<R, PL::R2_REG>(tile, v, b2);  // in place
  pair_sync();  // rounds 2 and 3 share warp bits 9-11: data moves inside a warp pair
  const uint32_t b3 = pdep(lane, PL::R3_LANE) | pdep(warp, PL::R3_WARP);
  el8_load<R, PL::R3_REG, true>(tile, v, b3);
  el8_bflys<R>(v, t);
  el8_store_swz<R, PL::R3_REG>(tile, v, b3);  // in place
  __syncthreads();
  const uint32_t b4 = pdep(lane, PL::R4_LANE) | pdep(warp, PL::R4_WARP);
  el8_load<R, PL::R4_REG, true>(tile, v, b4);
  el8_bflys<R>(v, t);
  const uint64_t pol = D.a1_evict_first ? policy_evict_first() : policy_evict_last();
#pragma unroll
  for (int j = 0; j < 8; ++j) E::stg(D.state + 16ull * (tile_base | b4 | pdep((uint32_t)j, PL::R4_REG)), v[j], pol);
  if (slot >= 0)
    compute_reduce<kA1WideThreads / 32>(acc, D.partials, D.ticket, D.results, slot, t_idx, D.n_a1, red, &last_flag);
}

// ---------------------------------------------------------------------------
// Grid variant: one CTA per tile of one pass (kind = TASK_A1 / TASK_S2 /
// TASK_S3 / TASK_M), no dependencies (the kernel boundary orders the passes).
// Same tile arithmetic as the persistent engine; blockIdx.x is the tile. The
// descriptor is a kernel parameter (constant bank), so the TMA coordinates need
// no dependent global loads.
// ---------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(kComputeThreads, 2)
    tile_pass_kernel(const __grid_constant__ InstDesc<R> D, int kind, uint32_t step, int* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t full_bar;
  __shared__ int last_flag;
  unsigned char* stage = smem;
  unsigned char* phase_smem = smem + PersistSmem::kPhaseOff;
  double* red = reinterpret_cast<double*>(smem + PersistSmem::kRedOff);
  const int tid = threadIdx.x;
  const uint32_t fb = smem_addr(&full_bar);
  StageMeta m;
  m.kind = kind;
  m.inst = 0;
  m.tile = blockIdx.x;
  m.step = step;
  // the tile load goes out first; the phase tables are staged while it is in flight
  if (tid == 0) {
    mbar_init(fb, 1);
    fence_barrier_init();
    issue_task_load(D, m, stage, fb);
  }
  if (kind == TASK_A1) PhaseV<R>::stage(D.phase, phase_smem, tid, kComputeThreads);
  __syncthreads();
  const bool ok = mbar_wait_bounded(fb, 0, err);
  if (__syncthreads_or(!ok)) return;
  auto none = []() {};
  if (kind == TASK_A1) {
    process_a1<R, false>(stage, stage + kStageTileBytes, D, m.tile, step, phase_smem, red, &last_flag, none);
  } else if (kind == TASK_M) {
    process_a1<R, true>(stage, stage + kStageTileBytes, D, m.tile, step, phase_smem, red, &last_flag, none);
  } else {
    const bool s2 = (kind == TASK_S2);
    const int w = s2 ? D.w2 : D.w3;
    const int mb = s2 ? D.s2_mid_bits : D.s3_mid_bits;
    const uint32_t h0 = s2 ? (uint32_t)D.a1_bits : (uint32_t)(D.a1_bits + D.w2);
    const uint32_t cp = (uint32_t)(kElemBits - w);
    const uint32_t mid = m.tile & ((1u << mb) - 1u), hi = m.tile >> mb;
    const uint32_t tile_base = (mid << cp) | (hi << (h0 + (uint32_t)w));
    process_s_dispatch<R>(w, stage, D.state, tile_base, h0, D.tan[step], none);
  }
}

// The 256-thread A1 (BK_OPT_A1_WIDE = 0) as its own grid kernel with the full
// phase table (complex64): three rounds of 16 elements per thread move each
// element through shared memory five times against seven in the 512-thread A1,
// which matters once the table's lookups share the shared-memory pipe.
template <class R>
__global__ void __launch_bounds__(kComputeThreads, 2)
    tile_a1_tab_kernel(const __grid_constant__ InstDesc<R> D, uint32_t step, int* err) {
  static_assert(sizeof(R) == 4, "the full phase table is complex64 only");
  using SM = A1Smem<true>;
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t full_bar;
  __shared__ int last_flag;
  unsigned char* stage = smem;
  unsigned char* phase_smem = smem + SM::kPhaseOff;
  double* red = reinterpret_cast<double*>(smem + SM::kRedOff);
  const uint32_t fb = smem_addr(&full_bar);
  StageMeta m;
  m.kind = TASK_A1;
  m.inst = 0;
  m.tile = blockIdx.x;
  m.step = step;
  if (threadIdx.x == 0) {
    mbar_init(fb, 1);
    fence_barrier_init();
    const uint32_t tb = phase_tab_bytes(D.phase);
    issue_task_load(D, m, stage, fb, tb);
    bulk_load(smem_addr(phase_smem), D.phase.tab, tb, fb);
  }
  __syncthreads();
  const bool ok = mbar_wait_bounded(fb, 0, err);
  if (__syncthreads_or(!ok)) return;
  auto none = []() {};
  process_a1<R, false, true>(stage, stage + kStageTileBytes, D, m.tile, step, phase_smem, red, &last_flag, none);
}

// ---------------------------------------------------------------------------
// Warp-local A1 (per-pass schedule, up to 27 element bits): the pass butterflies
// element bits 0-8 (+ amplitude bit 0 for complex64), so every warp owns the
// contiguous 512-element block of the tile with its warp bits 9-11 and both
// rounds stay inside the warp: no CTA barrier. The tile arrives through the
// 128-byte TMA swizzle (16-byte chunk address bits 4-6 ^= bits 7-9), which makes
// round 1 (register bits 0-2, 6; lane bits 3-5, 7, 8) conflict free; round 2
// (register bits 3-5, 7; lane bits 0-2, 6, 8) reads the engine's XOR swizzle
// and does bit 8 across lanes 16 apart, then stores 128-byte runs. The strided
// passes cover element bits 9 and up.
// ---------------------------------------------------------------------------
struct PlanA1Warp {
  static constexpr uint32_t R1_REG = 0x047, R1_LANE = 0x1B8;
  static constexpr uint32_t R2_REG = 0x0B8, R2_LANE = 0x147;
  static constexpr uint32_t WARP = 0xE00;
  static constexpr int kShuffleLanes = 16;  // tile bit 8 = round-2 lane bit 4
};
constexpr int kA1WarpBits = 9;
constexpr int kA1WarpSmem = PersistSmem::kBytes + 1024;  // + room to align the stage to 1024 bytes

// E of 8 consecutive elements starting at `e` (a multiple of 8): complex64 a
// uint32 pair per element, complex128 a uint16
template <class R>
__device__ __forceinline__ void load_e8(const unsigned char* etile, uint32_t e, uint32_t (&ev)[8]) {
  if constexpr (sizeof(R) == 4) {
    const uint4 a = *reinterpret_cast<const uint4*>(etile + 4u * e);
    const uint4 b = *reinterpret_cast<const uint4*>(etile + 4u * e + 16u);
    ev[0] = a.x; ev[1] = a.y; ev[2] = a.z; ev[3] = a.w;
    ev[4] = b.x; ev[5] = b.y; ev[6] = b.z; ev[7] = b.w;
  } else {
    const uint4 a = *reinterpret_cast<const uint4*>(etile + 2u * e);
    const uint32_t w[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      ev[2 * q] = w[q] & 0xFFFFu;
      ev[2 * q + 1] = w[q] >> 16;
    }
  }
}

// Shared-memory layout of the half-tile (4-warp) warp-local A1: a 32 KB tile,
// then its E values (8 KB for complex64), the phase table and reduction scratch.
struct HalfA1Smem {
  static constexpr int kTileBytes = kStageTileBytes / 2;
  static constexpr int kEOff = kTileBytes;
  static constexpr int kPhaseOff = kEOff + kStageEBytes / 2;
  static constexpr int kRedOff = kPhaseOff + 3328;
  static constexpr int kBytes = kRedOff + 512 + 1024;  // + room to align the stage to 1024 bytes
};

// NW = 8: one CTA per 4096-element tile (64 KB); NW = 4: one CTA per half tile
// (2048 elements, 32 KB; four CTAs per SM instead of two, so more independent
// load -> compute -> store chains overlap on each SM). Each warp owns a 512-element
// block either way: same arithmetic per element, bit-identical results.
// shared memory of the warp-local A1 (NW warps; kTab: room for the full phase
// table), + room to align the stage to 1024 bytes
template <int NW, bool kTab>
struct WarpA1Smem {
  static constexpr int kEOff = (NW == 8) ? kStageTileBytes : HalfA1Smem::kEOff;
  static constexpr int kPhaseOff = (NW == 8) ? PersistSmem::kPhaseOff : HalfA1Smem::kPhaseOff;
  static constexpr int kRedOff = kPhaseOff + (kTab ? kPhaseTabBytes : 3328);
  static constexpr int kBytes = kRedOff + 512 + 1024;
};
static_assert(WarpA1Smem<8, false>::kBytes == kA1WarpSmem && WarpA1Smem<4, false>::kBytes == HalfA1Smem::kBytes,
              "the warp-local layouts without the table are the original ones");

template <class R, int NW, bool kTab>
__global__ void __launch_bounds__(NW * 32, 8 / NW * 2)
    tile_a1_warp_kernel(const __grid_constant__ InstDesc<R> D, uint32_t step, int* err) {
  using PL = PlanA1Warp;
  using E = El<R>;
  static_assert(NW == 8 || NW == 4, "");
  static_assert(!kTab || sizeof(R) == 4, "the full phase table is complex64 only");
  constexpr int kTB = kA1WarpBits + (NW == 8 ? 3 : 2);   // element bits of the CTA's tile
  constexpr uint32_t kWarpMask = (NW == 8) ? PL::WARP : 0x600u;
  constexpr uint32_t kTileBytes = 16u << kTB;
  using SM = WarpA1Smem<NW, kTab>;
  constexpr int kEOff = SM::kEOff;
  constexpr int kPhaseOff = SM::kPhaseOff;
  constexpr int kRedOff = SM::kRedOff;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full_bar;
  __shared__ int last_flag;
  // the swizzled TMA destination must sit on a 1024-byte boundary
  unsigned char* smem = smem_raw + ((1024u - (smem_addr(smem_raw) & 1023u)) & 1023u);
  unsigned char* tile = smem;
  const unsigned char* etile = smem + kEOff;
  unsigned char* phase_smem = smem + kPhaseOff;
  double* red = reinterpret_cast<double*>(smem + kRedOff);
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t fb = smem_addr(&full_bar);
  const uint32_t t_idx = blockIdx.x;
  const uint32_t tile_base = t_idx << kTB;
  if (tid == 0) {
    mbar_init(fb, 1);
    fence_barrier_init();
    const bool e_tile = !D.e_recompute;
    uint32_t tb = 0u;
    if constexpr (kTab) tb = phase_tab_bytes(D.phase);
    mbar_arrive_expect_tx(fb, kTileBytes + (e_tile ? (kTileBytes / 16u) * 2u * (uint32_t)E::kAmps : 0u) + tb);
    if constexpr (kTab) bulk_load(smem_addr(phase_smem), D.phase.tab, tb, fb);
    const uint64_t pol = policy_evict_first();
    if constexpr (NW == 8) {
      tma_load_5d_hint(smem_addr(tile), D.map_a1s, 0, 0, 0, (int)t_idx, 0, fb, pol);
      if (e_tile) tma_load_5d_hint(smem_addr(tile + kEOff), D.map_e, 0, 0, (int)t_idx, 0, 0, fb, pol);
    } else {
      // half-tile maps: the A1 tile map with a box of one half, the E map with 2^12-amplitude tiles
      tma_load_5d_hint(smem_addr(tile), D.map_a1s, 0, 0, (int)(t_idx & 1u), (int)(t_idx >> 1), 0, fb, pol);
      if (e_tile) tma_load_5d_hint(smem_addr(tile + kEOff), D.map_e_half, 0, 0, (int)t_idx, 0, 0, fb, pol);
    }
  }
  if constexpr (!kTab) PhaseV<R>::stage(D.phase, phase_smem, (int)tid, NW * 32);
  __syncthreads();
  const bool ok = mbar_wait_bounded(fb, 0, err);
  if (__syncthreads_or(!ok)) return;
  typename E::T v[16];
  const R t = D.tan[step];
  const int slot = D.slot[step];
  MeasureAcc acc;
  // round 1 through the TMA swizzle (tile is 1024-byte aligned, so the swizzle
  // is a function of the tile offset)
  const uint32_t b1 = pdep(lane, PL::R1_LANE) | pdep(warp, kWarpMask);
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const uint32_t e = b1 | pdep((uint32_t)j, PL::R1_REG);
    v[j] = E::ld(tile + 16u * (e ^ ((e >> 3) & 7u)));
  }
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uint32_t eb = b1 | ((uint32_t)h << 6);
    uint32_t ev[8];
    if (D.e_recompute) {
#pragma unroll
      for (int q = 0; q < 8; ++q) ev[q] = recompute_e<R>(tile_base | eb | (uint32_t)q, D.n);
    } else {
      load_e8<R>(etile, eb, ev);
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int j = 8 * h + q;
      if (slot >= 0) measure_el(acc, v[j], ev[q], tile_base | eb | (uint32_t)q, D.e0, D.s0);
      a1_phase<R, kTab>(v[j], ev[q], D, phase_smem);
      E::bfly_inner(v[j], t);
    }
  }
  const R sc = D.scale[step];
  if (sc != (R)1) {
#pragma unroll
    for (int j = 0; j < 16; ++j) E::scale(v[j], sc);
  }
  el_bflys<R, PL::R1_REG, PL::R1_REG>(v, t);
  warp_sync();  // round-1 reads vs swizzled stores: same warp
  el_store_swz<R, PL::R1_REG>(tile, v, b1);
  warp_sync();  // rounds 1 and 2 share the warp bits
  const uint32_t b2 = pdep(lane, PL::R2_LANE) | pdep(warp, kWarpMask);
  el_load<R, PL::R2_REG, true>(tile, v, b2);
  el_bflys<R, PL::R2_REG, PL::R2_REG>(v, t);
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const typename E::T q = E::shfl_xor(v[j], PL::kShuffleLanes);
    E::bfly_partner(v[j], q, t);
  }
  el_gstore<R, PL::R2_REG, kElemBits>(D.state, v, tile_base, b2, 0,
                                      D.a1_evict_first ? policy_evict_first() : policy_evict_last());
  if (slot >= 0)
    compute_reduce<NW>(acc, D.partials, D.ticket, D.results, slot, t_idx, D.n_a1 * (8u / NW), red, &last_flag);
}

}  // namespace bk
