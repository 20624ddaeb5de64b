// Reverse sweep of the adjoint gradient (sm_100a).
//
// Objective O = <psi_T| W |psi_T> with a diagonal W (P_<: [E(s) < e0];
// <d_H>: popcount(s ^ s0)). For the step psi_{k+1} = M(g_k) D psi_k with
// M(g) = prod_q exp(+i g dt X_q) the adjoint method gives
//   lambda_T = W psi_T,   lambda_k = (M(g_k) D)^dagger lambda_{k+1},
//   dO/dg_k = -2 dt Im <lambda_{k+1}| G |psi_{k+1}>,   G = sum_q X_q.
// No trajectory is stored: psi_{k+1} is rebuilt from psi_T by the same inverse
// steps that carry lambda (U^dagger = D^dagger M^dagger), and replaced by a
// stored checkpoint every K steps to bound the drift of the inverse steps.
//
// Both statevectors go through every inverse step together: a task loads the
// same tile of psi and of lambda, keeps both in registers and applies the same
// rounds to both. G needs no extra pass: X_q commutes with every Rx factor, so
// <lambda|X_q|psi> can be read in any common frame, and each round reads it off
// the butterfly pairs (psi_s, psi_s'), (lambda_s, lambda_s') just before it
// rotates them:  Im(conj(lambda_s) psi_s' + conj(lambda_s') psi_s).
// The butterflies apply (I - i t X_q) = R_q^dagger / cos(g dt), which scales
// <lambda|X_q'|psi> by (1 + t^2) per qubit already rotated in this step; each
// round's sum is divided by (1 + t^2)^m for its m, the whole-step scale of both
// vectors is divided out on the host.
//
// Reverse step j (j = 0 .. T - 1, undoing forward step k = T - 1 - j) is laid
// out like a forward step: A1 applies D^dagger (skipped for j = 0), the exact
// power-of-two rescale and the low-qubit butterflies; S2 / S3 the high ones.
// After reverse step j the buffers hold D psi_k and D lambda_k (the D^dagger
// that completes the inverse step opens reverse step j + 1), so a checkpoint
// psi_k is put back as D psi_k.
//
// One CTA per SM (two 64 KB tiles and the E tile in shared memory), every CTA
// loops over the pass's tiles and issues the next tile's loads as soon as the
// last shared-memory read of the current one is done. Per-tile partial sums are
// reduced in index order by the last CTA of the step's last pass
// (deterministic).
#pragma once
#include "bk_persist.cuh"

namespace bk {

template <class R>
struct AdjDesc {
  unsigned char* psi;             // 16-byte elements
  unsigned char* lam;
  const CUtensorMap* map_a1;      // [2]: psi, lambda
  const CUtensorMap* map_e;
  const CUtensorMap* map_s2;      // [2]
  const CUtensorMap* map_s3;      // [2]
  int np, n, w2, w3;
  int a1_hi_dim;
  int s2_mid_dim, s2_hi_dim, s2_mid_bits;
  int s3_mid_dim, s3_hi_dim, s3_mid_bits;
  typename PhaseV<R>::params phase;
  const R* tan;                   // [T] tangent of reverse step j (the negated forward tangent)
  const R* scale;                 // [T] exact power of two applied in A1 of reverse step j
  const double* lg1t2;            // [T] log2(1 + t^2) of that tangent
  double* partials;               // [n_a1 + n_s2 + n_s3] per-tile sums of the current step
  unsigned int* ticket;
  double* cross;                  // [T] sum over rounds of the weighted Im <lambda|G|psi>
  uint32_t n_a1, n_s2, n_s3;
  const CUtensorMap* map_a1s;     // [2]: warp-local A1 tiles of psi, lambda (128-byte TMA swizzle)
};

struct AdjSmem {
  static constexpr int kPsiOff = 0;
  static constexpr int kLamOff = kStageTileBytes;
  static constexpr int kEOff = 2 * kStageTileBytes;
  static constexpr int kPhaseOff = kEOff + kStageEBytes;
  static constexpr int kRedOff = kPhaseOff + 3328;
  static constexpr int kBytes = kRedOff + 256;
  static constexpr int kAlloc = kBytes + 1024;  // + room to align the stage to 1024 bytes (swizzled TMA)
  // complex64 A1 with the full phase table (BK_OPT_PHASE_TABLE): a larger phase room
  static constexpr int kRedOffTab = kPhaseOff + kPhaseTabBytes;
  static constexpr int kAllocTab = kRedOffTab + 256 + 1024;
};

// D^dagger on the same element of psi (v) and lambda (u): one set of rotation
// coefficients for both; kTab (complex64): from the full phase table, the two
// half-angle shear rotations negated (a shear triple with (-a, -b) undoes (a, b))
template <class R, bool kTab>
__device__ __forceinline__ void adj_phase_inv(typename El<R>::T& v, typename El<R>::T& u, uint32_t e,
                                              const typename PhaseV<R>::params& P, const unsigned char* phase_smem) {
  if constexpr (kTab) {
    const float2* tab = reinterpret_cast<const float2*>(phase_smem);
    const uint32_t c0 = (uint32_t)P.c0;
    const float2 H0 = tab[((e & 0xFFFFu) - c0) >> 2], H1 = tab[((e >> 16) - c0) >> 2];
    const float2 A = make_float2(-H0.x, -H1.x), B = make_float2(-H0.y, -H1.y);
    PhaseV<float>::shear2(v.re, v.im, A, B);
    PhaseV<float>::shear2(v.re, v.im, A, B);
    PhaseV<float>::shear2(u.re, u.im, A, B);
    PhaseV<float>::shear2(u.re, u.im, A, B);
  } else {
    const typename PhaseV<R>::Coef cf = PhaseV<R>::coef(e, P, phase_smem, true);
    PhaseV<R>::rotate(v, cf, true);
    PhaseV<R>::rotate(u, cf, true);
  }
}

__host__ __device__ constexpr int popc_c(uint32_t x) { return x ? (int)(x & 1u) + popc_c(x >> 1) : 0; }

// cross-term accumulators of one round: sum of Im(conj(y) x) over ordered pairs
template <class R>
struct CrossAcc;
template <>
struct CrossAcc<float> {
  using T = El<float>::T;
  float2 p = make_float2(0.f, 0.f), q = make_float2(0.f, 0.f);  // sum y.re x.im, sum y.im x.re
  __device__ __forceinline__ void one(const T& x, const T& y) {
    p = __ffma2_rn(y.re, x.im, p);
    q = __ffma2_rn(y.im, x.re, q);
  }
  __device__ __forceinline__ void pair(const T& x0, const T& x1, const T& y0, const T& y1) {
    one(x1, y0);
    one(x0, y1);
  }
  // amplitude bit 0 (inside the element): conj(y_0) x_1 + conj(y_1) x_0
  __device__ __forceinline__ void inner(const T& x, const T& y) {
    p.x = fmaf(y.re.x, x.im.y, p.x);
    q.x = fmaf(y.im.x, x.re.y, q.x);
    p.y = fmaf(y.re.y, x.im.x, p.y);
    q.y = fmaf(y.im.y, x.re.x, q.y);
  }
  __device__ __forceinline__ double take() {
    const double r = ((double)p.x - (double)q.x) + ((double)p.y - (double)q.y);
    p = q = make_float2(0.f, 0.f);
    return r;
  }
};
template <>
struct CrossAcc<double> {
  using T = El<double>::T;
  double a = 0.0;
  __device__ __forceinline__ void one(const T& x, const T& y) {
    a = fma(y.v.x, x.v.y, a);
    a = fma(-y.v.y, x.v.x, a);
  }
  __device__ __forceinline__ void pair(const T& x0, const T& x1, const T& y0, const T& y1) {
    one(x1, y0);
    one(x0, y1);
  }
  __device__ __forceinline__ void inner(const T&, const T&) {}
  __device__ __forceinline__ double take() {
    const double r = a;
    a = 0.0;
    return r;
  }
};

// Im <y|X_q|x> of every register bit whose tile bit is in ACT
template <class R, uint32_t REG, uint32_t ACT>
__device__ __forceinline__ void el_cross(const typename El<R>::T (&x)[16], const typename El<R>::T (&y)[16],
                                         CrossAcc<R>& ca) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if ((ACT & pdep(1u << k, REG)) != 0u) {
#pragma unroll
      for (int j = 0; j < 16; ++j)
        if (!(j & (1 << k))) ca.pair(x[j], x[j | (1 << k)], y[j], y[j | (1 << k)]);
    }
  }
}

template <class R, uint32_t REG, int CP>
__device__ __forceinline__ void el_gstore_plain(unsigned char* g, const typename El<R>::T (&v)[16],
                                                uint32_t tile_base, uint32_t base, uint32_t h0) {
  const uint32_t gb = tile_base | tile_to_global<CP>(base, h0);
#pragma unroll
  for (int j = 0; j < 16; ++j) El<R>::st(g + 16ull * (gb | tile_to_global<CP>(pdep((uint32_t)j, REG), h0)), v[j]);
}

// the round weight (1 + t^2)^-m
__device__ __forceinline__ double round_weight(int m, double lg1t2) { return exp2(-(double)m * lg1t2); }

// reverse A1 on a staged (psi, lambda, E) tile: D^dagger, rescale, low-qubit
// butterflies with their cross terms. Returns this thread's weighted sum.
template <class R, bool kTab, class F>
__device__ __forceinline__ double adj_a1(unsigned char* sp, unsigned char* sl, const unsigned char* etile,
                                         const AdjDesc<R>& D, uint32_t t_idx, uint32_t j, bool phase_on,
                                         const unsigned char* phase_smem, F&& stage_free) {
  using PL = Plan<double>;
  using E = El<R>;
  constexpr bool kC64 = sizeof(R) == 4;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t tile_base = t_idx << kElemBits;
  const R t = D.tan[j];
  const R sc = D.scale[j];
  const double L = D.lg1t2[j];
  typename E::T v[16], u[16];
  CrossAcc<R> ca;
  double acc = 0.0;
  const uint32_t b1 = pdep(lane, PL::A1_R1_LANE) | pdep(warp, PL::A1_R1_WARP);
  el_load<R, PL::A1_R1_REG, false>(sp, v, b1);
  el_load<R, PL::A1_R1_REG, false>(sl, u, b1);
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    if (phase_on) {
      const uint32_t e = load_e<R>(etile, b1 | pdep((uint32_t)q, PL::A1_R1_REG));
      adj_phase_inv<R, kTab>(v[q], u[q], e, D.phase, phase_smem);
    }
    if (sc != (R)1) {
      E::scale(v[q], sc);
      E::scale(u[q], sc);
    }
  }
  int m = 0;
  if constexpr (kC64) {
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      ca.inner(v[q], u[q]);
      E::bfly_inner(v[q], t);
      E::bfly_inner(u[q], t);
    }
    acc += ca.take();  // m = 0
    m = 1;
  }
  el_cross<R, PL::A1_R1_REG, PL::A1_R1_REG>(v, u, ca);
  acc += round_weight(m, L) * ca.take();
  m += popc_c(PL::A1_R1_REG);
  el_bflys<R, PL::A1_R1_REG, PL::A1_R1_REG>(v, t);
  el_bflys<R, PL::A1_R1_REG, PL::A1_R1_REG>(u, t);
  warp_sync();  // round-1 reads vs swizzled stores: same warp
  el_store_swz<R, PL::A1_R1_REG>(sp, v, b1);
  el_store_swz<R, PL::A1_R1_REG>(sl, u, b1);
  warp_sync();  // rounds 1 and 2 share the warp bits
  const uint32_t b2 = pdep(lane, PL::A1_R2_LANE) | pdep(warp, PL::A1_R2_WARP);
  el_load<R, PL::A1_R2_REG, true>(sp, v, b2);
  el_load<R, PL::A1_R2_REG, true>(sl, u, b2);
  el_cross<R, PL::A1_R2_REG, PL::A1_R2_REG>(v, u, ca);
  acc += round_weight(m, L) * ca.take();
  m += popc_c(PL::A1_R2_REG);
  el_bflys<R, PL::A1_R2_REG, PL::A1_R2_REG>(v, t);
  el_bflys<R, PL::A1_R2_REG, PL::A1_R2_REG>(u, t);
  el_store_swz<R, PL::A1_R2_REG>(sp, v, b2);  // in place
  el_store_swz<R, PL::A1_R2_REG>(sl, u, b2);
  __syncthreads();
  const uint32_t b3 = pdep(lane, PL::A1_R3_LANE) | pdep(warp, PL::A1_R3_WARP);
  el_load<R, PL::A1_R3_REG, true>(sp, v, b3);
  el_load<R, PL::A1_R3_REG, true>(sl, u, b3);
  __syncthreads();
  stage_free();
  el_cross<R, PL::A1_R3_REG, PL::A1_R3_ACT>(v, u, ca);
  acc += round_weight(m, L) * ca.take();
  el_bflys<R, PL::A1_R3_REG, PL::A1_R3_ACT>(v, t);
  el_bflys<R, PL::A1_R3_REG, PL::A1_R3_ACT>(u, t);
  el_gstore_plain<R, PL::A1_R3_REG, kElemBits>(D.psi, v, tile_base, b3, 0);
  el_gstore_plain<R, PL::A1_R3_REG, kElemBits>(D.lam, u, tile_base, b3, 0);
  return acc;
}

// Warp-local reverse A1 (element bits 0-8, one warp per 512-element block of
// both statevectors; the tile layout of the forward warp-local A1): D^dagger,
// rescale, amplitude bit 0, round 1 (register bits 0-2, 6) and round 2
// (register bits 3-5, 7) with their cross terms, bit 8 across lanes 16 apart.
// The only CTA barrier releases the stage after round 2's reads.
template <class R, bool kTab, class F>
__device__ __forceinline__ double adj_a1_warp(unsigned char* sp, unsigned char* sl, const unsigned char* etile,
                                              const AdjDesc<R>& D, uint32_t t_idx, uint32_t j, bool phase_on,
                                              const unsigned char* phase_smem, F&& stage_free) {
  using PL = PlanA1Warp;
  using E = El<R>;
  constexpr bool kC64 = sizeof(R) == 4;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t tile_base = t_idx << kElemBits;
  const R t = D.tan[j];
  const R sc = D.scale[j];
  const double L = D.lg1t2[j];
  typename E::T v[16], u[16];
  CrossAcc<R> ca;
  double acc = 0.0;
  const uint32_t b1 = pdep(lane, PL::R1_LANE) | pdep(warp, PL::WARP);
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const uint32_t e = b1 | pdep((uint32_t)q, PL::R1_REG);
    const uint32_t o = 16u * (e ^ ((e >> 3) & 7u));  // 128-byte TMA swizzle (stage 1024-byte aligned)
    v[q] = E::ld(sp + o);
    u[q] = E::ld(sl + o);
  }
  if (phase_on) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      uint32_t ev[8];
      load_e8<R>(etile, b1 | ((uint32_t)h << 6), ev);
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        adj_phase_inv<R, kTab>(v[8 * h + q], u[8 * h + q], ev[q], D.phase, phase_smem);
      }
    }
  }
  if (sc != (R)1) {
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      E::scale(v[q], sc);
      E::scale(u[q], sc);
    }
  }
  int m = 0;
  if constexpr (kC64) {
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      ca.inner(v[q], u[q]);
      E::bfly_inner(v[q], t);
      E::bfly_inner(u[q], t);
    }
    acc += ca.take();  // m = 0
    m = 1;
  }
  el_cross<R, PL::R1_REG, PL::R1_REG>(v, u, ca);
  acc += round_weight(m, L) * ca.take();
  m += popc_c(PL::R1_REG);
  el_bflys<R, PL::R1_REG, PL::R1_REG>(v, t);
  el_bflys<R, PL::R1_REG, PL::R1_REG>(u, t);
  warp_sync();  // round-1 reads vs swizzled stores: same warp
  el_store_swz<R, PL::R1_REG>(sp, v, b1);
  el_store_swz<R, PL::R1_REG>(sl, u, b1);
  warp_sync();  // rounds 1 and 2 share the warp bits
  const uint32_t b2 = pdep(lane, PL::R2_LANE) | pdep(warp, PL::WARP);
  el_load<R, PL::R2_REG, true>(sp, v, b2);
  el_load<R, PL::R2_REG, true>(sl, u, b2);
  __syncthreads();
  stage_free();
  el_cross<R, PL::R2_REG, PL::R2_REG>(v, u, ca);
  acc += round_weight(m, L) * ca.take();
  m += popc_c(PL::R2_REG);
  el_bflys<R, PL::R2_REG, PL::R2_REG>(v, t);
  el_bflys<R, PL::R2_REG, PL::R2_REG>(u, t);
  // tile bit 8 across lanes: each thread adds its own ordered term
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const typename E::T pv = E::shfl_xor(v[q], PL::kShuffleLanes);
    const typename E::T pu = E::shfl_xor(u[q], PL::kShuffleLanes);
    ca.one(pv, u[q]);
    E::bfly_partner(v[q], pv, t);
    E::bfly_partner(u[q], pu, t);
  }
  acc += round_weight(m, L) * ca.take();
  el_gstore_plain<R, PL::R2_REG, kElemBits>(D.psi, v, tile_base, b2, 0);
  el_gstore_plain<R, PL::R2_REG, kElemBits>(D.lam, u, tile_base, b2, 0);
  return acc;
}

// reverse strided pass of width W (element bits [0, 12 - W) u [h0, h0 + W));
// m0 = qubits already rotated in this step by the earlier passes
template <class R, int W, class F>
__device__ __forceinline__ double adj_s(unsigned char* sp, unsigned char* sl, const AdjDesc<R>& D,
                                        uint32_t tile_base, uint32_t h0, uint32_t j, int m0, F&& stage_free) {
  using PL = Plan<double>;
  using E = El<R>;
  constexpr int CP = kElemBits - W;
  constexpr uint32_t ACT_ALL = ((1u << W) - 1u) << CP;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const R t = D.tan[j];
  const double L = D.lg1t2[j];
  typename E::T v[16], u[16];
  CrossAcc<R> ca;
  double acc = 0.0;
  int m = m0;
  const uint32_t b1 = pdep(lane, PL::S_R1_LANE) | pdep(warp, PL::S_R1_WARP);
  el_load<R, PL::S_R1_REG, false>(sp, v, b1);
  el_load<R, PL::S_R1_REG, false>(sl, u, b1);
  if constexpr (W <= 4) {
    __syncthreads();
    stage_free();
  }
  el_cross<R, PL::S_R1_REG, ACT_ALL>(v, u, ca);
  acc += round_weight(m, L) * ca.take();
  m += popc_c(PL::S_R1_REG & ACT_ALL);
  el_bflys<R, PL::S_R1_REG, ACT_ALL>(v, t);
  el_bflys<R, PL::S_R1_REG, ACT_ALL>(u, t);
  if constexpr (W <= 4) {
    el_gstore_plain<R, PL::S_R1_REG, CP>(D.psi, v, tile_base, b1, h0);
    el_gstore_plain<R, PL::S_R1_REG, CP>(D.lam, u, tile_base, b1, h0);
  } else {
    using R2 = StridedR2<double, W>;
    warp_sync();  // round-1 reads vs swizzled stores: same warp
    el_store_swz<R, PL::S_R1_REG>(sp, v, b1);
    el_store_swz<R, PL::S_R1_REG>(sl, u, b1);
    __syncthreads();
    const uint32_t b2 = pdep(lane, R2::LANE) | pdep(warp, R2::WARP);
    el_load<R, R2::REG, true>(sp, v, b2);
    el_load<R, R2::REG, true>(sl, u, b2);
    __syncthreads();
    stage_free();
    el_cross<R, R2::REG, R2::ACT>(v, u, ca);
    acc += round_weight(m, L) * ca.take();
    m += popc_c(R2::REG & R2::ACT);
    el_bflys<R, R2::REG, R2::ACT>(v, t);
    el_bflys<R, R2::REG, R2::ACT>(u, t);
    if constexpr (R2::kShuffleLaneBit >= 0) {
      // the tile bit held across lanes: each thread adds its own ordered term
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const typename E::T pv = E::shfl_xor(v[q], 1 << R2::kShuffleLaneBit);
        const typename E::T pu = E::shfl_xor(u[q], 1 << R2::kShuffleLaneBit);
        ca.one(pv, u[q]);
        E::bfly_partner(v[q], pv, t);
        E::bfly_partner(u[q], pu, t);
      }
      acc += round_weight(m, L) * ca.take();
    }
    el_gstore_plain<R, R2::REG, CP>(D.psi, v, tile_base, b2, h0);
    el_gstore_plain<R, R2::REG, CP>(D.lam, u, tile_base, b2, h0);
  }
  return acc;
}

template <class R, bool kWarpA1>
__device__ __forceinline__ void adj_issue(const AdjDesc<R>& D, int kind, uint32_t tile, unsigned char* stage,
                                          uint32_t fb) {
  if (kind == TASK_A1) {
    mbar_arrive_expect_tx(fb, (uint32_t)(2 * kStageTileBytes + 4096 * 2 * El<R>::kAmps));
    if (kWarpA1) {
      tma_load_5d(smem_addr(stage + AdjSmem::kPsiOff), D.map_a1s + 0, 0, 0, 0, (int)tile, 0, fb);
      tma_load_5d(smem_addr(stage + AdjSmem::kLamOff), D.map_a1s + 1, 0, 0, 0, (int)tile, 0, fb);
    } else {
      const int hd = D.a1_hi_dim;
      const int c2 = hd == 2 ? (int)tile : 0, c3 = hd == 3 ? (int)tile : 0;
      tma_load_5d(smem_addr(stage + AdjSmem::kPsiOff), D.map_a1 + 0, 0, 0, c2, c3, 0, fb);
      tma_load_5d(smem_addr(stage + AdjSmem::kLamOff), D.map_a1 + 1, 0, 0, c2, c3, 0, fb);
    }
    tma_load_5d(smem_addr(stage + AdjSmem::kEOff), D.map_e, 0, 0, (int)tile, 0, 0, fb);
  } else {
    const bool s2 = (kind == TASK_S2);
    const int mb = s2 ? D.s2_mid_bits : D.s3_mid_bits;
    const int md = s2 ? D.s2_mid_dim : D.s3_mid_dim;
    const int hd = s2 ? D.s2_hi_dim : D.s3_hi_dim;
    const CUtensorMap* mp = s2 ? D.map_s2 : D.map_s3;
    const int mid = (int)(tile & ((1u << mb) - 1u)), hi = (int)(tile >> mb);
    mbar_arrive_expect_tx(fb, (uint32_t)(2 * kStageTileBytes));
#pragma unroll
    for (int s = 0; s < 2; ++s)
      tma_load_5d(smem_addr(stage + (s ? AdjSmem::kLamOff : AdjSmem::kPsiOff)), mp + s, tile_coord(0, md, mid, hd, hi),
                  tile_coord(1, md, mid, hd, hi), tile_coord(2, md, mid, hd, hi), tile_coord(3, md, mid, hd, hi),
                  tile_coord(4, md, mid, hd, hi), fb);
  }
}

// One reverse pass (kind = TASK_A1 / TASK_S2 / TASK_S3) of reverse step j.
// Grid: at most one CTA per SM, each loops over tiles blockIdx.x + i gridDim.x.
// last_pass: the step's last pass also reduces the step's per-tile sums.
// kWarpA1: every pass of a warp-local run (A1 in the warp-local layout, strided
// passes from element bit 9); its own instantiation, so the 12-bit kernel keeps
// its register allocation.
// kW: 0 = the A1 pass; 1..9 = a strided pass of that width (kind TASK_S2 or
// TASK_S3, whose width the host has matched to kW). One width per instantiation
// keeps each kernel's code small: a CTA runs only a few tiles per launch, so
// code that does not fit the instruction cache stalls every warp on fetches.
template <class R, bool kWarpA1, int kW, bool kTab = false>
__global__ void __launch_bounds__(kComputeThreads, 1)
    adj_pass_kernel(const __grid_constant__ AdjDesc<R> D, int kind, uint32_t j, int phase_on, int last_pass,
                    int* err) {
  static_assert(kW >= 0 && kW <= 9, "strided widths 1..9");
  static_assert(!kTab || (kW == 0 && sizeof(R) == 4), "the full phase table: complex64 A1 passes only");
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full_bar;
  __shared__ int is_last;
  // warp-local runs: the stage sits on a 1024-byte boundary (swizzled TMA)
  unsigned char* smem = kWarpA1 ? smem_raw + ((1024u - (smem_addr(smem_raw) & 1023u)) & 1023u) : smem_raw;
  unsigned char* stage = smem;
  unsigned char* phase_smem = smem + AdjSmem::kPhaseOff;
  double* red = reinterpret_cast<double*>(smem + (kTab ? AdjSmem::kRedOffTab : AdjSmem::kRedOff));
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t fb = smem_addr(&full_bar);
  const uint32_t ntiles = kind == TASK_A1 ? D.n_a1 : (kind == TASK_S2 ? D.n_s2 : D.n_s3);
  const uint32_t part0 = kind == TASK_A1 ? 0u : (kind == TASK_S2 ? D.n_a1 : D.n_a1 + D.n_s2);
  constexpr int w = kW;
  constexpr int kA1Bits = kWarpA1 ? kA1WarpBits : kElemBits;  // element bits of the step's A1 pass
  const uint32_t h0 = kind == TASK_S2 ? (uint32_t)kA1Bits : (uint32_t)(kA1Bits + D.w2);
  const int mb = kind == TASK_S2 ? D.s2_mid_bits : D.s3_mid_bits;
  // qubits rotated by the earlier passes of the step (complex64: + amplitude bit 0)
  const int m0 = (sizeof(R) == 4 ? 1 : 0) + kA1Bits + (kind == TASK_S3 ? D.w2 : 0);
  uint32_t tile = blockIdx.x;
  // Launched as a programmatic dependent of the previous pass: the barrier and
  // the phase tables (constant over the sweep) are set up while that pass
  // finishes; everything the previous passes write (psi, lambda, the step's
  // partials and ticket) is touched only after the grid-dependency wait.
  if (tid == 0) {
    mbar_init(fb, 1);
    fence_barrier_init();
  }
  if (kind == TASK_A1 && phase_on) {
    if constexpr (kTab) {
      float2* tab = reinterpret_cast<float2*>(phase_smem);
      for (int i = tid; i < D.phase.n_j; i += kComputeThreads) tab[i] = D.phase.tab[i];
    } else {
      PhaseV<R>::stage(D.phase, phase_smem, tid, kComputeThreads);
    }
  }
  grid_dependency_wait();
  if (tid == 0 && tile < ntiles) adj_issue<R, kWarpA1>(D, kind, tile, stage, fb);
  __syncthreads();
  uint32_t parity = 0;
  for (; tile < ntiles; tile += gridDim.x) {
    const bool ok = mbar_wait_bounded(fb, parity, err);
    if (__syncthreads_or(!ok)) return;
    parity ^= 1u;
    const uint32_t nxt = tile + gridDim.x;
    // the CTA's last tile: the next pass may be scheduled onto SMs as they free up
    if (nxt >= ntiles) grid_dependents_launch();
    auto stage_free = [&]() {
      if (tid == 0 && nxt < ntiles) adj_issue<R, kWarpA1>(D, kind, nxt, stage, fb);
    };
    double acc;
    if constexpr (kW == 0 && kWarpA1) {
      acc = adj_a1_warp<R, kTab>(stage + AdjSmem::kPsiOff, stage + AdjSmem::kLamOff, stage + AdjSmem::kEOff, D, tile, j,
                           phase_on != 0, phase_smem, stage_free);
    } else if constexpr (kW == 0) {
      acc = adj_a1<R, kTab>(stage + AdjSmem::kPsiOff, stage + AdjSmem::kLamOff, stage + AdjSmem::kEOff, D, tile, j,
                      phase_on != 0, phase_smem, stage_free);
    } else {
      const uint32_t cp = (uint32_t)(kElemBits - w);
      const uint32_t mid = tile & ((1u << mb) - 1u), hi = tile >> mb;
      const uint32_t tile_base = (mid << cp) | (hi << (h0 + (uint32_t)w));
      acc = adj_s<R, kW>(stage + AdjSmem::kPsiOff, stage + AdjSmem::kLamOff, D, tile_base, h0, j, m0, stage_free);
    }
    acc = warp_sum(acc);
    if (lane == 0) red[warp] = acc;
    __syncthreads();
    if (tid == 0) {
      double s = 0.0;
      for (int i = 0; i < kComputeThreads / 32; ++i) s += red[i];
      D.partials[part0 + tile] = s;
    }
    __syncthreads();
  }
  if (!last_pass) return;
  // the last CTA of the step's last pass sums every tile of the step in index order
  if (tid == 0) {
    __threadfence();
    is_last = (atomicAdd(D.ticket, 1u) == gridDim.x - 1u);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  const uint32_t total = D.n_a1 + D.n_s2 + D.n_s3;
  double s = 0.0;
  for (uint32_t i = tid; i < total; i += kComputeThreads) s += __ldcg(&D.partials[i]);
  s = warp_sum(s);
  if (lane == 0) red[warp] = s;
  __syncthreads();
  if (tid == 0) {
    double r = 0.0;
    for (int i = 0; i < kComputeThreads / 32; ++i) r += red[i];
    D.cross[j] = r;
    *D.ticket = 0u;
  }
}

// lambda_T = W psi_T on 16-byte elements (objective 0: [E < e0], 1: popcount(s ^ s0))
template <class R>
__global__ void adj_lambda_init_kernel(const unsigned char* __restrict__ psi, unsigned char* __restrict__ lam,
                                       const uint16_t* __restrict__ E, uint32_t n_el, int objective, int e0,
                                       uint32_t s0) {
  using El_ = El<R>;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_el; i += gridDim.x * blockDim.x) {
    typename El_::T v = El_::ld(psi + 16ull * i);
    if constexpr (sizeof(R) == 4) {
      const uint32_t a0 = 2u * i, a1 = a0 + 1u;
      const float w0 = objective == 0 ? ((int)E[a0] < e0 ? 1.f : 0.f) : (float)__popc(a0 ^ s0);
      const float w1 = objective == 0 ? ((int)E[a1] < e0 ? 1.f : 0.f) : (float)__popc(a1 ^ s0);
      v.re.x *= w0;
      v.im.x *= w0;
      v.re.y *= w1;
      v.im.y *= w1;
    } else {
      const double w0 = objective == 0 ? ((int)E[i] < e0 ? 1.0 : 0.0) : (double)__popc(i ^ s0);
      v.v.x *= w0;
      v.v.y *= w0;
    }
    El_::st(lam + 16ull * i, v);
  }
}

// Checkpoint put back: psi <- D ckpt (the reverse sweep holds D psi_k at this
// point); dev_partials[blockIdx.x] = sum |a psi_rebuilt - b D ckpt|^2, the drift
// of the inverse steps since the previous checkpoint (a, b undo the scales).
template <class R>
__global__ void __launch_bounds__(kComputeThreads)
    adj_reset_kernel(unsigned char* __restrict__ psi, const unsigned char* __restrict__ ckpt,
                     const uint16_t* __restrict__ E, uint32_t n_el, typename PhaseV<R>::params ph, double a,
                     double b, double* __restrict__ dev_partials) {
  __shared__ __align__(16) unsigned char tab[3328];
  __shared__ double red[kComputeThreads / 32];
  using El_ = El<R>;
  PhaseV<R>::stage(ph, tab, threadIdx.x, blockDim.x);
  __syncthreads();
  double dev = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_el; i += gridDim.x * blockDim.x) {
    typename El_::T c = El_::ld(ckpt + 16ull * i);
    const typename El_::T r = El_::ld(psi + 16ull * i);
    if constexpr (sizeof(R) == 4) {
      const uint32_t e2 = (uint32_t)E[2u * i] | ((uint32_t)E[2u * i + 1u] << 16);
      PhaseV<R>::apply(c, e2, ph, tab, false);
      const double d0 = a * r.re.x - b * c.re.x, d1 = a * r.im.x - b * c.im.x;
      const double d2 = a * r.re.y - b * c.re.y, d3 = a * r.im.y - b * c.im.y;
      dev += d0 * d0 + d1 * d1 + d2 * d2 + d3 * d3;
    } else {
      PhaseV<R>::apply(c, (uint32_t)E[i], ph, tab, false);
      const double d0 = a * r.v.x - b * c.v.x, d1 = a * r.v.y - b * c.v.y;
      dev += d0 * d0 + d1 * d1;
    }
    El_::st(psi + 16ull * i, c);
  }
  dev = warp_sum(dev);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dev;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < kComputeThreads / 32; ++i) s += red[i];
    dev_partials[blockIdx.x] = s;
  }
}

}  // namespace bk
