// Two-pass Trotter step on thread-block clusters (sm_100a).
//
// With 64 KB tiles a step over 27 element bits needs three HBM round trips
// (A1 12 bits + two strided passes). A cluster of 8 CTAs holds a 512 KB
// super-tile in distributed shared memory, so 15 qubits fit one pass and the
// step needs two:
//   pass L  element bits [0, 15): CTA rank r loads A1 tile (cluster << 3) | r
//           (bits 0..11 local, r = bits 12..14); measurement, diagonal phase and
//           the 12 (+ amplitude bit 0) local qubits as in A1; then tile bits
//           9..11 are exchanged with the rank bits through DSMEM and the three
//           remaining qubits are rotated locally;
//   pass H  element bits [0, 3) u [15, 27): CTA rank r loads the strided tile
//           (bits 0..2 contiguous, 15..23 local; cluster = bits 3..14, r = bits
//           24..26); the 9 local high qubits as in a W = 9 strided pass; then tile
//           bits 9..11 (element bits 21..23) are exchanged with the rank bits and
//           element bits 24..26 are rotated.
// Exchange: element at local position p goes to CTA d = p[9..11], position
// (p & ~0xE00) | (r << 9), by 16-byte st.shared::cluster stores; two cluster
// barriers bracket it (every CTA done reading its stage / every write landed).
// Every CTA executes both barriers whatever happens before them (a failed
// bounded TMA wait records an error and skips the work, never the barrier).
// No TMA multicast; each CTA loads only its own tile of this GPU's memory.
#pragma once
#include "bk_persist.cuh"

namespace bk {

constexpr int kClusterSize = 8;
constexpr uint32_t kXchgBits = 0xE00u;  // tile bits 9..11, swapped with the cluster rank

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_index() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cluster_barrier() {
  asm volatile(
      "barrier.cluster.arrive.release.aligned;\n\t"
      "barrier.cluster.wait.acquire.aligned;" ::
          : "memory");
}
__device__ __forceinline__ uint32_t map_to_rank(uint32_t smem_address, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_address), "r"(rank));
  return r;
}
template <class T>
__device__ __forceinline__ void st_cluster16(uint32_t addr, const T& v) {
  static_assert(sizeof(T) == 16, "16-byte elements");
  const uint4 w = *reinterpret_cast<const uint4*>(&v);
  asm volatile("st.shared::cluster.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(w.x), "r"(w.y), "r"(w.z),
               "r"(w.w)
               : "memory");
}

// Global element index of local position q after the exchange.
__device__ __forceinline__ uint32_t cl_global_L(uint32_t q, uint32_t c, uint32_t r) {
  return (c << 15) | (q & 0x1FFu) | (r << 9) | (((q >> 9) & 7u) << 12);
}
__device__ __forceinline__ uint32_t cl_global_H(uint32_t q, uint32_t c, uint32_t r) {
  return (q & 7u) | (c << 3) | (((q >> 3) & 0x3Fu) << 15) | (r << 21) | (((q >> 9) & 7u) << 24);
}

// Sends the 16 elements held in layout REG (positions base | pdep(j, REG)) to
// their owners: CTA p[9..11], position (p & ~0xE00) | (r << 9).
template <class R, uint32_t REG>
__device__ __forceinline__ void cl_exchange(unsigned char* stage, const typename El<R>::T (&v)[16], uint32_t base,
                                            uint32_t r) {
  const uint32_t s0 = smem_addr(stage);
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const uint32_t p = base | pdep((uint32_t)j, REG);
    const uint32_t d = (p >> 9) & 7u;
    const uint32_t p2 = (p & ~kXchgBits) | (r << 9);
    st_cluster16(map_to_rank(s0 + 16u * swz<double>(p2), d), v[j]);
  }
}

// Pass L rounds up to the exchange: measurement (if flagged), D, rescale,
// amplitude bit 0, tile bits 0..11. Leaves v in the A1_R3 layout (base b3).
template <class R>
__device__ __forceinline__ void cl_rounds_L(unsigned char* tile, const unsigned char* etile, const InstDesc<R>& D,
                                            uint32_t t_idx, uint32_t step, const unsigned char* phase_smem,
                                            typename El<R>::T (&v)[16], uint32_t& b3, MeasureAcc& acc, int slot) {
  using PL = Plan<double>;
  using E = El<R>;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t tile_base = t_idx << kElemBits;
  const uint32_t b1 = pdep(lane, PL::A1_R1_LANE) | pdep(warp, PL::A1_R1_WARP);
  el_load<R, PL::A1_R1_REG, false>(tile, v, b1);
  const R t = D.tan[step];
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const uint32_t i = b1 | pdep((uint32_t)j, PL::A1_R1_REG);
    const uint32_t e = load_e<R>(etile, i);
    if (slot >= 0) measure_el(acc, v[j], e, tile_base | i, D.e0, D.s0);
    PhaseV<R>::apply(v[j], e, D.phase, phase_smem, false);
    E::bfly_inner(v[j], t);
  }
  const R sc = D.scale[step];
  if (sc != (R)1) {
#pragma unroll
    for (int j = 0; j < 16; ++j) E::scale(v[j], sc);
  }
  el_bflys<R, PL::A1_R1_REG, PL::A1_R1_REG>(v, t);
  __syncthreads();
  el_store_swz<R, PL::A1_R1_REG>(tile, v, b1);
  __syncthreads();
  const uint32_t b2 = pdep(lane, PL::A1_R2_LANE) | pdep(warp, PL::A1_R2_WARP);
  el_load<R, PL::A1_R2_REG, true>(tile, v, b2);
  el_bflys<R, PL::A1_R2_REG, PL::A1_R2_REG>(v, t);
  __syncthreads();
  el_store_swz<R, PL::A1_R2_REG>(tile, v, b2);
  __syncthreads();
  b3 = pdep(lane, PL::A1_R3_LANE) | pdep(warp, PL::A1_R3_WARP);
  el_load<R, PL::A1_R3_REG, true>(tile, v, b3);
  el_bflys<R, PL::A1_R3_REG, PL::A1_R3_ACT>(v, t);
}

// Pass H rounds up to the exchange: the 9 local high qubits (tile bits 3..11).
// Leaves v in the W = 9 second-round layout (base b2).
template <class R>
__device__ __forceinline__ void cl_rounds_H(unsigned char* tile, R t, typename El<R>::T (&v)[16], uint32_t& b2) {
  using PL = Plan<double>;
  using E = El<R>;
  using R2 = StridedR2<double, 9>;
  constexpr uint32_t ACT_ALL = 0xFF8u;  // tile bits 3..11
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t b1 = pdep(lane, PL::S_R1_LANE) | pdep(warp, PL::S_R1_WARP);
  el_load<R, PL::S_R1_REG, false>(tile, v, b1);
  el_bflys<R, PL::S_R1_REG, ACT_ALL>(v, t);
  __syncthreads();
  el_store_swz<R, PL::S_R1_REG>(tile, v, b1);
  __syncthreads();
  b2 = pdep(lane, R2::LANE) | pdep(warp, R2::WARP);
  el_load<R, R2::REG, true>(tile, v, b2);
  el_bflys<R, R2::REG, R2::ACT>(v, t);
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const typename E::T q = E::shfl_xor(v[j], 1 << R2::kShuffleLaneBit);
    E::bfly_partner(v[j], q, t);
  }
}

// One pass (kind 0 = L, 1 = H) of Trotter step `step`; grid = all tiles,
// clusters of 8 along x. D.map_s2 / s2_* describe the H geometry (c' = 3,
// h0 = 15, W = 9).
template <class R>
__global__ void __launch_bounds__(kComputeThreads, 2)
    cluster_pass_kernel(const InstDesc<R>* __restrict__ insts, int kind, uint32_t step, int* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t full_bar;
  __shared__ int last_flag;
  unsigned char* stage = smem;
  unsigned char* phase_smem = smem + PersistSmem::kPhaseOff;
  double* red = reinterpret_cast<double*>(smem + PersistSmem::kRedOff);
  const InstDesc<R>& D = insts[0];
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t r = cluster_rank(), c = cluster_index();
  const uint32_t fb = smem_addr(&full_bar);
  if (tid == 0) {
    mbar_init(fb, 1);
    fence_barrier_init();
  }
  if (kind == 0) PhaseV<R>::stage(D.phase, phase_smem, tid, kComputeThreads);
  __syncthreads();
  StageMeta m;
  m.inst = 0;
  m.step = step;
  if (kind == 0) {
    m.kind = TASK_A1;
    m.tile = (c << 3) | r;
  } else {
    m.kind = TASK_S2;
    m.tile = (r << D.s2_mid_bits) | c;  // mid = cluster (element bits 3..14), hi = rank
  }
  if (tid == 0) issue_task_load(D, m, stage, fb);
  const bool ok = mbar_wait_bounded(fb, 0, err);
  const bool bad = __syncthreads_or(!ok) != 0;
  typename El<R>::T v[16];
  uint32_t base = 0;
  const int slot = (kind == 0) ? D.slot[step] : -1;
  MeasureAcc acc;
  if (!bad) {
    if (kind == 0)
      cl_rounds_L<R>(stage, stage + kStageTileBytes, D, m.tile, step, phase_smem, v, base, acc, slot);
    else
      cl_rounds_H<R>(stage, D.tan[step], v, base);
  }
  cluster_barrier();  // every CTA has read its stage into registers
  if (!bad) {
    if (kind == 0)
      cl_exchange<R, Plan<double>::A1_R3_REG>(stage, v, base, r);
    else
      cl_exchange<R, StridedR2<double, 9>::REG>(stage, v, base, r);
  }
  cluster_barrier();  // every element has landed in its owner's stage
  if (bad) return;
  const uint32_t bq = pdep(lane, 0x1Fu) | pdep(warp, 0xE0u);
  el_load<R, 0xF00u, true>(stage, v, bq);
  el_bflys<R, 0xF00u, kXchgBits>(v, D.tan[step]);
  const uint64_t pol = policy_evict_first();
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const uint32_t q = bq | pdep((uint32_t)j, 0xF00u);
    const uint32_t g = (kind == 0) ? cl_global_L(q, c, r) : cl_global_H(q, c, r);
    El<R>::stg(D.state + 16ull * g, v[j], pol);
  }
  if (kind == 0 && slot >= 0)
    compute_reduce(acc, D.partials, D.ticket, D.results, slot, m.tile, D.n_a1, red, &last_flag);
}

}  // namespace bk
