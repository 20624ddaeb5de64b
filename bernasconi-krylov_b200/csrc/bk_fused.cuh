// Fused tile passes of one Trotter step (sm_100a).
//
// A step psi <- M D psi (reference order, src/sampling/sampler.cuh:604-618) is
// split into passes over 64 KB tiles of the statevector:
//   A1       tile = index bits [0, T): fused measurement of psi (before D, since
//            |D psi|^2 = |psi|^2), diagonal phase D, and the Rx butterflies of the
//            T low qubits;
//   strided  tile = bits [0, c') u [h0, h0 + W): the Rx butterflies of the W high
//            qubits [h0, h0 + W); the c' = T - W contiguous low bits keep every
//            global access a >= 128 B segment.
// Qubit operations commute, so A1 + strided passes over disjoint high ranges
// apply M exactly once per qubit.
//
// Inside a tile every thread holds 2^r amplitudes in registers. A "round" names
// which tile bits are register bits (butterflied without data movement), lane
// bits and warp bits; between rounds the tile goes through shared memory with
// an XOR swizzle that keeps every round's accesses bank-conflict free. Loads
// come in by TMA (one 5-D box per tile, completion on an mbarrier with a
// bounded wait); results leave straight from registers as coalesced 128-bit
// (or 64-bit) global stores.
#pragma once
#include "bk_device.cuh"

namespace bk {

template <class R>
struct PassParams {
  typename AmpTraits<R>::amp* state;
  uint32_t n;         // qubits
  uint32_t cprime;    // contiguous low tile bits [0, cprime)
  uint32_t h0;        // first high tile bit (strided passes)
  uint32_t mid_bits;  // tile-id bits that sit in [cprime, h0)
  int32_t mid_dim;    // TMA dim carrying the [cprime, h0) coordinate (-1: none)
  int32_t hi_dim;     // TMA dim carrying the [h0 + W, n) coordinate (-1: none)
  R t;                // tan(g dt) of this step
  // A1 / measure-only
  typename PhaseOf<R>::params phase;
  R amp_scale;        // exact power of two applied with D (overflow guard); 1 = none
  int32_t measure;    // measure this step (A1) — measure-only kernels always do
  int32_t slot;       // results row
  int32_t e0;         // P_< threshold
  uint32_t s0;        // trap bits (Hamming reference)
  double* partials;
  unsigned int* ticket;
  double* results;
  int* err;
};

// ---- shared-memory swizzles (linear over GF(2), bijective on the tile) ----
// complex64: 8 B amps, pairs (bit 0) stay adjacent; bits [4,13) fold into bits 1..3.
// complex128: 16 B amps; bits [3,12) fold into bits 0..2.
template <class R>
__host__ __device__ constexpr uint32_t swz(uint32_t i);
template <>
__host__ __device__ constexpr uint32_t swz<float>(uint32_t i) {
  return i ^ ((((i >> 4) ^ (i >> 7) ^ (i >> 10)) & 7u) << 1);
}
template <>
__host__ __device__ constexpr uint32_t swz<double>(uint32_t i) {
  return i ^ (((i >> 3) ^ (i >> 6) ^ (i >> 9)) & 7u);
}

template <class R, uint32_t REG>
struct RegSet {
  static constexpr int kN = 1 << AmpTraits<R>::kRegBits;
  // 128-bit pair access for complex64 when tile bit 0 is the lowest register bit
  static constexpr bool kPair = sizeof(R) == 4 && (REG & 1u);
};

template <class R, uint32_t REG, bool SWZ>
__device__ __forceinline__ void smem_load(const typename AmpTraits<R>::amp* s,
                                          typename AmpTraits<R>::amp (&v)[RegSet<R, REG>::kN],
                                          uint32_t base) {
  constexpr int NR = RegSet<R, REG>::kN;
  const uint32_t sb = SWZ ? swz<R>(base) : base;
  if constexpr (RegSet<R, REG>::kPair) {
#pragma unroll
    for (int j = 0; j < NR; j += 2) {
      const uint32_t o = SWZ ? swz<R>(pdep((uint32_t)j, REG)) : pdep((uint32_t)j, REG);
      const float4 q = *reinterpret_cast<const float4*>(reinterpret_cast<const float2*>(s) + (sb ^ o));
      v[j] = make_float2(q.x, q.y);
      v[j + 1] = make_float2(q.z, q.w);
    }
  } else {
#pragma unroll
    for (int j = 0; j < NR; ++j) {
      const uint32_t o = SWZ ? swz<R>(pdep((uint32_t)j, REG)) : pdep((uint32_t)j, REG);
      v[j] = s[sb ^ o];
    }
  }
}

template <class R, uint32_t REG>
__device__ __forceinline__ void smem_store_swz(typename AmpTraits<R>::amp* s,
                                               const typename AmpTraits<R>::amp (&v)[RegSet<R, REG>::kN],
                                               uint32_t base) {
  constexpr int NR = RegSet<R, REG>::kN;
  const uint32_t sb = swz<R>(base);
  if constexpr (RegSet<R, REG>::kPair) {
#pragma unroll
    for (int j = 0; j < NR; j += 2) {
      const uint32_t o = swz<R>(pdep((uint32_t)j, REG));
      *reinterpret_cast<float4*>(reinterpret_cast<float2*>(s) + (sb ^ o)) =
          make_float4(v[j].x, v[j].y, v[j + 1].x, v[j + 1].y);
    }
  } else {
#pragma unroll
    for (int j = 0; j < NR; ++j) s[sb ^ swz<R>(pdep((uint32_t)j, REG))] = v[j];
  }
}

// Butterflies on every register bit whose tile bit is in ACT.
template <class R, uint32_t REG, uint32_t ACT>
__device__ __forceinline__ void butterflies(typename AmpTraits<R>::amp (&v)[RegSet<R, REG>::kN], R t) {
  constexpr int NR = RegSet<R, REG>::kN;
#pragma unroll
  for (int k = 0; k < AmpTraits<R>::kRegBits; ++k) {
    if ((ACT & pdep(1u << k, REG)) != 0u) {
#pragma unroll
      for (int j = 0; j < NR; ++j)
        if (!(j & (1 << k))) bfly(v[j], v[j | (1 << k)], t);
    }
  }
}

// Tile position -> global amplitude index for tile bits [0, CP) u [h0, h0 + T - CP).
template <int CP>
__device__ __forceinline__ uint32_t tile_to_global(uint32_t p, uint32_t h0) {
  return (p & ((1u << CP) - 1u)) | ((p >> CP) << h0);
}

template <class R, uint32_t REG, int CP>
__device__ __forceinline__ void global_store(typename AmpTraits<R>::amp* g,
                                             const typename AmpTraits<R>::amp (&v)[RegSet<R, REG>::kN],
                                             uint32_t tile_base, uint32_t base, uint32_t h0) {
  constexpr int NR = RegSet<R, REG>::kN;
  const uint32_t gb = tile_base | tile_to_global<CP>(base, h0);
  if constexpr (RegSet<R, REG>::kPair) {
#pragma unroll
    for (int j = 0; j < NR; j += 2) {
      const uint32_t gi = gb | tile_to_global<CP>(pdep((uint32_t)j, REG), h0);
      *reinterpret_cast<float4*>(reinterpret_cast<float2*>(g) + gi) =
          make_float4(v[j].x, v[j].y, v[j + 1].x, v[j + 1].y);
    }
  } else {
#pragma unroll
    for (int j = 0; j < NR; ++j) g[gb | tile_to_global<CP>(pdep((uint32_t)j, REG), h0)] = v[j];
  }
}

// ---- round plans (REG, LANE, WARP bit masks of the 2^T tile index) ----
template <class R>
struct Plan;
template <>
struct Plan<float> {  // T = 13, 32 amps / thread
  // A1 / measure
  static constexpr uint32_t A1_R1_REG = 0x1E01, A1_R1_LANE = 0x3E, A1_R1_WARP = 0x1C0;
  static constexpr uint32_t A1_R2_REG = 0x3E, A1_R2_LANE = 0x3C1, A1_R2_WARP = 0x1C00;
  static constexpr uint32_t A1_R3_REG = 0x3C1, A1_R3_LANE = 0x3E, A1_R3_WARP = 0x1C00;
  static constexpr uint32_t A1_R3_ACT = 0x1C0;
  // strided, first round (natural TMA layout)
  static constexpr uint32_t S_R1_REG = 0x1E01, S_R1_LANE = 0x3E, S_R1_WARP = 0x1C0;
};
template <>
struct Plan<double> {  // T = 12, 16 amps / thread
  static constexpr uint32_t A1_R1_REG = 0x78, A1_R1_LANE = 0x187, A1_R1_WARP = 0xE00;
  static constexpr uint32_t A1_R2_REG = 0x87, A1_R2_LANE = 0x178, A1_R2_WARP = 0xE00;
  static constexpr uint32_t A1_R3_REG = 0xF00, A1_R3_LANE = 0x1F, A1_R3_WARP = 0xE0;
  static constexpr uint32_t A1_R3_ACT = 0xF00;
  static constexpr uint32_t S_R1_REG = 0xF00, S_R1_LANE = 0x1F, S_R1_WARP = 0xE0;
};

template <class R>
struct SmemLayout {
  static constexpr int kTileBytes = (1 << AmpTraits<R>::kTileBits) * (int)sizeof(typename AmpTraits<R>::amp);
  static constexpr int kEBytes = (1 << AmpTraits<R>::kTileBits) * 2;
  static constexpr int kTablesBytes = PhaseOf<R>::kSmemBytes;
  static constexpr int kA1Bytes = kTileBytes + kEBytes + kTablesBytes + 16;
  static constexpr int kStridedBytes = kTileBytes + 16;
};

// Starts the TMA load of this CTA's tile (and its E tile), returns false when
// the bounded wait ran out (every thread then leaves the kernel).
// Tile coordinate of dim k: the tile-id parts go to mid_dim / hi_dim, every
// other dim is covered by the box (coordinate 0). Selects, no local arrays.
__device__ __forceinline__ int tile_coord(int k, int mid_dim, int mid, int hi_dim, int hi) {
  return (k == mid_dim ? mid : 0) + (k == hi_dim ? hi : 0);
}

template <class R>
__device__ __forceinline__ bool load_tile(const CUtensorMap* amap, const CUtensorMap* emap, void* tile,
                                          void* etile, uint64_t* bar, int mid_dim, int mid, int hi_dim,
                                          int hi, int* err, uint32_t bytes) {
  const uint32_t b = smem_addr(bar);
  if (threadIdx.x == 0) {
    mbar_init(b, 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_arrive_expect_tx(b, bytes);
    tma_load_5d(smem_addr(tile), amap, tile_coord(0, mid_dim, mid, hi_dim, hi),
                tile_coord(1, mid_dim, mid, hi_dim, hi), tile_coord(2, mid_dim, mid, hi_dim, hi),
                tile_coord(3, mid_dim, mid, hi_dim, hi), tile_coord(4, mid_dim, mid, hi_dim, hi), b);
    if (emap != nullptr) tma_load_5d(smem_addr(etile), emap, 0, 0, (int)blockIdx.x, 0, 0, b);
  }
  const bool ok = mbar_wait_bounded(b, 0, err);
  return !__syncthreads_or(!ok);
}

// KIND 0: measure (optional) + D + butterflies on the T low qubits.
// KIND 1: measurement only.
template <class R, int KIND>
__global__ void __launch_bounds__(kThreads, 2)
    a1_kernel(const __grid_constant__ CUtensorMap amap, const __grid_constant__ CUtensorMap emap,
              const PassParams<R> p) {
  using amp = typename AmpTraits<R>::amp;
  using PL = Plan<R>;
  using L = SmemLayout<R>;
  constexpr int T = AmpTraits<R>::kTileBits;
  constexpr int NR = 1 << AmpTraits<R>::kRegBits;
  extern __shared__ __align__(1024) unsigned char smem[];
  amp* tile = reinterpret_cast<amp*>(smem);
  uint16_t* etile = reinterpret_cast<uint16_t*>(smem + L::kTileBytes);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + L::kTileBytes + L::kEBytes + L::kTablesBytes);

  // tables for D (overlaps the TMA)
  typename PhaseOf<R>::Smem tabs{};
  if (KIND == 0) tabs = PhaseOf<R>::stage(p.phase, smem + L::kTileBytes + L::kEBytes);
  if (!load_tile<R>(&amap, &emap, tile, etile, bar, -1, 0, p.hi_dim, (int)blockIdx.x, p.err,
                    (uint32_t)(L::kTileBytes + L::kEBytes)))
    return;

  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t tile_base = (uint32_t)blockIdx.x << T;
  amp v[NR];

  // ---- round 1 (natural TMA layout): measure, D, butterflies ----
  const uint32_t b1 = pdep(lane, PL::A1_R1_LANE) | pdep(warp, PL::A1_R1_WARP);
  smem_load<R, PL::A1_R1_REG, false>(tile, v, b1);
  MeasureAcc acc;
  const bool do_measure = (KIND == 1) || p.measure;
#pragma unroll
  for (int j = 0; j < NR; ++j) {
    const uint32_t i = b1 | pdep((uint32_t)j, PL::A1_R1_REG);
    const int e = (int)etile[i];
    if (do_measure) acc.add(norm2d(v[j]), e < p.e0, __popc((tile_base | i) ^ p.s0));
    if (KIND == 0) v[j] = PhaseOf<R>::apply(v[j], e, p.phase, tabs);
  }
  if (KIND == 0 && p.amp_scale != (R)1) {
#pragma unroll
    for (int j = 0; j < NR; ++j) {
      v[j].x *= p.amp_scale;
      v[j].y *= p.amp_scale;
    }
  }
  if (KIND == 0) {
    butterflies<R, PL::A1_R1_REG, PL::A1_R1_REG>(v, p.t);
    __syncthreads();
    smem_store_swz<R, PL::A1_R1_REG>(tile, v, b1);
    __syncthreads();
    // ---- round 2 ----
    const uint32_t b2 = pdep(lane, PL::A1_R2_LANE) | pdep(warp, PL::A1_R2_WARP);
    smem_load<R, PL::A1_R2_REG, true>(tile, v, b2);
    butterflies<R, PL::A1_R2_REG, PL::A1_R2_REG>(v, p.t);
    __syncthreads();
    smem_store_swz<R, PL::A1_R2_REG>(tile, v, b2);
    __syncthreads();
    // ---- round 3 -> global ----
    const uint32_t b3 = pdep(lane, PL::A1_R3_LANE) | pdep(warp, PL::A1_R3_WARP);
    smem_load<R, PL::A1_R3_REG, true>(tile, v, b3);
    butterflies<R, PL::A1_R3_REG, PL::A1_R3_ACT>(v, p.t);
    global_store<R, PL::A1_R3_REG, T>(p.state, v, tile_base, b3, 0);
  }
  if (do_measure) block_reduce_and_finalize(acc, p.partials, p.ticket, p.results, p.slot, (int)gridDim.x);
}

// Second-round plans of the strided pass, by W (active high bits).
template <class R, int W>
struct StridedR2;
// complex64 (T = 13)
template <int W>
struct StridedR2<float, W> {
  static_assert(W >= 5 && W <= 9, "");
  static constexpr uint32_t REG = (W <= 7) ? 0x3C1u : (W == 8 ? 0x1E1u : 0x1F0u);
  static constexpr uint32_t LANE = (W <= 7) ? 0x3Eu : (W == 8 ? 0x21Eu : 0x20Fu);
  static constexpr uint32_t WARP = 0x1C00u;
  static constexpr uint32_t ACT = (((1u << (W - 4)) - 1u) << (13 - W));
  static constexpr int kShuffleLaneBit = -1;
};
// complex128 (T = 12)
template <int W>
struct StridedR2<double, W> {
  static_assert(W >= 5 && W <= 9, "");
  static constexpr uint32_t REG = (W <= 8) ? 0xF0u : 0x78u;
  static constexpr uint32_t LANE = (W <= 8) ? 0x10Fu : 0x187u;
  static constexpr uint32_t WARP = 0xE00u;
  static constexpr uint32_t ACT = (W <= 8) ? (((1u << (W - 4)) - 1u) << (12 - W)) : 0x78u;
  static constexpr int kShuffleLaneBit = (W <= 8) ? -1 : 3;  // tile bit 7 butterflied across lanes
};

template <class R, int W>
__global__ void __launch_bounds__(kThreads, 2)
    strided_kernel(const __grid_constant__ CUtensorMap amap, const PassParams<R> p) {
  using amp = typename AmpTraits<R>::amp;
  using PL = Plan<R>;
  using L = SmemLayout<R>;
  constexpr int T = AmpTraits<R>::kTileBits;
  constexpr int CP = T - W;
  constexpr int NR = 1 << AmpTraits<R>::kRegBits;
  extern __shared__ __align__(1024) unsigned char smem[];
  amp* tile = reinterpret_cast<amp*>(smem);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + L::kTileBytes);

  const uint32_t b = blockIdx.x;
  const uint32_t mid = b & ((1u << p.mid_bits) - 1u);
  const uint32_t hi = b >> p.mid_bits;
  if (!load_tile<R>(&amap, nullptr, tile, nullptr, bar, p.mid_dim, (int)mid, p.hi_dim, (int)hi, p.err,
                    (uint32_t)L::kTileBytes))
    return;

  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t tile_base = (mid << CP) | (hi << (p.h0 + W));
  amp v[NR];
  constexpr uint32_t ACT_ALL = ((1u << W) - 1u) << CP;
  const uint32_t b1 = pdep(lane, PL::S_R1_LANE) | pdep(warp, PL::S_R1_WARP);
  smem_load<R, PL::S_R1_REG, false>(tile, v, b1);
  butterflies<R, PL::S_R1_REG, ACT_ALL>(v, p.t);
  if constexpr (W <= 4) {
    global_store<R, PL::S_R1_REG, CP>(p.state, v, tile_base, b1, p.h0);
  } else {
    using R2 = StridedR2<R, W>;
    __syncthreads();
    smem_store_swz<R, PL::S_R1_REG>(tile, v, b1);
    __syncthreads();
    const uint32_t b2 = pdep(lane, R2::LANE) | pdep(warp, R2::WARP);
    smem_load<R, R2::REG, true>(tile, v, b2);
    butterflies<R, R2::REG, R2::ACT>(v, p.t);
    if constexpr (R2::kShuffleLaneBit >= 0) {
#pragma unroll
      for (int j = 0; j < NR; ++j) {
        amp q;
        q.x = __shfl_xor_sync(0xffffffffu, v[j].x, 1 << R2::kShuffleLaneBit);
        q.y = __shfl_xor_sync(0xffffffffu, v[j].y, 1 << R2::kShuffleLaneBit);
        bfly_partner(v[j], q, p.t);
      }
    }
    global_store<R, R2::REG, CP>(p.state, v, tile_base, b2, p.h0);
  }
}

}  // namespace bk
