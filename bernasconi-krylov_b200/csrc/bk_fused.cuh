// Tile geometry shared by the tile engines (sm_100a): the persistent / grid
// forward engine (bk_persist.cuh) and the adjoint sweep (bk_adjoint.cuh).
//
// A step psi <- M D psi (reference order, src/sampling/sampler.cuh:604-618) is
// split into passes over 64 KB tiles of 16-byte elements (one complex128
// amplitude, or a pair of complex64 amplitudes stored pair-planar):
//   A1       tile = element bits [0, 12): measurement, diagonal phase D and the
//            Rx butterflies of the low qubits;
//   strided  tile = element bits [0, c') u [h0, h0 + W): the Rx butterflies of
//            the W high qubits [h0, h0 + W); the c' = 12 - W >= 3 contiguous low
//            bits keep every global access a >= 128 B segment.
// Qubit operations commute, so A1 + strided passes over disjoint high ranges
// apply M exactly once per qubit.
//
// Inside a tile every thread holds 16 elements in registers. A "round" names
// which tile bits are register bits (butterflied without data movement), lane
// bits and warp bits; between rounds the tile goes through shared memory with
// an XOR swizzle that keeps every round's 128-bit accesses bank-conflict free.
#pragma once
#include "bk_device.cuh"

namespace bk {

// shared-memory swizzle on 16-byte elements (linear over GF(2), bijective on
// the tile): bits [3, 12) fold into bits 0..2
template <class R>
__host__ __device__ constexpr uint32_t swz(uint32_t i);
template <>
__host__ __device__ constexpr uint32_t swz<double>(uint32_t i) {
  return i ^ (((i >> 3) ^ (i >> 6) ^ (i >> 9)) & 7u);
}

// Tile position -> global element index for tile bits [0, CP) u [h0, h0 + 12 - CP).
template <int CP>
__device__ __forceinline__ uint32_t tile_to_global(uint32_t p, uint32_t h0) {
  return (p & ((1u << CP) - 1u)) | ((p >> CP) << h0);
}

// ---- round plans (REG, LANE, WARP bit masks of the 2^12-element tile) ----
template <class R>
struct Plan;
template <>
struct Plan<double> {  // 16 elements per thread, 256 threads
  static constexpr uint32_t A1_R1_REG = 0x78, A1_R1_LANE = 0x187, A1_R1_WARP = 0xE00;
  static constexpr uint32_t A1_R2_REG = 0x87, A1_R2_LANE = 0x178, A1_R2_WARP = 0xE00;
  static constexpr uint32_t A1_R3_REG = 0xF00, A1_R3_LANE = 0x1F, A1_R3_WARP = 0xE0;
  static constexpr uint32_t A1_R3_ACT = 0xF00;
  static constexpr uint32_t S_R1_REG = 0xF00, S_R1_LANE = 0x1F, S_R1_WARP = 0xE0;
};

// Tile coordinate of TMA dim k: the tile-id parts go to mid_dim / hi_dim, every
// other dim is covered by the box (coordinate 0). Selects, no local arrays.
__device__ __forceinline__ int tile_coord(int k, int mid_dim, int mid, int hi_dim, int hi) {
  return (k == mid_dim ? mid : 0) + (k == hi_dim ? hi : 0);
}

// Second-round plans of the strided pass, by W (active high bits).
template <class R, int W>
struct StridedR2;
template <int W>
struct StridedR2<double, W> {
  static_assert(W >= 5 && W <= 9, "");
  static constexpr uint32_t REG = (W <= 8) ? 0xF0u : 0x78u;
  static constexpr uint32_t LANE = (W <= 8) ? 0x10Fu : 0x187u;
  static constexpr uint32_t WARP = 0xE00u;
  static constexpr uint32_t ACT = (W <= 8) ? (((1u << (W - 4)) - 1u) << (12 - W)) : 0x78u;
  static constexpr int kShuffleLaneBit = (W <= 8) ? -1 : 3;  // tile bit 7 butterflied across lanes
};

}  // namespace bk
