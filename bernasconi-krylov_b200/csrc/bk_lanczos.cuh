// Full-space Hamiltonian matvec and Lanczos building blocks (sm_100a).
//
// The reference's full-space Krylov solver (src/subspace/diagonalizer.cuh:377-416,
// driver :418-560) multiplies by H = diag(scale E(s)) - g sum_j X_j with one
// thread per basis state gathering its N neighbours i ^ 2^j from global memory
// (fullspace_matvec_kernel_d, :60-77). On a B200 the 126 MB L2 already serves
// that form's neighbours up to ~2^23 states away, and the DRAM cost is the far
// neighbours. Here one product is:
//   block pass (fs_block_kernel): 8192-state blocks, the block of x staged in
//     shared memory by a bulk copy for the 13 low-bit neighbours, bits 13..22 as
//     coalesced sweeps of the partner blocks (L2 hits: partners <= 32 MB away),
//     the diagonal from the cached uint16 E table, y stored streaming;
//   strided pass (fs_tile_kernel, n > 23): tiles of index bits [0, 13 - w) u
//     [23, n), w = n - 23 <= 7 (runs of >= 64 doubles) loaded as one tensor-map
//     box, y -= g sum x[i ^ 2^j] for the far bits with every partner inside the tile.
// DRAM per state: x, E, y once (18 B) plus x, y, y (24 B) for the far bits.
//
// Lanczos steps (the driver's cuBLAS calls, :437-482) are fused element-wise
// kernels with per-block partial sums reduced in a fixed order (deterministic).
#pragma once
#include "bk_device.cuh"
#include "bk_fused.cuh"

namespace bk {

constexpr int kFsTileBits = 13;  // 8192 doubles per tile
constexpr int kFsThreads = 256;
constexpr int kLzBlocks = 296;   // partial-sum blocks of the Lanczos reductions (2 per SM on a B200)

// One neighbour-sum pass over a tile smaller than 8192 doubles (n < 13: the
// whole vector in one CTA). Tile position p -> state index: bits [0, cp) stay,
// bits [cp, tb) go to [h0, h0 + tb - cp); the tile id splits into mb "mid" bits
// (index bits [cp, h0)) and the bits above h0 + tb - cp. first: pass 0 (writes
// the diagonal term); act_lo: lowest tile bit whose neighbours this pass sums.
__global__ void __launch_bounds__(kFsThreads) fs_pass_kernel(const double* __restrict__ x, double* __restrict__ y,
                                                             const uint16_t* __restrict__ E, double scale, double g,
                                                             int tb, int cp, int h0, int mb, int first, int act_lo) {
  extern __shared__ __align__(16) double ft[];
  const uint32_t tile = blockIdx.x;
  const int w = tb - cp;
  const uint64_t mid = tile & ((1u << mb) - 1u), hi = tile >> mb;
  const uint64_t base = (mid << cp) | (hi << (h0 + w));
  const uint32_t size = 1u << tb, lo_mask = (1u << cp) - 1u;
  for (uint32_t p = threadIdx.x; p < size; p += kFsThreads)
    ft[p] = x[base | (p & lo_mask) | ((uint64_t)(p >> cp) << h0)];
  __syncthreads();
  for (uint32_t p = threadIdx.x; p < size; p += kFsThreads) {
    double s = 0.0;
    for (int b = act_lo; b < tb; ++b) s += ft[p ^ (1u << b)];
    const uint64_t gi = base | (p & lo_mask) | ((uint64_t)(p >> cp) << h0);
    y[gi] = first ? scale * (double)E[gi] * ft[p] - g * s : y[gi] - g * s;
  }
}


constexpr int kFsPer = (1 << kFsTileBits) / kFsThreads;  // 32 tile positions per thread
constexpr int kFsTileSmem = (1 << kFsTileBits) * (int)sizeof(double) + 128;  // strided pass: tile + alignment slack

// A neighbour-sum pass over a full 8192-double tile (the strided pass): the tile
// of x arrives as ONE tensor-map box (runs of 2^cp contiguous doubles, 2^w of
// them 2^h0 doubles apart) while every thread prefetches its 32 values of y (or
// of scale * E when first) into registers, so each SM keeps > 100 KB of loads in
// flight; then the neighbour sums over tile bits [act_lo, 13) are read from
// shared memory. (One bulk copy per run was measured 3-5x slower per byte than
// one box for runs of a few hundred bytes.)
__global__ void __launch_bounds__(kFsThreads, 2) fs_tile_kernel(const CUtensorMap* __restrict__ xmap,
                                                                double* __restrict__ y,
                                                                const uint16_t* __restrict__ E, double scale, double g,
                                                                int cp, int h0, int mb, int md, int hd, int first,
                                                                int act_lo, int* err) {
  // the tensor copy's destination must sit on a 128-byte boundary: the dynamic
  // area gets 128 bytes of slack (kFsTileSmem) and the tile is aligned here
  extern __shared__ __align__(128) unsigned char fs_raw[];
  double* ft = reinterpret_cast<double*>(fs_raw + ((128u - (smem_addr(fs_raw) & 127u)) & 127u));
  __shared__ __align__(8) uint64_t bar;
  const uint32_t tid = threadIdx.x, tile = blockIdx.x;
  if ((smem_addr(ft) & 127u) != 0u) {  // cannot happen after the alignment above; never issue a misaligned copy
    if (tid == 0) atomicCAS(err, 0, DEV_BAD_LAUNCH);
    return;
  }
  const int w = kFsTileBits - cp;
  const uint32_t mid = tile & ((1u << mb) - 1u), hi = tile >> mb;
  const uint64_t base = ((uint64_t)mid << cp) | ((uint64_t)hi << (h0 + w));
  const uint32_t lo_mask = (1u << cp) - 1u;
  const uint32_t fb = smem_addr(&bar);
  if (tid == 0) {
    mbar_init(fb, 1);
    fence_barrier_init();
    mbar_arrive_expect_tx(fb, 8u << kFsTileBits);
    tma_load_5d_hint(smem_addr(ft), xmap, tile_coord(0, md, (int)mid, hd, (int)hi),
                     tile_coord(1, md, (int)mid, hd, (int)hi), tile_coord(2, md, (int)mid, hd, (int)hi),
                     tile_coord(3, md, (int)mid, hd, (int)hi), tile_coord(4, md, (int)mid, hd, (int)hi), fb,
                     policy_evict_first());
  }
  // no thread may poll the barrier before thread 0 has initialised it
  __syncthreads();
  double pre[kFsPer];
#pragma unroll
  for (int k = 0; k < kFsPer; ++k) {
    const uint32_t p = tid + kFsThreads * (uint32_t)k;
    const uint64_t gi = base | (p & lo_mask) | ((uint64_t)(p >> cp) << h0);
    pre[k] = first ? scale * (double)E[gi] : y[gi];
  }
  const bool ok = mbar_wait_bounded(fb, 0, err);
  if (__syncthreads_or(!ok)) return;
#pragma unroll
  for (int k = 0; k < kFsPer; ++k) {
    const uint32_t p = tid + kFsThreads * (uint32_t)k;
    double s = 0.0;
    for (int b = act_lo; b < kFsTileBits; ++b) s += ft[p ^ (1u << b)];
    const uint64_t gi = base | (p & lo_mask) | ((uint64_t)(p >> cp) << h0);
    y[gi] = first ? pre[k] * ft[p] - g * s : pre[k] - g * s;
  }
}

// First pass for n >= 13: CTA = one 8192-state block (index bits 0-12). The
// block of x arrives in shared memory by one 64 KB bulk copy; the 13 low-bit
// neighbours are read there. Each bit j in [13, n_gather) pairs the block with
// the block 2^(j-13) away, read as one coalesced sweep (32 loads in flight per
// thread) into register accumulators: with blocks in index order and at most 512
// blocks (32 MB) between partners (n_gather <= 23), the partner is still in the
// 126 MB L2, so DRAM sees x, E and y once; y is stored streaming (evict-first) so
// it does not push x out of L2. Bits >= n_gather go to a strided tile pass.
constexpr int kFsGatherBits = 23;
__global__ void __launch_bounds__(kFsThreads, 2) fs_block_kernel(const double* __restrict__ x, double* __restrict__ y,
                                                                 const uint16_t* __restrict__ E, double scale, double g,
                                                                 int n_gather, int* err) {
  extern __shared__ __align__(128) double ft[];
  __shared__ __align__(8) uint64_t bar;
  const uint32_t tid = threadIdx.x;
  const uint64_t base = (uint64_t)blockIdx.x << kFsTileBits;
  const uint32_t fb = smem_addr(&bar);
  if (tid == 0) {
    mbar_init(fb, 1);
    fence_barrier_init();
    mbar_arrive_expect_tx(fb, 8u << kFsTileBits);
    bulk_load(smem_addr(ft), x + base, 8u << kFsTileBits, fb);
  }
  // no thread may poll the barrier before thread 0 has initialised it (an SM's
  // shared memory can still hold a completed barrier of an earlier CTA)
  __syncthreads();
  double acc[kFsPer];
#pragma unroll
  for (int k = 0; k < kFsPer; ++k) acc[k] = 0.0;
  // high bits first (global, mostly L2), while the block's own copy is in flight
  for (int j = kFsTileBits; j < n_gather; ++j) {
    const double* nb = x + (base ^ (1ull << j));
#pragma unroll
    for (int k = 0; k < kFsPer; ++k) acc[k] += __ldg(nb + tid + kFsThreads * k);
  }
  const bool ok = mbar_wait_bounded(fb, 0, err);
  if (__syncthreads_or(!ok)) return;
#pragma unroll
  for (int k = 0; k < kFsPer; ++k) {
    const uint32_t p = tid + kFsThreads * (uint32_t)k;
    double s = 0.0;
#pragma unroll
    for (int b = 0; b < kFsTileBits; ++b) s += ft[p ^ (1u << b)];
    const double v = scale * (double)E[base + p] * ft[p] - g * (s + acc[k]);
    __stcs(y + base + p, v);
  }
}

// The reference's form (diagonalizer.cuh:60-77): one thread per state, its n
// neighbours gathered from global memory in bit order (the BK_PLAIN comparison).
__global__ void __launch_bounds__(256) fs_plain_kernel(const double* __restrict__ x, double* __restrict__ y,
                                                       const uint16_t* __restrict__ E, double scale, double g, int n,
                                                       uint64_t N) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double yi = (double)E[i] * scale * x[i];
  for (int j = 0; j < n; ++j) yi -= g * x[i ^ (1ull << j)];
  y[i] = yi;
}

__device__ __forceinline__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
  return s;  // valid in thread 0
}

// w -= beta[jb] * vprev (jb >= 0); partials[block] = sum of v * w over the block's states
__global__ void __launch_bounds__(256) lz_orth_dot_kernel(double* __restrict__ w, const double* __restrict__ vprev,
                                                          const double* __restrict__ v, const double* __restrict__ beta,
                                                          int jb, uint64_t N, double* __restrict__ partials) {
  __shared__ double red[8];
  const double b = jb >= 0 ? beta[jb] : 0.0;
  double acc = 0.0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (uint64_t)gridDim.x * blockDim.x) {
    double wi = w[i];
    if (jb >= 0) wi -= b * vprev[i];
    w[i] = wi;
    acc += v[i] * wi;
  }
  const double s = block_sum(acc, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// w -= alpha[ja] * v; partials[block] = sum of w^2
// w and v may be the same vector (the start vector's norm): no __restrict__ on them
__global__ void __launch_bounds__(256) lz_axpy_nrm_kernel(double* w, const double* v,
                                                          const double* __restrict__ alpha, int ja, uint64_t N,
                                                          double* __restrict__ partials) {
  __shared__ double red[8];
  const double a = ja >= 0 ? alpha[ja] : 0.0;
  double acc = 0.0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (uint64_t)gridDim.x * blockDim.x) {
    const double wi = w[i] - a * v[i];
    if (ja >= 0) w[i] = wi;
    acc += wi * wi;
  }
  const double s = block_sum(acc, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// out[slot] = sum of partials[0..count) in a fixed order (sqrt of it when take_sqrt)
__global__ void lz_reduce_kernel(const double* __restrict__ partials, int count, double* __restrict__ out, int slot,
                                 int take_sqrt) {
  __shared__ double red[8];
  double acc = 0.0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) acc += partials[i];
  const double s = block_sum(acc, red);
  if (threadIdx.x == 0) out[slot] = take_sqrt ? sqrt(s) : s;
}

// dst = src * (1 / norm[slot]); dst may equal src (in-place normalisation), so
// neither is __restrict__
__global__ void __launch_bounds__(256) lz_scale_kernel(double* dst, const double* src,
                                                       const double* __restrict__ norm, int slot, uint64_t N) {
  const double inv = 1.0 / norm[slot];
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (uint64_t)gridDim.x * blockDim.x)
    dst[i] = src[i] * inv;
}

// x = sum_j V[j] * coef[j] (a Ritz vector from the Krylov basis)
__global__ void __launch_bounds__(256) lz_combine_kernel(const double* __restrict__ V, const double* __restrict__ coef,
                                                         int m, uint64_t N, double* __restrict__ x) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (uint64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < m; ++j) s += V[(uint64_t)j * N + i] * coef[j];
    x[i] = s;
  }
}

}  // namespace bk
