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
constexpr int kPhaseLoBits = 7;  // phase(E) = hi[E >> 7] * lo[E & 127]
constexpr int kPhaseLo = 1 << kPhaseLoBits;

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
