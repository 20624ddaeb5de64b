// Auxiliary kernels: E table, p_blind count, state init, the whole-state kernel
// for n <= T (all steps in one launch), the plain per-qubit path, state export
// and projective sampling.
#pragma once
#include "bk_device.cuh"

namespace bk {

// E(s) for all s as uint16 (reference keeps doubles: src/sampling/sampler.cuh:54-70).
// Each thread writes 8 consecutive states (one 16-byte store).
__global__ void energy_table_kernel(uint16_t* __restrict__ out, int n, uint32_t count) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t s0 = g * 8u;
  if (s0 >= count) return;
  if (count - s0 >= 8u) {
    uint16_t e[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) e[k] = (uint16_t)labs_energy(s0 + k, n);
    uint4 q;
    q.x = e[0] | ((uint32_t)e[1] << 16);
    q.y = e[2] | ((uint32_t)e[3] << 16);
    q.z = e[4] | ((uint32_t)e[5] << 16);
    q.w = e[6] | ((uint32_t)e[7] << 16);
    *reinterpret_cast<uint4*>(out + s0) = q;
  } else {
    for (uint32_t s = s0; s < count; ++s) out[s] = (uint16_t)labs_energy(s, n);
  }
}

// #{s : E(s) < e0} (src/sampling/sampler.cuh:198-227); integer atomics are order-independent.
__global__ void count_below_kernel(const uint16_t* __restrict__ E, uint32_t count, int e0,
                                   unsigned long long* out) {
  unsigned long long c = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    c += ((int)E[i] < e0) ? 1ull : 0ull;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

template <class A>
__global__ void set_basis_kernel(A* psi, uint32_t idx) {
  A one;
  one.x = 1;
  one.y = 0;
  psi[idx] = one;
}

// complex64 pair-planar storage: float4 k = (re[2k], re[2k+1], im[2k], im[2k+1])
struct Planar64 {};
__global__ void set_basis_planar_kernel(float* psi, uint32_t idx) { psi[4u * (idx >> 1) + (idx & 1u)] = 1.0f; }
__device__ __forceinline__ double norm2_at(const float2* psi, uint32_t i) { return norm2d(psi[i]); }
__device__ __forceinline__ double norm2_at(const double2* psi, uint32_t i) { return norm2d(psi[i]); }
__device__ __forceinline__ double norm2_at(const Planar64* psi, uint32_t i) {
  const float* f = reinterpret_cast<const float*>(psi) + 4u * (i >> 1) + (i & 1u);
  return (double)fmaf(f[0], f[0], f[2] * f[2]);
}
__device__ __forceinline__ double2 amp_at(const float2* psi, uint32_t i) {
  return make_double2(psi[i].x, psi[i].y);
}
__device__ __forceinline__ double2 amp_at(const double2* psi, uint32_t i) { return psi[i]; }
__device__ __forceinline__ double2 amp_at(const Planar64* psi, uint32_t i) {
  const float* f = reinterpret_cast<const float*>(psi) + 4u * (i >> 1) + (i & 1u);
  return make_double2(f[0], f[2]);
}

// ---------------------------------------------------------------------------
// Whole-state kernel (n <= T): one CTA keeps the 2^n amplitudes in shared
// memory and runs every step (measure if flagged, D, Rx on each qubit) in one
// launch. Per-step tangents, D scale factors, measure flags and result slots
// come from device arrays.
// ---------------------------------------------------------------------------
template <class R>
struct SmallParams {
  typename AmpTraits<R>::amp* state;
  int n, n_steps;
  const R* t;            // n_steps tangents
  const R* amp_scale;    // n_steps exact powers of two folded into D
  const int* slot;       // n_steps + 1: results row, or -1
  typename PhaseOf<R>::params phase;
  int e0;
  uint32_t s0;
  double* results;
  int inverse;           // 1: apply the adjoint step (butterflies with -t, then conj(D))
  int measure_last;      // measure the entry at step n_steps (else the caller does later)
};

template <class R>
__global__ void __launch_bounds__(kThreads, 1) small_state_kernel(const SmallParams<R> p) {
  using amp = typename AmpTraits<R>::amp;
  extern __shared__ __align__(1024) unsigned char smem[];
  const int A = 1 << p.n;
  amp* s = reinterpret_cast<amp*>(smem);
  const auto tabs = PhaseOf<R>::stage(p.phase, smem);
  s = reinterpret_cast<amp*>(smem + PhaseOf<R>::kSmemBytes);
  uint16_t* E = reinterpret_cast<uint16_t*>(smem + PhaseOf<R>::kSmemBytes + (size_t)A * sizeof(amp));
  __shared__ double red[3][kThreads / 32];
  for (int i = threadIdx.x; i < A; i += kThreads) {
    s[i] = p.state[i];
    E[i] = (uint16_t)labs_energy((uint32_t)i, p.n);
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int step = 0; step <= p.n_steps; ++step) {
    const int slot = (step < p.n_steps || p.measure_last) ? p.slot[step] : -1;
    if (slot >= 0) {
      MeasureAcc acc;
      for (int i = threadIdx.x; i < A; i += kThreads)
        acc.add(norm2d(s[i]), (int)E[i] < p.e0, __popc((uint32_t)i ^ p.s0));
      double a = warp_sum(acc.norm), b = warp_sum(acc.p_less), c = warp_sum(acc.d_h);
      if (lane == 0) {
        red[0][warp] = a;
        red[1][warp] = b;
        red[2][warp] = c;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double x = 0, y = 0, z = 0;
        for (int w = 0; w < kThreads / 32; ++w) {
          x += red[0][w];
          y += red[1][w];
          z += red[2][w];
        }
        p.results[4 * (size_t)slot + 0] = y;
        p.results[4 * (size_t)slot + 1] = z;
        p.results[4 * (size_t)slot + 2] = x;
      }
      __syncthreads();
    }
    if (step == p.n_steps) break;
    const R t = p.inverse ? -p.t[step] : p.t[step];
    if (!p.inverse) {
      const R sc = p.amp_scale[step];
      for (int i = threadIdx.x; i < A; i += kThreads) {
        const int e = E[i];
        amp v = PhaseOf<R>::apply(s[i], e, p.phase, tabs);
        v.x *= sc;
        v.y *= sc;
        s[i] = v;
      }
      __syncthreads();
    }
    for (int q = 0; q < p.n; ++q) {
      for (int k = threadIdx.x; k < A / 2; k += kThreads) {
        const int a = ((k >> q) << (q + 1)) | (k & ((1 << q) - 1));
        bfly(s[a], s[a | (1 << q)], t);
      }
      __syncthreads();
    }
    if (p.inverse) {
      const R sc = p.amp_scale[step];
      for (int i = threadIdx.x; i < A; i += kThreads) {
        const int e = E[i];
        amp v = PhaseOf<R>::apply_inverse(s[i], e, p.phase, tabs);
        v.x *= sc;
        v.y *= sc;
        s[i] = v;
      }
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < A; i += kThreads) p.state[i] = s[i];
}

// ---------------------------------------------------------------------------
// Plain path: the reference's launch structure (src/sampling/sampler.cuh:604-618)
// — one diagonal-phase kernel per step with FP64 sincos (:73-91), then one
// 2x2 kernel per qubit with the matrix [[c, i s], [i s, c]] (:451-457).
// ---------------------------------------------------------------------------
template <class A>
__global__ void plain_phase_kernel(A* __restrict__ psi, const uint16_t* __restrict__ E, uint32_t count,
                                   double dt_over_n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const double th = -dt_over_n * (double)E[i];
  double sn, cs;
  sincos(th, &sn, &cs);
  const A a = psi[i];
  A r;
  r.x = (double)a.x * cs - (double)a.y * sn;
  r.y = (double)a.x * sn + (double)a.y * cs;
  psi[i] = r;
}

template <class A>
__global__ void plain_rx_kernel(A* __restrict__ psi, uint32_t half, int q, double c, double s) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= half) return;
  const uint32_t lo = k & ((1u << q) - 1u);
  const uint32_t a = ((k >> q) << (q + 1)) | lo;
  const uint32_t b = a | (1u << q);
  const A x = psi[a], y = psi[b];
  A xa, yb;
  // [a'; b'] = [[c, i s], [i s, c]] [a; b]
  xa.x = c * (double)x.x - s * (double)y.y;
  xa.y = c * (double)x.y + s * (double)y.x;
  yb.x = c * (double)y.x - s * (double)x.y;
  yb.y = c * (double)y.y + s * (double)x.x;
  psi[a] = xa;
  psi[b] = yb;
}

// Measurement over the whole state (plain path and any state the tiled A1 pass
// does not cover): fixed grid, FP64 per-block partials, ordered finalize.
template <class A>
__global__ void measure_kernel(const A* __restrict__ psi, const uint16_t* __restrict__ E, uint32_t count,
                               int e0, uint32_t s0, double* partials, unsigned int* ticket, double* results,
                               int slot) {
  MeasureAcc acc;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    acc.add(norm2d(psi[i]), (int)E[i] < e0, __popc(i ^ s0));
  block_reduce_and_finalize(acc, partials, ticket, results, slot, (int)gridDim.x);
}

// Export as interleaved (re, im) doubles, optionally multiplied by a diagonal
// phase exp(-i angle_unit * E(s)) (Strang convention) and a real scale.
template <class A>
__global__ void export_kernel(const A* __restrict__ psi, const uint16_t* __restrict__ E, uint32_t count,
                              double angle_unit, double scale, double2* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const double2 a = amp_at(psi, i);
  double2 r = make_double2(a.x * scale, a.y * scale);
  if (angle_unit != 0.0) {
    double sn, cs;
    sincos(-angle_unit * (double)E[i], &sn, &cs);
    r = make_double2(r.x * cs - r.y * sn, r.x * sn + r.y * cs);
  }
  out[i] = r;
}

// ---------------------------------------------------------------------------
// Projective sampling by inverse CDF (the reference calls the closed
// custatevecSampler*, src/sampling/sampler.cuh:464-466, 564-573): chunk sums of
// |psi|^2 in FP64, an exclusive scan over chunks, then per shot a binary search
// over chunks and a warp scan inside the chunk. Shot k returns the smallest s
// with u_k * total < cdf(s).
// ---------------------------------------------------------------------------
constexpr int kSampleChunkBits = 12;

template <class A>
__global__ void chunk_sums_kernel(const A* __restrict__ psi, uint32_t count, double* __restrict__ sums) {
  const uint32_t chunk = blockIdx.x;
  const uint32_t base = chunk << kSampleChunkBits;
  const uint32_t len = min(1u << kSampleChunkBits, count - base);
  double acc = 0.0;
  for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) acc += norm2_at(psi, base + i);
  __shared__ double red[kThreads / 32];
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) s += red[w];
    sums[chunk] = s;
  }
}

// In-place exclusive scan of `m` chunk sums by one block; total written to sums[m].
__global__ void scan_chunks_kernel(double* sums, uint32_t m) {
  __shared__ double carry;
  __shared__ double wsum[32];
  if (threadIdx.x == 0) carry = 0.0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t base = 0; base < m; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const double x = (i < m) ? sums[i] : 0.0;
    double inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const double y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
      double w = (lane < (int)(blockDim.x / 32)) ? wsum[lane] : 0.0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      wsum[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const double before = carry + (warp > 0 ? wsum[warp - 1] : 0.0);
    if (i < m) sums[i] = before + inc - x;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = before + inc;
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[m] = carry;
}

// One warp per shot.
template <class A>
__global__ void sample_kernel(const A* __restrict__ psi, uint32_t count, const double* __restrict__ prefix,
                              uint32_t m, const double* __restrict__ randnums, int64_t shots,
                              unsigned long long* __restrict__ out) {
  const int64_t shot = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (shot >= shots) return;
  const double total = prefix[m];
  const double target = randnums[shot] * total;
  // last chunk whose exclusive prefix is <= target
  uint32_t lo = 0, hi = m;  // answer in [lo, hi)
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (prefix[mid] <= target) lo = mid; else hi = mid;
  }
  const uint32_t base = lo << kSampleChunkBits;
  const uint32_t len = min(1u << kSampleChunkBits, count - base);
  const uint32_t per = (len + 31) / 32;
  const uint32_t mine0 = min(len, lane * per), mine1 = min(len, mine0 + per);
  double part = 0.0;
  for (uint32_t i = mine0; i < mine1; ++i) part += norm2_at(psi, base + i);
  double inc = part;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  const double start = prefix[lo] + inc - part;
  const double end = prefix[lo] + inc;
  // first lane whose inclusive cumulative exceeds the target
  const unsigned ballot = __ballot_sync(0xffffffffu, target < end && mine1 > mine0);
  uint32_t result = base + len - 1;  // rounding guard: clamp to the chunk's last state
  if (ballot) {
    const int owner = __ffs(ballot) - 1;
    if (lane == owner) {
      double c = start;
      uint32_t r = mine1 - 1;
      for (uint32_t i = mine0; i < mine1; ++i) {
        c += norm2_at(psi, base + i);
        if (target < c) {
          r = i;
          break;
        }
      }
      out[shot] = base + r;
    }
  } else if (lane == 0) {
    out[shot] = result;
  }
}

}  // namespace bk

namespace bk {

// ---------------------------------------------------------------------------
// d_min (reference: src/labs_energy/labs_energy.hpp:175-207): is there a state
// with E < target on the Hamming sphere of radius d around s? Each thread
// unranks masks of weight d (combinatorial number system, colex order) in a
// grid-stride loop; the first hit raises *found and the others stop early.
// binom[c * 32 + k] = C(c, k) for c, k < 32.
// ---------------------------------------------------------------------------
__global__ void dmin_sphere_kernel(int n, uint32_t s, int target, int d, unsigned long long count,
                                   const unsigned long long* __restrict__ binom, int* found) {
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long r = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; r < count; r += stride) {
    if (*reinterpret_cast<volatile int*>(found)) return;
    uint32_t mask = 0;
    unsigned long long rem = r;
    int c = n - 1;
    for (int k = d; k >= 1; --k) {
      while (binom[c * 32 + k] > rem) --c;
      mask |= 1u << c;
      rem -= binom[c * 32 + k];
      --c;
    }
    if (labs_energy(s ^ mask, n) < target) atomicExch(found, 1);
  }
}

// ---------------------------------------------------------------------------
// Batched single-flip steepest descent (reference: batch_steepest_descent_kernel,
// src/classical/classical.cuh:459-540; CPU form :625-712). One warp per start:
// lane l scores the flips p = l, l + 32 from the shared autocorrelations C_k
// (C_k + d_k(p))^2 summed over k, the warp keeps the lowest energy and, among
// equal energies, the lowest p — the flip the sequential scan (first strictly
// better) takes; lanes own C_k for k = l, l + 32 for the update. An iteration
// costs n evaluations and runs only while evals + n <= budget, as in the reference.
// ---------------------------------------------------------------------------
constexpr int kDescentWarps = 8;

__device__ __forceinline__ int spin_of(uint64_t x, int i) { return ((x >> i) & 1ull) ? -1 : 1; }

__global__ void __launch_bounds__(32 * kDescentWarps)
    descent_kernel(int n, const uint64_t* __restrict__ starts, long long count, unsigned long long budget,
                   uint64_t* __restrict__ final_states, long long* __restrict__ final_energies,
                   unsigned long long* __restrict__ evals_out) {
  __shared__ int Cs[kDescentWarps][64];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const long long i = (long long)blockIdx.x * kDescentWarps + wib;
  if (i >= count) return;  // the whole warp leaves together
  int* C = Cs[wib];
  const uint64_t mask = (1ull << n) - 1ull;
  uint64_t x = starts[i] & mask;
  int part = 0;
  for (int k = 1 + lane; k < n; k += 32) {
    const int c = (n - k) - 2 * __popcll((x ^ (x >> k)) & ((1ull << (n - k)) - 1ull));
    C[k] = c;
    part += c * c;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  int e = part;
  __syncwarp();
  unsigned long long evals = 1;
  while (evals + (unsigned long long)n <= budget) {
    int best_e = e, best_p = 0x7fffffff;
    for (int p = lane; p < n; p += 32) {
      const int sp = spin_of(x, p);
      int ne = 0;
      for (int k = 1; k < n; ++k) {
        int d = 0;
        if (p + k < n) d -= 2 * sp * spin_of(x, p + k);
        if (p - k >= 0) d -= 2 * sp * spin_of(x, p - k);
        const int c = C[k] + d;
        ne += c * c;
      }
      if (ne < best_e) {
        best_e = ne;
        best_p = p;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const int oe = __shfl_xor_sync(0xffffffffu, best_e, o);
      const int op = __shfl_xor_sync(0xffffffffu, best_p, o);
      if (oe < best_e || (oe == best_e && op < best_p)) {
        best_e = oe;
        best_p = op;
      }
    }
    evals += (unsigned long long)n;
    if (best_p == 0x7fffffff) break;  // no strictly better neighbour: a local minimum
    const int sp = spin_of(x, best_p);
    __syncwarp();
    for (int k = 1 + lane; k < n; k += 32) {
      int d = 0;
      if (best_p + k < n) d -= 2 * sp * spin_of(x, best_p + k);
      if (best_p - k >= 0) d -= 2 * sp * spin_of(x, best_p - k);
      C[k] += d;
    }
    __syncwarp();
    x ^= 1ull << best_p;
    e = best_e;
  }
  if (lane == 0) {
    final_states[i] = x;
    final_energies[i] = e;
    if (evals_out) evals_out[i] = evals;
  }
}

// Per-shot energy and Hamming distance to the start state for drawn basis
// states (the reference evaluates both on the host for every shot,
// src/sampling/sampler.cuh:575-596): one thread per shot, exact integers.
__global__ void shot_stats_kernel(const unsigned long long* __restrict__ states, long long count, int n,
                                  unsigned long long s0, int* __restrict__ energies, int* __restrict__ flips) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const unsigned long long b = states[i];
  energies[i] = labs_energy((uint32_t)b, n);
  flips[i] = __popcll(b ^ s0);
}

}  // namespace bk
