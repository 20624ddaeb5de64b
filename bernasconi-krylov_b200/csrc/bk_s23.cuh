// Fused strided pass (sm_100a): the S2 and S3 tile passes of one Trotter step in
// ONE persistent launch, so that every element crosses HBM once per step in the
// strided part instead of twice.
//
// Slabs. S2 tiles cover element bits [0, cp2) u [a1, a1 + w2), S3 tiles
// [0, cp3) u [a1 + w2, np) (cp = 12 - w, a1 = the bits the A1 pass covers). The
// bits [cpm, a1) with cpm = max(cp2, cp3) lie in neither tile: fixing them
// gives a slab that both passes tile completely. The Rx gates of different
// qubits commute, so either pass may go first; the high-bit pass S3 goes first
// because its tiles (rows 2^(a1 + w2) elements apart, a power of two of
// megabytes) read at full speed from DRAM but poorly from L2, where such rows
// crowd few L2 sets, while S2's rows (2^a1 elements apart) read from L2 at well
// over twice DRAM speed. An S2 tile of slab v needs every S3 tile of slab v and
// nothing else, so with the tasks ordered
//   S3(slab 0 .. L-1), then S2(slab v) before S3(slab v + L), ...
// S2 re-reads a slab that S3 wrote a few slabs earlier, while it is still in
// L2 (S3 stores evict-last; at N = 28 complex64 a slab is 16 MB). DRAM sees S3's
// reads and S2's writes only.
//
// Warp roles, one CTA per SM:
//   warp 0 (producer): claims tasks one at a time from a global counter in
//     order (the next claim already in flight), waits
//     (bounded) for an S3 task's slab counter, and issues the TMA load into a
//     ring of three 64 KB stages; a full barrier per stage carries the bytes,
//     so two tiles are in flight from HBM while the third is computed.
//   warps 1-8 (the compute group, 256 threads): the rounds of a tile run
//     between the group's named barrier; after the tile's last shared-memory
//     read the group frees the stage (empty barrier) and stores straight from
//     registers. An S3 tile then releases its slab counter (one thread,
//     red.release.gpu after the group barrier that orders all the group's
//     stores before it), deferred to the next tile's stage-free point so the
//     group does not wait for its own stores to drain.
// Nine warps keep each SM sub-partition at three warps or fewer, so the tile
// code keeps its registers (a second compute group would put five warps on
// one sub-partition and cap every thread at 96 registers, spilling).
// The producer never waits on a dependency before its earlier tasks are loaded,
// and claims are global and in order, so the smallest unfinished task always
// has its dependencies done, its stage free and its group idle: no deadlock.
// Every wait is bounded; a timeout sets the error word and the abort flag that
// every other wait polls, so the launch always ends.
#pragma once
#include "bk_persist.cuh"

namespace bk {

constexpr int kS23Stages = 3;
constexpr int kS23Groups = 1;
constexpr int kS23Threads = 32 + kS23Groups * kComputeThreads;  // 288
constexpr int kS23Smem = kS23Stages * kStageTileBytes;          // 192 KB
static_assert(kS23Stages == 3, "the producer tracks three stages by name");

enum S23Kind : uint32_t { S23_S2 = 1, S23_S3 = 2, S23_END = 0xFF };

// one launch = the strided part of one Trotter step
struct S23Program {
  // task order (claim index g -> task): for h = 0 .. slabs + lag - 1, the S3
  // tiles of slab h (h < slabs), then the S2 tiles of slab h - lag (h >= lag),
  // 2^lb tiles each in increasing tile id; decoded in closed form (s23_decode)
  uint32_t slabs, lag, lb;          // slab count, S2 -> S3 lag in slabs, log2 tiles per slab and pass
  uint32_t x, y, mb2, bits;         // cpm - cp2, cpm - cp3, S2 mid bits, slab bits
  uint32_t n_tasks;
  uint32_t step;                    // Trotter step (tangent index, slab-counter epoch)
  unsigned int* next;               // claim counter (reset by the last CTA to leave)
  unsigned int* ctas_done;
  unsigned int* slab_done;          // S3 completions per slab, cumulative over the steps of a call
  int* err;
  int* abort;
  uint32_t poll_limit;
};

struct S23Task {
  uint32_t kind, slab, tile;
};

// Task g of the launch's claim order (g < n_tasks): per slab the S3 tiles first,
// the S2 tiles `lag` slabs later. S2 tiles of slab v are
// mid | hi << mb2 with mid = v << x | low; S3 tiles are low | v << y | up << (y + bits).
__host__ __device__ inline S23Task s23_decode(const S23Program& P, uint32_t g) {
  const uint32_t B = 1u << P.lb;
  bool first;  // the slab's first sub-pass (S3) or its second (S2)
  uint32_t v, i;
  if (g < P.lag * B) {
    first = true;
    v = g >> P.lb;
    i = g & (B - 1u);
  } else {
    const uint32_t g1 = g - P.lag * B;
    if (g1 < 2u * B * (P.slabs - P.lag)) {
      const uint32_t pr = g1 >> (P.lb + 1u), r = g1 & (2u * B - 1u);
      first = r < B;
      v = first ? P.lag + pr : pr;
      i = r & (B - 1u);
    } else {
      const uint32_t g2 = g1 - 2u * B * (P.slabs - P.lag);
      first = false;
      v = P.slabs - P.lag + (g2 >> P.lb);
      i = g2 & (B - 1u);
    }
  }
  S23Task t;
  t.kind = first ? (uint32_t)S23_S3 : (uint32_t)S23_S2;
  t.slab = v;
  if (first)
    t.tile = (i & ((1u << P.y) - 1u)) | (v << P.y) | ((i >> P.y) << (P.y + P.bits));
  else
    t.tile = (v << P.x) | (i & ((1u << P.x) - 1u)) | ((i >> P.x) << P.mb2);
  return t;
}

__device__ __forceinline__ void red_release_add(unsigned int* p, unsigned int v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void s23_raise(const S23Program& P, int code) {
  atomicCAS(P.err, 0, code);
  atomicExch(P.abort, 1);
}
__device__ __forceinline__ bool s23_aborted(const S23Program& P) {
  return *reinterpret_cast<const volatile int*>(P.abort) != 0;
}
// bounded wait on a stage barrier phase that also gives up on a global abort
__device__ __forceinline__ bool s23_wait(uint32_t bar, uint32_t parity, const S23Program& P) {
  for (uint32_t i = 0; i < kWaitPolls; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255u) == 255u && s23_aborted(P)) return false;
  }
  s23_raise(P, DEV_TIMEOUT);
  return false;
}

template <class R>
__global__ void __launch_bounds__(kS23Threads, 1)
    s23_kernel(const __grid_constant__ InstDesc<R> D, const __grid_constant__ S23Program P) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t full_bar[kS23Stages];
  __shared__ __align__(8) uint64_t empty_bar[kS23Stages];
  __shared__ S23Task meta[kS23Stages];
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  if (tid == 0) {
    for (int s = 0; s < kS23Stages; ++s) {
      mbar_init(smem_addr(&full_bar[s]), 1);
      mbar_init(smem_addr(&empty_bar[s]), 1);
    }
    fence_barrier_init();
  }
  __syncthreads();

  if (warp == 0) {
    if (tid != 0) return;
    // ---- producer ----
    // One task claimed at a time (the GPU's window of tasks in progress stays
    // a few per SM, so S3 tiles find their slab finished and in L2), with the
    // next claim's atomic in flight while this task waits for its stage; the
    // task itself is decoded from its index (no memory read), and a slab
    // counter seen complete is not read again for the same slab.
    uint32_t armed0 = 0u, armed1 = 0u, armed2 = 0u;  // uses of each stage whose full phase was armed
    uint32_t ends = 0;                                // END markers published (one per compute group)
    uint32_t ok_slab = 0xFFFFFFFFu;                   // slab whose S2 tiles are known complete this step
    const uint32_t target = (1u << P.lb) * (P.step + 1u);
    uint32_t g_next = s23_aborted(P) ? P.n_tasks : atomicAdd(P.next, 1u);
    for (uint32_t j = 0; ends < (uint32_t)kS23Groups; ++j) {
      const uint32_t s = j % kS23Stages, u = j / kS23Stages;
      const uint32_t g = g_next;
      if (ends == 0u) g_next = (g >= P.n_tasks || s23_aborted(P)) ? P.n_tasks : atomicAdd(P.next, 1u);
      if (u > 0 && !s23_wait(smem_addr(&empty_bar[s]), (u - 1u) & 1u, P)) break;
      S23Task t{S23_END, 0u, 0u};
      if (ends == 0u && g < P.n_tasks && !s23_aborted(P)) t = s23_decode(P, g);
      if (t.kind == S23_S2 && t.slab != ok_slab) {
        // every S3 tile of the slab, this step, must be in memory
        const unsigned int* ctr = P.slab_done + t.slab;
        uint32_t polls = 0;
        bool ok = true;
        while (ld_acquire(ctr) < target) {
          if (++polls > P.poll_limit) {
            s23_raise(P, DEV_TIMEOUT);
            ok = false;
            break;
          }
          if ((polls & 63u) == 0u && s23_aborted(P)) {
            ok = false;
            break;
          }
          __nanosleep(64);
        }
        if (!ok) {
          t.kind = S23_END;
        } else {
          fence_proxy_async_global();  // the TMA reads what the counter released
          ok_slab = t.slab;
        }
      }
      meta[s] = t;
      const uint32_t fb = smem_addr(&full_bar[s]);
      if (t.kind == S23_END) {
        ++ends;
        mbar_arrive(fb);  // releases meta[s]; no bytes
      } else {
        StageMeta m;
        m.kind = (t.kind == S23_S2) ? TASK_S2 : TASK_S3;  // geometry of the tile
        m.inst = 0;
        m.tile = t.tile;
        m.step = P.step;
        issue_task_load(D, m, smem + (size_t)s * kStageTileBytes, fb);
      }
      if (s == 0) armed0 = u + 1u;
      else if (s == 1) armed1 = u + 1u;
      else armed2 = u + 1u;
    }
    // loads still in flight land before the CTA leaves
    if (armed0 > 0u) mbar_wait_bounded(smem_addr(&full_bar[0]), (armed0 - 1u) & 1u, P.err);
    if (armed1 > 0u) mbar_wait_bounded(smem_addr(&full_bar[1]), (armed1 - 1u) & 1u, P.err);
    if (armed2 > 0u) mbar_wait_bounded(smem_addr(&full_bar[2]), (armed2 - 1u) & 1u, P.err);
    // the last CTA out resets the claim counter for the next launch
    __threadfence();
    if (atomicAdd(P.ctas_done, 1u) == gridDim.x - 1u) {
      *P.next = 0u;
      *P.ctas_done = 0u;
    }
    return;
  }

  // ---- compute group(s): group g takes the CTA's tasks g, g + kS23Groups, ... ----
  const uint32_t grp = (warp - 1u) / 8u;
  const uint32_t tg = tid - 32u - (uint32_t)kComputeThreads * grp;
  const GroupSync sy{1u + grp};
  const R t = D.tan[P.step];
  // The release of an S3 tile's slab counter is deferred to the group's next
  // stage-free point: a release makes the releasing thread wait until every
  // store it covers is performed, and by then the previous tile's stores have
  // had a whole tile's compute to drain, while the current tile's are not yet
  // issued. It is never held across a wait: if the next tile is not loaded yet
  // (its load may depend on this very slab), the release goes out first.
  // Only thread 0 of the group tracks it; the group barrier at the end of the
  // S3 tile has made every thread's stores visible to it.
  constexpr uint32_t kNone = 0xFFFFFFFFu;
  uint32_t pending = kNone;
  for (uint32_t j = grp;; j += (uint32_t)kS23Groups) {
    const uint32_t s = j % kS23Stages, u = j / kS23Stages;
    const uint32_t fb = smem_addr(&full_bar[s]);
    if (tg == 0 && pending != kNone && !mbar_try_wait(fb, u & 1u)) {
      red_release_add(P.slab_done + pending, 1u);
      pending = kNone;
    }
    if (!s23_wait(fb, u & 1u, P)) break;
    const S23Task task = meta[s];
    if (task.kind == S23_END) break;
    unsigned char* stage = smem + (size_t)s * kStageTileBytes;
    const uint32_t eb = smem_addr(&empty_bar[s]);
    auto stage_free = [&]() {
      if (tg == 0) {
        mbar_arrive(eb);
        if (pending != kNone) {
          red_release_add(P.slab_done + pending, 1u);
          pending = kNone;
        }
      }
    };
    const bool s2 = (task.kind == S23_S2);
    const int w = s2 ? D.w2 : D.w3;
    const int mb = s2 ? D.s2_mid_bits : D.s3_mid_bits;
    const uint32_t h0 = s2 ? (uint32_t)D.a1_bits : (uint32_t)(D.a1_bits + D.w2);
    const uint32_t cp = (uint32_t)(kElemBits - w);
    const uint32_t mid = task.tile & ((1u << mb) - 1u), hi = task.tile >> mb;
    const uint32_t tile_base = (mid << cp) | (hi << (h0 + (uint32_t)w));
    // S3 (first) output is re-read by S2 from L2; S2 (second) output streams to DRAM
    process_s_dispatch<R>(w, stage, D.state, tile_base, h0, t, stage_free, tg, sy,
                          s2 ? policy_evict_first() : policy_evict_last());
    if (!s2) {
      sy.sync();  // every store of the group's tile precedes the (deferred) release
      if (tg == 0) pending = task.slab;
    }
  }
  if (tg == 0 && pending != kNone) red_release_add(P.slab_done + pending, 1u);
}

// ---------------------------------------------------------------------------
// Fused strided pass without a producer warp (engine mode 3): two compute
// groups of 8 warps per CTA (512 threads, so the tile code keeps 128 registers),
// each serving itself from a private 64 KB stage. A group's leader claims its
// next task one task ahead (the atomic's latency hides behind a tile), issues
// the task's load into the group's stage as soon as the current tile's last
// shared-memory read is done, and releases an S3 tile's slab counter at the
// next such point (the stores have had a tile's compute to drain). A group never
// waits on a slab counter while it holds an unfinished or unreleased task: when
// the next task's slab is not complete at the stage-free point, its load is
// deferred to the end of the current task, after the release. Claims are global
// and in order, so the smallest unfinished task always has its dependencies
// released and its group free: no deadlock. Same tile arithmetic as s23_kernel
// (bit-identical results); every wait is bounded.
// ---------------------------------------------------------------------------
constexpr int kS23gThreads = 2 * kComputeThreads;  // 512

// true in every thread of the 256-thread group (named barrier `id`) when any of them passes true
__device__ __forceinline__ bool group_any(uint32_t id, bool v) {
  uint32_t r;
  asm volatile(
      "{ .reg .pred p, q; setp.ne.u32 p, %1, 0; bar.red.or.pred q, %2, 256, p; selp.u32 %0, 1, 0, q; }"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(id)
      : "memory");
  return r != 0u;
}
__device__ __forceinline__ void fence_proxy_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
constexpr int kS23gSmem = 2 * kStageTileBytes;      // 128 KB

template <class R>
__global__ void __launch_bounds__(kS23gThreads, 1)
    s23g_kernel(const __grid_constant__ InstDesc<R> D, const __grid_constant__ S23Program P) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t full_bar[2];
  __shared__ uint32_t s_task[2];  // the group's current claim index, published by its leader
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  const uint32_t grp = warp >> 3, tg = tid & 255u;
  const bool leader = (tg == 0u);
  const GroupSync sy{1u + grp};
  unsigned char* stage = smem + (size_t)grp * kStageTileBytes;
  const uint32_t fb = smem_addr(&full_bar[grp]);
  const uint32_t target = (1u << P.lb) * (P.step + 1u);
  constexpr uint32_t kNone = 0xFFFFFFFFu;
  // leader state
  uint32_t pending = kNone;  // slab whose counter this group still owes a release
  uint32_t ok_slab = kNone;  // slab seen complete
  uint32_t ahead = 0u;       // the claim after the current one (issued one task early)
  bool armed = false;        // a load is in flight into the stage
  auto claim = [&]() -> uint32_t { return s23_aborted(P) ? P.n_tasks : atomicAdd(P.next, 1u); };
  // leader: the slab of an S2 task complete (polls once if `block` is false)
  auto slab_ready = [&](const S23Task& t, bool block) -> int {
    if (t.kind != S23_S2 || t.slab == ok_slab) return 1;
    const unsigned int* ctr = P.slab_done + t.slab;
    uint32_t polls = 0;
    while (ld_acquire(ctr) < target) {
      if (!block) return 0;
      if (++polls > P.poll_limit) {
        s23_raise(P, DEV_TIMEOUT);
        return -1;
      }
      if ((polls & 63u) == 0u && s23_aborted(P)) return -1;
      __nanosleep(64);
    }
    fence_proxy_async_global();  // the TMA reads what the counter released
    ok_slab = t.slab;
    return 1;
  };
  auto issue = [&](const S23Task& t) {
    fence_proxy_async_shared();  // the group's generic-proxy accesses of the stage precede the TMA's writes
    StageMeta m;
    m.kind = (t.kind == S23_S2) ? TASK_S2 : TASK_S3;
    m.inst = 0;
    m.tile = t.tile;
    m.step = P.step;
    issue_task_load(D, m, stage, fb);
    armed = true;
  };
  if (tid == 0) {
    mbar_init(smem_addr(&full_bar[0]), 1);
    mbar_init(smem_addr(&full_bar[1]), 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (leader) {
    uint32_t first = claim();
    ahead = claim();
    if (first < P.n_tasks) {
      const S23Task t = s23_decode(P, first);
      const int r = slab_ready(t, true);
      if (r > 0) issue(t);
      else first = P.n_tasks;
    }
    s_task[grp] = first;
  }
  sy.sync();
  const R tn = D.tan[P.step];
  uint32_t parity = 0;
  for (;;) {
    const uint32_t cur = s_task[grp];
    if (cur >= P.n_tasks) break;
    const bool landed = s23_wait(fb, parity, P);
    if (group_any(1u + grp, !landed)) break;  // the whole group leaves together
    parity ^= 1u;
    if (leader) armed = false;
    const S23Task task = s23_decode(P, cur);
    bool deferred = false;
    uint32_t nxt = P.n_tasks;
    auto stage_free = [&]() {
      if (!leader) return;
      // the stage is free: the next task's load goes out now unless its slab is not complete yet
      nxt = ahead;
      ahead = (nxt < P.n_tasks) ? claim() : P.n_tasks;
      if (nxt < P.n_tasks) {
        const S23Task t = s23_decode(P, nxt);
        if (slab_ready(t, false) > 0) issue(t);
        else deferred = true;
      }
      if (pending != kNone) {
        red_release_add(P.slab_done + pending, 1u);
        pending = kNone;
      }
    };
    const bool s2 = (task.kind == S23_S2);
    const int w = s2 ? D.w2 : D.w3;
    const int mb = s2 ? D.s2_mid_bits : D.s3_mid_bits;
    const uint32_t h0 = s2 ? (uint32_t)D.a1_bits : (uint32_t)(D.a1_bits + D.w2);
    const uint32_t cp = (uint32_t)(kElemBits - w);
    const uint32_t mid = task.tile & ((1u << mb) - 1u), hi = task.tile >> mb;
    const uint32_t tile_base = (mid << cp) | (hi << (h0 + (uint32_t)w));
    process_s_dispatch<R>(w, stage, D.state, tile_base, h0, tn, stage_free, tg, sy,
                          s2 ? policy_evict_first() : policy_evict_last());
    if (!s2) {
      sy.sync();  // every store of the group's tile precedes the (deferred) release
      if (leader) pending = task.slab;
    }
    if (leader) {
      if (deferred) {
        // nothing of this group is unfinished or unreleased while it waits for the slab
        if (pending != kNone) {
          red_release_add(P.slab_done + pending, 1u);
          pending = kNone;
        }
        const int r = slab_ready(s23_decode(P, nxt), true);
        if (r > 0) issue(s23_decode(P, nxt));
        else nxt = P.n_tasks;
      }
      s_task[grp] = nxt;
    }
    sy.sync();  // publishes the next claim (and orders this tile's reads of s_task before the write)
  }
  if (leader) {
    if (pending != kNone) red_release_add(P.slab_done + pending, 1u);
    if (armed) mbar_wait_bounded(fb, parity, P.err);  // a load in flight lands before the CTA leaves
  }
  __syncthreads();
  if (tid == 0) {
    // the last CTA out resets the claim counter for the next launch
    __threadfence();
    if (atomicAdd(P.ctas_done, 1u) == gridDim.x - 1u) {
      *P.next = 0u;
      *P.ctas_done = 0u;
    }
  }
}

}  // namespace bk
