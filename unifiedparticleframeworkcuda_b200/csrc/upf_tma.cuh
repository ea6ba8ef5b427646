// upf_tma.cuh — TMA (cp.async.bulk.tensor) streaming of the neighbour lists
// into shared memory, one pipeline per warp.
//
// The neighbour lists are column-major [row k][particle i], so the rows
// k..k+R-1 of a warp's 32 consecutive particles form a 2D box of 32 x R
// elements. Lane 0 of each warp issues one 2D tensor copy per box into a ring
// of kStages shared-memory stages; every lane waits on the stage's mbarrier
// (bounded: a wait that runs out records ERR_TIMEOUT, and the warp stops its
// walk, drains the copies it issued and goes on without that data rather
// than hanging). Only loads from this GPU's own
// memory, no cluster multicast.
#pragma once

#include <cuda.h>
#include <stdint.h>

#include "upf_common.cuh"

namespace upf {

constexpr int kListRows = 8;     // default list rows per stage (a launch shape parameter)
constexpr int kListStages = 3;   // ring depth
constexpr uint32_t kWaitSpins = 1u << 24;          // bounded wait: at most this many polls ...
constexpr uint64_t kWaitLimitNs = 1000000000ull;    // ... and at most 1 s of device time

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bounded wait, by poll count and by device time; returns false (and the
// caller records a timeout) if the phase did not complete
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns = kWaitLimitNs) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  for (uint32_t s = 0; s < kWaitSpins; ++s) {
    if (mbar_try_wait(bar, parity)) return true;
    if (globaltimer_ns() - t0 > limit_ns) return false;
  }
  return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// One warp's ring of list stages. Stage s holds rows [c*R, c*R+R) of chunk c
// (c % kListStages == s) for the warp's 32 columns: codes (uint32) and,
// when kWithVals, the entries' list values (uint32). R = kRows, the box
// height of the tensor map.
template <bool kWithVals, int kRows = kListRows>
struct __align__(128) WarpListRing {
  uint32_t codes[kListStages][kRows][32];                   // 128 B per row
  uint32_t vals[kWithVals ? kListStages : 1][kRows][32];     // 128 B per row
  uint64_t full[kListStages];
};

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

template <bool kWithVals, int kRows>
__device__ __forceinline__ void ring_issue(WarpListRing<kWithVals, kRows>& r, const CUtensorMap* cmap,
                                           const CUtensorMap* vmap, int chunk, int col0) {
  const int s = chunk % kListStages;
  const uint32_t bytes = kRows * 32 * (4 + (kWithVals ? 4 : 0));
  fence_proxy_async_smem();  // the stage's previous contents were read through the generic proxy
  mbar_arrive_expect_tx(&r.full[s], bytes);
  tma_load_2d(&r.codes[s][0][0], cmap, &r.full[s], col0, chunk * kRows);
  if (kWithVals) tma_load_2d(&r.vals[s][0][0], vmap, &r.full[s], col0, chunk * kRows);
}

// Walks the warp's lists chunk by chunk. `body(s, rows)` consumes stage s
// (rows valid rows); lanes index their own column. Returns false if a wait
// ran out: the warp then issues no further copy, skips the remaining chunks,
// and waits (again bounded) for the copies it already issued, so that none
// lands in the ring after the warp has moved on.
constexpr uint64_t kDrainLimitNs = 100000000ull;  // 0.1 s per issued stage when draining after a timeout

template <bool kWithVals, int kRows, class Body>
__device__ __forceinline__ bool ring_walk(WarpListRing<kWithVals, kRows>& r, const CUtensorMap* cmap,
                                          const CUtensorMap* vmap, int col0, uint32_t warp_max_cnt, Body&& body) {
  const int lane = threadIdx.x & 31;
  const int nchunks = (int)((warp_max_cnt + kRows - 1) / kRows);
  if (lane == 0) {
    for (int c = 0; c < kListStages && c < nchunks; ++c) ring_issue(r, cmap, vmap, c, col0);
  }
  int c = 0;
  for (; c < nchunks; ++c) {
    const int s = c % kListStages;
    const uint32_t parity = (uint32_t)(c / kListStages) & 1u;
    // warp-uniform decision: every lane consumes the stage, or none does
    if (!__all_sync(0xffffffffu, mbar_wait(&r.full[s], parity))) break;
    body(s, c * kRows);
    __syncwarp();
    if (lane == 0 && c + kListStages < nchunks) ring_issue(r, cmap, vmap, c + kListStages, col0);
  }
  if (c == nchunks) return true;
  // chunks c .. issued-1 were issued and not consumed
  const int issued = (c + kListStages < nchunks) ? c + kListStages : nchunks;
  for (int d = c; d < issued; ++d)
    (void)mbar_wait(&r.full[d % kListStages], (uint32_t)(d / kListStages) & 1u, kDrainLimitNs);
  __syncwarp();
  return false;
}

template <bool kWithVals, int kRows>
__device__ __forceinline__ void ring_init(WarpListRing<kWithVals, kRows>& r) {
  if ((threadIdx.x & 31) == 0) {
    for (int s = 0; s < kListStages; ++s) mbar_init(&r.full[s], 1);
    fence_barrier_init();
  }
  __syncwarp();
}

}  // namespace upf
