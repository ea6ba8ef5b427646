// upf_sort.cu — stable LSD radix sort of (key, value) pairs, Morton keys and
// cell ranges.
//
// Replaces the reference's 2006 SDK sort (RadixSum / RadixPrefixSum /
// RadixAddOffsetsAndShuffle, src/gpu/radixsort_kernel.cu:64-540, driver
// src/gpu/particles.cu:31-60), which runs a fixed 48-CTA grid. Here each pass
// is three launches sized to the input, one CTA per tile of 512, 2048 or 8192
// keys (radix_tile_keys: the smallest tile that needs at most kRadixTileCap
// tiles):
//   upsweep   per-tile digit histograms (shared-memory atomics)
//   scan      per digit, exclusive scan of its row of tile counts (one CTA
//             per digit) and the digit's total
//   downsweep per-tile stable ranking with warp match/ballot (each warp owns
//             a contiguous segment of 32, 128 or 512 keys, rounds run in key
//             order), a local sort through shared memory, and coalesced runs
//             to global memory.
// Stability: warps own consecutive segments and rank in order, so equal
// digits keep their input order; an LSD sort of stable passes is stable.
#include <cuda_runtime.h>

#include <mutex>

#include "upf_common.cuh"
#include "upf_internal.h"

namespace upf {

namespace {

constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kThreads = 512;               // 16 warps
constexpr int kWarps = kThreads / 32;
static_assert(kRadix == (int)kRadixDigits, "scratch layout constants");

// kItems keys per lane: a warp ranks 32 * kItems consecutive keys, a tile is
// kWarps warps' segments
template <int kItems>
__global__ void __launch_bounds__(kThreads) k_upsweep(const uint32_t* __restrict__ keys, uint32_t n,
                                                       int shift, uint32_t ntiles,
                                                       uint32_t* __restrict__ counts) {
  constexpr int kTile = kWarps * 32 * kItems;
  __shared__ uint32_t hist[kRadix];
  for (int d = threadIdx.x; d < kRadix; d += kThreads) hist[d] = 0;
  __syncthreads();
  const uint32_t base = blockIdx.x * (uint32_t)kTile;
#pragma unroll 4
  for (int r = 0; r < kTile / kThreads; ++r) {
    uint32_t i = base + r * kThreads + threadIdx.x;
    if (i < n) atomicAdd(&hist[(keys[i] >> shift) & (kRadix - 1)], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadix; d += kThreads) counts[(size_t)d * ntiles + blockIdx.x] = hist[d];
}

// Exclusive scan of each digit's row of tile counts, one CTA of 256 threads
// per digit: counts[d][t] becomes the number of keys with digit d in tiles
// before t, and totals[d] the digit's count over all tiles. The downsweep
// adds the digit's base (the exclusive scan of the totals).
__global__ void __launch_bounds__(256) k_scan_rows(uint32_t* __restrict__ counts, uint32_t ntiles,
                                                   uint32_t* __restrict__ totals) {
  __shared__ uint32_t warp_sums[8];
  __shared__ uint32_t carry;
  uint32_t* row = counts + (size_t)blockIdx.x * ntiles;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t base = 0; base < ntiles; base += 256 * 4) {
    uint32_t v[4];
    const uint32_t idx0 = base + threadIdx.x * 4;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      v[k] = (idx0 + k < ntiles) ? row[idx0 + k] : 0u;
      s += v[k];
    }
    uint32_t incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const uint32_t w = lane < 8 ? warp_sums[lane] : 0u;
      uint32_t wi = w;
#pragma unroll
      for (int o = 1; o < 8; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += t;
      }
      if (lane < 8) warp_sums[lane] = wi - w;  // exclusive
    }
    __syncthreads();
    uint32_t run = carry + warp_sums[warp] + (incl - s);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (idx0 + k < ntiles) row[idx0 + k] = run;
      run += v[k];
    }
    __syncthreads();
    if (threadIdx.x == 255) carry = run;
    __syncthreads();
  }
  if (threadIdx.x == 0) totals[blockIdx.x] = carry;
}

template <int kItems>
constexpr size_t down_smem() {
  return sizeof(uint32_t) * (kWarps * kRadix + 2 * (kWarps * 32 * kItems) + 3 * kRadix);
}

template <bool kIotaValues, int kItems>
__global__ void __launch_bounds__(kThreads) k_downsweep(const uint32_t* __restrict__ keys_in,
                                                         const uint32_t* __restrict__ vals_in,
                                                         uint32_t* __restrict__ keys_out,
                                                         uint32_t* __restrict__ vals_out, uint32_t n,
                                                         int shift, uint32_t ntiles,
                                                         const uint32_t* __restrict__ counts,
                                                         const uint32_t* __restrict__ totals) {
  constexpr int kItemsPerLane = kItems;
  constexpr int kWarpItems = 32 * kItems;
  constexpr int kTile = kWarps * kWarpItems;
  extern __shared__ uint32_t smem[];
  uint32_t* whist = smem;                                  // [kWarps][kRadix]
  uint32_t* skeys = whist + kWarps * kRadix;               // [kTile]
  uint32_t* svals = skeys + kTile;                         // [kTile]
  uint32_t* digit_off = svals + kTile;                     // [kRadix] tile-local digit offsets
  uint32_t* gbase = digit_off + kRadix;                    // [kRadix] global bases
  uint32_t* dbase = gbase + kRadix;                        // [kRadix] digit bases over all tiles

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int d = threadIdx.x; d < kWarps * kRadix; d += kThreads) whist[d] = 0;
  __syncthreads();

  const uint32_t tile_base = blockIdx.x * (uint32_t)kTile;
  const uint32_t seg_base = tile_base + warp * kWarpItems;
  uint32_t* wh = whist + warp * kRadix;
  uint32_t k[kItemsPerLane], v[kItemsPerLane];
  uint32_t local[kItemsPerLane];
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int r = 0; r < kItemsPerLane; ++r) {
    uint32_t i = seg_base + r * 32 + lane;
    bool valid = i < n;
    k[r] = valid ? keys_in[i] : 0xffffffffu;
    v[r] = valid ? (kIotaValues ? i : vals_in[i]) : 0u;
    uint32_t d = (k[r] >> shift) & (kRadix - 1);
    uint32_t vmask = __ballot_sync(0xffffffffu, valid);
    local[r] = 0;
    if (valid) {
      uint32_t peers = __match_any_sync(vmask, d);
      uint32_t rank = __popc(peers & lt);
      uint32_t prior = wh[d];
      local[r] = prior + rank;
      __syncwarp(vmask);
      if (rank == 0) wh[d] = prior + __popc(peers);
    }
    __syncwarp();
  }
  __syncthreads();
  // per digit: exclusive prefix over warps, and the tile's digit totals
  for (int d = threadIdx.x; d < kRadix; d += kThreads) {
    uint32_t acc = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      uint32_t t = whist[w * kRadix + d];
      whist[w * kRadix + d] = acc;
      acc += t;
    }
    digit_off[d] = acc;  // total for now
    gbase[d] = counts[(size_t)d * ntiles + blockIdx.x];
    dbase[d] = totals[d];
  }
  __syncthreads();
  // digit bases: exclusive scan of the 256 digit totals (warp 1, 8 per lane)
  if (warp == 1) {
    uint32_t t[8], s = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      t[q] = dbase[lane * 8 + q];
      s += t[q];
    }
    uint32_t incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    uint32_t run = incl - s;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      gbase[lane * 8 + q] += run;
      run += t[q];
    }
  }
  // the tile's digit offsets: exclusive scan of its 256 digit totals (warp 0)
  if (warp == 0) {
    uint32_t t[8], s = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      t[q] = digit_off[lane * 8 + q];
      s += t[q];
    }
    uint32_t incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    uint32_t run = incl - s;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      digit_off[lane * 8 + q] = run;
      run += t[q];
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kItemsPerLane; ++r) {
    uint32_t i = seg_base + r * 32 + lane;
    if (i < n) {
      uint32_t d = (k[r] >> shift) & (kRadix - 1);
      uint32_t pos = digit_off[d] + whist[warp * kRadix + d] + local[r];
      skeys[pos] = k[r];
      svals[pos] = v[r];
    }
  }
  __syncthreads();
  const uint32_t tile_n = (n - tile_base < (uint32_t)kTile) ? (n - tile_base) : (uint32_t)kTile;
  for (uint32_t i = threadIdx.x; i < tile_n; i += kThreads) {
    uint32_t key = skeys[i];
    uint32_t d = (key >> shift) & (kRadix - 1);
    uint32_t g = gbase[d] + (i - digit_off[d]);
    keys_out[g] = key;
    vals_out[g] = svals[i];
  }
}

}  // namespace

// scratch layout: keys_alt[pad64(n)] | vals_alt[pad64(n)] | counts[256 * tiles]
size_t radix_temp_words(uint32_t n) {
  size_t pad = ((size_t)n + 63) & ~size_t(63);
  return 2 * pad + radix_count_words(n);
}

size_t radix_temp_bytes(uint32_t n) { return radix_temp_words(n) * sizeof(uint32_t); }

// Opt the downsweep kernel into its 82 KB of dynamic shared memory on the
// current device, once per device (before any launch on it, and so before
// any stream capture that launches it).
cudaError_t radix_init() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  if (dev >= 0 && dev < 64 && done[dev]) return cudaSuccess;
  e = cudaFuncSetAttribute(k_downsweep<true, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)down_smem<16>());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_downsweep<false, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)down_smem<16>());
  if (e == cudaSuccess && dev >= 0 && dev < 64) done[dev] = true;
  return e;
}

cudaError_t radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt,
                             uint32_t* counts, uint32_t n, int key_bits, bool iota_values,
                             cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const uint32_t ntiles = radix_tiles(n);
  const uint32_t tile = radix_tile_keys(n);
  // the digit totals follow the [256][ntiles] counts
  uint32_t* totals = counts + (size_t)kRadix * ntiles;
  int passes = (key_bits + kRadixBits - 1) / kRadixBits;
  if (passes < 1) passes = 1;
  uint32_t *ki = keys, *vi = vals, *ko = keys_alt, *vo = vals_alt;
  for (int p = 0; p < passes; ++p) {
    int shift = p * kRadixBits;
    const bool iota = p == 0 && iota_values;
#define UPF_PASS(I)                                                                                          \
  k_upsweep<I><<<ntiles, kThreads, 0, st>>>(ki, n, shift, ntiles, counts);                                   \
  k_scan_rows<<<kRadix, 256, 0, st>>>(counts, ntiles, totals);                                               \
  if (iota)                                                                                                  \
    k_downsweep<true, I><<<ntiles, kThreads, down_smem<I>(), st>>>(ki, vi, ko, vo, n, shift, ntiles, counts,  \
                                                                    totals);                                  \
  else                                                                                                       \
    k_downsweep<false, I><<<ntiles, kThreads, down_smem<I>(), st>>>(ki, vi, ko, vo, n, shift, ntiles, counts, \
                                                                     totals);
    if (tile == 8192u) {
      UPF_PASS(16)
    } else if (tile == 2048u) {
      UPF_PASS(4)
    } else {
      UPF_PASS(1)
    }
#undef UPF_PASS
    uint32_t* t;
    t = ki; ki = ko; ko = t;
    t = vi; vi = vo; vo = t;
  }
  // an odd number of passes leaves the result in the alternate buffers
  if (passes & 1) {
    cudaError_t e = cudaMemcpyAsync(keys, ki, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(vals, vi, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

int radix_launches(int key_bits) {
  int passes = (key_bits + kRadixBits - 1) / kRadixBits;
  if (passes < 1) passes = 1;
  return 3 * passes;
}

// ---- Morton keys ------------------------------------------------------------
__global__ void k_morton_keys(const float4* __restrict__ pos, uint32_t n, float3 origin, float3 scales,
                              uint32_t* __restrict__ keys) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) keys[i] = morton_key(pos[i], origin, scales);
}

cudaError_t morton_keys(const float4* pos, uint32_t n, float3 origin, float3 scales, uint32_t* keys,
                        cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_morton_keys<<<(n + 255) / 256, 256, 0, st>>>(pos, n, origin, scales, keys);
  return cudaGetLastError();
}

// ---- cell ranges ------------------------------------------------------------
// ClearIndexArrays + CalculateBlocksKernel (src/gpu/particles_kernel.cu:656-726)
// become a boundary scan over the sorted keys: deterministic, no atomics.
__global__ void k_cell_ranges(const uint32_t* __restrict__ keys, uint32_t n, int shift, uint32_t ncells,
                              uint32_t* __restrict__ start, uint32_t* __restrict__ end) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t c = keys[i] >> shift;
  if (c >= ncells) return;
  if (i == 0 || (keys[i - 1] >> shift) != c) start[c] = i;
  if (i == n - 1 || (keys[i + 1] >> shift) != c) end[c] = i + 1;
}

cudaError_t cell_ranges(const uint32_t* keys, uint32_t n, int shift, uint32_t ncells, uint32_t* start,
                        uint32_t* end, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(start, 0, sizeof(uint32_t) * ncells, st);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(end, 0, sizeof(uint32_t) * ncells, st);
  if (e != cudaSuccess) return e;
  if (n == 0) return cudaSuccess;
  k_cell_ranges<<<(n + 255) / 256, 256, 0, st>>>(keys, n, shift, ncells, start, end);
  return cudaGetLastError();
}

}  // namespace upf
