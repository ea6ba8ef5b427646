// upf_pipeline.cu — the per-step kernels.
//
// Step = sort (Morton keys -> radix sort -> reorder -> cell ranges)
//      -> neighbour lists
//      -> WCSPH: density/pressure, then force + integration
//         PCISPH: external forces, then the predict-correct loop
//                 (predicted density + pressure update, pressure force +
//                 next prediction, loop control), then integration.
// Every kernel is one thread per particle over the sorted working set; the
// neighbour loops read the column-major lists, so a warp's list reads are
// coalesced and its position gathers hit the Morton-ordered neighbourhood in
// L1/L2.
//
// Reference kernels replaced (src/gpu/particles_kernel.cu):
//   FillZindicesKernel 3360, CopySortedParticleValuesKernel* 543-654,
//   ClearIndexArrays/CalculateBlocksKernel/RedistributeBlocks* 656-810,
//   CalculateDensitiesInBlocksKernelWCSPH 1529-1708,
//   CalculateForcesInBlocksKernelWCSPH 2399-2653,
//   CalculateExternalForcesInBlocksKernelPCISPH 3397-3621,
//   PredictPositionAndVelocityBlocksKernelPCISPH 3624-3660,
//   ComputePredictedDensityAndPressureBlocksKernelPCISPH 3662-3842,
//   ComputeCorrectivePressureForceBlocksKernelPCISPH 4034-4211,
//   ReduceMax + GetReductionFinalMax (particles.cu:2840-2932, kernel.cu:3381),
//   TimeIntegrationBlocksKernelPCISPHPureFluid 5033-5104.
// The arithmetic follows the reference's CPU path (src/cpu/UnifiedPhysics.cpp),
// which is the parity target; each kernel cites the function it restates.
#include <cuda_runtime.h>

#include "upf_sys.h"
#include "upf_tma.cuh"

namespace upf {

namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ float mx0(float a, float b) { return (a >= b) ? a : b; }  // MAX macro

__device__ __forceinline__ float lut_at(const float* s, float d, float factor) {
  int idx = lut_index(d, factor);
  return idx >= kLut ? 0.0f : s[idx];
}

__device__ __forceinline__ void stage_lut(float* dst, const float* __restrict__ src) {
  for (int k = threadIdx.x; k < UPF_LUT_ENTRIES; k += blockDim.x) dst[k] = src[k];
}

__device__ __forceinline__ float4 f4(float x, float y, float z) { return make_float4(x, y, z, 0.0f); }

// Neighbour loop with memory-level parallelism: the list entries of a batch
// of kUnroll neighbours are loaded together, then their gathers, then the
// arithmetic runs in list order (so floating-point sums keep the reference's
// sequential order). `load(code)` gathers a neighbour's data, `use(code, v)`
// accumulates it.
constexpr int kUnroll = 8;
// The external-force pass gathers 36 bytes per neighbour (position,
// velocity, type): batches of 2 hold it to 64 registers a thread (batches of
// 8 took 128, a quarter of the SM's warps resident), which measured 0.24
// against 0.38-0.45 ms per launch on the 1M dam.
constexpr int kExternalUnroll = 2;
// The list build gathers candidate positions 4 at a time: 40 registers a
// thread against 56 with 8 (1.22 against 1.35 ms per build on the 1M dam).
constexpr int kNlistUnroll = 4;

template <int kU = kUnroll, class Load, class Use>
__device__ __forceinline__ void for_neighbors(const uint32_t* __restrict__ col, uint32_t stride, uint32_t cnt,
                                              Load&& load, Use&& use) {
  using T = decltype(load(0u));
  uint32_t k = 0;
  for (; k + kU <= cnt; k += kU) {
    uint32_t code[kU];
    T v[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) code[u] = __ldg(col + (size_t)(k + u) * stride);
#pragma unroll
    for (int u = 0; u < kU; ++u) v[u] = load(code[u]);
#pragma unroll
    for (int u = 0; u < kU; ++u) use(code[u], v[u]);
  }
  if (k < cnt) {
    uint32_t code[kU];
    T v[kU];
    const uint32_t rem = cnt - k;
#pragma unroll
    for (int u = 0; u < kU; ++u)
      if (u < rem) code[u] = __ldg(col + (size_t)(k + u) * stride);
#pragma unroll
    for (int u = 0; u < kU; ++u)
      if (u < rem) v[u] = load(code[u]);
#pragma unroll
    for (int u = 0; u < kU; ++u)
      if (u < rem) use(code[u], v[u]);
  }
}

// The same, also handing each entry's stored list value (the kernel-table
// bin, in the WCSPH passes) to `use`.
template <class Load, class Use>
__device__ __forceinline__ void for_neighbors_bin(const uint32_t* __restrict__ col, const uint32_t* __restrict__ bcol,
                                                  uint32_t stride, uint32_t cnt, Load&& load, Use&& use) {
  using T = decltype(load(0u));
  uint32_t k = 0;
  for (; k + kUnroll <= cnt; k += kUnroll) {
    uint32_t code[kUnroll];
    uint32_t bin[kUnroll];
    T v[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      code[u] = __ldg(col + (size_t)(k + u) * stride);
      bin[u] = __ldg(bcol + (size_t)(k + u) * stride);
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) v[u] = load(code[u]);
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) use(code[u], bin[u], v[u]);
  }
  for (; k < cnt; ++k) {
    const uint32_t code = __ldg(col + (size_t)k * stride);
    const uint32_t bin = __ldg(bcol + (size_t)k * stride);
    use(code, bin, load(code));
  }
}

struct PosP {
  float4 x;
  float p;
};

// What a CTA works on: one system (plain launch) or, in a batched launch,
// the scene its slots belong to (BatchView). Batched CTAs copy the scene's
// parameters to shared memory; `end` bounds the particle index.
struct Scope {
  const DevParams* P;
  const float* luts;
  DevState* st;
  uint32_t end;
  uint32_t scene;
  bool skip;  // a loop pass of a scene whose loop has finished
};

// batched scenes: the key of a padding slot (above every 30-bit Morton key)
constexpr uint32_t kPadKeyBatch = 1u << 30;

// The scope of virtual block `block` (blockIdx.x, or a group taken from a
// list of work by a resident grid).
template <bool kBatch>
__device__ __forceinline__ Scope enter_scope_at(uint32_t block, const DevParams& Pk, const float* luts, DevState* st,
                                                uint32_t n, const BatchView& bv, DevParams* sP, bool loop_pass) {
  if constexpr (!kBatch) {
    return Scope{&Pk, luts, st, n, 0u, false};
  } else {
    const uint32_t s = bv.group_scene[(block * blockDim.x) / kSegAlign];
    const uint32_t* src = reinterpret_cast<const uint32_t*>(bv.params + s);
    for (uint32_t k = threadIdx.x; k < sizeof(DevParams) / 4; k += blockDim.x)
      reinterpret_cast<uint32_t*>(sP)[k] = src[k];
    DevState* sst = bv.st + s;
    const bool skip = loop_pass && !*reinterpret_cast<volatile int32_t*>(&sst->loop_active);
    return Scope{sP, bv.luts + (size_t)s * kLutFloats, sst, bv.seg_end[s], s, skip};
  }
}

template <bool kBatch>
__device__ __forceinline__ Scope enter_scope(const DevParams& Pk, const float* luts, DevState* st, uint32_t n,
                                             const BatchView& bv, DevParams* sP, bool loop_pass) {
  return enter_scope_at<kBatch>(blockIdx.x, Pk, luts, st, n, bv, sP, loop_pass);
}

// The list walk of the loop passes, in one of two modes:
//  * TMA ring (kDirect = false): each warp streams its 32 columns' list rows
//    through a shared-memory ring of kRows-row stages (upf_tma.cuh), waits on
//    the stage's mbarrier, and hands the rows to `body`;
//  * direct loads (kDirect = true): each thread loads its own list entries
//    kRows at a time with coalesced global loads (consecutive threads read
//    consecutive words of a row) and no barriers.
// body(code, val, k0) consumes entries k0 .. k0 + kRows - 1 (those below
// the thread's count); code(r) / val(r) give entry k0 + r and its list
// value (read from the shared-memory stage when it is used, in the ring
// mode). Returns false if a ring wait ran out.
struct ListArgs {
  const CUtensorMap* cmap;
  const CUtensorMap* vmap;
  const uint32_t* nbr;
  const uint32_t* vals;
  uint32_t stride;
};

template <bool kDirect, bool kWithVals, int kThreads, int kRows, class Body>
__device__ __forceinline__ bool walk_lists(const ListArgs& L, uint32_t block, uint32_t i, uint32_t cnt, Body&& body) {
  if constexpr (kDirect) {
    const uint32_t* __restrict__ col = L.nbr + i;
    const uint32_t* __restrict__ vcol = L.vals + i;
    for (uint32_t k0 = 0; k0 < cnt; k0 += kRows) {
      uint32_t code[kRows], val[kRows];
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        if (k0 + r < cnt) {
          code[r] = __ldg(col + (size_t)(k0 + r) * L.stride);
          if (kWithVals) val[r] = __ldg(vcol + (size_t)(k0 + r) * L.stride);
        }
      }
      body([&](int r) { return code[r]; }, [&](int r) { return val[r]; }, (int)k0);
    }
    return true;
  } else {
    __shared__ WarpListRing<kWithVals, kRows> rings[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    WarpListRing<kWithVals, kRows>& ring = rings[warp];
    ring_init(ring);
    const uint32_t wcnt = __reduce_max_sync(0xffffffffu, cnt);
    return ring_walk(ring, L.cmap, L.vmap, (int)(block * blockDim.x + warp * 32), wcnt, [&](int s, int k0) {
      body([&](int r) { return ring.codes[s][r][lane]; }, [&](int r) { return ring.vals[s][r][lane]; }, k0);
    });
  }
}

// ---------------------------------------------------------------- reorder
// CopySortedParticleValuesKernel* (particles_kernel.cu:543-654): gather the
// state into sorted order.
__global__ void __launch_bounds__(kBlock) k_reorder(uint32_t n, const uint32_t* __restrict__ perm,
                                                     DynArrays A, DynArrays B, bool with_lag) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t j = perm[i];
  B.pos[i] = A.pos[j];
  B.vel[i] = A.vel[j];
  B.id[i] = A.id[j];
  B.type[i] = A.type[j];
  if (with_lag) B.lag[i] = A.lag[j];
}

// ---------------------------------------------------------------- neighbours
// Squared distance with the rounding of dist3 (no sqrt).
__device__ __forceinline__ float dist2(float4 a, float4 b) {
  float dx = fsub(a.x, b.x), dy = fsub(a.y, b.y), dz = fsub(a.z, b.z);
  return fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz));
}
// The same with x and y as one packed pair (axy = pk2(a.x, a.y)): the same
// operations, the same roundings.
__device__ __forceinline__ float dist2_xy(unsigned long long axy, float az, float4 b) {
  const float2 s = up2(mul2(sub2(axy, pk2(b.x, b.y)), sub2(axy, pk2(b.x, b.y))));
  const float dz = fsub(az, b.z);
  return fadd(fadd(s.x, s.y), fmul(dz, dz));
}

// GetNeighbors (UnifiedPhysics.cpp:2242-2280) with ZIndex::BoxQuery
// (zIndex.cpp:43-73), one thread per particle: candidates are the search
// cells (aligned Morton blocks of 2^cell_shift grid units, at most the
// reference's block size) covering the query box with a one-grid-unit
// margin. Every particle within h lies in the reference's query box, hence in
// these cells, so the candidate set holds all of the reference's
// neighbours. Cells are visited in ascending Morton order, each a contiguous
// key range; within a cell the dynamic and boundary ranges are merged by
// key. The list therefore comes out in the reference's ascending
// sorted-index order, and membership is the reference's exact test: j != i
// and |x_i - x_j| < h in float. Candidate positions are gathered kNlistUnroll at
// a time. Each entry also records a list value at the current positions:
// its kernel-table bin (WCSPH: the density and force passes read their
// tables by it), or the pressure-gradient table's value at that bin
// (PCISPH: the pressure-force pass, which evaluates at the current
// positions, then reads no table).
//
// kWarpUnion: the 32 lanes of a warp (32 consecutive Morton-sorted particles,
// close together) walk the union of their query boxes, when it spans at
// most 64 cells, instead of each lane its own box: every lane then visits
// the same cells and candidates in the same order (no divergence; each
// candidate position is one broadcast load) and keeps those within h of its
// own particle. A lane's list is unchanged: all its neighbours lie in its own
// box, a subset of the union, and the union's cells are still visited in
// ascending Morton order.
template <bool kBatch, int kThreads, bool kWarpUnion>
__global__ void __launch_bounds__(kThreads) k_build_nlist(
    const __grid_constant__ DevParams Pk, const BatchView bv, uint32_t n, const float4* __restrict__ pos,
    const uint32_t* __restrict__ keys, const uint32_t* __restrict__ cstart, const uint32_t* __restrict__ cend,
    uint32_t ns, const float4* __restrict__ spos, const uint32_t* __restrict__ skeys,
    const uint32_t* __restrict__ sstart, const uint32_t* __restrict__ send, uint32_t* __restrict__ nbr,
    uint32_t* __restrict__ lval, uint32_t* __restrict__ ncnt, const float* __restrict__ luts,
    DevState* __restrict__ st_plain) {
  __shared__ DevParams sP;
  __shared__ float thr[kThresholds];
  __shared__ float pg[UPF_LUT_ENTRIES];
  const Scope sc = enter_scope<kBatch>(Pk, luts, st_plain, n, bv, &sP, false);
  for (int k = threadIdx.x; k < kThresholds; k += blockDim.x) thr[k] = sc.luts[5 * UPF_LUT_ENTRIES + k];
  stage_lut(pg, sc.luts + LUT_PGRAD * UPF_LUT_ENTRIES);
  __syncthreads();
  const DevParams& P = *sc.P;
  DevState* st = sc.st;
  if (kBatch) {
    // the scene's own cell table (keys are the scene's Morton keys)
    cstart += bv.cell_base[sc.scene];
    cend += bv.cell_base[sc.scene];
  }
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = i < sc.end;
  if (!kWarpUnion && !active) return;
  if (kWarpUnion && !__any_sync(0xffffffffu, active)) return;  // uniform over the warp
  const float4 xi = active ? pos[i] : make_float4(0, 0, 0, 0);
  const float h = P.h;
  int lo[3], hi[3];
  float cg[3];  // the particle's grid position, clamped to the grid as keys are
  {
    const float c[3] = {(xi.x - P.origin.x) * P.scales.x, (xi.y - P.origin.y) * P.scales.y,
                        (xi.z - P.origin.z) * P.scales.z};
    const float r[3] = {h * P.scales.x, h * P.scales.y, h * P.scales.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float l = c[a] - r[a] - 1.0f, u = c[a] + r[a] + 1.0f;
      int li = (l <= 0.0f) ? 0 : (l >= 1023.0f ? 1023 : (int)l);
      int ui = (u <= 0.0f) ? 0 : (u >= 1023.0f ? 1023 : (int)u);
      lo[a] = li >> P.cell_shift;
      hi[a] = ui >> P.cell_shift;
      cg[a] = fminf(fmaxf(c[a], 0.0f), 1024.0f);
    }
  }
  // Cells of the query box whose nearest point lies farther than h from the
  // particle hold no neighbour and are skipped. A particle's key cell holds
  // its clamped grid position to within float rounding, so the cell's box is
  // widened by one grid unit; clamping shortens no distance, and h^2 gets
  // a 1e-5 relative margin: the test only drops cells that cannot hold a
  // particle within h. Lanes that walk the warp's union of boxes skip none.
  const int cs = 1 << P.cell_shift;
  const float cull_h2 = h * h * 1.00001f;
  bool cull = !kWarpUnion;
  auto may_hold = [&](int bx, int by, int bz) {
    if (!cull) return true;
    const int b[3] = {bx, by, bz};
    const float sc[3] = {P.scales.x, P.scales.y, P.scales.z};
    float s = 0.0f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float blo = (float)(b[a] * cs) - 1.0f, bhi = (float)((b[a] + 1) * cs) + 1.0f;
      const float d = fmaxf(0.0f, fmaxf(blo - cg[a], cg[a] - bhi)) / sc[a];
      s += d * d;
    }
    return s <= cull_h2;
  };
  if (kWarpUnion) {
    int ulo[3], uhi[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      ulo[a] = __reduce_min_sync(0xffffffffu, active ? lo[a] : 0x7fffffff);
      uhi[a] = __reduce_max_sync(0xffffffffu, active ? hi[a] : -1);
    }
    if ((uhi[0] - ulo[0] + 1) * (uhi[1] - ulo[1] + 1) * (uhi[2] - ulo[2] + 1) <= 64) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        lo[a] = ulo[a];
        hi[a] = uhi[a];
      }
    }
  }
  const uint32_t maxn = P.maxn, stride = P.nstride;
  uint32_t cnt = 0;
  uint32_t* __restrict__ out = nbr + i;
  uint32_t* __restrict__ ov = lval + i;
  const bool grad = P.list_grad != 0;
  // An append stores the entry and its squared distance; the list value
  // (bin_of_r2 and the table) follows in one pass over the finished list,
  // where the lanes of a warp run together instead of one append at a time.
  auto append = [&](uint32_t code, float r2) {
    if (!active) return;
    if (cnt < maxn) {
      out[(size_t)cnt * stride] = code;
      ov[(size_t)cnt * stride] = __float_as_uint(r2);
    }
    cnt++;
  };
  // one contiguous range of one set; `base` turns a set index into a
  // neighbour index (0 for dynamic, static_base for boundary particles)
  auto scan_range = [&](const float4* __restrict__ set, uint32_t b, uint32_t e, uint32_t base, bool skip_self) {
    for (; b + kNlistUnroll <= e; b += kNlistUnroll) {
      float4 xj[kNlistUnroll];
#pragma unroll
      for (int u = 0; u < kNlistUnroll; ++u) xj[u] = __ldg(set + b + u);
#pragma unroll
      for (int u = 0; u < kNlistUnroll; ++u) {
        const uint32_t j = b + u;
        const float r2 = dist2(xi, xj[u]);
        if (!(skip_self && j == i) && r2 < thr[kThresholds - 1]) append(j + base, r2);
      }
    }
    for (; b < e; ++b) {
      const float r2 = dist2(xi, __ldg(set + b));
      if (!(skip_self && b == i) && r2 < thr[kThresholds - 1]) append(b + base, r2);
    }
  };
  auto visit = [&](uint32_t c) {
    uint32_t ds = cstart[c], de = cend[c];
    uint32_t ss = 0, se = 0;
    if (ns) {
      ss = sstart[c];
      se = send[c];
    }
    if (ss == se) {
      scan_range(pos, ds, de, 0u, true);
      return;
    }
    if (ds == de) {
      scan_range(spos, ss, se, P.static_base, false);
      return;
    }
    while (ds < de || ss < se) {  // both sets present: merge by key
      bool take_dyn = (ds < de) && (ss >= se || keys[ds] <= skeys[ss]);
      if (take_dyn) {
        uint32_t j = ds++;
        const float r2 = dist2(xi, pos[j]);
        if (j != i && r2 < thr[kThresholds - 1]) append(j, r2);
      } else {
        uint32_t j = ss++;
        const float r2 = dist2(xi, spos[j]);
        if (r2 < thr[kThresholds - 1]) append(j + P.static_base, r2);
      }
    }
  };
  const int nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1, nz = hi[2] - lo[2] + 1;
  const int nblk = nx * ny * nz;
  if (nblk <= 64) {
    uint32_t codes[64];
    int m = 0;
    for (int bz = lo[2]; bz <= hi[2]; ++bz)
      for (int by = lo[1]; by <= hi[1]; ++by)
        for (int bx = lo[0]; bx <= hi[0]; ++bx) {
          if (!may_hold(bx, by, bz)) continue;
          uint32_t c = morton3(bx, by, bz);
          int q = m++;
          while (q > 0 && codes[q - 1] > c) {
            codes[q] = codes[q - 1];
            --q;
          }
          codes[q] = c;
        }
    for (int q = 0; q < m; ++q) visit(codes[q]);
  } else {
    for (int bz = lo[2]; bz <= hi[2]; ++bz)
      for (int by = lo[1]; by <= hi[1]; ++by)
        for (int bx = lo[0]; bx <= hi[0]; ++bx)
          if (may_hold(bx, by, bz)) visit(morton3(bx, by, bz));
  }
  if (!active) return;
  const uint32_t m = cnt < maxn ? cnt : maxn;
  // the list values at the entries' squared distances, four entries' loads
  // in flight at a time
  uint32_t k = 0;
  for (; k + 4 <= m; k += 4) {
    float r2[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) r2[u] = __uint_as_float(ov[(size_t)(k + u) * stride]);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int bin = bin_of_r2(r2[u], P.lut_factor, thr);
      ov[(size_t)(k + u) * stride] = grad ? __float_as_uint(pg[bin]) : (uint32_t)bin;
    }
  }
  for (; k < m; ++k) {
    const int bin = bin_of_r2(__uint_as_float(ov[(size_t)k * stride]), P.lut_factor, thr);
    ov[(size_t)k * stride] = grad ? __float_as_uint(pg[bin]) : (uint32_t)bin;
  }
  ncnt[i] = m;
  if (cnt > maxn) atomicOr(&st->error_flags, (uint32_t)ERR_OVERFLOW);
  atomicMax(&st->max_neighbors, cnt);
}

// ---------------------------------------------------------------- WCSPH
// DistanceToWall (UnifiedPhysics.cpp:5926-5990) and WallWeight (6032-6060)
__device__ float wall_weight(const DevParams& P, const float* m4, float4 x) {
  const float L = P.wmax.x - P.wmin.x, H = P.wmax.y - P.wmin.y, W = P.wmax.z - P.wmin.z;
  float res = mx0(L, mx0(H, W));
  float d;
  d = mx0(x.y - P.wmin.y, 0.0f); res = (res <= d) ? res : d;
  d = mx0(P.wmax.y - x.y, 0.0f); res = (res <= d) ? res : d;
  d = mx0(x.x - P.wmin.x, 0.0f); res = (res <= d) ? res : d;
  d = mx0(P.wmax.x - x.x, 0.0f); res = (res <= d) ? res : d;
  d = mx0(x.z - P.wmin.z, 0.0f); res = (res <= d) ? res : d;
  d = mx0(P.wmax.z - x.z, 0.0f); res = (res <= d) ? res : d;
  const float eff = P.h - P.radius;
  if (res >= eff) return 0.0f;
  const float s = P.spacing;
  float d1 = res + P.radius;
  float d2 = d1 + s;
  float d3 = sqrtf(d1 * d1 + s * s);
  float d4 = sqrtf(d1 * d1 + (s * 2) * (s * 2));
  float d5 = sqrtf(d2 * d2 + s * s);
  float d6 = sqrtf(d2 * d2 + (s * 2) * (s * 2));
  float k1 = lut_at(m4, d1, P.lut_factor), k2 = lut_at(m4, d2, P.lut_factor),
        k3 = lut_at(m4, d3, P.lut_factor), k4 = lut_at(m4, d4, P.lut_factor),
        k5 = lut_at(m4, d5, P.lut_factor), k6 = lut_at(m4, d6, P.lut_factor);
  return P.mass * (k1 + k2 + 2 * (k3 + k4 + k5 + k6));
}

// CalculateDensityPressurePureFluidSPH + CalculatePressureWCSPH
// (UnifiedPhysics.cpp:2408-2501), liquid particles.
__global__ void __launch_bounds__(kBlock) k_wcsph_density(
    DevParams P, uint32_t n, const float4* __restrict__ pos, const int32_t* __restrict__ type,
    const uint32_t* __restrict__ lval, const uint32_t* __restrict__ ncnt, const float* __restrict__ luts,
    float* __restrict__ rho, float* __restrict__ press) {
  __shared__ float m4[UPF_LUT_ENTRIES];
  stage_lut(m4, luts + LUT_M4 * UPF_LUT_ENTRIES);
  __syncthreads();
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (type[i] != UPF_LIQUID) return;
  const float4 xi = pos[i];
  const float m = P.mass;
  float den = P.kernel_self * m;
  // densities at the positions the list was built at: every entry is within
  // h and carries its kernel-table bin, so only the bins are read (list values)
  const uint32_t* __restrict__ b = lval + i;
  const uint32_t c = ncnt[i];
  uint32_t k = 0;
  for (; k + kUnroll <= c; k += kUnroll) {
    uint32_t bb[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) bb[u] = __ldg(b + (size_t)(k + u) * P.nstride);
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) den += m4[bb[u]] * m;
  }
  for (; k < c; ++k) den += m4[__ldg(b + (size_t)k * P.nstride)] * m;
  if (P.flags & UPF_FLAG_WALL_WEIGHT) den += wall_weight(P, m4, xi);
  const float frac = den / P.rho0;
  // pow(float, float) of the reference's host build is glibc powf, which
  // evaluates in double and rounds once; the double pow rounded to float
  // gives the same float (CUDA's single-precision powf may differ by ulps,
  // which the stiff Tait equation amplifies over many steps)
  const float powg = (float)pow((double)frac, (double)P.gamma);
  const float pr = P.gas_b * (powg - 1.0f);
  rho[i] = den;
  press[i] = (0.0f >= pr) ? 0.0f : pr;
}

// WeightingKernel::kernelSplineSurfaceTension (WeightingKernel.cpp:210-231)
__device__ float cohesion_spline(float dist, float sr) {
  const float c = 32.0f / ((3.14159274f * sr * sr * sr * sr * sr * sr * sr * sr * sr));
  if (dist > 0.5 * sr && dist <= sr) return c * (sr - dist) * (sr - dist) * (sr - dist) * dist * dist * dist;
  if (dist > 0 && dist <= 0.5 * sr)
    return c * (2.0f * (sr - dist) * (sr - dist) * (sr - dist) * dist * dist * dist -
                sr * sr * sr * sr * sr * sr / 64.0f);
  return 0.0f;
}

// BoundaryHandlingBoxPerNonRigidParticle (UnifiedPhysics.cpp:4000-4044)
__device__ __forceinline__ void clamp_box(const DevParams& P, float4& x, float4& v, float damping) {
  if (x.y < P.cmin.y) { x.y = P.cmin.y; v.y *= damping; }
  if (x.y > P.cmax.y) { x.y = P.cmax.y; v.y *= damping; }
  if (x.x < P.cmin.x) { x.x = P.cmin.x; v.x *= damping; }
  if (x.x > P.cmax.x) { x.x = P.cmax.x; v.x *= damping; }
  if (x.z < P.cmin.z) { x.z = P.cmin.z; v.z *= damping; }
  if (x.z > P.cmax.z) { x.z = P.cmax.z; v.z *= damping; }
}

__device__ __forceinline__ void block_stats(DevState* st, double ke, double mx, double my, double mz) {
  __shared__ double red[4][kBlock / 32];
  ke = warp_sum(ke);
  mx = warp_sum(mx);
  my = warp_sum(my);
  mz = warp_sum(mz);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][w] = ke; red[1][w] = mx; red[2][w] = my; red[3][w] = mz;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0, c = 0, d = 0;
    for (int k = 0; k < (int)(blockDim.x / 32); ++k) {
      a += red[0][k]; b += red[1][k]; c += red[2][k]; d += red[3][k];
    }
    atomicAdd(&st->ke, a);
    atomicAdd(&st->mom[0], b);
    atomicAdd(&st->mom[1], c);
    atomicAdd(&st->mom[2], d);
  }
}

// UpdateLiquidParticlePosVelSphCPU (UnifiedPhysics.cpp:3705-3742) + boundary
// handling with damping -0.5 + new key (UnifiedPhysics.cpp:3972-3998):
// writes the A copy.
__device__ __forceinline__ void integrate_store(const DevParams& P, uint32_t i, float4 x, float4 v, float3 F,
                                                DynArrays& A, uint32_t* keysA, const DynArrays& B,
                                                double& ke, double& mx, double& my, double& mz) {
  v.x = v.x + F.x * P.inv_mass * P.dt;
  v.y = v.y + F.y * P.inv_mass * P.dt;
  v.z = v.z + F.z * P.inv_mass * P.dt;
  x.x = x.x + v.x * P.dt;
  x.y = x.y + v.y * P.dt;
  x.z = x.z + v.z * P.dt;
  clamp_box(P, x, v, -0.5f);
  A.pos[i] = x;
  A.vel[i] = v;
  keysA[i] = morton_key(x, P.origin, P.scales);
  const double m = P.mass;
  ke = 0.5 * m * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
  mx = m * v.x;
  my = m * v.y;
  mz = m * v.z;
  if (isnan(x.x) || isnan(x.y) || isnan(x.z)) ke = nan("");
}

// CalculateLiquidParticleForces (UnifiedPhysics.cpp:3009-3083) + gravity +
// integration (the reference's GPU path fuses these too,
// CalculateForcesInBlocksKernelWCSPH particles_kernel.cu:2399-2653).
__global__ void __launch_bounds__(kBlock) k_wcsph_force_integrate(
    DevParams P, uint32_t n, DynArrays B, DynArrays A, uint32_t* __restrict__ keysA,
    const uint32_t* __restrict__ nbr, const uint32_t* __restrict__ lval, const uint32_t* __restrict__ ncnt,
    const float* __restrict__ luts, const float* __restrict__ rho, const float* __restrict__ press,
    float4* __restrict__ force, DevState* __restrict__ st) {
  __shared__ float pg[UPF_LUT_ENTRIES], vl[UPF_LUT_ENTRIES];
  stage_lut(pg, luts + LUT_PGRAD * UPF_LUT_ENTRIES);
  stage_lut(vl, luts + LUT_VISC * UPF_LUT_ENTRIES);
  __syncthreads();
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  double ke = 0, mx = 0, my = 0, mz = 0;
  if (i < n) {
    const int32_t ti = B.type[i];
    float4 xi = B.pos[i], vi = B.vel[i];
    if (ti == UPF_LIQUID) {
      const float m = P.mass, h = P.h;
      const float di = rho[i], pi = press[i];
      const float invD = (float)(1.0 / (double)di);
      const float pVol = m * invD;
      float fx = 0, fy = 0, fz = 0;
      struct WNb {
        float4 x, v;
        float d, p;
        int32_t t;
      };
      const float4* __restrict__ bpos = B.pos;
      const float4* __restrict__ bvel = B.vel;
      const int32_t* __restrict__ btype = B.type;
      // positions are those the list was built at: entries are within h and
      // carry their kernel-table bin
      for_neighbors_bin(
          nbr + i, lval + i, P.nstride, ncnt[i],
          [&](uint32_t code) {
            WNb s;
            // boundary particles (array tails) are FROZEN and skipped below
            s.t = __ldg(btype + code);
            s.x = __ldg(bpos + code);
            s.v = __ldg(bvel + code);
            s.d = __ldg(rho + code);
            s.p = __ldg(press + code);
            return s;
          },
          [&](uint32_t, uint32_t bin, const WNb& s) {
        if (s.t != UPF_LIQUID) return;
        const float4 xj = s.x;
        const float kv = vl[bin];
        const float dj = s.d, pj = s.p;
        const float nVol = m / dj;
        const float dvx = xi.x - xj.x, dvy = xi.y - xj.y, dvz = xi.z - xj.z;
        const float g = pg[bin];
        const float grad = pi * invD * invD + pj / (dj * dj);
        fx = fx - dvx * g * grad * m * m;
        fy = fy - dvy * g * grad * m * m;
        fz = fz - dvz * g * grad * m * m;
        const float4 vj = s.v;
        const float vx = vi.x - vj.x, vy = vi.y - vj.y, vz = vi.z - vj.z;
        fx = fx - vx * pVol * nVol * P.visc * kv;
        fy = fy - vy * pVol * nVol * P.visc * kv;
        fz = fz - vz * pVol * nVol * P.visc * kv;
        if (P.flags & UPF_FLAG_SURFACE_TENSION) {
          const float d = dist3(xi, xj);
          if (!(d >= h * 0.25f)) return;
          const float sp = cohesion_spline(d, h);
          const float inv = 1.0f / d;
          fx = fx - dvx * P.st_gamma * m * m * sp * inv;
          fy = fy - dvy * P.st_gamma * m * m * sp * inv;
          fz = fz - dvz * P.st_gamma * m * m * sp * inv;
        }
          });
      fy -= m * P.gravity;
      force[i] = f4(fx, fy, fz);
      integrate_store(P, i, xi, vi, make_float3(fx, fy, fz), A, keysA, B, ke, mx, my, mz);
    } else {
      A.pos[i] = xi;
      A.vel[i] = vi;
      keysA[i] = morton_key(xi, P.origin, P.scales);
      force[i] = f4(0, 0, 0);
    }
    A.id[i] = B.id[i];
    A.type[i] = ti;
  }
  if (!(ke == ke)) {
    atomicOr(&st->error_flags, (uint32_t)ERR_NAN);
    ke = 0;
  }
  block_stats(st, ke, mx, my, mz);
}

// ---------------------------------------------------------------- PCISPH
// CalculateBoundaryForcePerLiquidParticleHost (UnifiedPhysics.cpp:2032-2069):
// the scalar is evaluated in double because of the 2.0 literal.
__device__ __forceinline__ float wall_term(float t, const DevParams& P) {
  return (float)((double)(t * P.inv_force_dist) * 2.0 * (double)P.max_boundary_force);
}

__device__ __forceinline__ void penalty_walls(const DevParams& P, float4 x, float& fx, float& fy, float& fz) {
  const float fd = P.force_dist;
  if (x.x < P.cmin.x + fd) fx += wall_term(P.cmin.x + fd - x.x, P);
  if (x.x > P.cmax.x - fd) fx += -1.0f * wall_term(x.x + fd - P.cmax.x, P);
  if (x.y < P.cmin.y + fd) fy += wall_term(P.cmin.y + fd - x.y, P);
  if (x.y > P.cmax.y - fd) fy += -1.0f * wall_term(x.y + fd - P.cmax.y, P);
  if (x.z < P.cmin.z + fd) fz += wall_term(P.cmin.z + fd - x.z, P);
  if (x.z > P.cmax.z - fd) fz += -1.0f * wall_term(x.z + fd - P.cmax.z, P);
}

// PredictPositionAndVelocity + CollisionHandling (UnifiedPhysics.cpp:5426-5454, 5739-5757)
__device__ __forceinline__ float4 predict(const DevParams& P, float4 x, float4 v, float3 F, float3 Fp,
                                          bool& bad) {
  const float inv = 1.0f / P.mass;  // vmml: vector / scalar multiplies by the reciprocal
  float vx = v.x + (F.x + Fp.x) * P.dt * inv;
  float vy = v.y + (F.y + Fp.y) * P.dt * inv;
  float vz = v.z + (F.z + Fp.z) * P.dt * inv;
  float4 xs = make_float4(x.x + vx * P.dt, x.y + vy * P.dt, x.z + vz * P.dt, 0.0f);
  if (xs.x < P.cmin.x) xs.x = P.cmin.x;
  if (xs.x > P.cmax.x) xs.x = P.cmax.x;
  if (xs.y < P.cmin.y) xs.y = P.cmin.y;
  if (xs.y > P.cmax.y) xs.y = P.cmax.y;
  if (xs.z < P.cmin.z) xs.z = P.cmin.z;
  if (xs.z > P.cmax.z) xs.z = P.cmax.z;
  bad = isnan(xs.x) || isnan(xs.y) || isnan(xs.z);
  return xs;
}

// CalculateBoundaryFluidPressureForceHost (UnifiedPhysics.cpp:4240-4250),
// indexed by distance; lagged pressure and predicted density of the liquid
// particle, Akinci volume of the boundary particle.
__device__ __forceinline__ void boundary_pressure(const DevParams& P, const float* pg, float d, float4 xi,
                                                  float4 xj, float rho_prev, float p_prev, float wvol,
                                                  float& fx, float& fy, float& fz) {
  const float inv_den = 1.0f / rho_prev;
  const float g = lut_at(pg, d, P.lut_factor);
  const float kx = (xi.x - xj.x) * g, ky = (xi.y - xj.y) * g, kz = (xi.z - xj.z) * g;
  const float pgd = p_prev * inv_den * inv_den;
  fx = fx + kx * pgd * P.mass * P.rho0 * wvol * (-1.0f);
  fy = fy + ky * pgd * P.mass * P.rho0 * wvol * (-1.0f);
  fz = fz + kz * pgd * P.mass * P.rho0 * wvol * (-1.0f);
}

// The reaction of boundary_pressure on the solid particle: the same vector as
// the liquid particle receives, subtracted (the pair force is antisymmetric).
__device__ __forceinline__ void boundary_pressure_reaction(const DevParams& P, const float* pg, float d,
                                                           float4 xl, float4 xs_, float rho_prev, float p_prev,
                                                           float wvol, float& fx, float& fy, float& fz) {
  const float inv_den = 1.0f / rho_prev;
  const float g = lut_at(pg, d, P.lut_factor);
  const float kx = (xl.x - xs_.x) * g, ky = (xl.y - xs_.y) * g, kz = (xl.z - xs_.z) * g;
  const float pgd = p_prev * inv_den * inv_den;
  fx = fx - kx * pgd * P.mass * P.rho0 * wvol * (-1.0f);
  fy = fy - ky * pgd * P.mass * P.rho0 * wvol * (-1.0f);
  fz = fz - kz * pgd * P.mass * P.rho0 * wvol * (-1.0f);
}

// CalculateBoundaryForcePerRigidParticleHost (UnifiedPhysics.cpp:2071-2131):
// spring against each box face the particle's sphere crosses, damping once if
// any face is hit; added to the force as one vector.
__device__ __forceinline__ void rigid_box_force(const DevParams& P, float4 x, float4 v, float& fx, float& fy,
                                                float& fz) {
  const float r = P.radius, ks = P.spring_boundary, kd = P.damping;
  float f[3] = {0.0f, 0.0f, 0.0f};
  const float xv[3] = {x.x, x.y, x.z};
  const float mn[3] = {P.cmin.x, P.cmin.y, P.cmin.z}, mx[3] = {P.cmax.x, P.cmax.y, P.cmax.z};
  bool hit = false;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (xv[a] - r < mn[a]) {
      hit = true;
      f[a] += (mn[a] + r - xv[a]) * ks;
    }
    if (xv[a] + r > mx[a]) {
      hit = true;
      f[a] += (-1.0f * (xv[a] + r - mx[a])) * ks;
    }
  }
  if (hit) {
    f[0] -= kd * v.x;
    f[1] -= kd * v.y;
    f[2] -= kd * v.z;
  }
  fx = fx + f[0];
  fy = fy + f[1];
  fz = fz + f[2];
}

// Vector3::normalize: scales v to unit length with a reciprocal taken in
// double, returns the length (0 leaves v unchanged).
__device__ __forceinline__ float normalize3(float& x, float& y, float& z) {
  const float l = __fsqrt_rn(x * x + y * y + z * z);
  if (l == 0.0f) return 0.0f;
  const float ll = (float)(1.0 / (double)l);
  x *= ll;
  y *= ll;
  z *= ll;
  return l;
}

// External forces on a rigid or granular particle (rigid branch of
// CalculateExternalForcesVersatilCouplingPCISPH, UnifiedPhysics.cpp:5300-5348;
// granular contact of CalculateForcesWithContactForces, UnifiedPhysics.cpp:3219-3338).
// Rigid: spring-damper against rigid particles of other bodies, the reaction
// of the liquid's boundary pressure (and adhesion), the box penalty.
// Granular: Bell et al. contact (normal spring-damper, Coulomb-bounded
// tangential friction) against grains, rigid and boundary particles closer
// than 2 r, the liquid reaction, gravity, the box penalty. Solid particles are
// a minority, so the loop is plain (no batching) to keep registers for the
// liquid path. `id_body` is null when no bodies are set.
__device__ __forceinline__ float3 solid_external(const DevParams& P, uint32_t i, int32_t ti, float4 xi, float4 vi,
                                              const DynArrays& B, const int32_t* __restrict__ id_body,
                                              const uint32_t* __restrict__ nbr, uint32_t cnt, const float* pg,
                                              const float* adl) {
  const float m = P.mass, h = P.h, rv = P.rest_volume;
  const float dc = 2.0f * P.radius;
  const int32_t bi = (ti == UPF_RIGID && id_body) ? id_body[B.id[i]] : -1;
  float fx = 0.0f, fy = 0.0f, fz = 0.0f;
  for (uint32_t k = 0; k < cnt; ++k) {
    const uint32_t code = __ldg(nbr + (size_t)k * P.nstride + i);
    const float4 xj = __ldg(B.pos + code);
    const float d = dist3(xi, xj);
    if (!(d < h)) continue;
    const unsigned dl = dist_lut(d, h);
    const int32_t tj = __ldg(B.type + code);
    if (ti == UPF_RIGID) {
      if (tj == UPF_RIGID) {
        // dynamic rigid neighbours have code < stride, inside the id array
        const int32_t bj = id_body ? id_body[B.id[code]] : -1;
        if (bj == bi) continue;
        // CalculateSpringForceHost / CalculateDampingForceHost (UnifiedPhysics.cpp:2010-2030)
        const float overlap = 2.0f * P.radius - d;
        if (overlap > 0.00001f) {
          const float4 vj = __ldg(B.vel + code);
          const float sx = -1.0f * P.spring * overlap * (xj.x - xi.x) / d;
          const float sy = -1.0f * P.spring * overlap * (xj.y - xi.y) / d;
          const float sz = -1.0f * P.spring * overlap * (xj.z - xi.z) / d;
          fx = fx + (sx + P.damping * (vj.x - vi.x));
          fy = fy + (sy + P.damping * (vj.y - vi.y));
          fz = fz + (sz + P.damping * (vj.z - vi.z));
        }
        continue;
      }
    } else if ((tj == UPF_GRANULAR || tj == UPF_RIGID || tj == UPF_FROZEN) && d < dc) {
      const float4 vj = __ldg(B.vel + code);
      const float ksi = (dc - d < 0.0f) ? 0.0f : dc - d;
      float nx = (xi.x - xj.x) * -1.0f, ny = (xi.y - xj.y) * -1.0f, nz = (xi.z - xj.z) * -1.0f;
      normalize3(nx, ny, nz);
      const float Vx = vi.x - vj.x, Vy = vi.y - vj.y, Vz = vi.z - vj.z;
      const float ksi_dot = Vx * nx + Vy * ny + Vz * nz;
      float tx = Vx - nx * ksi_dot, ty = Vy - ny * ksi_dot, tz = Vz - nz * ksi_dot;
      const float fn = -P.gran_kd * ksi_dot - P.gran_kr * ksi;
      const float vtl = normalize3(tx, ty, tz);
      const float a = P.gran_mu * fabsf(fn), b = P.gran_kt * vtl;
      const float t = (b < a) ? b : a;
      fx = fx + (nx * fn + tx * (-t));
      fy = fy + (ny * fn + ty * (-t));
      fz = fz + (nz * fn + tz * (-t));
      continue;
    }
    if (tj == UPF_LIQUID) {
      // the liquid neighbour's lagged pressure and density, its rest volume
      const float4 lj = __ldg(B.lag + code);
      if (P.flags & UPF_FLAG_BOUNDARY_PRESSURE)
        boundary_pressure_reaction(P, pg, d, xj, xi, lj.z, lj.x, rv, fx, fy, fz);
      if ((P.flags & UPF_FLAG_ADHESION) && d >= h * 0.25f) {
        const float sp = adl[dl];
        const float inv = 1.0f / d;
        fx = fx + (xj.x - xi.x) * P.adh_beta * m * P.rho0 * rv * sp * inv;
        fy = fy + (xj.y - xi.y) * P.adh_beta * m * P.rho0 * rv * sp * inv;
        fz = fz + (xj.z - xi.z) * P.adh_beta * m * P.rho0 * rv * sp * inv;
      }
    }
  }
  if (ti == UPF_GRANULAR) fy -= m * P.gravity;
  rigid_box_force(P, xi, vi, fx, fy, fz);
  return make_float3(fx, fy, fz);
}

// CalculateExternalForcesVersatilCouplingPCISPH (UnifiedPhysics.cpp:5252-5365):
// liquid particles (then the first prediction of the loop), rigid and
// granular particles (solid_external).
// Held to five CTAs of 256 threads an SM (48 registers, a few dozen bytes of
// spill) for one system: 0.223 against 0.240 ms a launch at four CTAs and 60
// registers on the 1M dam. The batched pass, which spills more at that cap,
// keeps the compiler's choice.
constexpr int external_min_blocks(bool batch, int threads) { return batch ? 1 : 1280 / threads; }

template <bool kBatch, int kThreads>
__global__ void __launch_bounds__(kThreads, external_min_blocks(kBatch, kThreads)) k_pcisph_external(
    const __grid_constant__ DevParams Pk, const BatchView bv, uint32_t n, DynArrays B,
    const float* __restrict__ wvol, const int32_t* __restrict__ id_body, const uint32_t* __restrict__ nbr,
    const uint32_t* __restrict__ ncnt, const float* __restrict__ luts_plain, float4* __restrict__ force,
    float4* __restrict__ pforce, float4* __restrict__ xs, float* __restrict__ press, float4* __restrict__ pq,
    DevState* __restrict__ st_plain) {
  __shared__ DevParams sP;
  __shared__ float vl[UPF_LUT_ENTRIES], pg[UPF_LUT_ENTRIES], stl[UPF_LUT_ENTRIES], adl[UPF_LUT_ENTRIES];
  const Scope sc = enter_scope<kBatch>(Pk, luts_plain, st_plain, n, bv, &sP, false);
  const float* luts = sc.luts;
  stage_lut(vl, luts + LUT_VISC * UPF_LUT_ENTRIES);
  stage_lut(pg, luts + LUT_PGRAD * UPF_LUT_ENTRIES);
  stage_lut(stl, luts + LUT_ST * UPF_LUT_ENTRIES);
  stage_lut(adl, luts + LUT_ADH * UPF_LUT_ENTRIES);
  __syncthreads();
  const DevParams& P = *sc.P;
  DevState* st = sc.st;
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= sc.end) return;
  const int32_t ti = B.type[i];
  const float4 xi = B.pos[i];
  press[i] = 0.0f;
  pq[i] = make_float4(xi.x, xi.y, xi.z, 0.0f);  // position, p / rho0^2 (updated by the density pass)
  pforce[i] = f4(0, 0, 0);
  if (ti != UPF_LIQUID) {
    // predicted position of a non-liquid particle: its current position
    xs[i] = xi;
    if (ti == UPF_RIGID || ti == UPF_GRANULAR) {
      const float3 F = solid_external(P, i, ti, xi, B.vel[i], B, id_body, nbr, ncnt[i], pg, adl);
      force[i] = f4(F.x, F.y, F.z);
    } else {
      force[i] = f4(0, 0, 0);
    }
    return;
  }
  const float4 vi = B.vel[i];
  const float4 lag = B.lag[i];
  const float m = P.mass, h = P.h, rv = P.rest_volume;
  const uint32_t flags = P.flags;
  float fx = 0, fy = 0, fz = 0;
  struct NbState {
    float4 x, v;
    int32_t t;
  };
  const float4* __restrict__ bpos = B.pos;
  const float4* __restrict__ bvel = B.vel;
  const int32_t* __restrict__ btype = B.type;
  // boundary particles sit in the tails of the B arrays (type FROZEN, velocity 0)
  for_neighbors<kExternalUnroll>(
      nbr + i, P.nstride, ncnt[i],
      [&](uint32_t code) {
        NbState s;
        s.x = __ldg(bpos + code);
        s.v = __ldg(bvel + code);
        s.t = __ldg(btype + code);
        return s;
      },
      [&](uint32_t code, const NbState& s) {
    const float4 xj = s.x;
    const float d = dist3(xi, xj);
    if (!(d < h)) return;
    const unsigned dl = dist_lut(d, h);
    const int32_t tj = s.t;
    if (tj == UPF_LIQUID) {
      const float kv = lut_at(vl, d, P.lut_factor);
      const float4 vj = s.v;
      fx = fx - (vi.x - vj.x) * rv * rv * P.visc * kv;
      fy = fy - (vi.y - vj.y) * rv * rv * P.visc * kv;
      fz = fz - (vi.z - vj.z) * rv * rv * P.visc * kv;
      if ((flags & UPF_FLAG_SURFACE_TENSION) && d >= h * 0.25f) {
        const float sp = stl[dl];
        const float inv = 1.0f / d;
        fx = fx - (xi.x - xj.x) * P.st_gamma * m * m * sp * inv;
        fy = fy - (xi.y - xj.y) * P.st_gamma * m * m * sp * inv;
        fz = fz - (xi.z - xj.z) * P.st_gamma * m * m * sp * inv;
      }
    } else if (tj == UPF_FROZEN || tj == UPF_RIGID || tj == UPF_GRANULAR) {
      // granular grains count as boundary, as rigid particles do
      const float wv = wvol[code];
      // the reference passes the liquid particle's own weighted volume (its
      // rest volume) to the pressure term, UnifiedPhysics.cpp:5292
      if (flags & UPF_FLAG_BOUNDARY_PRESSURE)
        boundary_pressure(P, pg, d, xi, xj, lag.z, lag.x, rv, fx, fy, fz);
      if ((flags & UPF_FLAG_ADHESION) && d >= h * 0.25f) {
        const float sp = adl[dl];
        const float inv = 1.0f / d;
        fx = fx - (xi.x - xj.x) * P.adh_beta * m * P.rho0 * wv * sp * inv;
        fy = fy - (xi.y - xj.y) * P.adh_beta * m * P.rho0 * wv * sp * inv;
        fz = fz - (xi.z - xj.z) * P.adh_beta * m * P.rho0 * wv * sp * inv;
      }
    }
      });
  fy -= m * P.gravity;
  if (flags & UPF_FLAG_PENALTY_WALLS) penalty_walls(P, xi, fx, fy, fz);
  force[i] = f4(fx, fy, fz);
  bool bad;
  xs[i] = predict(P, xi, vi, make_float3(fx, fy, fz), make_float3(0, 0, 0), bad);
  if (bad) atomicOr(&st->error_flags, (uint32_t)ERR_NAN);
}

// ComputePredictedDensityAndPressure (UnifiedPhysics.cpp:5456-5491) with the
// maximum for the loop test reduced in the same pass. The list entries come
// by the TMA ring or by direct loads (walk_lists); each lane gathers kRows
// neighbours' predicted positions at once and accumulates them in list order.
template <bool kBatch, bool kDirect, int kThreads, int kRows>
__device__ __forceinline__ void density_block(
    uint32_t block, const DevParams& Pk, const BatchView& bv, uint32_t n, const int32_t* __restrict__ type,
    const float4* __restrict__ xs, const CUtensorMap& cmap, const uint32_t* __restrict__ nbr,
    const uint32_t* __restrict__ ncnt, const float* __restrict__ luts_plain, float* __restrict__ rho,
    float* __restrict__ press, float4* __restrict__ pq, DevState* __restrict__ st_plain) {
  __shared__ DevParams sP;
  __shared__ float m4[UPF_LUT_ENTRIES];
  __shared__ uint32_t wmax[kThreads / 32];
  const Scope sc = enter_scope_at<kBatch>(block, Pk, luts_plain, st_plain, n, bv, &sP, true);
  if (sc.skip) return;  // uniform over the CTA: the scene's loop has finished
  const int lane = threadIdx.x & 31;
  // the table times the mass: each pair adds the same rounded product
  // m4[bin] * m as the reference's kernelM4Lut(d) * mass
  const float mass = kBatch ? __ldg(&bv.params[sc.scene].mass) : Pk.mass;
  for (int k = threadIdx.x; k < UPF_LUT_ENTRIES; k += blockDim.x)
    m4[k] = fmul(__ldg(sc.luts + LUT_M4 * UPF_LUT_ENTRIES + k), mass);
  // the first r2 of the zero entry (thresholds follow the five tables)
  const float r2_edge = __ldg(sc.luts + 5 * UPF_LUT_ENTRIES + kLut);
  __syncthreads();
  const DevParams& P = *sc.P;
  DevState* st = sc.st;
  uint32_t i = block * blockDim.x + threadIdx.x;
  uint32_t best = 0;
  const bool active = i < sc.end && type[i] == UPF_LIQUID;
  const uint32_t cnt = active ? ncnt[i] : 0u;
  const float4 xi = active ? xs[i] : make_float4(0, 0, 0, 0);
  const unsigned long long xiy = pk2(xi.x, xi.y);
  const float m = P.mass;
  float den = P.kernel_self * m;
  const ListArgs L{&cmap, &cmap, nbr, nullptr, P.nstride};
  const bool ok = walk_lists<kDirect, false, kThreads, kRows>(L, block, i, cnt, [&](auto code, auto, int k0) {
    // predicted positions; boundary particles sit in the array's tail at
    // their fixed positions
    float4 xj[kRows];
#pragma unroll
    for (int r = 0; r < kRows; ++r)
      if (k0 + r < (int)cnt) xj[r] = __ldg(xs + code(r));
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      if (k0 + r < (int)cnt) {
        // the table bin of d from d^2 (exact); at or beyond h the bin is 300,
        // whose entry 0 adds +0 exactly as the reference's skipped term does
        const float r2 = dist2_xy(xiy, xi.z, xj[r]);
        den += m4[bin_of_r2_edge(r2, P.lut_factor, r2_edge)];  // table times mass
      }
    }
  });
  if (!ok && lane == 0) atomicOr(&st->error_flags, (uint32_t)ERR_TIMEOUT);
  if (active) {
    const float err = mx0(den - P.rho0, 0.0f);
    const float pnew = press[i] + mx0(err * P.delta, 0.0f);
    press[i] = pnew;
    // p / (rho0 * rho0): the pressure-force pass divides every neighbour's
    // pressure by the same constant; dividing once here is bit-identical
    reinterpret_cast<float*>(pq + i)[3] = pnew / (P.rho0 * P.rho0);  // .w only: the position stays
    rho[i] = den;
    best = __float_as_uint(den);  // densities are positive: uint order == float order
  }
  best = warp_max(best);
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x < 32) {
    uint32_t v = threadIdx.x < (blockDim.x >> 5) ? wmax[threadIdx.x] : 0u;
    v = warp_max(v);
    if (threadIdx.x == 0 && v) atomicMax(&st->max_rho_bits, v);
  }
}

template <bool kBatch, bool kDirect, int kThreads, int kRows>
__global__ void __launch_bounds__(kThreads) k_pcisph_density(
    const __grid_constant__ DevParams Pk, const BatchView bv, uint32_t n, const int32_t* __restrict__ type,
    const float4* __restrict__ xs, const __grid_constant__ CUtensorMap cmap, const uint32_t* __restrict__ nbr,
    const uint32_t* __restrict__ ncnt, const float* __restrict__ luts_plain, float* __restrict__ rho,
    float* __restrict__ press, float4* __restrict__ pq, DevState* __restrict__ st_plain) {
  density_block<kBatch, kDirect, kThreads, kRows>(blockIdx.x, Pk, bv, n, type, xs, cmap, nbr, ncnt, luts_plain, rho,
                                                  press, pq, st_plain);
}

// Batched scenes once most have finished their loop: a resident grid takes
// the 256-slot groups of the scenes still iterating from the list the loop
// control wrote (direct list loads: the TMA ring's barriers belong to one
// walk), instead of a CTA for every group of every scene.
template <int kRows>
__global__ void __launch_bounds__(kSegAlign) k_pcisph_density_active(
    const BatchView bv, uint32_t n, const uint32_t* __restrict__ groups, const uint32_t* __restrict__ ngroups,
    const int32_t* __restrict__ type, const float4* __restrict__ xs, const uint32_t* __restrict__ nbr,
    const uint32_t* __restrict__ ncnt, float* __restrict__ rho, float* __restrict__ press,
    float4* __restrict__ pq) {
  const uint32_t count = *ngroups;
  for (uint32_t g = blockIdx.x; g < count; g += gridDim.x) {
    density_block<true, true, kSegAlign, kRows>(groups[g], DevParams{}, bv, n, type, xs, CUtensorMap{}, nbr, ncnt,
                                                 nullptr, rho, press, pq, nullptr);
    __syncthreads();  // the next group reuses the shared scope and table
  }
}

// ComputeCorrectivePressureForce (UnifiedPhysics.cpp:5493-5522), then the
// prediction of the next iteration (PredictPositionAndVelocity). The
// positions are the step's, at which the list was built: every entry lies
// within h and carries the pressure-gradient table's value at its bin as its
// list value, so the pass reads no table. List entries and values come by
// the TMA ring or by direct loads (walk_lists).
// Short TMA rings (at most 4 rows a stage) are held to 64 registers a thread
// (four 256-thread CTAs an SM): two chunks of gathers in flight need them
// (held to 40, the 4-row rings spilled). The batched pass keeps one chunk in
// flight at 40 registers: its scenes converge unevenly, and the occupancy
// pays more there than the second chunk.
__host__ __device__ constexpr bool pforce_two_chunks(bool batch) { return !batch; }
constexpr int pforce_min_blocks(bool batch, bool direct, int threads, int rows) {
  return (!direct && rows <= 4) ? (pforce_two_chunks(batch) ? 1024 : 1536) / threads : 1;
}

template <bool kBatch, bool kDirect, int kThreads, int kRows>
__device__ __forceinline__ void pforce_block(
    uint32_t block, const DevParams& Pk, const BatchView& bv, uint32_t n, const DynArrays& B,
    const CUtensorMap& cmap, const CUtensorMap& vmap, const uint32_t* __restrict__ nbr,
    const uint32_t* __restrict__ lval, const uint32_t* __restrict__ ncnt, const float* __restrict__ luts_plain,
    const float4* __restrict__ pq, const float4* __restrict__ force, float4* __restrict__ pforce,
    float4* __restrict__ xs, DevState* __restrict__ st_plain) {
  __shared__ DevParams sP;
  const Scope sc = enter_scope_at<kBatch>(block, Pk, luts_plain, st_plain, n, bv, &sP, true);
  if (sc.skip) return;  // uniform over the CTA: the scene's loop has finished
  const int lane = threadIdx.x & 31;
  if (kBatch) __syncthreads();  // the scene's parameters in shared memory
  const DevParams& P = *sc.P;
  DevState* st = sc.st;
  uint32_t i = block * blockDim.x + threadIdx.x;
  const bool active = i < sc.end && B.type[i] == UPF_LIQUID;
  const uint32_t cnt = active ? ncnt[i] : 0u;
  const float4 xi = active ? B.pos[i] : make_float4(0, 0, 0, 0);
  const float m = P.mass;
  // grad = p_i / rho0^2 + p_j / rho0^2, both quotients precomputed by the
  // density pass (pq.w); boundary particles have p = 0, so 0 / rho0^2 = 0
  const float qi = active ? pq[i].w : 0.0f;
  // Scalar arithmetic on purpose: a packed (f32x2) multiply whose product
  // feeds a packed subtract did not reproduce the scalar roundings on the
  // device (measured: the pass drifted from the oracle by an ulp in rare
  // pairs, then the loop by whole iterations), and the packed form was no
  // faster.
  float fx = 0, fy = 0, fz = 0;
  const ListArgs L{&cmap, &vmap, nbr, lval, P.nstride};
  // One gather per neighbour: position and p / rho0^2 packed in pq
  // (boundary particles sit in the tail, w = 0 there), with the entry's
  // list value, kernelPressureGradLut at its bin. Each chunk's gathers are
  // issued before the previous chunk's arithmetic (two chunks in flight a
  // lane: 0.085-0.086 against 0.088 ms a launch on the 1M dam); the sums
  // stay in list order.
  float4 xp[kRows];
  float gp[kRows];
  int kp = -1;
  auto accumulate = [&](const float4* xj, const float* g, int k0) {
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      if (k0 + r < (int)cnt) {
        // k = (x_i - x_j) * g; f -= ((k * grad) * m) * m, per component
        const float kx = (xi.x - xj[r].x) * g[r], ky = (xi.y - xj[r].y) * g[r], kz = (xi.z - xj[r].z) * g[r];
        const float grad = qi + xj[r].w;
        fx = fx - kx * grad * m * m;
        fy = fy - ky * grad * m * m;
        fz = fz - kz * grad * m * m;
      }
    }
  };
  const bool ok = walk_lists<kDirect, true, kThreads, kRows>(L, block, i, cnt, [&](auto code, auto val, int k0) {
    float4 xn[kRows];
    float gn[kRows];
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      if (k0 + r < (int)cnt) {
        xn[r] = __ldg(pq + code(r));
        gn[r] = __uint_as_float(val(r));
      }
    }
    if constexpr (pforce_two_chunks(kBatch)) {
      if (kp >= 0) accumulate(xp, gp, kp);
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        xp[r] = xn[r];
        gp[r] = gn[r];
      }
      kp = k0;
    } else {
      accumulate(xn, gn, k0);
    }
  });
  if (kp >= 0) accumulate(xp, gp, kp);
  if (!ok && lane == 0) atomicOr(&st->error_flags, (uint32_t)ERR_TIMEOUT);
  if (!active) return;
  pforce[i] = f4(fx, fy, fz);
  const float4 F = force[i];
  bool bad;
  xs[i] = predict(P, xi, B.vel[i], make_float3(F.x, F.y, F.z), make_float3(fx, fy, fz), bad);
  if (bad) atomicOr(&st->error_flags, (uint32_t)ERR_NAN);
}

template <bool kBatch, bool kDirect, int kThreads, int kRows>
__global__ void __launch_bounds__(kThreads, pforce_min_blocks(kBatch, kDirect, kThreads, kRows)) k_pcisph_pressure_force(
    const __grid_constant__ DevParams Pk, const BatchView bv, uint32_t n, DynArrays B,
    const __grid_constant__ CUtensorMap cmap, const __grid_constant__ CUtensorMap vmap,
    const uint32_t* __restrict__ nbr, const uint32_t* __restrict__ lval, const uint32_t* __restrict__ ncnt,
    const float* __restrict__ luts_plain, const float4* __restrict__ pq, const float4* __restrict__ force,
    float4* __restrict__ pforce, float4* __restrict__ xs, DevState* __restrict__ st_plain) {
  pforce_block<kBatch, kDirect, kThreads, kRows>(blockIdx.x, Pk, bv, n, B, cmap, vmap, nbr, lval, ncnt, luts_plain,
                                                 pq, force, pforce, xs, st_plain);
}

// The pressure-force pass over the active groups (k_pcisph_density_active).
template <int kRows>
__global__ void __launch_bounds__(kSegAlign) k_pcisph_pressure_force_active(
    const BatchView bv, uint32_t n, const uint32_t* __restrict__ groups, const uint32_t* __restrict__ ngroups,
    DynArrays B, const uint32_t* __restrict__ nbr, const uint32_t* __restrict__ lval,
    const uint32_t* __restrict__ ncnt, const float4* __restrict__ pq, const float4* __restrict__ force,
    float4* __restrict__ pforce, float4* __restrict__ xs) {
  const uint32_t count = *ngroups;
  for (uint32_t g = blockIdx.x; g < count; g += gridDim.x) {
    pforce_block<true, true, kSegAlign, kRows>(groups[g], DevParams{}, bv, n, B, CUtensorMap{}, CUtensorMap{}, nbr,
                                                lval, ncnt, nullptr, pq, force, pforce, xs, nullptr);
    __syncthreads();  // the next group reuses the shared scope
  }
}

// ---------------------------------------------------------------- staged neighbourhoods
// Loop-pass mode 2. The 256 particles of a chunk (one CTA) sit close together
// in Morton order, so their lists draw on one small neighbourhood: about 830
// distinct neighbours on the 1M dam against 256 x 29 list entries. Once per
// step k_stage_lists writes that union and rewrites the chunk's list entries
// as positions in it; each loop pass then copies the union's data into
// shared memory (one gather per distinct neighbour instead of one per list
// entry) and reads every neighbour from there. The entries keep their list
// order, so every sum keeps the reference's order and the results are
// bit-identical to the other modes.
// The union is kept as a set of 8-index blocks (a block id and a mask of the
// indices present), so that neighbour indices that follow one another get
// consecutive positions: the k-th neighbours of a warp's consecutive
// particles are mostly consecutive indices, and consecutive 16-byte entries
// in shared memory fall in different banks.
constexpr uint32_t kStageBlocks = 1024;  // block slots, open addressing
constexpr uint32_t kMaxStageBlocks = kStageBlocks / 2;
constexpr uint32_t kHashEmpty = 0xffffffffu;

__device__ __forceinline__ uint32_t stage_hash(uint32_t blk) {
  return (blk * 2654435761u) >> (32 - 10);  // Fibonacci hashing onto kStageBlocks = 1024 slots
}
static_assert(kStageBlocks == 1024, "stage_hash maps onto 1024 slots");
static_assert((kUnionMax & (kUnionMax - 1)) == 0, "union positions are masked with kUnionMax - 1");

// One CTA per chunk: (1) insert the chunk's neighbour indices into the block
// set in shared memory, stopping at more than kMaxStageBlocks blocks;
// (2) number the indices (blocks in slot order, indices in a block in
// order), stopping at more than `cap`, and write the union; (3) rewrite each
// list entry as its index's number. Liquid particles only (the loop passes
// read no other lists).
__global__ void __launch_bounds__(kStageChunk) k_stage_lists(uint32_t n, const int32_t* __restrict__ type,
                                                              const uint32_t* __restrict__ nbr,
                                                              const uint32_t* __restrict__ ncnt, uint32_t stride,
                                                              uint32_t cap, uint32_t* __restrict__ ucodes,
                                                              uint32_t* __restrict__ ucount,
                                                              unsigned long long* __restrict__ lloc) {
  __shared__ uint32_t bkey[kStageBlocks];
  __shared__ uint32_t bmask[kStageBlocks];
  __shared__ uint16_t bbase[kStageBlocks];
  __shared__ uint32_t warp_tot[kStageChunk / 32];
  __shared__ uint32_t nblocks;
  __shared__ int over;
  const uint32_t chunk = blockIdx.x, tid = threadIdx.x;
  for (uint32_t k = tid; k < kStageBlocks; k += kStageChunk) {
    bkey[k] = kHashEmpty;
    bmask[k] = 0u;
  }
  if (tid == 0) {
    nblocks = 0;
    over = 0;
  }
  __syncthreads();
  const uint32_t i = chunk * kStageChunk + tid;
  const bool active = i < n && type[i] == UPF_LIQUID;
  const uint32_t cnt = active ? ncnt[i] : 0u;
  const uint32_t* __restrict__ col = nbr + i;
  unsigned long long* __restrict__ out = lloc + i;
  volatile int* vover = &over;
  volatile uint32_t* vkey = bkey;
  // each entry's (block slot, index in the block) goes to lloc for now, four
  // to a word; step (3) turns them into union positions in place
  // the codes come four at a time, the next four loaded before these are
  // inserted (the insertions' shared-memory atomics keep the compiler from
  // moving later loads ahead of them)
  uint32_t nxt[4];
#pragma unroll
  for (uint32_t r = 0; r < 4; ++r) nxt[r] = r < cnt ? __ldg(col + (size_t)r * stride) : 0u;
  for (uint32_t k0 = 0; k0 < cnt && !*vover; k0 += 4) {
    uint32_t codes[4];
#pragma unroll
    for (uint32_t r = 0; r < 4; ++r) {
      codes[r] = nxt[r];
      if (k0 + 4 + r < cnt) nxt[r] = __ldg(col + (size_t)(k0 + 4 + r) * stride);
    }
    unsigned long long w = 0;
#pragma unroll
    for (uint32_t r = 0; r < 4; ++r) {
      if (k0 + r >= cnt) break;
      const uint32_t code = codes[r];
      const uint32_t blk = code >> 3, bit = 1u << (code & 7u);
      uint32_t slot = stage_hash(blk);
      // a plain read first: most entries find their block present (each
      // neighbour is in about nine lists of the chunk), and the atomics of a
      // warp's lanes on one shared-memory word serialise. At most
      // kMaxStageBlocks + kStageChunk < kStageBlocks blocks are ever
      // inserted, so an empty slot is always found; the probes are bounded
      // all the same.
      for (uint32_t probe = 0; probe < kStageBlocks; ++probe) {
        const uint32_t cur = vkey[slot];
        if (cur == blk) break;
        if (cur == kHashEmpty) {
          const uint32_t prev = atomicCAS(&bkey[slot], kHashEmpty, blk);
          if (prev == kHashEmpty) {
            if (atomicAdd(&nblocks, 1u) >= kMaxStageBlocks) *vover = 1;
            break;
          }
          if (prev == blk) break;
        }
        slot = (slot + 1) & (kStageBlocks - 1);
      }
      if (!(bmask[slot] & bit)) atomicOr(&bmask[slot], bit);
      w |= (unsigned long long)((slot << 3) | (code & 7u)) << (16 * r);
    }
    out[(size_t)(k0 / 4) * stride] = w;
  }
  __syncthreads();
  if (over) {
    if (tid == 0) ucount[chunk] = kUnionOverflow;
    return;  // uniform: the chunk's passes read the plain lists
  }
  // (2) thread t numbers the blocks in slots [t * 4, t * 4 + 4); an exclusive
  // scan over the threads' index counts gives each block its first position
  constexpr uint32_t kPer = kStageBlocks / kStageChunk;
  uint32_t mine = 0;
#pragma unroll
  for (uint32_t j = 0; j < kPer; ++j) mine += __popc(bmask[tid * kPer + j]);
  const uint32_t lane = tid & 31, warp = tid >> 5;
  uint32_t incl = mine;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= (uint32_t)d) incl += v;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kStageChunk / 32 ? warp_tot[lane] : 0u;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, w, d);
      if (lane >= (uint32_t)d) w += v;
    }
    if (lane < kStageChunk / 32) warp_tot[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  const uint32_t total = warp_tot[kStageChunk / 32 - 1];
  if (total > cap) {
    if (tid == 0) ucount[chunk] = kUnionOverflow;
    return;  // uniform
  }
  uint32_t at = (warp ? warp_tot[warp - 1] : 0u) + incl - mine;
  uint32_t* __restrict__ uc = ucodes + (size_t)chunk * kUnionMax;
#pragma unroll
  for (uint32_t j = 0; j < kPer; ++j) {
    const uint32_t slot = tid * kPer + j;
    uint32_t m = bmask[slot];
    bbase[slot] = (uint16_t)at;
    const uint32_t base = bkey[slot] << 3;
    while (m) {
      const uint32_t b = __ffs(m) - 1;
      m &= m - 1;
      uc[at++] = base + b;
    }
  }
  if (tid == 0) ucount[chunk] = total;
  __syncthreads();
  // (3) the chunk's entries as union positions, four to a word, in place
  // (the next word loaded before this one is rewritten)
  unsigned long long vn = cnt ? out[0] : 0ull;
  for (uint32_t k0 = 0; k0 < cnt; k0 += 4) {
    const unsigned long long v = vn;
    if (k0 + 4 < cnt) vn = out[(size_t)(k0 / 4 + 1) * stride];
    unsigned long long w2 = 0;
#pragma unroll
    for (uint32_t r = 0; r < 4; ++r) {
      if (k0 + r < cnt) {
        const uint32_t e = (uint32_t)(v >> (16 * r)) & 0xffffu;
        const uint32_t slot = e >> 3, b = e & 7u;
        const uint32_t posn = bbase[slot] + __popc(bmask[slot] & ((1u << b) - 1u));
        w2 |= (unsigned long long)posn << (16 * r);
      }
    }
    out[(size_t)(k0 / 4) * stride] = w2;
  }
}

// The staged list walk of one lane: batches of kRows entries (kRows / 4
// words of lloc, the next batch's words loaded before this batch's
// arithmetic); `body(pos, k0)` gets the union positions of the batch.
template <int kRows, class Body>
__device__ __forceinline__ void walk_staged(const unsigned long long* __restrict__ col, uint32_t stride, uint32_t cnt,
                                            Body&& body) {
  constexpr int kWords = kRows / 4;
  unsigned long long w[kWords];
#pragma unroll
  for (int q = 0; q < kWords; ++q) w[q] = (4 * q < (int)cnt) ? __ldg(col + (size_t)q * stride) : 0ull;
  for (uint32_t k0 = 0; k0 < cnt; k0 += kRows) {
    unsigned long long cur[kWords];
#pragma unroll
    for (int q = 0; q < kWords; ++q) {
      cur[q] = w[q];
      const uint32_t kn = k0 + kRows + 4 * q;
      if (kn < cnt) w[q] = __ldg(col + (size_t)(kn / 4) * stride);
    }
    // (positions are below kUnionMax by construction; the mask keeps every
    // shared-memory read in bounds even on lists staged for another step)
    body([&](int r) { return (uint32_t)(cur[r >> 2] >> (16 * (r & 3))) & (kUnionMax - 1); }, (int)k0);
  }
}

// The predicted-density pass over staged neighbourhoods (density_block's
// arithmetic, ComputePredictedDensityAndPressure, UnifiedPhysics.cpp:5456-5491).
// Register caps (CTAs an SM the launch bounds ask for; six fit the shared
// memory, 33-34 KB each): 4-entry batches of the density pass are held to 40
// registers (six CTAs an SM; 8 bytes of spill, and 0.083 against 0.085 ms a
// launch at five CTAs and 48 registers on the 1M dam), of the pressure-force
// pass to 48; 8-entry batches to 64 (density) and 80 (pressure force), the
// caps below which they spill.
constexpr int density_staged_min_blocks(int rows) { return rows == 4 ? 6 : 4; }
constexpr int pforce_staged_min_blocks(int rows) { return rows == 4 ? 5 : 3; }

template <int kRows>
__global__ void __launch_bounds__(kStageChunk, density_staged_min_blocks(kRows)) k_pcisph_density_staged(
    const __grid_constant__ DevParams P, uint32_t n, const int32_t* __restrict__ type,
    const float4* __restrict__ xs, const uint32_t* __restrict__ nbr, const uint32_t* __restrict__ ncnt,
    const uint32_t* __restrict__ ucodes, const uint32_t* __restrict__ ucount,
    const unsigned long long* __restrict__ lloc, const float* __restrict__ luts, float* __restrict__ rho,
    float* __restrict__ press, float4* __restrict__ pq, DevState* __restrict__ st) {
  __shared__ float4 xsm[kUnionMax];
  __shared__ float m4[UPF_LUT_ENTRIES];
  __shared__ uint32_t wmax[kStageChunk / 32];
  const uint32_t chunk = blockIdx.x;
  const uint32_t U = ucount[chunk];
  const bool staged = U != kUnionOverflow;
  // the table times the mass, as in density_block
  for (int k = threadIdx.x; k < UPF_LUT_ENTRIES; k += kStageChunk)
    m4[k] = fmul(__ldg(luts + LUT_M4 * UPF_LUT_ENTRIES + k), P.mass);
  if (staged) {
    const uint32_t* __restrict__ uc = ucodes + (size_t)chunk * kUnionMax;
    const uint32_t nu = U < kUnionMax ? U : kUnionMax;
    for (uint32_t l = threadIdx.x; l < nu; l += kStageChunk) xsm[l] = __ldg(xs + __ldg(uc + l));
  }
  const float r2_edge = __ldg(luts + 5 * UPF_LUT_ENTRIES + kLut);
  __syncthreads();
  const uint32_t i = chunk * kStageChunk + threadIdx.x;
  const bool active = i < n && type[i] == UPF_LIQUID;
  const uint32_t cnt = active ? ncnt[i] : 0u;
  const float4 xi = active ? xs[i] : make_float4(0, 0, 0, 0);
  const unsigned long long xiy = pk2(xi.x, xi.y);
  float den = P.kernel_self * P.mass;
  auto add = [&](float4 xj) {
    const float r2 = dist2_xy(xiy, xi.z, xj);
    den += m4[bin_of_r2_edge(r2, P.lut_factor, r2_edge)];
  };
  if (staged) {
    walk_staged<kRows>(lloc + i, P.nstride, cnt, [&](auto pos, int k0) {
      float4 xj[kRows];
#pragma unroll
      for (int r = 0; r < kRows; ++r)
        if (k0 + r < (int)cnt) xj[r] = xsm[pos(r)];
#pragma unroll
      for (int r = 0; r < kRows; ++r)
        if (k0 + r < (int)cnt) add(xj[r]);
    });
  } else {
    const uint32_t* __restrict__ col = nbr + i;
    for (uint32_t k0 = 0; k0 < cnt; k0 += 4) {
      float4 xj[4];
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (k0 + r < cnt) xj[r] = __ldg(xs + __ldg(col + (size_t)(k0 + r) * P.nstride));
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (k0 + r < cnt) add(xj[r]);
    }
  }
  uint32_t best = 0;
  if (active) {
    const float err = mx0(den - P.rho0, 0.0f);
    const float pnew = press[i] + mx0(err * P.delta, 0.0f);
    press[i] = pnew;
    reinterpret_cast<float*>(pq + i)[3] = pnew / (P.rho0 * P.rho0);
    rho[i] = den;
    best = __float_as_uint(den);
  }
  best = warp_max(best);
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x < 32) {
    uint32_t v = threadIdx.x < kStageChunk / 32 ? wmax[threadIdx.x] : 0u;
    v = warp_max(v);
    if (threadIdx.x == 0 && v) atomicMax(&st->max_rho_bits, v);
  }
}

// The pressure-force pass over staged neighbourhoods (pforce_block's
// arithmetic, ComputeCorrectivePressureForce, UnifiedPhysics.cpp:5493-5522,
// then the next prediction): the union's (position, p / rho0^2) in shared
// memory, the entries' pressure-gradient values from the list values.
template <int kRows>
__global__ void __launch_bounds__(kStageChunk, pforce_staged_min_blocks(kRows)) k_pcisph_pressure_force_staged(
    const __grid_constant__ DevParams P, uint32_t n, DynArrays B, const uint32_t* __restrict__ nbr,
    const uint32_t* __restrict__ lval, const uint32_t* __restrict__ ncnt, const uint32_t* __restrict__ ucodes,
    const uint32_t* __restrict__ ucount, const unsigned long long* __restrict__ lloc,
    const float4* __restrict__ pq, const float4* __restrict__ force, float4* __restrict__ pforce,
    float4* __restrict__ xs, DevState* __restrict__ st) {
  __shared__ float4 qsm[kUnionMax];
  const uint32_t chunk = blockIdx.x;
  const uint32_t U = ucount[chunk];
  const bool staged = U != kUnionOverflow;
  if (staged) {
    const uint32_t* __restrict__ uc = ucodes + (size_t)chunk * kUnionMax;
    const uint32_t nu = U < kUnionMax ? U : kUnionMax;
    for (uint32_t l = threadIdx.x; l < nu; l += kStageChunk) qsm[l] = __ldg(pq + __ldg(uc + l));
  }
  __syncthreads();
  const uint32_t i = chunk * kStageChunk + threadIdx.x;
  const bool active = i < n && B.type[i] == UPF_LIQUID;
  if (!active) return;  // no barrier follows
  const uint32_t cnt = ncnt[i];
  const float4 xi = B.pos[i];
  const float m = P.mass;
  const float qi = pq[i].w;
  // scalar arithmetic, as in pforce_block
  float fx = 0, fy = 0, fz = 0;
  const uint32_t* __restrict__ vcol = lval + i;
  auto add = [&](float4 xj, float g) {
    const float kx = (xi.x - xj.x) * g, ky = (xi.y - xj.y) * g, kz = (xi.z - xj.z) * g;
    const float grad = qi + xj.w;
    fx = fx - kx * grad * m * m;
    fy = fy - ky * grad * m * m;
    fz = fz - kz * grad * m * m;
  };
  if (staged) {
    // the list values of the next batch are loaded with its positions,
    // before this batch's arithmetic (walk_staged's prefetch, extended)
    float gn[kRows];
#pragma unroll
    for (int r = 0; r < kRows; ++r) gn[r] = r < (int)cnt ? __uint_as_float(__ldg(vcol + (size_t)r * P.nstride)) : 0.0f;
    walk_staged<kRows>(lloc + i, P.nstride, cnt, [&](auto pos, int k0) {
      float4 xj[kRows];
      float g[kRows];
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        g[r] = gn[r];
        const uint32_t kn = (uint32_t)k0 + kRows + r;
        if (kn < cnt) gn[r] = __uint_as_float(__ldg(vcol + (size_t)kn * P.nstride));
      }
#pragma unroll
      for (int r = 0; r < kRows; ++r)
        if (k0 + r < (int)cnt) xj[r] = qsm[pos(r)];
#pragma unroll
      for (int r = 0; r < kRows; ++r)
        if (k0 + r < (int)cnt) add(xj[r], g[r]);
    });
  } else {
    const uint32_t* __restrict__ col = nbr + i;
    for (uint32_t k0 = 0; k0 < cnt; k0 += 4) {
      float4 xj[4];
      float g[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        if (k0 + r < cnt) {
          g[r] = __uint_as_float(__ldg(vcol + (size_t)(k0 + r) * P.nstride));
          xj[r] = __ldg(pq + __ldg(col + (size_t)(k0 + r) * P.nstride));
        }
      }
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (k0 + r < cnt) add(xj[r], g[r]);
    }
  }
  pforce[i] = f4(fx, fy, fz);
  const float4 F = force[i];
  bool bad;
  xs[i] = predict(P, xi, B.vel[i], make_float3(F.x, F.y, F.z), make_float3(fx, fy, fz), bad);
  if (bad) atomicOr(&st->error_flags, (uint32_t)ERR_NAN);
}

__global__ void k_loop_init(DevState* st) {
  st->iteration = 0;
  st->too_large = 1;
  st->max_rho_bits = 0;
  st->ke = 0;
  st->mom[0] = st->mom[1] = st->mom[2] = 0;
}

__global__ void k_step_init(DevState* st, int count_step) {
  st->ke = 0;
  st->mom[0] = st->mom[1] = st->mom[2] = 0;
  st->max_neighbors = 0;
  if (count_step) st->total_steps += 1;  // PCISPH counts its steps in the loop control
}

// Loop control of PredictionCorrectionStep (UnifiedPhysics.cpp:5376-5420):
// continue while iteration < min_loops, or the error is still too large and
// iteration < max_loops. The "too large" flag is sticky-false, as in the
// reference. Runs on the device and feeds the graph's conditional node.
__device__ __forceinline__ int loop_ctl(const DevParams& P, DevState* st) {
  const int it = st->iteration + 1;
  st->iteration = it;
  const float maxd = __uint_as_float(st->max_rho_bits);
  const float e = mx0(P.err_scale * maxd - 100.0f, 0.0f);
  if (it <= 64) st->iter_max_rho[it - 1] = maxd;
  if (e < P.max_err) st->too_large = 0;
  int cont = (it < P.min_loops) || (st->too_large && it < P.max_loops);
  if (st->error_flags & ERR_NAN) cont = 0;
  st->final_iterations = it;
  st->final_max_rho = maxd;
  st->final_err = e;
  st->max_rho_bits = 0;
  if (!cont) {
    st->total_steps += 1;
    st->total_iterations += it;
    if (it >= P.max_loops) st->steps_at_max += 1;
    if (e > st->max_step_err) st->max_step_err = e;
  }
  return cont;
}

__global__ void k_loop_ctl(DevParams P, DevState* st, cudaGraphConditionalHandle h, int use_handle) {
  const int cont = loop_ctl(P, st);
  if (use_handle) cudaGraphSetConditional(h, cont ? 1u : 0u);
}

// ---------------------------------------------------------------- batched scenes
constexpr uint32_t kPadKey = kPadKeyBatch;

// Set-up of a batch after upload: keys of every slot (particles: Morton key
// in the scene's grid; padding: kPadKey) and the lagged PCISPH state.
__global__ void __launch_bounds__(kBlock) k_batch_init(const BatchView bv, uint32_t nslots, DynArrays A,
                                                        uint32_t* __restrict__ keys, int with_lag) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nslots) return;
  const uint32_t s = bv.group_scene[i / kSegAlign];
  if (i < bv.seg_end[s]) {
    const DevParams& P = bv.params[s];
    keys[i] = morton_key(A.pos[i], P.origin, P.scales);
    if (with_lag) A.lag[i] = make_float4(0.0f, 0.0f, P.rho0, 0.0f);
  } else {
    keys[i] = kPadKey;
  }
}

// Second sort stage key: the scene of the slot each element came from.
__global__ void __launch_bounds__(kBlock) k_scene_digits(uint32_t nslots, const uint32_t* __restrict__ perm,
                                                          const uint32_t* __restrict__ group_scene,
                                                          uint32_t* __restrict__ digits) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nslots) digits[i] = group_scene[perm[i] / kSegAlign];
}

// Reorder of a batch: the gather of k_reorder, plus each slot's sorted key
// (the scene's Morton key of the gathered position; kPadKey for padding).
__global__ void __launch_bounds__(kBlock) k_reorder_batch(const BatchView bv, uint32_t nslots,
                                                           const uint32_t* __restrict__ perm, DynArrays A,
                                                           DynArrays B, uint32_t* __restrict__ keys) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nslots) return;
  const uint32_t j = perm[i];
  const float4 x = A.pos[j];
  B.pos[i] = x;
  B.vel[i] = A.vel[j];
  B.id[i] = A.id[j];
  B.type[i] = A.type[j];
  B.lag[i] = A.lag[j];
  const uint32_t s = bv.group_scene[i / kSegAlign];
  const DevParams& P = bv.params[s];
  keys[i] = i < bv.seg_end[s] ? morton_key(x, P.origin, P.scales) : kPadKey;
}

// Cell ranges of every scene into its own table (CalculateBlocksKernel,
// particles_kernel.cu:693-726, per scene).
__global__ void __launch_bounds__(kBlock) k_cell_ranges_batch(const BatchView bv, const uint32_t* __restrict__ seg_begin,
                                                               uint32_t nslots, const uint32_t* __restrict__ keys,
                                                               uint32_t* __restrict__ cstart,
                                                               uint32_t* __restrict__ cend) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nslots) return;
  const uint32_t s = bv.group_scene[i / kSegAlign];
  const uint32_t b = seg_begin[s], e = bv.seg_end[s];
  if (i >= e) return;
  const int shift = 3 * (int)bv.params[s].cell_shift;
  const uint32_t c = keys[i] >> shift;
  const uint32_t base = bv.cell_base[s];
  if (i == b || (keys[i - 1] >> shift) != c) cstart[base + c] = i;
  if (i + 1 == e || (keys[i + 1] >> shift) != c) cend[base + c] = i + 1;
}

__global__ void k_step_init_batch(DevState* st, uint32_t nscenes) {
  for (uint32_t s = threadIdx.x; s < nscenes; s += blockDim.x) {
    st[s].ke = 0;
    st[s].mom[0] = st[s].mom[1] = st[s].mom[2] = 0;
    st[s].max_neighbors = 0;
  }
}

__global__ void k_loop_init_batch(DevState* st, uint32_t nscenes, int32_t* any_active) {
  for (uint32_t s = threadIdx.x; s < nscenes; s += blockDim.x) {
    st[s].iteration = 0;
    st[s].too_large = 1;
    st[s].max_rho_bits = 0;
    st[s].loop_active = 1;
  }
  if (threadIdx.x == 0) *any_active = nscenes > 0;
}

// Loop control of every scene still iterating (each exactly as k_loop_ctl);
// the while-node continues while any scene does.
// Loop control of the batch: the loop test of every scene still iterating;
// the 256-slot groups of the scenes that go on, listed in scene order for
// the resident passes; and for the next iteration, whether the passes run
// over the full grid (while at least half of the groups iterate) or over the
// list. One CTA of 1024 threads.
__global__ void __launch_bounds__(1024) k_loop_ctl_batch(const BatchView bv, uint32_t nscenes, int32_t* any_active,
                                                         const uint32_t* __restrict__ seg_begin, uint32_t total_groups,
                                                         uint32_t* __restrict__ groups, uint32_t* __restrict__ ngroups,
                                                         cudaGraphConditionalHandle h,
                                                         cudaGraphConditionalHandle h_full,
                                                         cudaGraphConditionalHandle h_list, int use_handle) {
  __shared__ uint32_t warp_sums[32];
  int any = 0;
  uint32_t mine = 0;  // groups of this thread's active scenes
  for (uint32_t s = threadIdx.x; s < nscenes; s += blockDim.x) {
    DevState* st = bv.st + s;
    if (!st->loop_active) continue;
    const int cont = loop_ctl(bv.params[s], st);
    st->loop_active = cont;
    any |= cont;
    if (cont) mine += (bv.seg_end[s] - seg_begin[s] + kSegAlign - 1) / kSegAlign;
  }
  any = __syncthreads_or(any);
  // exclusive scan of the threads' group counts
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = mine;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += v;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0u;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, w, d);
      if (lane >= d) w += v;
    }
    warp_sums[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  uint32_t at = (warp ? warp_sums[warp - 1] : 0u) + incl - mine;
  for (uint32_t s = threadIdx.x; s < nscenes; s += blockDim.x) {
    if (!bv.st[s].loop_active) continue;
    const uint32_t g0 = seg_begin[s] / kSegAlign;
    const uint32_t ng = (bv.seg_end[s] - seg_begin[s] + kSegAlign - 1) / kSegAlign;
    for (uint32_t k = 0; k < ng; ++k) groups[at++] = g0 + k;
  }
  if (threadIdx.x == 0) {
    const uint32_t total = warp_sums[(blockDim.x >> 5) - 1];
    *ngroups = total;
    *any_active = any;
    if (use_handle) {
      const bool full = 2 * total >= total_groups;
      cudaGraphSetConditional(h, any ? 1u : 0u);
      cudaGraphSetConditional(h_full, (any && full) ? 1u : 0u);
      cudaGraphSetConditional(h_list, (any && !full) ? 1u : 0u);
    }
  }
}

// Integration for PCISPH: force + pressure force (UnifiedPhysics.cpp:3710-3712),
// and the lagged pressure state carried to the next step.
template <bool kBatch>
__global__ void __launch_bounds__(kBlock) k_pcisph_integrate(
    const __grid_constant__ DevParams Pk, const BatchView bv, uint32_t n, DynArrays B, DynArrays A,
    uint32_t* __restrict__ keysA, const float4* __restrict__ force, const float4* __restrict__ pforce,
    const float* __restrict__ rho, const float* __restrict__ press, DevState* __restrict__ st_plain) {
  __shared__ DevParams sP;
  const Scope sc = enter_scope<kBatch>(Pk, nullptr, st_plain, n, bv, &sP, false);
  if (kBatch) __syncthreads();
  const DevParams& P = *sc.P;
  DevState* st = sc.st;
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  double ke = 0, mx = 0, my = 0, mz = 0;
  if (i < sc.end) {
    const int32_t ti = B.type[i];
    const float4 xi = B.pos[i], vi = B.vel[i];
    const float4 lag = B.lag[i];
    if (ti == UPF_LIQUID) {
      const float4 F = force[i], Fp = pforce[i];
      integrate_store(P, i, xi, vi, make_float3(F.x + Fp.x, F.y + Fp.y, F.z + Fp.z), A, keysA, B, ke, mx, my,
                      mz);
      A.lag[i] = make_float4(lag.y, press[i], rho[i], 0.0f);
    } else if (ti == UPF_GRANULAR) {
      // integrated and clamped like liquid, without a pressure force; not
      // part of the liquid statistics
      const float4 F = force[i];
      integrate_store(P, i, xi, vi, make_float3(F.x, F.y, F.z), A, keysA, B, ke, mx, my, mz);
      if (ke == ke) ke = 0;
      mx = my = mz = 0;
      A.lag[i] = lag;
    } else {
      // rigid particles are placed by the body sync that follows
      A.pos[i] = xi;
      A.vel[i] = vi;
      keysA[i] = morton_key(xi, P.origin, P.scales);
      A.lag[i] = lag;
    }
    A.id[i] = B.id[i];
    A.type[i] = ti;
  } else if (kBatch && i < n) {
    keysA[i] = kPadKeyBatch;  // padding slots sort after the scene's particles
  }
  if (!(ke == ke)) {
    atomicOr(&st->error_flags, (uint32_t)ERR_NAN);
    ke = 0;
  }
  block_stats(st, ke, mx, my, mz);
}

// Akinci volume of the static boundary (CalculateWeightedVolume,
// UnifiedPhysics.cpp:2703-2746): V_b = 1 / sum over boundary neighbours of W.
__global__ void __launch_bounds__(kBlock) k_static_wvol(DevParams P, uint32_t ns, const float4* __restrict__ spos,
                                                         const uint32_t* __restrict__ sstart,
                                                         const uint32_t* __restrict__ send,
                                                         const float* __restrict__ luts, float* __restrict__ wvol) {
  __shared__ float m4[UPF_LUT_ENTRIES];
  stage_lut(m4, luts + LUT_M4 * UPF_LUT_ENTRIES);
  __syncthreads();
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  const float4 xi = spos[i];
  const float h = P.h;
  int lo[3], hi[3];
  const float c[3] = {(xi.x - P.origin.x) * P.scales.x, (xi.y - P.origin.y) * P.scales.y,
                      (xi.z - P.origin.z) * P.scales.z};
  const float r[3] = {h * P.scales.x, h * P.scales.y, h * P.scales.z};
  for (int a = 0; a < 3; ++a) {
    float l = c[a] - r[a] - 1.0f, u = c[a] + r[a] + 1.0f;
    int li = (l <= 0.0f) ? 0 : (l >= 1023.0f ? 1023 : (int)l);
    int ui = (u <= 0.0f) ? 0 : (u >= 1023.0f ? 1023 : (int)u);
    lo[a] = li >> P.cell_shift;
    hi[a] = ui >> P.cell_shift;
  }
  // accumulate in the reference's ascending order: blocks by Morton code
  uint32_t codes[64];
  int m = 0;
  const int nblk = (hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
  float inv = 0.0f;
  auto visit = [&](uint32_t cc) {
    for (uint32_t j = sstart[cc]; j < send[cc]; ++j) {
      if (j == i) continue;
      float d = dist3(xi, spos[j]);
      if (d < h) inv += lut_at(m4, d, P.lut_factor);
    }
  };
  if (nblk <= 64) {
    for (int bz = lo[2]; bz <= hi[2]; ++bz)
      for (int by = lo[1]; by <= hi[1]; ++by)
        for (int bx = lo[0]; bx <= hi[0]; ++bx) {
          uint32_t cc = morton3(bx, by, bz);
          int q = m++;
          while (q > 0 && codes[q - 1] > cc) {
            codes[q] = codes[q - 1];
            --q;
          }
          codes[q] = cc;
        }
    for (int q = 0; q < m; ++q) visit(codes[q]);
  } else {
    for (int bz = lo[2]; bz <= hi[2]; ++bz)
      for (int by = lo[1]; by <= hi[1]; ++by)
        for (int bx = lo[0]; bx <= hi[0]; ++bx) visit(morton3(bx, by, bz));
  }
  if (inv != 0.0f) wvol[i] = (float)(1.0 / (double)inv);
}

inline uint32_t grid_of(uint32_t n) { return (n + kBlock - 1) / kBlock; }

// ---- launches of the tunable passes at a LaunchShape
template <bool kBatch>
cudaError_t run_nlist(const LaunchShape& sh, cudaStream_t st, const DevParams& P, const BatchView& bv, uint32_t n,
                      const float4* pos, const uint32_t* keys, const uint32_t* cstart, const uint32_t* cend,
                      uint32_t ns, const float4* spos, const uint32_t* skeys, const uint32_t* sstart,
                      const uint32_t* send, uint32_t* nbr, uint32_t* lval, uint32_t* ncnt, const float* luts,
                      DevState* stp) {
#define UPF_NL(T, W)                                                                                          \
  k_build_nlist<kBatch, T, W><<<(n + T - 1) / T, T, 0, st>>>(P, bv, n, pos, keys, cstart, cend, ns, spos, skeys, \
                                                             sstart, send, nbr, lval, ncnt, luts, stp)
  switch (sh.nlist_threads * 10 + sh.nlist_mode) {
    case 640: UPF_NL(64, false); break;
    case 1280: UPF_NL(128, false); break;
    case 2560: UPF_NL(256, false); break;
    case 641: UPF_NL(64, true); break;
    case 1281: UPF_NL(128, true); break;
    case 2561: UPF_NL(256, true); break;
    default: return cudaErrorInvalidConfiguration;
  }
#undef UPF_NL
  return cudaGetLastError();
}

template <bool kBatch>
cudaError_t run_external(const LaunchShape& sh, cudaStream_t st, const DevParams& P, const BatchView& bv, uint32_t n,
                         const DynArrays& B, const float* wvol, const int32_t* id_body, const uint32_t* nbr,
                         const uint32_t* ncnt, const float* luts, float4* force, float4* pforce, float4* xs,
                         float* press, float4* pq, DevState* stp) {
#define UPF_EXT(T)                                                                                        \
  k_pcisph_external<kBatch, T><<<(n + T - 1) / T, T, 0, st>>>(P, bv, n, B, wvol, id_body, nbr, ncnt, luts, \
                                                              force, pforce, xs, press, pq, stp)
  switch (sh.external_threads) {
    case 128: UPF_EXT(128); break;
    case 256: UPF_EXT(256); break;
    default: return cudaErrorInvalidConfiguration;
  }
#undef UPF_EXT
  return cudaGetLastError();
}

// (mode, threads, rows): TMA ring pairs and direct-load pairs (see kLoopShapes)
#define UPF_SHAPE_SWITCH(mode, threads, rows, CALL)        \
  switch ((mode) * 1000000 + (threads) * 100 + (rows)) {   \
    case 12804: CALL(false, 128, 4); break;                \
    case 12808: CALL(false, 128, 8); break;                \
    case 12816: CALL(false, 128, 16); break;               \
    case 25602: CALL(false, 256, 2); break;                \
    case 25604: CALL(false, 256, 4); break;                \
    case 25608: CALL(false, 256, 8); break;                \
    case 51202: CALL(false, 512, 2); break;                \
    case 51204: CALL(false, 512, 4); break;                \
    case 102402: CALL(false, 1024, 2); break;              \
    case 1012804: CALL(true, 128, 4); break;               \
    case 1012808: CALL(true, 128, 8); break;               \
    case 1025604: CALL(true, 256, 4); break;               \
    case 1025608: CALL(true, 256, 8); break;               \
    case 1051204: CALL(true, 512, 4); break;               \
    case 1051208: CALL(true, 512, 8); break;               \
    default: return cudaErrorInvalidConfiguration;          \
  }

template <bool kBatch>
cudaError_t run_density(const LaunchShape& sh, cudaStream_t st, const DevParams& P, const BatchView& bv, uint32_t n,
                        const int32_t* type, const float4* xs, const CUtensorMap* cmaps, const uint32_t* nbr,
                        const uint32_t* ncnt, const float* luts, float* rho, float* press, float4* pq,
                        DevState* stp) {
#define UPF_DEN(D, T, R)                                                                                   \
  k_pcisph_density<kBatch, D, T, R><<<(n + T - 1) / T, T, 0, st>>>(P, bv, n, type, xs, cmaps[rows_index(R)], \
                                                                   nbr, ncnt, luts, rho, press, pq, stp)
  UPF_SHAPE_SWITCH(sh.density_mode, sh.density_threads, sh.density_rows, UPF_DEN)
#undef UPF_DEN
  return cudaGetLastError();
}

template <bool kBatch>
cudaError_t run_pforce(const LaunchShape& sh, cudaStream_t st, const DevParams& P, const BatchView& bv, uint32_t n,
                       const DynArrays& B, const CUtensorMap* cmaps, const CUtensorMap* vmaps, const uint32_t* nbr,
                       const uint32_t* lval, const uint32_t* ncnt, const float* luts, const float4* pq,
                       const float4* force, float4* pforce, float4* xs, DevState* stp) {
  // shapes whose ring does not fit are neither built nor launched
#define UPF_PF(D, T, R)                                                                                             \
  if constexpr (pforce_ring_fits(D ? 1 : 0, T, R)) {                                                                \
    k_pcisph_pressure_force<kBatch, D, T, R><<<(n + T - 1) / T, T, 0, st>>>(                                        \
        P, bv, n, B, cmaps[rows_index(R)], vmaps[rows_index(R)], nbr, lval, ncnt, luts, pq, force, pforce, xs, stp); \
  } else {                                                                                                          \
    return cudaErrorInvalidConfiguration;                                                                          \
  }
  UPF_SHAPE_SWITCH(sh.pforce_mode, sh.pforce_threads, sh.pforce_rows, UPF_PF)
#undef UPF_PF
  return cudaGetLastError();
}
#undef UPF_SHAPE_SWITCH

}  // namespace

// ----------------------------------------------------------------- launchers
cudaError_t launch_sort_phase(System& s, cudaStream_t st) {
  const uint32_t n = s.n_dyn;
  if (n == 0) return cudaSuccess;
  uint32_t* kalt = s.sort_tmp;
  uint32_t* valt = kalt + ((n + 63) & ~63u);
  uint32_t* counts = valt + ((n + 63) & ~63u);
  cudaError_t e = radix_sort_pairs(s.keysA, s.perm, kalt, valt, counts, n, s.key_bits, true, st);
  if (e != cudaSuccess) return e;
  k_reorder<<<grid_of(n), kBlock, 0, st>>>(n, s.perm, s.A, s.B, s.prm.method == UPF_METHOD_PCISPH);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = launch_rigid_slots(s, st)) != cudaSuccess) return e;
  return cell_ranges(s.keysA, n, 3 * (int)s.dp.cell_shift, s.ncells, s.cstart, s.cend, st);
}

// The union and union positions of each chunk's lists (k_stage_lists).
static cudaError_t launch_stage_lists(System& s, cudaStream_t st) {
  const uint32_t n = s.n_dyn;
  k_stage_lists<<<(n + kStageChunk - 1) / kStageChunk, kStageChunk, 0, st>>>(
      n, s.B.type, s.nbr, s.ncnt, s.nstride, s.stage_cap, s.ucodes, s.ucount, s.lloc);
  s.lists_staged = true;
  return cudaGetLastError();
}

cudaError_t launch_list_staging(System& s, cudaStream_t st) {
  return s.n_dyn && s.ucodes ? launch_stage_lists(s, st) : cudaSuccess;
}

// the lists are staged when a loop pass reads staged neighbourhoods (or
// while the autotuner times every mode)
static bool stages_lists(const System& s) {
  return s.ucodes && (s.stage_always || loop_mode_staged(s.shape.density_mode) ||
                      loop_mode_staged(s.shape.pforce_mode));
}

cudaError_t launch_neighbor_phase(System& s, cudaStream_t st) {
  const uint32_t n = s.n_dyn;
  k_step_init<<<1, 1, 0, st>>>(s.st, s.prm.method == UPF_METHOD_WCSPH ? 1 : 0);
  if (n == 0) return cudaGetLastError();
  s.lists_staged = false;
  cudaError_t e = run_nlist<false>(s.shape, st, s.dp, BatchView{}, n, s.B.pos, s.keysA, s.cstart, s.cend, s.n_static,
                                   s.spos, s.skeys, s.sstart, s.send, s.nbr, s.lval, s.ncnt, s.luts, s.st);
  if (e != cudaSuccess || !stages_lists(s)) return e;
  return launch_stage_lists(s, st);
}

cudaError_t launch_force_phase(System& s, cudaStream_t st) {
  const uint32_t n = s.n_dyn;
  if (n == 0) return cudaSuccess;
  if (s.prm.method == UPF_METHOD_WCSPH) {
    k_wcsph_density<<<grid_of(n), kBlock, 0, st>>>(s.dp, n, s.B.pos, s.B.type, s.lval, s.ncnt, s.luts, s.rho,
                                                   s.press);
  } else {
    return run_external<false>(s.shape, st, s.dp, BatchView{}, n, s.B, s.wvol, s.rb.id_body, s.nbr, s.ncnt, s.luts,
                               s.force, s.pforce, s.xs, s.press, s.pq, s.st);
  }
  return cudaGetLastError();
}

cudaError_t launch_loop_init(System& s, cudaStream_t st) {
  k_loop_init<<<1, 1, 0, st>>>(s.st);
  return cudaGetLastError();
}

cudaError_t launch_loop_density(System& s, cudaStream_t st) {
  const uint32_t n = s.n_dyn;
  if (n && loop_mode_staged(s.shape.density_mode)) {
    // lists built under another shape (phase by phase) are staged first
    if (!s.lists_staged) {
      cudaError_t e = launch_stage_lists(s, st);
      if (e != cudaSuccess) return e;
    }
    const uint32_t g = (n + kStageChunk - 1) / kStageChunk;
    if (s.shape.density_rows == 4)
      k_pcisph_density_staged<4><<<g, kStageChunk, 0, st>>>(s.dp, n, s.B.type, s.xs, s.nbr, s.ncnt, s.ucodes,
                                                           s.ucount, s.lloc, s.luts, s.rho, s.press, s.pq, s.st);
    else if (s.shape.density_rows == 8)
      k_pcisph_density_staged<8><<<g, kStageChunk, 0, st>>>(s.dp, n, s.B.type, s.xs, s.nbr, s.ncnt, s.ucodes,
                                                           s.ucount, s.lloc, s.luts, s.rho, s.press, s.pq, s.st);
    else
      return cudaErrorInvalidConfiguration;
    return cudaGetLastError();
  }
  if (n)
    return run_density<false>(s.shape, st, s.dp, BatchView{}, n, s.B.type, s.xs, s.nbr_maps, s.nbr, s.ncnt, s.luts, s.rho,
                              s.press, s.pq, s.st);
  return cudaGetLastError();
}

cudaError_t launch_loop_pforce(System& s, cudaStream_t st) {
  const uint32_t n = s.n_dyn;
  if (n && loop_mode_staged(s.shape.pforce_mode)) {
    if (!s.lists_staged) {
      cudaError_t e = launch_stage_lists(s, st);
      if (e != cudaSuccess) return e;
    }
    const uint32_t g = (n + kStageChunk - 1) / kStageChunk;
    if (s.shape.pforce_rows == 4)
      k_pcisph_pressure_force_staged<4><<<g, kStageChunk, 0, st>>>(s.dp, n, s.B, s.nbr, s.lval, s.ncnt, s.ucodes,
                                                                  s.ucount, s.lloc, s.pq, s.force, s.pforce, s.xs,
                                                                  s.st);
    else if (s.shape.pforce_rows == 8)
      k_pcisph_pressure_force_staged<8><<<g, kStageChunk, 0, st>>>(s.dp, n, s.B, s.nbr, s.lval, s.ncnt, s.ucodes,
                                                                  s.ucount, s.lloc, s.pq, s.force, s.pforce, s.xs,
                                                                  s.st);
    else
      return cudaErrorInvalidConfiguration;
    return cudaGetLastError();
  }
  if (n)
    return run_pforce<false>(s.shape, st, s.dp, BatchView{}, n, s.B, s.nbr_maps, s.lval_maps, s.nbr, s.lval, s.ncnt, s.luts, s.pq,
                             s.force, s.pforce, s.xs, s.st);
  return cudaGetLastError();
}

cudaError_t launch_loop_ctl(System& s, cudaStream_t st, cudaGraphConditionalHandle h, bool use_handle) {
  k_loop_ctl<<<1, 1, 0, st>>>(s.dp, s.st, h, use_handle ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_loop_body(System& s, cudaStream_t st, cudaGraphConditionalHandle h, bool use_handle) {
  cudaError_t e = launch_loop_density(s, st);
  if (e != cudaSuccess) return e;
  if ((e = launch_loop_pforce(s, st)) != cudaSuccess) return e;
  return launch_loop_ctl(s, st, h, use_handle);
}

cudaError_t launch_upload_keys(System& s, cudaStream_t st) {
  return morton_keys(s.A.pos, s.n_dyn, s.dp.origin, s.dp.scales, s.keysA, st);
}

cudaError_t launch_integrate_phase(System& s, cudaStream_t st) {
  const uint32_t n = s.n_dyn;
  if (n == 0) return cudaSuccess;
  if (s.prm.method == UPF_METHOD_WCSPH) {
    k_wcsph_force_integrate<<<grid_of(n), kBlock, 0, st>>>(s.dp, n, s.B, s.A, s.keysA, s.nbr, s.lval, s.ncnt,
                                                           s.luts, s.rho, s.press, s.force, s.st);
  } else {
    k_pcisph_integrate<false><<<grid_of(n), kBlock, 0, st>>>(s.dp, BatchView{}, n, s.B, s.A, s.keysA, s.force, s.pforce, s.rho, s.press,
                                                      s.st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_rigid_phase(s, st);
  }
  return cudaGetLastError();
}

cudaError_t launch_static_setup(System& s, cudaStream_t st) {
  // boundary set: keys -> stable sort -> gather -> cell ranges -> Akinci volumes
  const uint32_t ns = s.n_static;
  cudaError_t e = cudaMemsetAsync(s.sstart, 0, sizeof(uint32_t) * s.ncells, st);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(s.send, 0, sizeof(uint32_t) * s.ncells, st);
  if (e != cudaSuccess) return e;
  if (ns == 0) return cudaSuccess;
  e = cell_ranges(s.skeys, ns, 3 * (int)s.dp.cell_shift, s.ncells, s.sstart, s.send, st);
  if (e != cudaSuccess) return e;
  k_static_wvol<<<grid_of(ns), kBlock, 0, st>>>(s.dp, ns, s.spos, s.sstart, s.send, s.luts,
                                                 s.wvol + s.dp.static_base);
  return cudaGetLastError();
}

// Neighbour lists of one sorted set with no boundary set (the adjoint's
// per-step lists); P.nstride is the list stride, P.maxn its rows.
cudaError_t launch_nlist_plain(const DevParams& P, uint32_t n, const float4* pos, const uint32_t* keys,
                               const uint32_t* cstart, const uint32_t* cend, uint32_t* nbr, uint32_t* lval,
                               uint32_t* ncnt, const float* luts, DevState* st, cudaStream_t stream) {
  if (!n) return cudaSuccess;
  return run_nlist<false>(LaunchShape{}, stream, P, BatchView{}, n, pos, keys, cstart, cend, 0u, nullptr, nullptr,
                          nullptr, nullptr, nbr, lval, ncnt, luts, st);
}

// ----------------------------------------------------------- batched launchers
cudaError_t batch_launch_init(BatchSystem& b, cudaStream_t st) {
  if (!b.n_slots) return cudaSuccess;
  k_batch_init<<<grid_of(b.n_slots), kBlock, 0, st>>>(b.view, b.n_slots, b.A, b.keysA, 1);
  return cudaGetLastError();
}

cudaError_t batch_launch_keys(BatchSystem& b, cudaStream_t st) {
  if (!b.n_slots) return cudaSuccess;
  k_batch_init<<<grid_of(b.n_slots), kBlock, 0, st>>>(b.view, b.n_slots, b.A, b.keysA, 0);
  return cudaGetLastError();
}

// Two stable LSD stages: the Morton keys (padding above them), then the
// scene index; each scene's particles end up in its own segment in Morton
// order, exactly the order a sort of that scene alone gives.
cudaError_t batch_launch_sort(BatchSystem& b, cudaStream_t st) {
  const uint32_t n = b.n_slots;
  if (!n) return cudaSuccess;
  uint32_t* kalt = b.sort_tmp;
  uint32_t* valt = kalt + ((n + 63) & ~63u);
  uint32_t* counts = valt + ((n + 63) & ~63u);
  cudaError_t e = radix_sort_pairs(b.keysA, b.perm, kalt, valt, counts, n, 31, true, st);
  if (e != cudaSuccess) return e;
  k_scene_digits<<<grid_of(n), kBlock, 0, st>>>(n, b.perm, b.group_scene_d, b.digits);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  e = radix_sort_pairs(b.digits, b.perm, kalt, valt, counts, n, b.scene_bits, false, st);
  if (e != cudaSuccess) return e;
  k_reorder_batch<<<grid_of(n), kBlock, 0, st>>>(b.view, n, b.perm, b.A, b.B, b.keysA);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(b.cstart, 0, sizeof(uint32_t) * b.n_cells, st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(b.cend, 0, sizeof(uint32_t) * b.n_cells, st)) != cudaSuccess) return e;
  k_cell_ranges_batch<<<grid_of(n), kBlock, 0, st>>>(b.view, b.seg_begin_d, n, b.keysA, b.cstart, b.cend);
  return cudaGetLastError();
}

cudaError_t batch_launch_neighbors(BatchSystem& b, cudaStream_t st) {
  const uint32_t n = b.n_slots;
  k_step_init_batch<<<1, 256, 0, st>>>(b.st_d, b.n_scenes);
  if (!n) return cudaGetLastError();
  return run_nlist<true>(b.shape, st, DevParams{}, b.view, n, b.B.pos, b.keysA, b.cstart, b.cend, 0u, nullptr, nullptr,
                         nullptr, nullptr, b.nbr, b.lval, b.ncnt, nullptr, nullptr);
}

cudaError_t batch_launch_forces(BatchSystem& b, cudaStream_t st) {
  const uint32_t n = b.n_slots;
  if (!n) return cudaSuccess;
  return run_external<true>(b.shape, st, DevParams{}, b.view, n, b.B, nullptr, nullptr, b.nbr, b.ncnt, nullptr,
                            b.force, b.pforce, b.xs, b.press, b.pq, nullptr);
}

cudaError_t batch_launch_loop_init(BatchSystem& b, cudaStream_t st) {
  k_loop_init_batch<<<1, 256, 0, st>>>(b.st_d, b.n_scenes, b.any_active_d);
  return cudaGetLastError();
}

cudaError_t batch_launch_loop_density(BatchSystem& b, cudaStream_t st) {
  const uint32_t n = b.n_slots;
  if (n)
    return run_density<true>(b.shape, st, DevParams{}, b.view, n, b.B.type, b.xs, b.nbr_maps, b.nbr, b.ncnt, nullptr, b.rho,
                             b.press, b.pq, nullptr);
  return cudaGetLastError();
}

cudaError_t batch_launch_loop_pforce(BatchSystem& b, cudaStream_t st) {
  const uint32_t n = b.n_slots;
  if (n)
    return run_pforce<true>(b.shape, st, DevParams{}, b.view, n, b.B, b.nbr_maps, b.lval_maps, b.nbr, b.lval, b.ncnt, nullptr, b.pq,
                            b.force, b.pforce, b.xs, nullptr);
  return cudaGetLastError();
}

cudaError_t batch_launch_loop_ctl(BatchSystem& b, cudaStream_t st, cudaGraphConditionalHandle h, bool use_handle) {
  k_loop_ctl_batch<<<1, 1024, 0, st>>>(b.view, b.n_scenes, b.any_active_d, b.seg_begin_d, b.n_slots / kSegAlign,
                                       b.active_groups_d, b.n_active_groups_d, h, 0, 0, 0);
  (void)use_handle;  // the host-driven loop reads any_active
  return cudaGetLastError();
}

// The loop passes over the active groups only, on a resident grid.
constexpr int kActiveRows = 4;
static cudaError_t active_grid_of(BatchSystem& b) {
  constexpr int kR = kActiveRows;
  if (!b.active_grid) {
    int dev = 0, sms = 0, per_sm_d = 0, per_sm_p = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_d, k_pcisph_density_active<kR>, kSegAlign, 0);
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_p, k_pcisph_pressure_force_active<kR>, kSegAlign, 0);
    if (e != cudaSuccess) return e;
    b.active_grid = (uint32_t)(sms * std::max(1, std::min(per_sm_d, per_sm_p)));
  }
  return cudaSuccess;
}

cudaError_t batch_launch_loop_density_active(BatchSystem& b, cudaStream_t st) {
  cudaError_t e = active_grid_of(b);
  if (e != cudaSuccess) return e;
  k_pcisph_density_active<kActiveRows><<<b.active_grid, kSegAlign, 0, st>>>(
      b.view, b.n_slots, b.active_groups_d, b.n_active_groups_d, b.B.type, b.xs, b.nbr, b.ncnt, b.rho, b.press, b.pq);
  return cudaGetLastError();
}

cudaError_t batch_launch_loop_pforce_active(BatchSystem& b, cudaStream_t st) {
  cudaError_t e = active_grid_of(b);
  if (e != cudaSuccess) return e;
  k_pcisph_pressure_force_active<kActiveRows><<<b.active_grid, kSegAlign, 0, st>>>(
      b.view, b.n_slots, b.active_groups_d, b.n_active_groups_d, b.B, b.nbr, b.lval, b.ncnt, b.pq, b.force, b.pforce,
      b.xs);
  return cudaGetLastError();
}

cudaError_t batch_launch_loop_active(BatchSystem& b, cudaStream_t st) {
  cudaError_t e = batch_launch_loop_density_active(b, st);
  return e == cudaSuccess ? batch_launch_loop_pforce_active(b, st) : e;
}

// An IF node at the capture point of `st` (capturing into a graph) whose
// body `fn` captures; the capture goes on after the node.
template <class Fn>
cudaError_t capture_if(cudaStream_t st, unsigned int default_value, cudaGraphConditionalHandle* h, Fn&& fn) {
  cudaStreamCaptureStatus cst;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  cudaError_t e = cudaStreamGetCaptureInfo(st, &cst, nullptr, &g, &deps, &ndeps);
  if (e != cudaSuccess) return e;
  if ((e = cudaGraphConditionalHandleCreate(h, g, default_value, cudaGraphCondAssignDefault)) != cudaSuccess) return e;
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = *h;
  np.conditional.type = cudaGraphCondTypeIf;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  if ((e = cudaGraphAddNode(&node, g, deps, ndeps, &np)) != cudaSuccess) return e;
  cudaGraph_t body = np.conditional.phGraph_out[0];
  if ((e = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies)) != cudaSuccess)
    return e;
  cudaStream_t bs = nullptr;
  if ((e = cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking)) != cudaSuccess) return e;
  e = cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    const cudaError_t eb = fn(bs);
    cudaGraph_t out = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(bs, &out);
    e = eb != cudaSuccess ? eb : ee;
  }
  cudaStreamDestroy(bs);
  return e;
}

cudaError_t batch_capture_loop_body(BatchSystem& b, cudaStream_t st, cudaGraphConditionalHandle h) {
  // every scene iterates in the first iteration: the full grid by default
  cudaGraphConditionalHandle h_full = 0, h_list = 0;
  cudaError_t e = capture_if(st, 1u, &h_full, [&](cudaStream_t bs) {
    cudaError_t r = batch_launch_loop_density(b, bs);
    return r == cudaSuccess ? batch_launch_loop_pforce(b, bs) : r;
  });
  if (e != cudaSuccess) return e;
  e = capture_if(st, 0u, &h_list, [&](cudaStream_t bs) { return batch_launch_loop_active(b, bs); });
  if (e != cudaSuccess) return e;
  k_loop_ctl_batch<<<1, 1024, 0, st>>>(b.view, b.n_scenes, b.any_active_d, b.seg_begin_d, b.n_slots / kSegAlign,
                                       b.active_groups_d, b.n_active_groups_d, h, h_full, h_list, 1);
  return cudaGetLastError();
}

cudaError_t batch_launch_loop_body(BatchSystem& b, cudaStream_t st, cudaGraphConditionalHandle h, bool use_handle) {
  cudaError_t e = batch_launch_loop_density(b, st);
  if (e == cudaSuccess) e = batch_launch_loop_pforce(b, st);
  if (e == cudaSuccess) e = batch_launch_loop_ctl(b, st, h, use_handle);
  return e;
}

cudaError_t batch_launch_integrate(BatchSystem& b, cudaStream_t st) {
  const uint32_t n = b.n_slots;
  if (!n) return cudaSuccess;
  k_pcisph_integrate<true><<<grid_of(n), kBlock, 0, st>>>(DevParams{}, b.view, n, b.B, b.A, b.keysA, b.force,
                                                          b.pforce, b.rho, b.press, nullptr);
  return cudaGetLastError();
}

int pipeline_launches_per_step(const System& s, int iterations) {
  int sort = radix_launches(s.key_bits) + 1 /*reorder*/ + 1 /*cells*/ + (s.rb.n_rigid ? 1 : 0) /*rigid slots*/;
  int nl = 2 + (stages_lists(s) ? 1 : 0);  // step init + neighbour lists (+ staging)
  if (s.prm.method == UPF_METHOD_WCSPH) return sort + nl + 2;
  return sort + nl + 1 /*external*/ + 1 /*loop init*/ + 3 * iterations + 1 /*integrate*/ + rigid_launches_per_step(s);
}

}  // namespace upf
