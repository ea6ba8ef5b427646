// upf_common.cuh — device-side types and helpers shared by the kernels.
//
// Every operation that decides something discrete (neighbour membership,
// lookup-table bin, Morton cell, clamp) is written with explicit
// round-to-nearest intrinsics in the reference CPU path's operation order, so
// that those decisions are bit-identical to the CPU path. The library is
// additionally compiled with -fmad=false so that continuous sums also round
// operation by operation like the CPU path (no contraction into FMA).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/upf.h"

namespace upf {

constexpr int kLut = UPF_LUT_SIZE;
// Bin thresholds: kBinThresholds[b] (b = 1..300) is the smallest float r2 whose
// bin lut_index(sqrt_rn(r2)) is >= b; entry 301 is the smallest r2 with
// sqrt_rn(r2) >= h (outside the support). Built on the host bit-exactly.
constexpr int kThresholds = UPF_LUT_ENTRIES + 1;

enum LutId { LUT_M4 = 0, LUT_PGRAD = 1, LUT_VISC = 2, LUT_ST = 3, LUT_ADH = 4 };

// Error flag bits in DevState::error_flags
enum : uint32_t { ERR_OVERFLOW = 1u, ERR_NAN = 2u, ERR_TIMEOUT = 4u };

// Everything a kernel needs from upf_params, by value.
struct DevParams {
  float h;            // support radius
  float lut_factor;   // (float)(1.0 / h): the reference's function-static factor
  float mass;
  float inv_mass;     // (float)(1.0 / mass)
  float rho0;
  float kernel_self;  // KernelM4(0, h)
  float gas_b;        // rest_density * gas_constant / gamma
  float gamma;
  float visc;
  float rest_volume;  // mass / rho0
  float gravity;
  float dt;
  float delta;        // PCISPH density error factor
  float err_scale;    // 100 / rho0
  float max_err;
  int min_loops, max_loops;
  float st_gamma, adh_beta;
  float force_dist, inv_force_dist, max_boundary_force;
  float radius, spacing;
  float spring, spring_boundary, damping, terminal_speed;
  float gran_kr, gran_kd, gran_kt, gran_mu;
  float3 origin, scales;
  float3 cmin, cmax;       // collision box
  float3 wmin, wmax;       // real container
  uint32_t block_shift;    // log2(block_size)
  uint32_t cell_shift;     // log2(search cell edge): the cell tables and the neighbour search
  uint32_t flags;
  uint32_t maxn;
  uint32_t nstride;        // neighbour-list column stride
  uint32_t static_base;    // neighbour index of boundary particle j is static_base + j
  uint32_t list_grad;      // list values hold the pressure-gradient table value (PCISPH), else the bin
};

// One rigid body (RigidBody, src/cpu/RigidBody.h:105-134): float state as in
// the reference; force and torque arrive from an FP64 reduction.
struct DevBody {
  float mass;
  float3 pos, vel, P, L, omega;
  float q[4];              // (s, x, y, z)
  float rot[3][3];
  float iinv_local[3][3];
  float iinv_world[3][3];
  double force[3];
  double torque[3];
};

// Device-side scalars of one system.
struct DevState {
  uint32_t max_rho_bits;   // running max predicted density (positive floats order as uints)
  int32_t iteration;
  int32_t too_large;
  uint32_t error_flags;
  uint32_t max_neighbors;
  int32_t final_iterations;
  float final_max_rho;
  float final_err;
  double ke;
  double mom[3];
  float iter_max_rho[64];
  int32_t total_steps;
  int32_t total_iterations;
  int32_t steps_at_max;
  float max_step_err;      // largest final density error (percent) of the steps counted above
  int32_t loop_active;     // batched scenes: the scene's predict-correct loop still runs
};

// ---- exact float helpers --------------------------------------------------
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }

// Packed pairs of floats (sm_100's f32x2 arithmetic): one instruction for two
// lanes, each rounded as the scalar operation (round to nearest, no flush of
// subnormals). Used only where a packed product is unpacked before the next
// operation (the density pass's squared distance): a packed product feeding a
// packed add or subtract was measured not to reproduce the scalar results.
__device__ __forceinline__ unsigned long long pk2(float a, float b) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ float2 up2(unsigned long long v) {
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
  return r;
}
__device__ __forceinline__ unsigned long long sub2(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long mul2(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}

// |a - b| as vmml computes it: sqrtf((dx*dx + dy*dy) + dz*dz)
__device__ __forceinline__ float dist3(float4 a, float4 b) {
  float dx = fsub(a.x, b.x), dy = fsub(a.y, b.y), dz = fsub(a.z, b.z);
  return __fsqrt_rn(fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz)));
}

// LUT bin of WeightingKernel::kernel*Lut: int index = dist * factor * 300
__device__ __forceinline__ int lut_index(float d, float factor) {
  return (int)fmul(fmul(d, factor), (float)kLut);
}
// lut_index(sqrt_rn(r2)) from r2 without the correctly rounded square root.
// rsqrtf is within 2 ulp, so r2 * rsqrtf(r2) is within 2^-21 of sqrt(r2);
// scaled down by (1 - 2^-19) it is below the true root and within 2^-18 of
// it. The reference's index, floor of sqrt_rn(r2) * factor * 300 with three
// float roundings, lies within 2^-22 of the exact product, so the guess taken
// from the scaled-down root is that index or one below it (the two differ by
// under 300 * 2^-17.9 < 1): one exact threshold `thr` (kThresholds entries,
// see above) decides. Returns 300 at or beyond the last bin (the tables' zero
// entry); r2 == 0 gives bin 0 (0 * inf = NaN converts to 0).
__device__ __forceinline__ int bin_of_r2(float r2, float factor, const float* thr) {
  const float d = r2 * rsqrtf(r2) * 0.999998092651367188f;  // 1 - 2^-19
  int g = (int)(d * factor * (float)kLut);
  g = g > kLut - 1 ? kLut - 1 : g;
  return g + (thr[g + 1] <= r2 ? 1 : 0);
}

// The same bin without reading the threshold table per pair. The bin
// position x = r2 * rsqrtf(r2) * factor * 300 lies within 300 * (2^-21 +
// 2^-22) < 2.2e-4 of the reference's sqrt_rn(r2) * factor * 300 (rsqrtf
// within 2 ulp, two more roundings here, three there), so wherever x is at
// least kBinEdge = 2^-10 from an integer both truncate to the same bin; only
// within kBinEdge of a bin edge (about 0.2% of pairs, or a non-finite x)
// does the correctly rounded root decide. r2_edge is thr[300], the first r2
// that takes the zero entry: pairs from there on return 300 exactly as
// bin_of_r2 does.
constexpr float kBinEdge = 1.0f / 1024.0f;
__device__ __forceinline__ float rsqrt_approx(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));  // within 2 ulp
  return r;
}
__device__ __forceinline__ int bin_of_r2_edge(float r2, float factor, float r2_edge) {
  // (a subnormal r2 flushes to 0 in the root: x is then NaN or infinite, and
  // the exact root decides)
  const float x = r2 * rsqrt_approx(r2) * factor * (float)kLut;
  int g = (int)x;
  if (!(fabsf(x - (float)g - 0.5f) <= 0.5f - kBinEdge)) g = lut_index(__fsqrt_rn(r2), factor);
  g = g > kLut - 1 ? kLut - 1 : g;
  return r2 < r2_edge ? g : kLut;
}

// PCISPH dist_lut: uint(dist * 300 / h), clamped to 300
__device__ __forceinline__ unsigned dist_lut(float d, float h) {
  unsigned dl = (unsigned)__fdiv_rn(fmul(d, (float)kLut), h);
  return dl > (unsigned)kLut ? (unsigned)kLut : dl;
}

// Morton interleave of a 10-bit coordinate (x -> bits 3i, y -> 3i+1, z -> 3i+2),
// the z_table_ of ZIndex::ZIndex (src/cpu/zIndex.cpp:10-24).
__host__ __device__ __forceinline__ uint32_t spread3(uint32_t v) {
  v &= 0x3FFu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}
__host__ __device__ __forceinline__ uint32_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}

// float -> unsigned short truncation of the key coordinate, clamped to the grid
__device__ __forceinline__ uint32_t grid_coord(float c) {
  if (!(c > 0.0f)) return 0;
  if (c >= 1023.0f) return 1023;
  return (uint32_t)c;
}

// zIndex.CalcIndex(scales * (x - origin))
__device__ __forceinline__ uint32_t morton_key(float4 x, const float3& origin, const float3& scales) {
  uint32_t cx = grid_coord(fmul(scales.x, fsub(x.x, origin.x)));
  uint32_t cy = grid_coord(fmul(scales.y, fsub(x.y, origin.y)));
  uint32_t cz = grid_coord(fmul(scales.z, fsub(x.z, origin.z)));
  return morton3(cx, cy, cz);
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <class T>
__device__ __forceinline__ T warp_max(T v) {
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace upf
