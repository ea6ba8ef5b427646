// upf_internal.h — declarations shared between the library's translation
// units (not part of the public ABI).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/upf.h"

namespace upf {

struct DevParams;
struct DevState;

// upf_params.cpp (host math, compiled with -ffp-contract=off)
void default_params(upf_params* p);
int derive_params(upf_params* p, double* delta_fp64);
void build_luts(const upf_params& p, float* out_5x301);
float kernel_self(float h);
void build_bin_thresholds(const upf_params& p, float* out_302);
int validate_params(const upf_params& p, const char** why);
uint32_t default_search_cell(const upf_params& p);
uint32_t effective_search_cell(const upf_params& p);  // p.search_cell, or the default when 0
double density_error_factor(const upf_params& p);

// upf_api.cu: test hook for allocation failures (upf_test_fail_allocation):
// true when the library's next device allocation is the one to fail
bool inject_alloc_failure();

// NVTX ranges around host entry points (header-only NVTX 3: a no-op unless a
// tool is attached)
struct NvtxRange {
  explicit NvtxRange(const char* name);
  ~NvtxRange();
};

// upf_sort.cu
// A sort pass runs one CTA per tile of keys. The tile is the smallest of
// 512, 2048 and 8192 keys (16 warps x 32, 128 or 512) that needs at most
// kRadixTileCap tiles: small inputs get more CTAs than 8192-key tiles would
// give them, while the single-CTA digit scan (256 counts per tile) stays short.
constexpr uint32_t kRadixDigits = 256;  // 8-bit digits
constexpr uint32_t kRadixTileCap = 512;
constexpr uint32_t radix_tile_keys(uint32_t n) {
  return n <= kRadixTileCap * 512u ? 512u : (n <= kRadixTileCap * 2048u ? 2048u : 8192u);
}
constexpr uint32_t radix_tiles(uint32_t n) { return (n + radix_tile_keys(n) - 1) / radix_tile_keys(n); }
// The most tiles of any count up to n: scratch sized for n serves every
// smaller count (a system sorts any number of particles up to its capacity).
constexpr uint32_t radix_tiles_upto(uint32_t n) {
  const uint32_t a = radix_tiles(n);
  const uint32_t b = radix_tiles(n < kRadixTileCap * 512u ? n : kRadixTileCap * 512u);
  const uint32_t c = radix_tiles(n < kRadixTileCap * 2048u ? n : kRadixTileCap * 2048u);
  return a > b ? (a > c ? a : c) : (b > c ? b : c);
}
// digit counts of a sort of up to n keys: [256][tiles] per tile, then the 256
// digit totals
constexpr size_t radix_count_words(uint32_t n) { return (size_t)kRadixDigits * (radix_tiles_upto(n) + 1); }
size_t radix_temp_words(uint32_t n);
size_t radix_temp_bytes(uint32_t n);
cudaError_t radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt,
                             uint32_t* counts, uint32_t n, int key_bits, bool iota_values,
                             cudaStream_t st);
int radix_launches(int key_bits);
cudaError_t radix_init();
cudaError_t morton_keys(const float4* pos, uint32_t n, float3 origin, float3 scales, uint32_t* keys,
                        cudaStream_t st);
cudaError_t cell_ranges(const uint32_t* keys, uint32_t n, int shift, uint32_t ncells, uint32_t* start,
                        uint32_t* end, cudaStream_t st);

// error reporting (upf_api.cu)
void set_error(const char* fmt, ...);

}  // namespace upf
