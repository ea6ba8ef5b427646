// upf_noalloc.cu — a radix sort entry point that allocates nothing.
//
// upf_radix_sort_pairs needs scratch of upf_radix_sort_temp_bytes(n), which
// its caller allocates. Some callers cannot call cudaMalloc: hosts that own all
// device memory through their own pool or arena and forbid libraries from
// allocating, and per-frame loops that must not pay cudaMalloc's implicit
// device synchronisation. upf_radix_sort_pairs_noalloc serves them with scratch
// in a file-scope __device__ array of fixed size, which every GPU that loads
// this library holds until the process exits.
#include <cuda_runtime.h>

#include <mutex>

#include "upf_internal.h"

namespace upf {
namespace {

constexpr uint32_t kNoAllocMaxPairs = UPF_NOALLOC_MAX_PAIRS;
constexpr size_t kPad = ((size_t)kNoAllocMaxPairs + 63) & ~size_t(63);
constexpr size_t kNoAllocWords = 2 * kPad + radix_count_words(kNoAllocMaxPairs);

// keys_alt | vals_alt | digit counts, laid out as upf_radix_sort_pairs lays out
// its caller's scratch (17 MB for the 2^21-pair maximum)
__device__ __align__(256) uint32_t g_sort_scratch[kNoAllocWords];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
uint32_t* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device. In host code
// g_sort_scratch names a host-side stand-in, so its device address is looked
// up once per device (with that device current) and cached.
upf_status scratch_for_current_device(uint32_t** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error("upf_radix_sort_pairs_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
    return UPF_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("upf_radix_sort_pairs_noalloc: device %d beyond the supported %d", dev, kMaxDevices);
    return UPF_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_addr[dev]) {
    e = radix_init();
    if (e != cudaSuccess) {
      set_error("upf_radix_sort_pairs_noalloc: set-up: %s", cudaGetErrorString(e));
      return UPF_ERR_CUDA;
    }
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_sort_scratch);
    if (e != cudaSuccess || !p) {
      set_error("upf_radix_sort_pairs_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      return UPF_ERR_CUDA;
    }
    g_scratch_addr[dev] = (uint32_t*)p;
  }
  *out = g_scratch_addr[dev];
  return UPF_OK;
}

}  // namespace
}  // namespace upf

using namespace upf;

extern "C" upf_status upf_radix_sort_pairs_noalloc(uint32_t* keys, uint32_t* vals, uint32_t n, int32_t key_bits,
                                                   void* stream) {
  if (n == 0) return UPF_OK;
  if (!keys || !vals || key_bits < 1 || key_bits > 32) {
    set_error("upf_radix_sort_pairs_noalloc: bad arguments");
    return UPF_ERR_INVALID_ARG;
  }
  if (n > kNoAllocMaxPairs) {
    set_error("upf_radix_sort_pairs_noalloc: %u pairs exceed the fixed scratch maximum of %u "
              "(use upf_radix_sort_pairs with caller scratch)",
              n, kNoAllocMaxPairs);
    return UPF_ERR_INVALID_ARG;
  }
  uint32_t* scratch = nullptr;
  upf_status st = scratch_for_current_device(&scratch);
  if (st != UPF_OK) return st;
  // the sort writes every word of the scratch it reads (the digit counts are
  // rebuilt by each pass's upsweep), so nothing has to be cleared between calls
  uint32_t* kalt = scratch;
  uint32_t* valt = kalt + ((n + 63) & ~63u);
  uint32_t* counts = valt + ((n + 63) & ~63u);
  cudaError_t e = radix_sort_pairs(keys, vals, kalt, valt, counts, n, key_bits, false, (cudaStream_t)stream);
  if (e != cudaSuccess) {
    set_error("upf_radix_sort_pairs_noalloc: %s", cudaGetErrorString(e));
    return UPF_ERR_CUDA;
  }
  return UPF_OK;
}
