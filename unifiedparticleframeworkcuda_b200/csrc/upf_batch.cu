// upf_batch.cu — batched scenes (include/upf.h, upf_batch_*): many
// independent PCISPH scenes of uneven sizes in one slot space, one launch
// per pass over all of them, one CUDA graph per step.
//
// The reference runs one simulation per process (its device state is
// file-scope, particles_kernel.cu:36-165), so it has no counterpart: a set of
// scenes there is a sequence of processes or of whole runs. Here each scene
// occupies a segment of the slot space that starts on a kSegAlign boundary;
// every CTA of every pass therefore works on one scene and takes that scene's
// parameters, tables and loop state from the batch tables (BatchView). The
// predict-correct loop runs as one while-node for the batch: a scene whose
// loop has finished skips the remaining iterations' passes at CTA entry, so
// each scene's iteration count and result are those of a single-scene run.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "upf_sys.h"

namespace upf {

namespace {

#define UPF_CUDA(call)                                                                       \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) {                                                                 \
      set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
      return UPF_ERR_CUDA;                                                                   \
    }                                                                                        \
  } while (0)

#define UPF_TRY(call)              \
  do {                             \
    upf_status st_ = (call);       \
    if (st_ != UPF_OK) return st_; \
  } while (0)

template <class T>
upf_status balloc(BatchSystem& b, T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  if (inject_alloc_failure()) {
    set_error("cudaMalloc of %zu bytes failed: injected by upf_test_fail_allocation", count * sizeof(T));
    return UPF_ERR_ALLOC;
  }
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e != cudaSuccess) {
    set_error("cudaMalloc of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
    *p = nullptr;
    return UPF_ERR_ALLOC;
  }
  b.allocations.push_back(*p);
  return UPF_OK;
}

uint32_t round_up(uint32_t v, uint32_t a) { return (v + a - 1) / a * a; }

// compact (host) index <-> slot: scatter a compact float4 array into the
// scenes' segments, or gather it back
__global__ void k_batch_scatter(const BatchView bv, const uint32_t* __restrict__ seg_begin,
                                const uint32_t* __restrict__ comp_begin, uint32_t nslots,
                                const float4* __restrict__ a, const float4* __restrict__ b, float4* __restrict__ da,
                                float4* __restrict__ db, int to_slots) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nslots) return;
  const uint32_t s = bv.group_scene[i / kSegAlign];
  if (i >= bv.seg_end[s]) return;
  const uint32_t c = comp_begin[s] + (i - seg_begin[s]);
  if (to_slots) {
    const float4 x = a[c], v = b[c];
    da[i] = make_float4(x.x, x.y, x.z, 0.0f);
    db[i] = make_float4(v.x, v.y, v.z, 0.0f);
  } else {
    da[c] = a[i];
    db[c] = b[i];
  }
}

struct BatchExtra {
  uint32_t* comp_begin_d = nullptr;
  float4* stage_a = nullptr;
  float4* stage_b = nullptr;
};

}  // namespace
}  // namespace upf

using namespace upf;

struct upf_batch : BatchSystem {
  BatchExtra x;
};

namespace {

void destroy_batch_graph(upf_batch* b) {
  if (b->step_exec) cudaGraphExecDestroy(b->step_exec);
  if (b->step_graph) cudaGraphDestroy(b->step_graph);
  b->step_exec = nullptr;
  b->step_graph = nullptr;
}

upf_status build_batch_graph(upf_batch* b) {
  destroy_batch_graph(b);
  GraphParts parts;
  parts.ctx = static_cast<BatchSystem*>(b);
  parts.pre = [](void* c, cudaStream_t st) {
    BatchSystem& B = *static_cast<BatchSystem*>(c);
    cudaError_t e = batch_launch_sort(B, st);
    if (e == cudaSuccess) e = batch_launch_neighbors(B, st);
    if (e == cudaSuccess) e = batch_launch_forces(B, st);
    if (e == cudaSuccess) e = batch_launch_loop_init(B, st);
    return e;
  };
  parts.loop = [](void* c, cudaStream_t st, cudaGraphConditionalHandle h) {
    return batch_capture_loop_body(*static_cast<BatchSystem*>(c), st, h);
  };
  parts.post = [](void* c, cudaStream_t st) { return batch_launch_integrate(*static_cast<BatchSystem*>(c), st); };
  return capture_step_graph(parts, &b->step_graph, &b->step_exec);
}

upf_status batch_guard(upf_batch* b, const char* where) {
  if (!b) {
    set_error("%s: null batch", where);
    return UPF_ERR_INVALID_ARG;
  }
  if (!b->have_particles) {
    set_error("%s: call upf_batch_set_particles first", where);
    return UPF_ERR_STATE;
  }
  return UPF_OK;
}

upf_status batch_check_errors(upf_batch* b) {
  UPF_CUDA(cudaMemcpyAsync(b->st_h, b->st_d, sizeof(DevState) * b->n_scenes, cudaMemcpyDeviceToHost, b->stream));
  UPF_CUDA(cudaStreamSynchronize(b->stream));
  for (uint32_t s = 0; s < b->n_scenes; ++s) {
    const uint32_t f = b->st_h[s].error_flags;
    if (f & ERR_NAN) {
      set_error("scene %u: a particle position became NaN", s);
      return UPF_ERR_NAN;
    }
    if (f & ERR_OVERFLOW) {
      set_error("scene %u: a particle has %u neighbours, more than max_neighbors=%u", s, b->st_h[s].max_neighbors,
                b->prm[s].max_neighbors);
      return UPF_ERR_NEIGHBOR_OVERFLOW;
    }
    if (f & ERR_TIMEOUT) {
      set_error("scene %u: a bounded device-side wait ran out", s);
      return UPF_ERR_TIMEOUT;
    }
  }
  return UPF_OK;
}

}  // namespace

extern "C" {

upf_status upf_batch_create(const upf_params* params, const uint32_t* counts, uint32_t num_scenes, int device,
                            upf_batch** out) {
  NvtxRange nvtx("upf_batch_create");
  if (!out || !params || !counts || num_scenes == 0) {
    set_error("upf_batch_create: null argument or no scenes");
    return UPF_ERR_INVALID_ARG;
  }
  *out = nullptr;
  if (num_scenes > 65536) {
    set_error("upf_batch_create: at most 65536 scenes");
    return UPF_ERR_INVALID_ARG;
  }
  uint64_t total = 0, slots = 0, cells = 0;
  for (uint32_t s = 0; s < num_scenes; ++s) {
    const char* why = nullptr;
    if (validate_params(params[s], &why) != 0) {
      set_error("upf_batch_create: scene %u: invalid parameters: %s", s, why);
      return UPF_ERR_INVALID_ARG;
    }
    if (params[s].method != UPF_METHOD_PCISPH) {
      set_error("upf_batch_create: scene %u: batched scenes use the PCISPH solver", s);
      return UPF_ERR_UNSUPPORTED;
    }
    total += counts[s];
    slots += round_up(counts[s] ? counts[s] : 1, kSegAlign);
    const uint64_t bpa = UPF_GRID_RESOLUTION / effective_search_cell(params[s]);
    cells += bpa * bpa * bpa;
  }
  if (slots >= (1ull << 31) || cells >= (1ull << 32)) {
    set_error("upf_batch_create: batch too large (%llu slots, %llu cells)", (unsigned long long)slots,
              (unsigned long long)cells);
    return UPF_ERR_INVALID_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("upf_batch_create: no CUDA device");
    return UPF_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) {
    set_error("upf_batch_create: device %d out of range (%d devices)", device, ndev);
    return UPF_ERR_INVALID_ARG;
  }
  UPF_CUDA(cudaSetDevice(device));
  UPF_CUDA(radix_init());
  upf_batch* b = new upf_batch();
  b->device = device;
  b->n_scenes = num_scenes;
  b->n_slots = (uint32_t)slots;
  b->n_particles = (uint32_t)total;
  b->n_cells = (uint32_t)cells;
  b->prm.assign(params, params + num_scenes);
  b->count.assign(counts, counts + num_scenes);
  auto bail = [&](upf_status st) {
    upf_batch_destroy(b);
    return st;
  };
  // layout
  std::vector<uint32_t> group_scene(b->n_slots / kSegAlign), comp_begin(num_scenes);
  b->seg_begin.resize(num_scenes);
  b->seg_end.resize(num_scenes);
  b->cell_base.resize(num_scenes);
  uint32_t off = 0, cb = 0, comp = 0, rows = 0;
  for (uint32_t s = 0; s < num_scenes; ++s) {
    const uint32_t padded = round_up(counts[s] ? counts[s] : 1, kSegAlign);
    b->seg_begin[s] = off;
    b->seg_end[s] = off + counts[s];
    for (uint32_t g = off / kSegAlign; g < (off + padded) / kSegAlign; ++g) group_scene[g] = s;
    off += padded;
    b->cell_base[s] = cb;
    const uint32_t bpa = UPF_GRID_RESOLUTION / effective_search_cell(params[s]);
    cb += bpa * bpa * bpa;
    comp_begin[s] = comp;
    comp += counts[s];
    rows = std::max(rows, params[s].max_neighbors);
  }
  b->list_rows = rows;
  int bits = 1;
  while ((1u << bits) < num_scenes) ++bits;
  b->scene_bits = bits;
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    set_error("cudaStreamCreate: %s", cudaGetErrorString(e));
    return bail(UPF_ERR_CUDA);
  }
  b->own_stream = true;
  const size_t n = b->n_slots;
  upf_status st = UPF_OK;
#define ALLOC(ptr, cnt) \
  if ((st = balloc(*b, &(ptr), (cnt))) != UPF_OK) return bail(st);
  ALLOC(b->A.pos, n); ALLOC(b->A.vel, n); ALLOC(b->A.lag, n); ALLOC(b->A.id, n); ALLOC(b->A.type, n);
  ALLOC(b->B.pos, n); ALLOC(b->B.vel, n); ALLOC(b->B.lag, n); ALLOC(b->B.id, n); ALLOC(b->B.type, n);
  ALLOC(b->keysA, n); ALLOC(b->perm, n); ALLOC(b->digits, n);
  ALLOC(b->sort_tmp, radix_temp_words((uint32_t)n));
  ALLOC(b->force, n); ALLOC(b->pforce, n); ALLOC(b->xs, n);
  ALLOC(b->rho, n); ALLOC(b->press, n); ALLOC(b->pq, n);
  ALLOC(b->nbr, n * rows); ALLOC(b->lval, n * rows); ALLOC(b->ncnt, n);
  ALLOC(b->cstart, b->n_cells); ALLOC(b->cend, b->n_cells);
  ALLOC(b->params_d, num_scenes); ALLOC(b->luts_d, (size_t)num_scenes * kLutFloats);
  ALLOC(b->st_d, num_scenes);
  ALLOC(b->group_scene_d, group_scene.size()); ALLOC(b->seg_begin_d, num_scenes); ALLOC(b->seg_end_d, num_scenes);
  ALLOC(b->cell_base_d, num_scenes); ALLOC(b->any_active_d, 1);
  ALLOC(b->active_groups_d, n / kSegAlign + 1); ALLOC(b->n_active_groups_d, 1);
  ALLOC(b->x.comp_begin_d, num_scenes); ALLOC(b->x.stage_a, std::max<size_t>(total, 1));
  ALLOC(b->x.stage_b, std::max<size_t>(total, 1));
#undef ALLOC
  if ((st = encode_list_maps(b->nbr_maps, b->lval_maps, b->nbr, b->lval, n, rows)) != UPF_OK) return bail(st);
  e = cudaMallocHost((void**)&b->st_h, sizeof(DevState) * num_scenes);
  if (e != cudaSuccess) {
    b->st_h = nullptr;
    set_error("cudaMallocHost: %s", cudaGetErrorString(e));
    return bail(UPF_ERR_ALLOC);
  }
  // per-scene parameters and tables
  std::vector<DevParams> dps(num_scenes);
  std::vector<float> luts((size_t)num_scenes * kLutFloats);
  for (uint32_t s = 0; s < num_scenes; ++s) {
    dps[s] = make_dev_params(params[s], (uint32_t)n);
    build_luts(params[s], luts.data() + (size_t)s * kLutFloats);
    build_bin_thresholds(params[s], luts.data() + (size_t)s * kLutFloats + 5 * UPF_LUT_ENTRIES);
  }
  e = cudaMemcpy(b->params_d, dps.data(), sizeof(DevParams) * num_scenes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->luts_d, luts.data(), sizeof(float) * luts.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(b->group_scene_d, group_scene.data(), sizeof(uint32_t) * group_scene.size(),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(b->seg_begin_d, b->seg_begin.data(), sizeof(uint32_t) * num_scenes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(b->seg_end_d, b->seg_end.data(), sizeof(uint32_t) * num_scenes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(b->cell_base_d, b->cell_base.data(), sizeof(uint32_t) * num_scenes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(b->x.comp_begin_d, comp_begin.data(), sizeof(uint32_t) * num_scenes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(b->st_d, 0, sizeof(DevState) * num_scenes);
  if (e == cudaSuccess) e = cudaMemset(b->A.type, 0xff, sizeof(int32_t) * n);  // padding: no type
  if (e == cudaSuccess) e = cudaMemset(b->A.pos, 0, sizeof(float4) * n);
  if (e == cudaSuccess) e = cudaMemset(b->A.vel, 0, sizeof(float4) * n);
  if (e == cudaSuccess) e = cudaMemset(b->A.id, 0xff, sizeof(uint32_t) * n);
  if (e != cudaSuccess) {
    set_error("upf_batch_create: upload: %s", cudaGetErrorString(e));
    return bail(UPF_ERR_CUDA);
  }
  b->view.params = b->params_d;
  b->view.luts = b->luts_d;
  b->view.st = b->st_d;
  b->view.group_scene = b->group_scene_d;
  b->view.seg_end = b->seg_end_d;
  b->view.cell_base = b->cell_base_d;
  *out = b;
  return UPF_OK;
}

upf_status upf_batch_destroy(upf_batch* b) {
  if (!b) return UPF_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  frame_streams_destroy(b->io);  // its buffers are in b->allocations
  destroy_batch_graph(b);
  for (void* p : b->allocations) cudaFree(p);
  for (void* p : b->checkpoint_slots)
    if (p) cudaFree(p);
  if (b->st_h) cudaFreeHost(b->st_h);
  if (b->stream && b->own_stream) cudaStreamDestroy(b->stream);
  delete b;
  return UPF_OK;
}

upf_status upf_batch_set_stream(upf_batch* b, void* stream) {
  if (!b) {
    set_error("upf_batch_set_stream: null");
    return UPF_ERR_INVALID_ARG;
  }
  UPF_CUDA(cudaStreamSynchronize(b->stream));
  if (b->own_stream) cudaStreamDestroy(b->stream);
  if (stream) {
    b->stream = (cudaStream_t)stream;
    b->own_stream = false;
  } else {
    UPF_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    b->own_stream = true;
  }
  return UPF_OK;
}

upf_status upf_batch_set_particles(upf_batch* b, const float* pos4, const float* vel4) {
  NvtxRange nvtx("upf_batch_set_particles");
  if (!b || (b->n_particles && (!pos4 || !vel4))) {
    set_error("upf_batch_set_particles: null argument");
    return UPF_ERR_INVALID_ARG;
  }
  UPF_CUDA(cudaSetDevice(b->device));
  cudaStream_t st = b->stream;
  UPF_CUDA(cudaStreamSynchronize(st));
  const size_t n = b->n_particles;
  if (n) {
    UPF_CUDA(cudaMemcpyAsync(b->x.stage_a, pos4, sizeof(float4) * n, cudaMemcpyHostToDevice, st));
    UPF_CUDA(cudaMemcpyAsync(b->x.stage_b, vel4, sizeof(float4) * n, cudaMemcpyHostToDevice, st));
  }
  // ids, types; positions w = 0
  std::vector<uint32_t> ids(b->n_slots, 0xffffffffu);
  std::vector<int32_t> types(b->n_slots, -1);
  for (uint32_t s = 0; s < b->n_scenes; ++s)
    for (uint32_t k = 0; k < b->count[s]; ++k) {
      ids[b->seg_begin[s] + k] = k;
      types[b->seg_begin[s] + k] = UPF_LIQUID;
    }
  UPF_CUDA(cudaMemcpyAsync(b->A.id, ids.data(), sizeof(uint32_t) * b->n_slots, cudaMemcpyHostToDevice, st));
  UPF_CUDA(cudaMemcpyAsync(b->A.type, types.data(), sizeof(int32_t) * b->n_slots, cudaMemcpyHostToDevice, st));
  k_batch_scatter<<<(b->n_slots + 255) / 256, 256, 0, st>>>(b->view, b->seg_begin_d, b->x.comp_begin_d, b->n_slots,
                                                            b->x.stage_a, b->x.stage_b, b->A.pos, b->A.vel, 1);
  UPF_CUDA(cudaGetLastError());
  UPF_CUDA(batch_launch_init(*b, st));
  UPF_CUDA(cudaMemsetAsync(b->st_d, 0, sizeof(DevState) * b->n_scenes, st));
  UPF_CUDA(cudaStreamSynchronize(st));  // host vectors go out of scope
  b->have_particles = true;
  for (void* p : b->checkpoint_slots)
    if (p) cudaFree(p);
  b->checkpoint_slots.clear();
  return build_batch_graph(b);
}

upf_status upf_batch_step(upf_batch* b, int32_t nsteps) {
  NvtxRange nvtx("upf_batch_step");
  UPF_TRY(batch_guard(b, "upf_batch_step"));
  if (nsteps < 0) {
    set_error("upf_batch_step: negative step count");
    return UPF_ERR_INVALID_ARG;
  }
  for (int32_t k = 0; k < nsteps; ++k) UPF_CUDA(cudaGraphLaunch(b->step_exec, b->stream));
  return UPF_OK;
}

upf_status upf_batch_synchronize(upf_batch* b) {
  UPF_TRY(batch_guard(b, "upf_batch_synchronize"));
  UPF_CUDA(cudaStreamSynchronize(b->stream));
  return batch_check_errors(b);
}

upf_status upf_batch_get_stats(upf_batch* b, upf_step_stats* out) {
  UPF_TRY(batch_guard(b, "upf_batch_get_stats"));
  if (!out) {
    set_error("upf_batch_get_stats: null");
    return UPF_ERR_INVALID_ARG;
  }
  const upf_status rc = batch_check_errors(b);
  for (uint32_t s = 0; s < b->n_scenes; ++s) {
    const DevState& d = b->st_h[s];
    upf_step_stats& o = out[s];
    std::memset(&o, 0, sizeof(o));
    o.iterations = d.final_iterations;
    o.hit_max_loops = d.final_iterations >= b->prm[s].max_loops;
    o.max_predicted_density = d.final_max_rho;
    o.density_error_percent = d.final_err;
    o.max_neighbor_count = d.max_neighbors;
    o.error_flags = d.error_flags;
    o.kinetic_energy = d.ke;
    for (int k = 0; k < 3; ++k) o.momentum[k] = d.mom[k];
    for (int k = 0; k < 64; ++k) o.iteration_max_density[k] = d.iter_max_rho[k];
    o.total_steps = d.total_steps;
    o.total_iterations = d.total_iterations;
    o.steps_at_max_loops = d.steps_at_max;
    o.max_step_density_error_percent = d.max_step_err;
  }
  return rc;
}

upf_status upf_batch_reset_counters(upf_batch* b) {
  UPF_TRY(batch_guard(b, "upf_batch_reset_counters"));
  std::vector<DevState> h(b->n_scenes);
  UPF_CUDA(cudaMemcpyAsync(h.data(), b->st_d, sizeof(DevState) * b->n_scenes, cudaMemcpyDeviceToHost, b->stream));
  UPF_CUDA(cudaStreamSynchronize(b->stream));
  for (DevState& d : h) {
    d.total_steps = d.total_iterations = d.steps_at_max = 0;
    d.max_step_err = 0.0f;
  }
  UPF_CUDA(cudaMemcpyAsync(b->st_d, h.data(), sizeof(DevState) * b->n_scenes, cudaMemcpyHostToDevice, b->stream));
  UPF_CUDA(cudaStreamSynchronize(b->stream));
  return UPF_OK;
}

upf_status upf_batch_get_particles(upf_batch* b, uint32_t scene, float* pos4, float* vel4, float* density,
                                   float* pressure, uint32_t* id, uint32_t* n_out) {
  UPF_TRY(batch_guard(b, "upf_batch_get_particles"));
  if (scene >= b->n_scenes) {
    set_error("upf_batch_get_particles: scene %u out of range", scene);
    return UPF_ERR_INVALID_ARG;
  }
  const uint32_t o = b->seg_begin[scene], n = b->count[scene];
  cudaStream_t st = b->stream;
  if (n) {
    if (pos4) UPF_CUDA(cudaMemcpyAsync(pos4, b->A.pos + o, sizeof(float4) * n, cudaMemcpyDeviceToHost, st));
    if (vel4) UPF_CUDA(cudaMemcpyAsync(vel4, b->A.vel + o, sizeof(float4) * n, cudaMemcpyDeviceToHost, st));
    if (density) UPF_CUDA(cudaMemcpyAsync(density, b->rho + o, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    if (pressure) UPF_CUDA(cudaMemcpyAsync(pressure, b->press + o, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    if (id) UPF_CUDA(cudaMemcpyAsync(id, b->A.id + o, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, st));
  }
  UPF_CUDA(cudaStreamSynchronize(st));
  if (n_out) *n_out = n;
  return UPF_OK;
}

// the dynamic state: A arrays + keys + per-scene device state
static size_t batch_state_bytes(const upf_batch* b) {
  const size_t n = b->n_slots;
  return n * (3 * sizeof(float4) + 3 * sizeof(uint32_t)) + sizeof(DevState) * b->n_scenes;
}

static upf_status batch_state_copy(upf_batch* b, char* flat, bool to_flat) {
  const size_t n = b->n_slots;
  struct Seg {
    void* p;
    size_t bytes;
  } seg[] = {{b->A.pos, n * sizeof(float4)}, {b->A.vel, n * sizeof(float4)}, {b->A.lag, n * sizeof(float4)},
             {b->A.id, n * sizeof(uint32_t)}, {b->A.type, n * sizeof(int32_t)}, {b->keysA, n * sizeof(uint32_t)},
             {b->st_d, sizeof(DevState) * b->n_scenes}};
  size_t off = 0;
  for (const Seg& s : seg) {
    UPF_CUDA(to_flat ? cudaMemcpyAsync(flat + off, s.p, s.bytes, cudaMemcpyDeviceToDevice, b->stream)
                     : cudaMemcpyAsync(s.p, flat + off, s.bytes, cudaMemcpyDeviceToDevice, b->stream));
    off += s.bytes;
  }
  return UPF_OK;
}

upf_status upf_batch_checkpoint(upf_batch* b, int32_t slot) {
  UPF_TRY(batch_guard(b, "upf_batch_checkpoint"));
  if (slot < 0 || slot > 4096) {
    set_error("upf_batch_checkpoint: slot %d out of range", slot);
    return UPF_ERR_INVALID_ARG;
  }
  if ((size_t)slot >= b->checkpoint_slots.size()) b->checkpoint_slots.resize(slot + 1, nullptr);
  if (!b->checkpoint_slots[slot]) {
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, batch_state_bytes(b));
    if (e != cudaSuccess) {
      set_error("upf_batch_checkpoint: cudaMalloc: %s", cudaGetErrorString(e));
      return UPF_ERR_ALLOC;
    }
    b->checkpoint_slots[slot] = p;
  }
  return batch_state_copy(b, (char*)b->checkpoint_slots[slot], true);
}

upf_status upf_batch_restore(upf_batch* b, int32_t slot) {
  UPF_TRY(batch_guard(b, "upf_batch_restore"));
  if (slot < 0 || (size_t)slot >= b->checkpoint_slots.size() || !b->checkpoint_slots[slot]) {
    set_error("upf_batch_restore: slot %d holds no checkpoint", slot);
    return UPF_ERR_INVALID_ARG;
  }
  return batch_state_copy(b, (char*)b->checkpoint_slots[slot], false);
}

upf_status upf_batch_upload_state(upf_batch* b, const float* pos4, const float* vel4) {
  UPF_TRY(batch_guard(b, "upf_batch_upload_state"));
  if (b->n_particles && (!pos4 || !vel4)) {
    set_error("upf_batch_upload_state: null argument");
    return UPF_ERR_INVALID_ARG;
  }
  cudaStream_t st = b->stream;
  const size_t n = b->n_particles;
  if (!n) return UPF_OK;
  UPF_CUDA(cudaMemcpyAsync(b->x.stage_a, pos4, sizeof(float4) * n, cudaMemcpyHostToDevice, st));
  UPF_CUDA(cudaMemcpyAsync(b->x.stage_b, vel4, sizeof(float4) * n, cudaMemcpyHostToDevice, st));
  k_batch_scatter<<<(b->n_slots + 255) / 256, 256, 0, st>>>(b->view, b->seg_begin_d, b->x.comp_begin_d, b->n_slots,
                                                            b->x.stage_a, b->x.stage_b, b->A.pos, b->A.vel, 1);
  UPF_CUDA(cudaGetLastError());
  // the keys of the uploaded positions (lagged state kept)
  UPF_CUDA(batch_launch_keys(*b, st));
  return UPF_OK;
}

upf_status upf_batch_download_state(upf_batch* b, float* pos4, float* vel4) {
  UPF_TRY(batch_guard(b, "upf_batch_download_state"));
  if (b->n_particles && (!pos4 || !vel4)) {
    set_error("upf_batch_download_state: null argument");
    return UPF_ERR_INVALID_ARG;
  }
  cudaStream_t st = b->stream;
  const size_t n = b->n_particles;
  if (!n) return UPF_OK;
  k_batch_scatter<<<(b->n_slots + 255) / 256, 256, 0, st>>>(b->view, b->seg_begin_d, b->x.comp_begin_d, b->n_slots,
                                                            b->A.pos, b->A.vel, b->x.stage_a, b->x.stage_b, 0);
  UPF_CUDA(cudaGetLastError());
  UPF_CUDA(cudaMemcpyAsync(pos4, b->x.stage_a, sizeof(float4) * n, cudaMemcpyDeviceToHost, st));
  UPF_CUDA(cudaMemcpyAsync(vel4, b->x.stage_b, sizeof(float4) * n, cudaMemcpyDeviceToHost, st));
  UPF_CUDA(cudaStreamSynchronize(st));
  return UPF_OK;
}

// Asynchronous counterparts of the per-frame upload and download (the
// single-system scheme of upf_upload_state_async): the host copies run on
// the batch's copy streams against staging buffers in the caller's
// scene-concatenated order; the scatter into the batch's slots (and back)
// runs in stream order on the compute stream.
static upf_status batch_frames_ready(BatchSystem& b) {
  FrameIO& io = b.io;
  if (io.ready) return UPF_OK;
  const size_t n = b.n_particles;
  UPF_TRY(balloc(b, &io.in_pos, n));
  UPF_TRY(balloc(b, &io.in_vel, n));
  UPF_TRY(balloc(b, &io.out_pos, n));
  UPF_TRY(balloc(b, &io.out_vel, n));
  UPF_CUDA(frame_streams_create(io, b.stream));
  io.ready = true;
  return UPF_OK;
}

upf_status upf_batch_upload_state_async(upf_batch* b, const float* pos4, const float* vel4) {
  UPF_TRY(batch_guard(b, "upf_batch_upload_state_async"));
  if (b->n_particles && (!pos4 || !vel4)) {
    set_error("upf_batch_upload_state_async: null argument");
    return UPF_ERR_INVALID_ARG;
  }
  const size_t n = b->n_particles;
  if (!n) return UPF_OK;
  UPF_TRY(batch_frames_ready(*b));
  FrameIO& io = b->io;
  cudaStream_t st = b->stream;
  UPF_CUDA(cudaStreamWaitEvent(io.up, io.consumed, 0));  // the last upload has left the staging buffers
  UPF_CUDA(cudaMemcpyAsync(io.in_pos, pos4, sizeof(float4) * n, cudaMemcpyHostToDevice, io.up));
  UPF_CUDA(cudaMemcpyAsync(io.in_vel, vel4, sizeof(float4) * n, cudaMemcpyHostToDevice, io.up));
  UPF_CUDA(cudaEventRecord(io.staged, io.up));
  UPF_CUDA(cudaStreamWaitEvent(st, io.staged, 0));
  k_batch_scatter<<<(b->n_slots + 255) / 256, 256, 0, st>>>(b->view, b->seg_begin_d, b->x.comp_begin_d, b->n_slots,
                                                            io.in_pos, io.in_vel, b->A.pos, b->A.vel, 1);
  UPF_CUDA(cudaGetLastError());
  UPF_CUDA(batch_launch_keys(*b, st));
  UPF_CUDA(cudaEventRecord(io.consumed, st));
  return UPF_OK;
}

upf_status upf_batch_download_state_async(upf_batch* b, float* pos4, float* vel4) {
  UPF_TRY(batch_guard(b, "upf_batch_download_state_async"));
  if (b->n_particles && (!pos4 || !vel4)) {
    set_error("upf_batch_download_state_async: null argument");
    return UPF_ERR_INVALID_ARG;
  }
  const size_t n = b->n_particles;
  if (!n) return UPF_OK;
  UPF_TRY(batch_frames_ready(*b));
  FrameIO& io = b->io;
  cudaStream_t st = b->stream;
  UPF_CUDA(cudaStreamWaitEvent(st, io.read_done, 0));  // the last download has left the snapshot
  k_batch_scatter<<<(b->n_slots + 255) / 256, 256, 0, st>>>(b->view, b->seg_begin_d, b->x.comp_begin_d, b->n_slots,
                                                            b->A.pos, b->A.vel, io.out_pos, io.out_vel, 0);
  UPF_CUDA(cudaGetLastError());
  UPF_CUDA(cudaEventRecord(io.snapped, st));
  UPF_CUDA(cudaStreamWaitEvent(io.down, io.snapped, 0));
  UPF_CUDA(cudaMemcpyAsync(pos4, io.out_pos, sizeof(float4) * n, cudaMemcpyDeviceToHost, io.down));
  UPF_CUDA(cudaMemcpyAsync(vel4, io.out_vel, sizeof(float4) * n, cudaMemcpyDeviceToHost, io.down));
  UPF_CUDA(cudaEventRecord(io.read_done, io.down));
  return UPF_OK;
}

upf_status upf_batch_wait_frames(upf_batch* b) {
  if (!b) {
    set_error("upf_batch_wait_frames: null");
    return UPF_ERR_INVALID_ARG;
  }
  if (!b->io.ready) return UPF_OK;
  UPF_CUDA(cudaStreamWaitEvent(b->stream, b->io.read_done, 0));
  UPF_CUDA(cudaEventSynchronize(b->io.staged));
  UPF_CUDA(cudaEventSynchronize(b->io.read_done));
  return UPF_OK;
}

upf_status upf_batch_get_launch_config(upf_batch* b, upf_launch_config* out) {
  if (!b || !out) {
    set_error("upf_batch_get_launch_config: null");
    return UPF_ERR_INVALID_ARG;
  }
  shape_to_config(b->shape, out);
  return UPF_OK;
}

upf_status upf_batch_set_launch_config(upf_batch* b, const upf_launch_config* cfg) {
  if (!b || !cfg) {
    set_error("upf_batch_set_launch_config: null");
    return UPF_ERR_INVALID_ARG;
  }
  const LaunchShape sh = config_to_shape(*cfg);
  const char* why = nullptr;
  if (!shape_valid(sh, true, &why)) {
    set_error("upf_batch_set_launch_config: %s", why);
    return UPF_ERR_INVALID_ARG;
  }
  UPF_CUDA(cudaStreamSynchronize(b->stream));
  b->shape = sh;
  return b->have_particles ? build_batch_graph(b) : UPF_OK;
}

namespace {
struct BatchTune {
  upf_batch* b;
  void* buf;
};
}  // namespace

upf_status upf_batch_autotune(upf_batch* b, int32_t repeats, upf_launch_config* chosen) {
  NvtxRange nvtx("upf_batch_autotune");
  UPF_TRY(batch_guard(b, "upf_batch_autotune"));
  UPF_CUDA(cudaStreamSynchronize(b->stream));
  BatchTune t{b, nullptr};
  TuneOps ops;
  ops.ctx = &t;
  ops.shape = &b->shape;
  ops.batched = true;
  ops.stream = b->stream;
  ops.save = [](void* c) -> upf_status {
    BatchTune& T = *static_cast<BatchTune*>(c);
    cudaError_t e = cudaMalloc(&T.buf, batch_state_bytes(T.b));
    if (e != cudaSuccess) {
      T.buf = nullptr;
      set_error("upf_batch_autotune: cudaMalloc: %s", cudaGetErrorString(e));
      return UPF_ERR_ALLOC;
    }
    return batch_state_copy(T.b, (char*)T.buf, true);
  };
  ops.restore = [](void* c) -> upf_status {
    BatchTune& T = *static_cast<BatchTune*>(c);
    if (!T.buf) return UPF_OK;
    upf_status rc = batch_state_copy(T.b, (char*)T.buf, false);
    cudaStreamSynchronize(T.b->stream);
    cudaFree(T.buf);
    T.buf = nullptr;
    return rc;
  };
  ops.prepare = [](void* c, cudaStream_t st) {
    BatchSystem& B = *static_cast<BatchTune*>(c)->b;
    cudaError_t e = batch_launch_sort(B, st);
    if (e == cudaSuccess) e = batch_launch_neighbors(B, st);
    if (e == cudaSuccess) e = batch_launch_forces(B, st);
    if (e == cudaSuccess) e = batch_launch_loop_init(B, st);
    return e;
  };
  ops.nlist = [](void* c, cudaStream_t st) { return batch_launch_neighbors(*static_cast<BatchTune*>(c)->b, st); };
  ops.external = [](void* c, cudaStream_t st) { return batch_launch_forces(*static_cast<BatchTune*>(c)->b, st); };
  ops.density = [](void* c, cudaStream_t st) { return batch_launch_loop_density(*static_cast<BatchTune*>(c)->b, st); };
  ops.pforce = [](void* c, cudaStream_t st) { return batch_launch_loop_pforce(*static_cast<BatchTune*>(c)->b, st); };
  UPF_TRY(autotune_shapes(ops, repeats, chosen));
  UPF_TRY(batch_check_errors(b));
  return build_batch_graph(b);
}

upf_status upf_batch_profile_step(upf_batch* b, upf_phase_times* out, uint64_t* active_particle_iterations) {
  UPF_TRY(batch_guard(b, "upf_batch_profile_step"));
  if (!out) {
    set_error("upf_batch_profile_step: null");
    return UPF_ERR_INVALID_ARG;
  }
  std::memset(out, 0, sizeof(*out));
  cudaStream_t st = b->stream;
  cudaEvent_t ev[8];
  for (auto& e : ev) UPF_CUDA(cudaEventCreate(&e));
  auto elapsed = [&](cudaEvent_t x, cudaEvent_t y) {
    float ms = 0;
    cudaEventElapsedTime(&ms, x, y);
    return ms;
  };
  uint64_t active = 0;
  std::vector<DevState> h(b->n_scenes);
  UPF_CUDA(cudaEventRecord(ev[0], st));
  UPF_CUDA(batch_launch_sort(*b, st));
  UPF_CUDA(cudaEventRecord(ev[1], st));
  UPF_CUDA(batch_launch_neighbors(*b, st));
  UPF_CUDA(cudaEventRecord(ev[2], st));
  UPF_CUDA(batch_launch_forces(*b, st));
  UPF_CUDA(cudaEventRecord(ev[3], st));
  UPF_CUDA(batch_launch_loop_init(*b, st));
  UPF_CUDA(cudaStreamSynchronize(st));
  out->sort_ms = elapsed(ev[0], ev[1]);
  out->neighbors_ms = elapsed(ev[1], ev[2]);
  out->forces_ms = elapsed(ev[2], ev[3]);
  int launches = 4 + 1 + 4 + 1 + 1 + 2 + 1 + 1 + 1;  // sort stages, digits, reorder, cells, init, nlist, ext, loop init
  float loop = 0;
  const uint32_t total_groups = b->n_slots / kSegAlign;
  for (int it = 0; it < 4096; ++it) {
    // scenes still iterating before this iteration, and the groups the last
    // loop control listed
    uint32_t ngroups = total_groups;
    UPF_CUDA(cudaMemcpyAsync(h.data(), b->st_d, sizeof(DevState) * b->n_scenes, cudaMemcpyDeviceToHost, st));
    if (it) UPF_CUDA(cudaMemcpyAsync(&ngroups, b->n_active_groups_d, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    UPF_CUDA(cudaStreamSynchronize(st));
    uint64_t act = 0;
    for (uint32_t s = 0; s < b->n_scenes; ++s)
      if (h[s].loop_active) act += b->count[s];
    if (!act) break;
    active += act;
    // the passes the step graph runs: the full grid in the first iteration
    // and while at least half of the groups iterate, then the resident
    // passes over the listed groups (k_loop_ctl_batch's choice)
    const bool full = 2 * ngroups >= total_groups;
    UPF_CUDA(cudaEventRecord(ev[4], st));
    UPF_CUDA(full ? batch_launch_loop_density(*b, st) : batch_launch_loop_density_active(*b, st));
    UPF_CUDA(cudaEventRecord(ev[5], st));
    UPF_CUDA(full ? batch_launch_loop_pforce(*b, st) : batch_launch_loop_pforce_active(*b, st));
    UPF_CUDA(cudaEventRecord(ev[6], st));
    UPF_CUDA(batch_launch_loop_ctl(*b, st));
    UPF_CUDA(cudaEventRecord(ev[7], st));
    UPF_CUDA(cudaStreamSynchronize(st));
    UPF_CUDA(cudaGetLastError());
    out->density_ms_total += elapsed(ev[4], ev[5]);
    out->pforce_ms_total += elapsed(ev[5], ev[6]);
    loop += elapsed(ev[4], ev[7]);
    out->iterations = it + 1;
    launches += 3;
  }
  out->loop_ms = loop;
  UPF_CUDA(cudaEventRecord(ev[0], st));
  UPF_CUDA(batch_launch_integrate(*b, st));
  UPF_CUDA(cudaEventRecord(ev[1], st));
  UPF_CUDA(cudaStreamSynchronize(st));
  out->integrate_ms = elapsed(ev[0], ev[1]);
  out->launches = launches + 1;
  for (auto& e : ev) cudaEventDestroy(e);
  if (active_particle_iterations) *active_particle_iterations = active;
  return batch_check_errors(b);
}

}  // extern "C"
