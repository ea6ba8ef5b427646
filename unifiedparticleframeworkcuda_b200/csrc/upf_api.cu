// upf_api.cu — the C ABI (include/upf.h): handle lifetime, uploads, the
// CUDA-graph step and readback.
//
// The reference allocates with MallocDeviceArraysParticles
// (src/gpu/particles.cu:100-166), uploads with Copy*HostToDevice
// (particles.cu:349-646), steps with ParticlePhysicsOnDevice*
// (particles.cu:1281-2769) and reads back with CopyParticlesCUDA
// (particles.cu:62-72). Its PCISPH loop is host-driven: one device-to-host
// read of the max predicted density per iteration (particles.cu:1917-1944,
// 2139-2154). Here one step is a single CUDA graph and the loop is a
// device-side conditional while-node fed by the loop-control kernel.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "upf_sys.h"
#include "upf_tma.cuh"

namespace upf {

namespace {
thread_local char g_err[512] = "";
}

namespace {
std::atomic<int64_t> g_fail_alloc_at{-1};  // allocations left before the injected failure; -1: none
}  // namespace

bool inject_alloc_failure() {
  int64_t v = g_fail_alloc_at.load();
  while (v >= 0) {
    if (g_fail_alloc_at.compare_exchange_weak(v, v - 1)) return v == 0;
  }
  return false;
}

NvtxRange::NvtxRange(const char* name) { nvtxRangePushA(name); }
NvtxRange::~NvtxRange() { nvtxRangePop(); }

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

namespace {

#define UPF_CUDA(call)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) {                                                            \
      set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
      return UPF_ERR_CUDA;                                                              \
    }                                                                                   \
  } while (0)

template <class T>
upf_status dalloc(System& s, T** p, size_t count) {
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
  s.allocations.push_back(*p);
  return UPF_OK;
}

#define UPF_TRY(call)              \
  do {                             \
    upf_status st_ = (call);       \
    if (st_ != UPF_OK) return st_; \
  } while (0)

uint32_t log2u(uint32_t v) {
  uint32_t r = 0;
  while ((1u << r) < v) ++r;
  return r;
}

}  // namespace

DevParams make_dev_params(const upf_params& p, uint32_t nstride) {
  DevParams d{};
  d.h = p.support_radius;
  d.lut_factor = (float)(1.0 / (double)p.support_radius);
  d.mass = p.mass;
  d.inv_mass = (float)(1.0 / (double)p.mass);
  d.rho0 = p.rest_density;
  d.kernel_self = kernel_self(p.support_radius);
  d.gas_b = p.rest_density * p.gas_constant / p.gamma;
  d.gamma = p.gamma;
  d.visc = p.viscosity;
  d.rest_volume = p.mass / p.rest_density;
  d.gravity = p.gravity;
  d.dt = p.dt;
  d.delta = p.density_error_factor;
  d.err_scale = 100.0f / p.rest_density;
  d.max_err = p.max_density_error;
  d.min_loops = p.min_loops;
  d.max_loops = p.max_loops;
  d.st_gamma = p.surface_tension_gamma;
  d.adh_beta = p.surface_adhesion_beta;
  d.force_dist = p.force_distance;
  d.inv_force_dist = 1.0f / p.force_distance;
  d.max_boundary_force = p.max_boundary_force;
  d.radius = p.particle_radius;
  d.spacing = p.particle_spacing;
  d.spring = p.spring_coefficient;
  d.spring_boundary = p.spring_coefficient_boundary;
  d.damping = p.damping_coefficient;
  d.terminal_speed = p.terminal_speed;
  d.gran_kr = p.granular_kr;
  d.gran_kd = p.granular_kd;
  d.gran_kt = p.granular_kt;
  d.gran_mu = p.granular_mu;
  d.origin = make_float3(p.zindex_origin[0], p.zindex_origin[1], p.zindex_origin[2]);
  d.scales = make_float3(p.scales[0], p.scales[1], p.scales[2]);
  d.cmin = make_float3(p.collision_min[0], p.collision_min[1], p.collision_min[2]);
  d.cmax = make_float3(p.collision_max[0], p.collision_max[1], p.collision_max[2]);
  d.wmin = make_float3(p.container_min[0], p.container_min[1], p.container_min[2]);
  d.wmax = make_float3(p.container_max[0], p.container_max[1], p.container_max[2]);
  d.block_shift = log2u(p.block_size);
  d.cell_shift = log2u(effective_search_cell(p));
  d.flags = p.flags;
  d.maxn = p.max_neighbors;
  d.nstride = nstride;
  d.static_base = nstride;
  d.list_grad = p.method == UPF_METHOD_PCISPH ? 1u : 0u;
  return d;
}

namespace {

}  // namespace

// 2D tensor map over a column-major neighbour array [rows][cols] for the
// TMA list stream: box = 32 columns (one warp) x kListRows rows.
upf_status encode_list_map(CUtensorMap* map, void* base, CUtensorMapDataType dt, uint32_t elem_bytes, uint64_t cols,
                           uint64_t rows, uint32_t box_rows) {
  typedef CUresult (*EncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static EncodeTiled encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || !fn || q != cudaDriverEntryPointSuccess) {
      set_error("cuTensorMapEncodeTiled unavailable: %s", cudaGetErrorString(e));
      return UPF_ERR_CUDA;
    }
    encode = (EncodeTiled)fn;
  }
  const cuuint64_t dims[2] = {cols, rows};
  const cuuint64_t strides[1] = {cols * elem_bytes};
  const cuuint32_t box[2] = {32, (cuuint32_t)box_rows};
  const cuuint32_t estride[2] = {1, 1};
  CUresult r = encode(map, dt, 2, base, dims, strides, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
    return UPF_ERR_CUDA;
  }
  return UPF_OK;
}

upf_status encode_list_maps(CUtensorMap* cmaps, CUtensorMap* vmaps, uint32_t* nbr, uint32_t* lval, uint64_t cols,
                            uint64_t rows) {
  const uint32_t box_rows[kListRowVariants] = {2, 4, 8, 16};
  for (int k = 0; k < kListRowVariants; ++k) {
    upf_status st = encode_list_map(&cmaps[k], nbr, CU_TENSOR_MAP_DATA_TYPE_UINT32, 4, cols, rows, box_rows[k]);
    if (st != UPF_OK) return st;
    st = encode_list_map(&vmaps[k], lval, CU_TENSOR_MAP_DATA_TYPE_UINT32, 4, cols, rows, box_rows[k]);
    if (st != UPF_OK) return st;
  }
  return UPF_OK;
}

bool shape_valid(const LaunchShape& s, bool batched, const char** why) {
  auto bad = [&](const char* w) {
    if (why) *why = w;
    return false;
  };
  auto pair_ok = [&](int mode, int t, int r) {
    for (const auto& p : kLoopShapes)
      if (p[0] == mode && p[1] == t && p[2] == r) return true;
    return false;
  };
  if (s.nlist_threads != 64 && s.nlist_threads != 128 && s.nlist_threads != 256)
    return bad("nlist_threads must be 64, 128 or 256");
  if (s.nlist_mode != 0 && s.nlist_mode != 1) return bad("nlist_mode must be 0 (lane boxes) or 1 (warp union)");
  if (s.external_threads != 128 && s.external_threads != 256) return bad("external_threads must be 128 or 256");
  if (!pair_ok(s.density_mode, s.density_threads, s.density_rows) ||
      !pair_ok(s.pforce_mode, s.pforce_threads, s.pforce_rows))
    return bad("(threads, rows) of a loop pass must be one of (128,4) (128,8) (128,16) (256,2) (256,4) (256,8) "
               "(512,2) (512,4) (1024,2) with the TMA ring (mode 0), (128,4) (128,8) (256,4) (256,8) (512,4) "
               "(512,8) with direct loads (mode 1), or (256,4) (256,8) with staged neighbourhoods (mode 2)");
  if (batched && (loop_mode_staged(s.density_mode) || loop_mode_staged(s.pforce_mode)))
    return bad("batched scenes: staged neighbourhoods (mode 2) are for single scenes");
  if (!pforce_ring_fits(s.pforce_mode, s.pforce_threads, s.pforce_rows))
    return bad("the pressure-force pass's TMA ring takes (128,4) (128,8) (256,2) (256,4) (512,2); its list values "
               "leave the larger rings no room in shared memory");
  if (batched && (s.density_threads > 256 || s.pforce_threads > 256))
    return bad("batched scenes: at most 256 threads per CTA (a CTA must stay within one scene's segment)");
  return true;
}

void shape_to_config(const LaunchShape& s, upf_launch_config* c) {
  std::memset(c, 0, sizeof(*c));
  c->nlist_threads = s.nlist_threads;
  c->external_threads = s.external_threads;
  c->density_threads = s.density_threads;
  c->density_rows = s.density_rows;
  c->pforce_threads = s.pforce_threads;
  c->pforce_rows = s.pforce_rows;
  c->density_mode = s.density_mode;
  c->pforce_mode = s.pforce_mode;
  c->nlist_mode = s.nlist_mode;
}

LaunchShape config_to_shape(const upf_launch_config& c) {
  LaunchShape s;
  s.nlist_threads = c.nlist_threads;
  s.external_threads = c.external_threads;
  s.density_threads = c.density_threads;
  s.density_rows = c.density_rows;
  s.pforce_threads = c.pforce_threads;
  s.pforce_rows = c.pforce_rows;
  s.density_mode = c.density_mode;
  s.pforce_mode = c.pforce_mode;
  s.nlist_mode = c.nlist_mode;
  return s;
}

upf_status autotune_shapes(const TuneOps& ops, int repeats, upf_launch_config* out) {
  if (repeats < 1) repeats = 1;
  cudaStream_t st = ops.stream;
  LaunchShape& sh = *ops.shape;
  cudaEvent_t e0, e1;
  UPF_CUDA(cudaEventCreate(&e0));
  UPF_CUDA(cudaEventCreate(&e1));
  float chosen_ms[4] = {0, 0, 0, 0};
  upf_status rc = UPF_OK;
  // ms per launch of `launch` at the current shape (one untimed launch first)
  auto time_pass = [&](cudaError_t (*launch)(void*, cudaStream_t), float* ms) -> upf_status {
    UPF_CUDA(launch(ops.ctx, st));
    UPF_CUDA(cudaEventRecord(e0, st));
    for (int r = 0; r < repeats; ++r) UPF_CUDA(launch(ops.ctx, st));
    UPF_CUDA(cudaEventRecord(e1, st));
    UPF_CUDA(cudaEventSynchronize(e1));
    float t = 0;
    UPF_CUDA(cudaEventElapsedTime(&t, e0, e1));
    *ms = t / repeats;
    return UPF_OK;
  };
  do {
    if ((rc = ops.save(ops.ctx)) != UPF_OK) break;
    if (ops.prepare) {
      cudaError_t e = ops.prepare(ops.ctx, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) {
        set_error("autotune: prepare: %s", cudaGetErrorString(e));
        rc = UPF_ERR_CUDA;
        break;
      }
    }
    // one pass at a time, the others at their current shapes
    if (ops.nlist) {
      const int cand[] = {64, 128, 256};
      int best = sh.nlist_threads, best_mode = sh.nlist_mode;
      float best_ms = 1e30f;
      for (int mode = 0; mode < 2 && rc == UPF_OK; ++mode)
        for (int t : cand) {
          sh.nlist_threads = t;
          sh.nlist_mode = mode;
          float ms;
          if ((rc = time_pass(ops.nlist, &ms)) != UPF_OK) break;
          if (ms < best_ms) best_ms = ms, best = t, best_mode = mode;
        }
      if (rc != UPF_OK) break;
      sh.nlist_threads = best;
      sh.nlist_mode = best_mode;
      chosen_ms[0] = best_ms;
      // the lists of the chosen shape (identical for every shape)
      if (cudaSuccess != ops.nlist(ops.ctx, st)) {
        rc = UPF_ERR_CUDA;
        break;
      }
    }
    if (ops.external) {
      const int cand[] = {128, 256};
      int best = sh.external_threads;
      float best_ms = 1e30f;
      for (int t : cand) {
        sh.external_threads = t;
        float ms;
        if ((rc = time_pass(ops.external, &ms)) != UPF_OK) break;
        if (ms < best_ms) best_ms = ms, best = t;
      }
      if (rc != UPF_OK) break;
      sh.external_threads = best;
      chosen_ms[1] = best_ms;
    }
    // the loop passes: the fastest shape of each pass, and the fastest that
    // reads the plain lists; staged shapes (mode 2) also cost the staging
    // kernel once per step, which the choice weighs against the passes'
    // saving times the iterations a step takes
    const auto& pairs = kLoopShapes;
    struct Pick {
      int mode, threads, rows;
      float ms;
    };
    Pick best_any[2], best_plain[2];
    bool tuned[2] = {false, false};
    for (int pass = 0; pass < 2 && rc == UPF_OK; ++pass) {
      cudaError_t (*launch)(void*, cudaStream_t) = pass == 0 ? ops.density : ops.pforce;
      if (!launch) continue;
      int& mode = pass == 0 ? sh.density_mode : sh.pforce_mode;
      int& threads = pass == 0 ? sh.density_threads : sh.pforce_threads;
      int& rows = pass == 0 ? sh.density_rows : sh.pforce_rows;
      best_any[pass] = best_plain[pass] = Pick{mode, threads, rows, 1e30f};
      for (const auto& pr : pairs) {
        if (ops.batched && (pr[1] > 256 || loop_mode_staged(pr[0]))) continue;
        if (!ops.stage && loop_mode_staged(pr[0])) continue;
        if (pass == 1 && !pforce_ring_fits(pr[0], pr[1], pr[2])) continue;
        mode = pr[0];
        threads = pr[1];
        rows = pr[2];
        float ms;
        if ((rc = time_pass(launch, &ms)) != UPF_OK) break;
        const Pick pk{pr[0], pr[1], pr[2], ms};
        if (ms < best_any[pass].ms) best_any[pass] = pk;
        if (!loop_mode_staged(pr[0]) && ms < best_plain[pass].ms) best_plain[pass] = pk;
      }
      tuned[pass] = rc == UPF_OK;
    }
    if (rc == UPF_OK && tuned[0] && tuned[1]) {
      Pick pick[2] = {best_any[0], best_any[1]};
      if (loop_mode_staged(pick[0].mode) || loop_mode_staged(pick[1].mode)) {
        float stage_ms = 0.0f;
        if ((rc = time_pass(ops.stage, &stage_ms)) != UPF_OK) break;
        const float it = ops.loop_iterations > 0.0f ? ops.loop_iterations : 1.0f;
        float best_cost = 1e30f;
        for (int a = 0; a < 2; ++a)
          for (int b = 0; b < 2; ++b) {
            const Pick& d = a ? best_any[0] : best_plain[0];
            const Pick& f = b ? best_any[1] : best_plain[1];
            const bool staged = loop_mode_staged(d.mode) || loop_mode_staged(f.mode);
            const float cost = it * (d.ms + f.ms) + (staged ? stage_ms : 0.0f);
            if (cost < best_cost) best_cost = cost, pick[0] = d, pick[1] = f;
          }
      }
      for (int pass = 0; pass < 2; ++pass) {
        (pass == 0 ? sh.density_mode : sh.pforce_mode) = pick[pass].mode;
        (pass == 0 ? sh.density_threads : sh.pforce_threads) = pick[pass].threads;
        (pass == 0 ? sh.density_rows : sh.pforce_rows) = pick[pass].rows;
        chosen_ms[2 + pass] = pick[pass].ms;
      }
    } else {
      for (int pass = 0; pass < 2; ++pass) {
        if (!tuned[pass]) continue;
        (pass == 0 ? sh.density_mode : sh.pforce_mode) = best_any[pass].mode;
        (pass == 0 ? sh.density_threads : sh.pforce_threads) = best_any[pass].threads;
        (pass == 0 ? sh.density_rows : sh.pforce_rows) = best_any[pass].rows;
        chosen_ms[2 + pass] = best_any[pass].ms;
      }
    }
  } while (0);
  const upf_status rr = ops.restore(ops.ctx);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != UPF_OK) return rc;
  if (rr != UPF_OK) return rr;
  if (out) {
    shape_to_config(sh, out);
    for (int k = 0; k < 4; ++k) out->measured_ms[k] = chosen_ms[k];
  }
  return UPF_OK;
}

// One step as a graph: pre -> [while: loop] -> post. The loop body is
// captured into the body graph of a conditional while-node; the body's last
// kernel sets the node's condition.
upf_status capture_step_graph(const GraphParts& parts, cudaGraph_t* graph_out, cudaGraphExec_t* exec_out) {
  *graph_out = nullptr;
  *exec_out = nullptr;
  cudaStream_t cs = nullptr, body_stream = nullptr;
  UPF_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  UPF_CUDA(cudaStreamCreateWithFlags(&body_stream, cudaStreamNonBlocking));
  auto cleanup = [&]() {
    cudaStreamDestroy(cs);
    cudaStreamDestroy(body_stream);
  };
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    cleanup();
    set_error("cudaStreamBeginCapture: %s", cudaGetErrorString(e));
    return UPF_ERR_CUDA;
  }
  auto fail = [&](const char* what, cudaError_t err) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(cs, &g);
    if (g) cudaGraphDestroy(g);
    cleanup();
    set_error("step graph: %s: %s", what, cudaGetErrorString(err));
    return UPF_ERR_CUDA;
  };
  if (parts.pre && (e = parts.pre(parts.ctx, cs)) != cudaSuccess) return fail("pre", e);
  if (parts.loop) {
    cudaStreamCaptureStatus cst;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    if ((e = cudaStreamGetCaptureInfo(cs, &cst, nullptr, &g, &deps, &ndeps)) != cudaSuccess)
      return fail("capture info", e);
    cudaGraphConditionalHandle handle;
    if ((e = cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault)) != cudaSuccess)
      return fail("conditional handle", e);
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = handle;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t cnode;
    if ((e = cudaGraphAddNode(&cnode, g, deps, ndeps, &np)) != cudaSuccess) return fail("while node", e);
    cudaGraph_t body = np.conditional.phGraph_out[0];
    if ((e = cudaStreamUpdateCaptureDependencies(cs, &cnode, 1, cudaStreamSetCaptureDependencies)) != cudaSuccess)
      return fail("capture dependencies", e);
    if ((e = cudaStreamBeginCaptureToGraph(body_stream, body, nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
      return fail("body capture", e);
    cudaError_t eb = parts.loop(parts.ctx, body_stream, handle);
    cudaGraph_t body_out = nullptr;
    cudaError_t ee = cudaStreamEndCapture(body_stream, &body_out);
    if (eb != cudaSuccess) return fail("loop body", eb);
    if (ee != cudaSuccess) return fail("body end capture", ee);
  }
  if (parts.post && (e = parts.post(parts.ctx, cs)) != cudaSuccess) return fail("post", e);
  cudaGraph_t graph = nullptr;
  e = cudaStreamEndCapture(cs, &graph);
  cleanup();
  if (e != cudaSuccess) {
    set_error("step graph end capture: %s", cudaGetErrorString(e));
    return UPF_ERR_CUDA;
  }
  e = cudaGraphInstantiate(exec_out, graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    set_error("step graph instantiate: %s", cudaGetErrorString(e));
    return UPF_ERR_CUDA;
  }
  *graph_out = graph;
  return UPF_OK;
}

namespace {

void destroy_graph(System& s) {
  if (s.step_exec) cudaGraphExecDestroy(s.step_exec);
  if (s.step_graph) cudaGraphDestroy(s.step_graph);
  s.step_exec = nullptr;
  s.step_graph = nullptr;
}

// One step of a system: sort -> neighbours -> forces -> [while: loop body] -> integrate.
upf_status build_step_graph(System& s) {
  destroy_graph(s);
  GraphParts parts;
  parts.ctx = &s;
  parts.pre = [](void* c, cudaStream_t st) {
    System& S = *static_cast<System*>(c);
    cudaError_t e = launch_sort_phase(S, st);
    if (e == cudaSuccess) e = launch_neighbor_phase(S, st);
    if (e == cudaSuccess) e = launch_force_phase(S, st);
    if (e == cudaSuccess && S.prm.method == UPF_METHOD_PCISPH) e = launch_loop_init(S, st);
    return e;
  };
  if (s.prm.method == UPF_METHOD_PCISPH)
    parts.loop = [](void* c, cudaStream_t st, cudaGraphConditionalHandle h) {
      return launch_loop_body(*static_cast<System*>(c), st, h, true);
    };
  parts.post = [](void* c, cudaStream_t st) { return launch_integrate_phase(*static_cast<System*>(c), st); };
  // capturing runs the launchers' host code without running the kernels:
  // the host-side record of whether the current lists are staged is kept,
  // and whether a step of this graph stages them is noted for upf_step
  const bool staged_now = s.lists_staged;
  const upf_status rc = capture_step_graph(parts, &s.step_graph, &s.step_exec);
  s.graph_stages = s.lists_staged;
  s.lists_staged = staged_now;
  return rc;
}

upf_status check_device_errors(System& s) {
  UPF_CUDA(cudaMemcpyAsync(s.st_host, s.st, sizeof(DevState), cudaMemcpyDeviceToHost, s.stream));
  UPF_CUDA(cudaStreamSynchronize(s.stream));
  const uint32_t f = s.st_host->error_flags;
  if (f & ERR_NAN) {
    set_error("a particle position became NaN");
    return UPF_ERR_NAN;
  }
  if (f & ERR_OVERFLOW) {
    set_error("a particle has %u neighbours, more than max_neighbors=%u", s.st_host->max_neighbors,
              s.prm.max_neighbors);
    return UPF_ERR_NEIGHBOR_OVERFLOW;
  }
  if (f & ERR_TIMEOUT) {
    set_error("a bounded device-side wait ran out");
    return UPF_ERR_TIMEOUT;
  }
  return UPF_OK;
}

void free_list(std::vector<void*>& v) {
  for (void* p : v)
    if (p) cudaFree(p);
  v.clear();
}

// checkpoints hold the state layout of the configuration they were taken in
void drop_checkpoints(System& s) { free_list(s.checkpoint_slots); }

void clear_rigid(System& s) {
  free_list(s.rigid_allocations);
  s.rb = RigidArrays{};
}

// One warp waits, with the library's bounded wait, on an mbarrier that no
// thread and no copy ever completes; the wait gives up after limit_ns and
// records ERR_TIMEOUT like the list stream's waits do.
__global__ void k_selftest_wait(uint64_t limit_ns, DevState* st) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_barrier_init();
  }
  __syncwarp();
  const bool ok = mbar_wait(&bar, 0, limit_ns);
  if (!ok && threadIdx.x == 0) atomicOr(&st->error_flags, (uint32_t)ERR_TIMEOUT);
}

// The table bins the density pass takes for squared distances r2
// (bin_of_r2_edge), checked against the list build's bin_of_r2 (thresholds
// staged in shared memory, as in that pass): -2 where the two disagree.
__global__ void k_selftest_support_bins(const float* __restrict__ thr_g, float factor, const float* __restrict__ r2,
                                        uint32_t n, int32_t* __restrict__ out) {
  __shared__ float thr[kThresholds];
  for (int k = threadIdx.x; k < kThresholds; k += blockDim.x) thr[k] = thr_g[k];
  __syncthreads();
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int a = bin_of_r2_edge(r2[i], factor, thr[kLut]);
    out[i] = a == bin_of_r2(r2[i], factor, thr) ? a : -2;
  }
}

__global__ void k_init_dyn(uint32_t n, DynArrays A, float rho0) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  A.lag[i] = make_float4(0.0f, 0.0f, rho0, 0.0f);
}

// Every particle of the last upf_set_particles call at its input index: the
// dynamic particles from the current state (position with its Morton key in
// w, as the reference keeps the z-index in pos.w), the boundary particles from
// the static set (at rest, rest density, zero pressure).
__global__ void k_scatter_input_order(uint32_t nd, DynArrays A, const float* __restrict__ rho,
                                      const float* __restrict__ press, uint32_t ns, const float4* __restrict__ spos,
                                      const uint32_t* __restrict__ sid, float3 origin, float3 scales, float rho0,
                                      uint32_t n_total, float4* __restrict__ opos, float4* __restrict__ ovel,
                                      float* __restrict__ orho, float* __restrict__ opress, int32_t* __restrict__ otype) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nd + ns) return;
  if (i < nd) {
    const uint32_t j = A.id[i];
    if (j >= n_total) return;
    const float4 x = A.pos[i];
    const float4 v = A.vel[i];
    opos[j] = make_float4(x.x, x.y, x.z, (float)morton_key(x, origin, scales));
    ovel[j] = make_float4(v.x, v.y, v.z, 0.0f);
    orho[j] = rho[i];
    opress[j] = press[i];
    otype[j] = A.type[i];
  } else {
    const uint32_t b = i - nd;
    const uint32_t j = sid[b];
    if (j >= n_total) return;
    const float4 x = spos[b];
    opos[j] = make_float4(x.x, x.y, x.z, (float)morton_key(x, origin, scales));
    ovel[j] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    orho[j] = rho0;
    opress[j] = 0.0f;
    otype[j] = UPF_FROZEN;
  }
}

// dst[k] = src[idx[k]] (gather) or dst[idx[k]] = src[k] (scatter), rows of
// one float or one float4: the halo exchange packs and unpacks with these
template <class T>
__global__ void k_rows(const T* __restrict__ src, const uint32_t* __restrict__ idx, uint32_t n, T* __restrict__ dst,
                       bool scatter) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  if (scatter)
    dst[idx[k]] = src[k];
  else
    dst[k] = src[idx[k]];
}

cudaError_t launch_rows(const void* src, uint32_t row_bytes, const uint32_t* idx, uint32_t n, void* dst,
                        bool scatter, cudaStream_t st) {
  const uint32_t grid = (n + 255) / 256;
  if (row_bytes == 16)
    k_rows<float4><<<grid, 256, 0, st>>>((const float4*)src, idx, n, (float4*)dst, scatter);
  else
    k_rows<uint32_t><<<grid, 256, 0, st>>>((const uint32_t*)src, idx, n, (uint32_t*)dst, scatter);
  return cudaGetLastError();
}

__global__ void k_gather_static(uint32_t n, const uint32_t* __restrict__ perm, const float4* __restrict__ in,
                                const uint32_t* __restrict__ in_id, float4* __restrict__ out,
                                uint32_t* __restrict__ out_id) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t j = perm[i];
  out[i] = in[j];
  out_id[i] = in_id[j];
}

}  // namespace
}  // namespace upf

using namespace upf;

struct upf_system : System {};

extern "C" {

const char* upf_last_error(void) { return g_err; }

const char* upf_status_string(upf_status st) {
  switch (st) {
    case UPF_OK: return "UPF_OK";
    case UPF_ERR_INVALID_ARG: return "UPF_ERR_INVALID_ARG";
    case UPF_ERR_CUDA: return "UPF_ERR_CUDA";
    case UPF_ERR_ALLOC: return "UPF_ERR_ALLOC";
    case UPF_ERR_NEIGHBOR_OVERFLOW: return "UPF_ERR_NEIGHBOR_OVERFLOW";
    case UPF_ERR_NAN: return "UPF_ERR_NAN";
    case UPF_ERR_TIMEOUT: return "UPF_ERR_TIMEOUT";
    case UPF_ERR_STATE: return "UPF_ERR_STATE";
    case UPF_ERR_UNSUPPORTED: return "UPF_ERR_UNSUPPORTED";
    case UPF_ERR_NO_DEVICE: return "UPF_ERR_NO_DEVICE";
    case UPF_ERR_IO: return "UPF_ERR_IO";
  }
  return "unknown";
}

int32_t upf_abi_version(void) { return UPF_ABI_VERSION; }

upf_status upf_test_stage_union_cap(upf_system* s, uint32_t cap) {
  if (!s || cap > kUnionMax) {
    set_error("upf_test_stage_union_cap: null system or cap above %u", kUnionMax);
    return UPF_ERR_INVALID_ARG;
  }
  UPF_CUDA(cudaStreamSynchronize(s->stream));
  s->stage_cap = cap;
  return s->have_particles ? build_step_graph(*s) : UPF_OK;
}

upf_status upf_test_fail_allocation(int32_t nth) {
  g_fail_alloc_at.store(nth < 0 ? -1 : (int64_t)nth);
  return UPF_OK;
}

upf_status upf_selftest_bounded_wait(int device, uint32_t limit_us) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("upf_selftest_bounded_wait: no CUDA device");
    return UPF_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev || limit_us == 0 || limit_us > 1000000) {
    set_error("upf_selftest_bounded_wait: bad device or limit (1..1e6 us)");
    return UPF_ERR_INVALID_ARG;
  }
  UPF_CUDA(cudaSetDevice(device));
  DevState* st = nullptr;
  UPF_CUDA(cudaMalloc(&st, sizeof(DevState)));
  cudaError_t e = cudaMemset(st, 0, sizeof(DevState));
  if (e == cudaSuccess) {
    k_selftest_wait<<<1, 32>>>((uint64_t)limit_us * 1000ull, st);
    e = cudaGetLastError();
  }
  DevState h{};
  if (e == cudaSuccess) e = cudaMemcpy(&h, st, sizeof(DevState), cudaMemcpyDeviceToHost);
  cudaFree(st);
  if (e != cudaSuccess) {
    set_error("upf_selftest_bounded_wait: %s", cudaGetErrorString(e));
    return UPF_ERR_CUDA;
  }
  if (h.error_flags & ERR_TIMEOUT) {
    set_error("a bounded device-side wait ran out (self-test)");
    return UPF_ERR_TIMEOUT;
  }
  return UPF_OK;
}

upf_status upf_selftest_support_bins(int device, const upf_params* p, const float* r2, uint32_t n, int32_t* bins) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("upf_selftest_support_bins: no CUDA device");
    return UPF_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev || !p || !(p->support_radius > 0.0f) || (n && (!r2 || !bins)) ||
      n > (1u << 26)) {
    set_error("upf_selftest_support_bins: bad arguments");
    return UPF_ERR_INVALID_ARG;
  }
  if (n == 0) return UPF_OK;
  UPF_CUDA(cudaSetDevice(device));
  float thr_h[kThresholds];
  build_bin_thresholds(*p, thr_h);
  const float factor = (float)(1.0 / (double)p->support_radius);
  float* d_thr = nullptr;
  float* d_r2 = nullptr;
  int32_t* d_out = nullptr;
  cudaError_t e = cudaMalloc(&d_thr, sizeof(thr_h));
  if (e == cudaSuccess) e = cudaMalloc(&d_r2, sizeof(float) * n);
  if (e == cudaSuccess) e = cudaMalloc(&d_out, sizeof(int32_t) * n);
  if (e == cudaSuccess) e = cudaMemcpy(d_thr, thr_h, sizeof(thr_h), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_r2, r2, sizeof(float) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    const uint32_t blocks = (n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184;
    k_selftest_support_bins<<<blocks, 256>>>(d_thr, factor, d_r2, n, d_out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(bins, d_out, sizeof(int32_t) * n, cudaMemcpyDeviceToHost);
  cudaFree(d_thr);
  cudaFree(d_r2);
  cudaFree(d_out);
  if (e != cudaSuccess) {
    set_error("upf_selftest_support_bins: %s", cudaGetErrorString(e));
    return UPF_ERR_CUDA;
  }
  return UPF_OK;
}

upf_status upf_default_params(upf_params* p) {
  if (!p) {
    set_error("upf_default_params: null");
    return UPF_ERR_INVALID_ARG;
  }
  default_params(p);
  return UPF_OK;
}

upf_status upf_params_derive(upf_params* p) {
  if (!p) {
    set_error("upf_params_derive: null");
    return UPF_ERR_INVALID_ARG;
  }
  if (derive_params(p, nullptr) != 0) {
    set_error("upf_params_derive: particle_spacing and zindex_extent must be > 0");
    return UPF_ERR_INVALID_ARG;
  }
  return UPF_OK;
}

upf_status upf_density_error_factor(const upf_params* p, double* out) {
  if (!p || !out) {
    set_error("upf_density_error_factor: null");
    return UPF_ERR_INVALID_ARG;
  }
  *out = density_error_factor(*p);
  return UPF_OK;
}

upf_status upf_build_luts(const upf_params* p, float* out) {
  if (!p || !out || !(p->support_radius > 0)) {
    set_error("upf_build_luts: bad arguments");
    return UPF_ERR_INVALID_ARG;
  }
  build_luts(*p, out);
  return UPF_OK;
}

upf_status upf_build_bin_thresholds(const upf_params* p, float* out) {
  if (!p || !out || !(p->support_radius > 0)) {
    set_error("upf_build_bin_thresholds: bad arguments");
    return UPF_ERR_INVALID_ARG;
  }
  build_bin_thresholds(*p, out);
  return UPF_OK;
}

upf_status upf_create(const upf_params* p, int device, uint32_t capacity, upf_system** out) {
  if (!p || !out || capacity == 0) {
    set_error("upf_create: null argument or zero capacity");
    return UPF_ERR_INVALID_ARG;
  }
  *out = nullptr;
  const char* why = nullptr;
  if (validate_params(*p, &why) != 0) {
    set_error("upf_create: invalid parameters: %s", why);
    return UPF_ERR_INVALID_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("upf_create: no CUDA device");
    return UPF_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) {
    set_error("upf_create: device %d out of range (%d devices)", device, ndev);
    return UPF_ERR_INVALID_ARG;
  }
  UPF_CUDA(cudaSetDevice(device));
  UPF_CUDA(radix_init());
  upf_system* s = new upf_system();
  s->prm = *p;
  s->device = device;
  s->capacity = capacity;
  s->nstride = (capacity + 31) & ~31u;
  s->dp = make_dev_params(*p, s->nstride);
  const uint32_t bpa = UPF_GRID_RESOLUTION / effective_search_cell(*p);
  s->ncells = bpa * bpa * bpa;
  auto bail = [&](upf_status st) {
    upf_destroy(s);
    return st;
  };
  cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    set_error("cudaStreamCreate: %s", cudaGetErrorString(e));
    return bail(UPF_ERR_CUDA);
  }
  s->own_stream = true;
  const uint32_t c = capacity;
  upf_status st = UPF_OK;
#define ALLOC(ptr, count)                   \
  if ((st = dalloc(*s, &(ptr), (count))) != UPF_OK) return bail(st);
  ALLOC(s->A.pos, c); ALLOC(s->A.vel, c); ALLOC(s->A.lag, c); ALLOC(s->A.id, c); ALLOC(s->A.type, c);
  // arrays gathered by neighbour index: [dynamic (stride) | boundary tail (capacity)]
  const size_t ct = (size_t)s->nstride + c;
  ALLOC(s->B.pos, ct); ALLOC(s->B.vel, ct); ALLOC(s->B.lag, c); ALLOC(s->B.id, c); ALLOC(s->B.type, ct);
  ALLOC(s->keysA, c); ALLOC(s->perm, c);
  ALLOC(s->sort_tmp, radix_temp_words(c));
  ALLOC(s->force, c); ALLOC(s->pforce, c); ALLOC(s->xs, ct);
  ALLOC(s->rho, ct); ALLOC(s->press, ct); ALLOC(s->pq, ct); ALLOC(s->wvol, ct);
  ALLOC(s->nbr, (size_t)s->nstride * p->max_neighbors);
  ALLOC(s->lval, (size_t)s->nstride * p->max_neighbors);
  ALLOC(s->ncnt, c);
  ALLOC(s->cstart, s->ncells); ALLOC(s->cend, s->ncells);
  ALLOC(s->sstart, s->ncells); ALLOC(s->send, s->ncells);
  ALLOC(s->spos, c); ALLOC(s->skeys, c); ALLOC(s->sid, c);
  ALLOC(s->luts, 5 * UPF_LUT_ENTRIES + kThresholds);
  ALLOC(s->st, 1);
  if (p->method == UPF_METHOD_PCISPH) {
    // staged neighbourhoods of the loop passes (loop-pass mode 2)
    const size_t chunks = ((size_t)c + kStageChunk - 1) / kStageChunk;
    ALLOC(s->ucodes, chunks * kUnionMax);
    ALLOC(s->ucount, chunks);
    ALLOC(s->lloc, (size_t)((p->max_neighbors + 3) / 4) * s->nstride);
  }
#undef ALLOC
  if ((st = encode_list_maps(s->nbr_maps, s->lval_maps, s->nbr, s->lval, s->nstride, p->max_neighbors)) != UPF_OK)
    return bail(st);
  e = cudaMallocHost((void**)&s->st_host, sizeof(DevState));
  if (e != cudaSuccess) {
    s->st_host = nullptr;
    set_error("cudaMallocHost: %s", cudaGetErrorString(e));
    return bail(UPF_ERR_ALLOC);
  }
  std::vector<float> lut(5 * UPF_LUT_ENTRIES + kThresholds);
  build_luts(*p, lut.data());
  build_bin_thresholds(*p, lut.data() + 5 * UPF_LUT_ENTRIES);
  e = cudaMemcpy(s->luts, lut.data(), sizeof(float) * lut.size(), cudaMemcpyHostToDevice);
  // boundary tails: zero velocity, pressure and pressure quotient
  if (e == cudaSuccess) e = cudaMemset(s->B.vel, 0, sizeof(float4) * ct);
  if (e == cudaSuccess) e = cudaMemset(s->pq, 0, sizeof(float4) * ct);
  if (e == cudaSuccess) e = cudaMemset(s->press, 0, sizeof(float) * ct);
  if (e == cudaSuccess) e = cudaMemset(s->rho, 0, sizeof(float) * ct);
  // no chunk is staged before the first staged list build: the passes read the plain lists
  if (e == cudaSuccess && s->ucount)
    e = cudaMemset(s->ucount, 0xff, sizeof(uint32_t) * (((size_t)c + kStageChunk - 1) / kStageChunk));
  if (e == cudaSuccess) e = cudaMemset(s->st, 0, sizeof(DevState));
  if (e != cudaSuccess) {
    set_error("upload: %s", cudaGetErrorString(e));
    return bail(UPF_ERR_CUDA);
  }
  *out = s;
  return UPF_OK;
}

upf_status upf_destroy(upf_system* s) {
  if (!s) return UPF_OK;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  frame_streams_destroy(s->io);  // its buffers are in s->allocations
  destroy_graph(*s);
  for (void* p : s->allocations) cudaFree(p);
  free_list(s->rigid_allocations);
  free_list(s->checkpoint_slots);
  if (s->st_host) cudaFreeHost(s->st_host);
  if (s->stream && s->own_stream) cudaStreamDestroy(s->stream);
  delete s;
  return UPF_OK;
}

upf_status upf_get_params(const upf_system* s, upf_params* out) {
  if (!s || !out) {
    set_error("upf_get_params: null");
    return UPF_ERR_INVALID_ARG;
  }
  *out = s->prm;
  return UPF_OK;
}

upf_status upf_set_stream(upf_system* s, void* stream) {
  if (!s) {
    set_error("upf_set_stream: null");
    return UPF_ERR_INVALID_ARG;
  }
  UPF_CUDA(cudaStreamSynchronize(s->stream));
  if (s->own_stream) cudaStreamDestroy(s->stream);
  if (stream) {
    s->stream = (cudaStream_t)stream;
    s->own_stream = false;
  } else {
    UPF_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    s->own_stream = true;
  }
  return UPF_OK;
}

upf_status upf_set_particles(upf_system* s, const float* pos4, const float* vel4, const int32_t* type,
                             uint32_t n) {
  NvtxRange nvtx("upf_set_particles");
  if (!s || (n && (!pos4 || !vel4 || !type))) {
    set_error("upf_set_particles: null argument");
    return UPF_ERR_INVALID_ARG;
  }
  if (n > s->capacity) {
    set_error("upf_set_particles: %u particles exceed capacity %u", n, s->capacity);
    return UPF_ERR_INVALID_ARG;
  }
  UPF_CUDA(cudaSetDevice(s->device));
  std::vector<float4> dpos, dvel, spos;
  std::vector<uint32_t> did, sid;
  std::vector<int32_t> dtype;
  for (uint32_t i = 0; i < n; ++i) {
    const int32_t t = type[i];
    if (t < 0 || t > UPF_FROZEN) {
      set_error("upf_set_particles: particle %u has unknown type %d", i, t);
      return UPF_ERR_INVALID_ARG;
    }
    const bool granular_ok = s->prm.method == UPF_METHOD_PCISPH;
    if (t != UPF_LIQUID && t != UPF_FROZEN && t != UPF_RIGID && !(t == UPF_GRANULAR && granular_ok)) {
      set_error("upf_set_particles: particle %u has type %d; supported: LIQUID, RIGID, FROZEN%s", i, t,
                granular_ok ? ", GRANULAR" : " (GRANULAR needs PCISPH)");
      return UPF_ERR_UNSUPPORTED;
    }
    float4 x = make_float4(pos4[4 * i], pos4[4 * i + 1], pos4[4 * i + 2], 0.0f);
    if (t == UPF_FROZEN) {
      spos.push_back(x);
      sid.push_back(i);
    } else {
      dpos.push_back(x);
      dvel.push_back(make_float4(vel4[4 * i], vel4[4 * i + 1], vel4[4 * i + 2], 0.0f));
      did.push_back(i);
      dtype.push_back(t);
    }
  }
  System& S = *s;
  cudaStream_t st = S.stream;
  UPF_CUDA(cudaStreamSynchronize(st));
  drop_checkpoints(S);
  clear_rigid(S);
  S.host_pos.resize(n);
  S.host_vel.resize(n);
  S.host_type.assign(type, type + n);
  for (uint32_t i = 0; i < n; ++i) {
    S.host_pos[i] = make_float4(pos4[4 * i], pos4[4 * i + 1], pos4[4 * i + 2], 0.0f);
    S.host_vel[i] = make_float4(vel4[4 * i], vel4[4 * i + 1], vel4[4 * i + 2], 0.0f);
  }
  S.n_dyn = (uint32_t)dpos.size();
  S.n_static = (uint32_t)spos.size();
  if (S.n_dyn) {
    UPF_CUDA(cudaMemcpyAsync(S.A.pos, dpos.data(), sizeof(float4) * S.n_dyn, cudaMemcpyHostToDevice, st));
    UPF_CUDA(cudaMemcpyAsync(S.A.vel, dvel.data(), sizeof(float4) * S.n_dyn, cudaMemcpyHostToDevice, st));
    UPF_CUDA(cudaMemcpyAsync(S.A.id, did.data(), sizeof(uint32_t) * S.n_dyn, cudaMemcpyHostToDevice, st));
    UPF_CUDA(cudaMemcpyAsync(S.A.type, dtype.data(), sizeof(int32_t) * S.n_dyn, cudaMemcpyHostToDevice, st));
    UPF_CUDA(morton_keys(S.A.pos, S.n_dyn, S.dp.origin, S.dp.scales, S.keysA, st));
    k_init_dyn<<<(S.n_dyn + 255) / 256, 256, 0, st>>>(S.n_dyn, S.A, S.prm.rest_density);
    UPF_CUDA(cudaGetLastError());
  }
  // boundary set: sort once by key (stable), gather positions and ids
  if (S.n_static) {
    float4* tmp_pos = S.xs;           // scratch: per-step fields are not live yet
    uint32_t* tmp_id = (uint32_t*)S.rho;
    uint32_t* perm = S.ncnt;
    UPF_CUDA(cudaMemcpyAsync(tmp_pos, spos.data(), sizeof(float4) * S.n_static, cudaMemcpyHostToDevice, st));
    UPF_CUDA(cudaMemcpyAsync(tmp_id, sid.data(), sizeof(uint32_t) * S.n_static, cudaMemcpyHostToDevice, st));
    UPF_CUDA(morton_keys(tmp_pos, S.n_static, S.dp.origin, S.dp.scales, S.skeys, st));
    uint32_t* kalt = S.sort_tmp;
    uint32_t* valt = kalt + ((S.n_static + 63) & ~63u);
    uint32_t* counts = valt + ((S.n_static + 63) & ~63u);
    UPF_CUDA(radix_sort_pairs(S.skeys, perm, kalt, valt, counts, S.n_static, S.key_bits, true, st));
    k_gather_static<<<(S.n_static + 255) / 256, 256, 0, st>>>(S.n_static, perm, tmp_pos, tmp_id, S.spos, S.sid);
    UPF_CUDA(cudaGetLastError());
    // boundary tails of the arrays gathered by neighbour index
    const size_t tb = S.dp.static_base;
    UPF_CUDA(cudaMemcpyAsync(S.B.pos + tb, S.spos, sizeof(float4) * S.n_static, cudaMemcpyDeviceToDevice, st));
    UPF_CUDA(cudaMemcpyAsync(S.xs + tb, S.spos, sizeof(float4) * S.n_static, cudaMemcpyDeviceToDevice, st));
    UPF_CUDA(cudaMemcpyAsync(S.pq + tb, S.spos, sizeof(float4) * S.n_static, cudaMemcpyDeviceToDevice, st));
    std::vector<int32_t> frozen(S.n_static, UPF_FROZEN);
    UPF_CUDA(cudaMemcpyAsync(S.B.type + tb, frozen.data(), sizeof(int32_t) * S.n_static, cudaMemcpyHostToDevice, st));
  }
  {
    // default Akinci volume: the rest volume (UnifiedParticle.cpp:24)
    std::vector<float> wv((size_t)S.dp.static_base + S.n_static, S.prm.mass / S.prm.rest_density);
    UPF_CUDA(cudaMemcpyAsync(S.wvol, wv.data(), sizeof(float) * wv.size(), cudaMemcpyHostToDevice, st));
    UPF_CUDA(cudaStreamSynchronize(st));  // host vectors go out of scope
  }
  UPF_CUDA(launch_static_setup(S, st));
  UPF_CUDA(cudaMemsetAsync(S.st, 0, sizeof(DevState), st));
  UPF_CUDA(cudaStreamSynchronize(st));
  S.have_particles = true;
  S.stepped = false;
  return build_step_graph(S);
}

upf_status upf_set_rigid_bodies(upf_system* s, const int32_t* body_of_particle, uint32_t n, uint32_t n_bodies) {
  if (!s) {
    set_error("upf_set_rigid_bodies: null");
    return UPF_ERR_INVALID_ARG;
  }
  System& S = *s;
  if (!S.have_particles || S.stepped) {
    set_error("upf_set_rigid_bodies: call it after upf_set_particles and before the first step");
    return UPF_ERR_STATE;
  }
  if (S.prm.method != UPF_METHOD_PCISPH) {
    set_error("upf_set_rigid_bodies: rigid bodies are coupled by the PCISPH solver only");
    return UPF_ERR_UNSUPPORTED;
  }
  if (n != S.host_type.size() || (n && !body_of_particle) || n_bodies > (1u << 20)) {
    set_error("upf_set_rigid_bodies: need one body index per particle of the last upload (%zu), at most 2^20 bodies",
              S.host_type.size());
    return UPF_ERR_INVALID_ARG;
  }
  const int32_t* bop = body_of_particle;
  // The rigid list: bodies in index order, each body's particles in input
  // order (a counting sort on the host, O(particles)); the bodies' mass,
  // centre, momenta and inertia (AddToRigidBody, UnifiedPhysics.cpp:825-885)
  // are summed on the device in FP64 (k_rigid_assemble).
  std::vector<uint32_t> start(n_bodies + 1, 0);
  for (uint32_t id = 0; id < n; ++id) {
    const int32_t b = bop[id];
    if (b < 0) continue;
    if (b >= (int32_t)n_bodies || S.host_type[id] != UPF_RIGID) {
      set_error("upf_set_rigid_bodies: particle %u: body %d is out of range or the particle is not RIGID", id, b);
      return UPF_ERR_INVALID_ARG;
    }
    start[b + 1] += 1;
  }
  for (uint32_t b = 0; b < n_bodies; ++b) {
    if (start[b + 1] == 0) {
      set_error("upf_set_rigid_bodies: body %u has no particles", b);
      return UPF_ERR_INVALID_ARG;
    }
    start[b + 1] += start[b];
  }
  const uint32_t n_rigid = start[n_bodies];
  std::vector<uint32_t> fill(start.begin(), start.end() - 1), id_entry(n, 0xffffffffu);
  std::vector<int32_t> id_body(n, -1), entry_body(n_rigid);
  std::vector<float4> entry_pos(n_rigid), entry_vel(n_rigid);
  for (uint32_t id = 0; id < n; ++id) {
    const int32_t b = bop[id];
    if (b < 0) continue;
    const uint32_t k = fill[b]++;
    entry_pos[k] = S.host_pos[id];
    entry_vel[k] = S.host_vel[id];
    entry_body[k] = b;
    id_entry[id] = k;
    id_body[id] = b;
  }
  UPF_CUDA(cudaSetDevice(S.device));
  UPF_CUDA(cudaStreamSynchronize(S.stream));
  drop_checkpoints(S);
  clear_rigid(S);
  if (n_bodies) {
    RigidArrays r;
    auto alloc = [&](auto** p, size_t count) -> upf_status {
      cudaError_t e = cudaMalloc((void**)p, (count ? count : 1) * sizeof(**p));
      if (e != cudaSuccess) {
        *p = nullptr;
        set_error("upf_set_rigid_bodies: cudaMalloc: %s", cudaGetErrorString(e));
        return UPF_ERR_ALLOC;
      }
      S.rigid_allocations.push_back(*p);
      return UPF_OK;
    };
    upf_status rc = UPF_OK;
    if ((rc = alloc(&r.bodies, n_bodies)) != UPF_OK || (rc = alloc(&r.start, n_bodies + 1)) != UPF_OK ||
        (rc = alloc(&r.id_body, n)) != UPF_OK || (rc = alloc(&r.id_entry, n)) != UPF_OK ||
        (rc = alloc(&r.entry_r0, n_rigid)) != UPF_OK || (rc = alloc(&r.entry_body, n_rigid)) != UPF_OK ||
        (rc = alloc(&r.entry_slot, n_rigid)) != UPF_OK) {
      clear_rigid(S);
      return rc;
    }
    r.n_bodies = n_bodies;
    r.n_rigid = n_rigid;
    r.n_ids = n;
    cudaStream_t st = S.stream;
    UPF_CUDA(cudaMemcpyAsync(r.start, start.data(), sizeof(uint32_t) * (n_bodies + 1), cudaMemcpyHostToDevice, st));
    UPF_CUDA(cudaMemcpyAsync(r.id_body, id_body.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
    UPF_CUDA(cudaMemcpyAsync(r.id_entry, id_entry.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, st));
    UPF_CUDA(cudaMemcpyAsync(r.entry_body, entry_body.data(), sizeof(int32_t) * n_rigid, cudaMemcpyHostToDevice, st));
    // the entries' positions and velocities for the assembly, in scratch
    // that is not live before the first step
    float4* epos = S.xs;
    float4* evel = S.pforce;
    UPF_CUDA(cudaMemcpyAsync(epos, entry_pos.data(), sizeof(float4) * n_rigid, cudaMemcpyHostToDevice, st));
    UPF_CUDA(cudaMemcpyAsync(evel, entry_vel.data(), sizeof(float4) * n_rigid, cudaMemcpyHostToDevice, st));
    UPF_CUDA(launch_rigid_assemble(S.prm.mass, r.bodies, n_bodies, r.start, epos, evel, r.entry_r0, st));
    UPF_CUDA(cudaStreamSynchronize(st));  // host vectors go out of scope
    S.rb = r;
  }
  return build_step_graph(S);
}

upf_status upf_get_rigid_bodies(upf_system* s, float* pos3, float* vel3, float* omega3, float* quat4,
                                uint32_t* n_out) {
  if (!s) {
    set_error("upf_get_rigid_bodies: null");
    return UPF_ERR_INVALID_ARG;
  }
  const uint32_t nb = s->rb.n_bodies;
  if (n_out) *n_out = nb;
  if (!nb) return UPF_OK;
  std::vector<DevBody> h(nb);
  UPF_CUDA(cudaMemcpyAsync(h.data(), s->rb.bodies, sizeof(DevBody) * nb, cudaMemcpyDeviceToHost, s->stream));
  UPF_CUDA(cudaStreamSynchronize(s->stream));
  for (uint32_t b = 0; b < nb; ++b) {
    const DevBody& B = h[b];
    if (pos3) { pos3[3 * b] = B.pos.x; pos3[3 * b + 1] = B.pos.y; pos3[3 * b + 2] = B.pos.z; }
    if (vel3) { vel3[3 * b] = B.vel.x; vel3[3 * b + 1] = B.vel.y; vel3[3 * b + 2] = B.vel.z; }
    if (omega3) { omega3[3 * b] = B.omega.x; omega3[3 * b + 1] = B.omega.y; omega3[3 * b + 2] = B.omega.z; }
    if (quat4)
      for (int k = 0; k < 4; ++k) quat4[4 * b + k] = B.q[k];
  }
  return UPF_OK;
}

upf_status upf_step(upf_system* s, int32_t nsteps) {
  NvtxRange nvtx("upf_step");
  if (!s || nsteps < 0) {
    set_error("upf_step: bad arguments");
    return UPF_ERR_INVALID_ARG;
  }
  if (!s->have_particles || !s->step_exec) {
    set_error("upf_step: call upf_set_particles first");
    return UPF_ERR_STATE;
  }
  if (s->graph_stale) {
    UPF_TRY(build_step_graph(*s));
    s->graph_stale = false;
  }
  s->stepped = true;
  for (int32_t k = 0; k < nsteps; ++k) UPF_CUDA(cudaGraphLaunch(s->step_exec, s->stream));
  if (nsteps > 0) s->lists_staged = s->graph_stages;
  return UPF_OK;
}

upf_status upf_synchronize(upf_system* s) {
  if (!s) {
    set_error("upf_synchronize: null");
    return UPF_ERR_INVALID_ARG;
  }
  UPF_CUDA(cudaStreamSynchronize(s->stream));
  return check_device_errors(*s);
}

upf_status upf_get_step_stats(upf_system* s, upf_step_stats* out) {
  if (!s || !out) {
    set_error("upf_get_step_stats: null");
    return UPF_ERR_INVALID_ARG;
  }
  upf_status st = check_device_errors(*s);
  const DevState& d = *s->st_host;
  std::memset(out, 0, sizeof(*out));
  out->iterations = s->prm.method == UPF_METHOD_PCISPH ? d.final_iterations : 0;
  out->hit_max_loops = (s->prm.method == UPF_METHOD_PCISPH && d.final_iterations >= s->prm.max_loops);
  out->max_predicted_density = d.final_max_rho;
  out->density_error_percent = d.final_err;
  out->max_neighbor_count = d.max_neighbors;
  out->error_flags = d.error_flags;
  out->kinetic_energy = d.ke;
  for (int k = 0; k < 3; ++k) out->momentum[k] = d.mom[k];
  for (int k = 0; k < 64; ++k) out->iteration_max_density[k] = d.iter_max_rho[k];
  out->total_steps = d.total_steps;
  out->total_iterations = d.total_iterations;
  out->steps_at_max_loops = d.steps_at_max;
  out->max_step_density_error_percent = d.max_step_err;
  return st;
}

upf_status upf_reset_counters(upf_system* s) {
  if (!s) {
    set_error("upf_reset_counters: null");
    return UPF_ERR_INVALID_ARG;
  }
  const size_t off = offsetof(DevState, total_steps);
  UPF_CUDA(cudaMemsetAsync((char*)s->st + off, 0, sizeof(DevState) - off, s->stream));
  return UPF_OK;
}

// ---- phases ---------------------------------------------------------------
static upf_status phase_guard(upf_system* s) {
  if (!s) {
    set_error("phase: null");
    return UPF_ERR_INVALID_ARG;
  }
  if (!s->have_particles) {
    set_error("phase: call upf_set_particles first");
    return UPF_ERR_STATE;
  }
  return UPF_OK;
}

upf_status upf_phase_sort(upf_system* s) {
  UPF_TRY(phase_guard(s));
  s->stepped = true;
  UPF_CUDA(launch_sort_phase(*s, s->stream));
  // The sort leaves the keys sorted in place and the state sorted in B, while
  // A keeps the previous order. In a step, integration rewrites A in sorted
  // order, together with its keys. Called on its own, the phase copies the
  // sorted state back into A instead. A and its keys then agree, and a
  // repeated sort (this phase again, or a step) finds them in order and
  // changes nothing, as re-sorting sorted arrays does in the reference.
  const size_t n = s->n_dyn;
  if (n) {
    UPF_CUDA(cudaMemcpyAsync(s->A.pos, s->B.pos, sizeof(float4) * n, cudaMemcpyDeviceToDevice, s->stream));
    UPF_CUDA(cudaMemcpyAsync(s->A.vel, s->B.vel, sizeof(float4) * n, cudaMemcpyDeviceToDevice, s->stream));
    UPF_CUDA(cudaMemcpyAsync(s->A.id, s->B.id, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s->stream));
    UPF_CUDA(cudaMemcpyAsync(s->A.type, s->B.type, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s->stream));
    if (s->prm.method == UPF_METHOD_PCISPH)
      UPF_CUDA(cudaMemcpyAsync(s->A.lag, s->B.lag, sizeof(float4) * n, cudaMemcpyDeviceToDevice, s->stream));
  }
  return UPF_OK;
}

upf_status upf_phase_neighbors(upf_system* s) {
  UPF_TRY(phase_guard(s));
  s->stepped = true;
  UPF_CUDA(launch_neighbor_phase(*s, s->stream));
  return UPF_OK;
}

upf_status upf_phase_forces(upf_system* s) {
  UPF_TRY(phase_guard(s));
  s->stepped = true;
  UPF_CUDA(launch_force_phase(*s, s->stream));
  return UPF_OK;
}

upf_status upf_phase_predict_correct(upf_system* s) {
  UPF_TRY(phase_guard(s));
  s->stepped = true;
  if (s->prm.method != UPF_METHOD_PCISPH) return UPF_OK;
  UPF_CUDA(launch_loop_init(*s, s->stream));
  // host-driven loop (the graph path runs the same body under a while-node)
  for (int it = 0; it < s->prm.max_loops + 1; ++it) {
    UPF_CUDA(launch_loop_body(*s, s->stream, 0, false));
    UPF_CUDA(cudaMemcpyAsync(s->st_host, s->st, sizeof(DevState), cudaMemcpyDeviceToHost, s->stream));
    UPF_CUDA(cudaStreamSynchronize(s->stream));
    const DevState& d = *s->st_host;
    int cont = (d.iteration < s->prm.min_loops) || (d.too_large && d.iteration < s->prm.max_loops);
    if (d.error_flags & ERR_NAN) cont = 0;
    if (!cont) break;
  }
  return UPF_OK;
}

upf_status upf_phase_integrate(upf_system* s) {
  UPF_TRY(phase_guard(s));
  s->stepped = true;
  UPF_CUDA(launch_integrate_phase(*s, s->stream));
  return UPF_OK;
}

// ---- the predict-correct loop pass by pass, and device access for a
// caller that exchanges fields between the passes (slab decomposition) -----
static upf_status pcisph_guard(upf_system* s, const char* who) {
  UPF_TRY(phase_guard(s));
  if (s->prm.method != UPF_METHOD_PCISPH) {
    set_error("%s: PCISPH systems only", who);
    return UPF_ERR_UNSUPPORTED;
  }
  return UPF_OK;
}

upf_status upf_phase_loop_begin(upf_system* s) {
  UPF_TRY(pcisph_guard(s, "upf_phase_loop_begin"));
  s->stepped = true;
  UPF_CUDA(launch_loop_init(*s, s->stream));
  return UPF_OK;
}

upf_status upf_phase_density(upf_system* s) {
  UPF_TRY(pcisph_guard(s, "upf_phase_density"));
  UPF_CUDA(launch_loop_density(*s, s->stream));
  return UPF_OK;
}

upf_status upf_phase_pressure_force(upf_system* s) {
  UPF_TRY(pcisph_guard(s, "upf_phase_pressure_force"));
  UPF_CUDA(launch_loop_pforce(*s, s->stream));
  return UPF_OK;
}

upf_status upf_phase_loop_control(upf_system* s, int32_t* cont) {
  UPF_TRY(pcisph_guard(s, "upf_phase_loop_control"));
  if (!cont) {
    set_error("upf_phase_loop_control: null");
    return UPF_ERR_INVALID_ARG;
  }
  UPF_CUDA(launch_loop_ctl(*s, s->stream, 0, false));
  UPF_CUDA(cudaMemcpyAsync(s->st_host, s->st, sizeof(DevState), cudaMemcpyDeviceToHost, s->stream));
  UPF_CUDA(cudaStreamSynchronize(s->stream));
  const DevState& d = *s->st_host;
  *cont = (d.final_iterations < s->prm.min_loops) ||
          (d.too_large && d.final_iterations < s->prm.max_loops);
  if (d.error_flags & ERR_NAN) *cont = 0;
  return UPF_OK;
}

upf_status upf_get_device_state(upf_system* s, upf_device_state* out) {
  UPF_TRY(phase_guard(s));
  if (!out) {
    set_error("upf_get_device_state: null");
    return UPF_ERR_INVALID_ARG;
  }
  std::memset(out, 0, sizeof(*out));
  out->pos4 = (float*)s->A.pos;
  out->vel4 = (float*)s->A.vel;
  out->lag4 = (float*)s->A.lag;
  out->type = s->A.type;
  out->id = s->A.id;
  out->n = s->n_dyn;
  out->capacity_dynamic = s->capacity - s->n_static;
  out->sorted_pos4 = (float*)s->B.pos;
  out->sorted_id = s->B.id;
  out->predicted_pos4 = (float*)s->xs;
  out->pressure = s->press;
  out->pq4 = (float*)s->pq;
  out->density = s->rho;
  out->loop_max_density_bits = &s->st->max_rho_bits;
  out->stream = (void*)s->stream;
  return UPF_OK;
}

upf_status upf_set_dynamic_device(upf_system* s, const float* pos4, const float* vel4, const float* lag4,
                                  const int32_t* type, const uint32_t* id, uint32_t n) {
  UPF_TRY(phase_guard(s));
  System& S = *s;
  if (n && (!pos4 || !vel4 || !lag4 || !type || !id)) {
    set_error("upf_set_dynamic_device: null argument");
    return UPF_ERR_INVALID_ARG;
  }
  if (n + S.n_static > S.capacity) {
    set_error("upf_set_dynamic_device: %u dynamic + %u boundary particles exceed capacity %u", n, S.n_static,
              S.capacity);
    return UPF_ERR_INVALID_ARG;
  }
  if (S.rb.n_bodies) {
    set_error("upf_set_dynamic_device: systems with rigid bodies keep their particle set");
    return UPF_ERR_UNSUPPORTED;
  }
  cudaStream_t st = S.stream;
  const float4* p4 = (const float4*)pos4;
  const float4* v4 = (const float4*)vel4;
  const float4* l4 = (const float4*)lag4;
  // the inputs may alias the system's own arrays: copy through B first
  if (n) {
    UPF_CUDA(cudaMemcpyAsync(S.B.pos, p4, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st));
    UPF_CUDA(cudaMemcpyAsync(S.B.vel, v4, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st));
    UPF_CUDA(cudaMemcpyAsync(S.B.lag, l4, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st));
    UPF_CUDA(cudaMemcpyAsync(S.B.type, type, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st));
    UPF_CUDA(cudaMemcpyAsync(S.B.id, id, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
    UPF_CUDA(cudaMemcpyAsync(S.A.pos, S.B.pos, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st));
    UPF_CUDA(cudaMemcpyAsync(S.A.vel, S.B.vel, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st));
    UPF_CUDA(cudaMemcpyAsync(S.A.lag, S.B.lag, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st));
    UPF_CUDA(cudaMemcpyAsync(S.A.type, S.B.type, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st));
    UPF_CUDA(cudaMemcpyAsync(S.A.id, S.B.id, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
  }
  S.n_dyn = n;  // the keys below cover the new count
  if (n) UPF_CUDA(launch_upload_keys(S, st));
  drop_checkpoints(S);
  S.graph_stale = true;
  return UPF_OK;
}

upf_status upf_gather_rows(const void* src, uint32_t row_bytes, const uint32_t* idx, uint32_t n, void* dst,
                           void* stream) {
  if (n == 0) return UPF_OK;
  if (!src || !idx || !dst || (row_bytes != 4 && row_bytes != 16)) {
    set_error("upf_gather_rows: null pointer or row size %u (4 or 16)", row_bytes);
    return UPF_ERR_INVALID_ARG;
  }
  UPF_CUDA(launch_rows(src, row_bytes, idx, n, dst, false, (cudaStream_t)stream));
  return UPF_OK;
}

upf_status upf_scatter_rows(const void* src, uint32_t row_bytes, const uint32_t* idx, uint32_t n, void* dst,
                            void* stream) {
  if (n == 0) return UPF_OK;
  if (!src || !idx || !dst || (row_bytes != 4 && row_bytes != 16)) {
    set_error("upf_scatter_rows: null pointer or row size %u (4 or 16)", row_bytes);
    return UPF_ERR_INVALID_ARG;
  }
  UPF_CUDA(launch_rows(src, row_bytes, idx, n, dst, true, (cudaStream_t)stream));
  return UPF_OK;
}

upf_status upf_upload_state(upf_system* s, const float* pos4, const float* vel4, uint32_t n) {
  UPF_TRY(phase_guard(s));
  if (n != s->n_dyn || (n && (!pos4 || !vel4))) {
    set_error("upf_upload_state: need %u dynamic particles and non-null arrays", s->n_dyn);
    return UPF_ERR_INVALID_ARG;
  }
  if (!n) return UPF_OK;
  UPF_CUDA(cudaMemcpyAsync(s->A.pos, pos4, sizeof(float4) * n, cudaMemcpyHostToDevice, s->stream));
  UPF_CUDA(cudaMemcpyAsync(s->A.vel, vel4, sizeof(float4) * n, cudaMemcpyHostToDevice, s->stream));
  UPF_CUDA(launch_upload_keys(*s, s->stream));
  return UPF_OK;
}

// ---- checkpoint / resume ---------------------------------------------------
// The dynamic state as contiguous segments (A copy + keys + device scalars).
namespace {
struct StateSeg {
  void* dev;
  size_t bytes;
};
int state_segments(System& s, StateSeg* seg) {
  const size_t n = s.n_dyn;
  seg[0] = {s.A.pos, sizeof(float4) * n};
  seg[1] = {s.A.vel, sizeof(float4) * n};
  seg[2] = {s.A.lag, sizeof(float4) * n};
  seg[3] = {s.A.id, sizeof(uint32_t) * n};
  seg[4] = {s.A.type, sizeof(int32_t) * n};
  seg[5] = {s.keysA, sizeof(uint32_t) * n};
  seg[6] = {s.st, sizeof(DevState)};
  seg[7] = {s.rb.bodies, sizeof(DevBody) * s.rb.n_bodies};
  return 8;
}
size_t state_total(System& s) {
  StateSeg seg[8];
  const int k = state_segments(s, seg);
  size_t t = 0;
  for (int i = 0; i < k; ++i) t += (seg[i].bytes + 255) & ~size_t(255);
  return t;
}
// copy all segments between the system and a flat buffer (device or host)
upf_status state_copy(System& s, char* flat, bool to_flat, cudaMemcpyKind kind) {
  StateSeg seg[8];
  const int k = state_segments(s, seg);
  size_t off = 0;
  for (int i = 0; i < k; ++i) {
    if (seg[i].bytes) {
      cudaError_t e = to_flat ? cudaMemcpyAsync(flat + off, seg[i].dev, seg[i].bytes, kind, s.stream)
                              : cudaMemcpyAsync(seg[i].dev, flat + off, seg[i].bytes, kind, s.stream);
      if (e != cudaSuccess) {
        set_error("state copy: %s", cudaGetErrorString(e));
        return UPF_ERR_CUDA;
      }
    }
    off += (seg[i].bytes + 255) & ~size_t(255);
  }
  return UPF_OK;
}
}  // namespace

upf_status upf_checkpoint(upf_system* s, int32_t slot) {
  UPF_TRY(phase_guard(s));
  if (slot < 0 || slot > 4096) {
    set_error("upf_checkpoint: slot %d out of range", slot);
    return UPF_ERR_INVALID_ARG;
  }
  if ((size_t)slot >= s->checkpoint_slots.size()) s->checkpoint_slots.resize(slot + 1, nullptr);
  if (!s->checkpoint_slots[slot]) {
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, state_total(*s));
    if (e != cudaSuccess) {
      set_error("upf_checkpoint: cudaMalloc: %s", cudaGetErrorString(e));
      return UPF_ERR_ALLOC;
    }
    s->checkpoint_slots[slot] = p;
  }
  return state_copy(*s, (char*)s->checkpoint_slots[slot], true, cudaMemcpyDeviceToDevice);
}

upf_status upf_restore(upf_system* s, int32_t slot) {
  UPF_TRY(phase_guard(s));
  if (slot < 0 || (size_t)slot >= s->checkpoint_slots.size() || !s->checkpoint_slots[slot]) {
    set_error("upf_restore: slot %d holds no checkpoint", slot);
    return UPF_ERR_INVALID_ARG;
  }
  return state_copy(*s, (char*)s->checkpoint_slots[slot], false, cudaMemcpyDeviceToDevice);
}

size_t upf_state_bytes(const upf_system* s) {
  if (!s || !s->have_particles) return 0;
  return state_total(*const_cast<upf_system*>(s));
}

upf_status upf_state_save(upf_system* s, void* host, size_t bytes) {
  UPF_TRY(phase_guard(s));
  if (!host || bytes < state_total(*s)) {
    set_error("upf_state_save: need %zu bytes", state_total(*s));
    return UPF_ERR_INVALID_ARG;
  }
  UPF_TRY(state_copy(*s, (char*)host, true, cudaMemcpyDeviceToHost));
  UPF_CUDA(cudaStreamSynchronize(s->stream));
  return UPF_OK;
}

upf_status upf_state_load(upf_system* s, const void* host, size_t bytes) {
  UPF_TRY(phase_guard(s));
  if (!host || bytes < state_total(*s)) {
    set_error("upf_state_load: need %zu bytes (same particle count as the saving system)", state_total(*s));
    return UPF_ERR_INVALID_ARG;
  }
  UPF_TRY(state_copy(*s, (char*)const_cast<void*>(host), false, cudaMemcpyHostToDevice));
  UPF_CUDA(cudaStreamSynchronize(s->stream));
  return UPF_OK;
}

upf_status upf_get_launch_config(upf_system* s, upf_launch_config* out) {
  if (!s || !out) {
    set_error("upf_get_launch_config: null");
    return UPF_ERR_INVALID_ARG;
  }
  shape_to_config(s->shape, out);
  return UPF_OK;
}

upf_status upf_set_launch_config(upf_system* s, const upf_launch_config* cfg) {
  if (!s || !cfg) {
    set_error("upf_set_launch_config: null");
    return UPF_ERR_INVALID_ARG;
  }
  const LaunchShape sh = config_to_shape(*cfg);
  const char* why = nullptr;
  if (!shape_valid(sh, false, &why)) {
    set_error("upf_set_launch_config: %s", why);
    return UPF_ERR_INVALID_ARG;
  }
  UPF_CUDA(cudaStreamSynchronize(s->stream));
  s->shape = sh;
  return s->have_particles ? build_step_graph(*s) : UPF_OK;
}

namespace {
struct SysTune {
  System* s;
  void* buf;
};
}  // namespace

upf_status upf_autotune(upf_system* s, int32_t repeats, upf_launch_config* chosen) {
  NvtxRange nvtx("upf_autotune");
  UPF_TRY(phase_guard(s));
  UPF_CUDA(cudaStreamSynchronize(s->stream));
  SysTune t{s, nullptr};
  TuneOps ops;
  ops.ctx = &t;
  ops.shape = &s->shape;
  ops.batched = false;
  ops.stream = s->stream;
  ops.save = [](void* c) -> upf_status {
    SysTune& T = *static_cast<SysTune*>(c);
    cudaError_t e = cudaMalloc(&T.buf, state_total(*T.s));
    if (e != cudaSuccess) {
      T.buf = nullptr;
      set_error("upf_autotune: cudaMalloc: %s", cudaGetErrorString(e));
      return UPF_ERR_ALLOC;
    }
    return state_copy(*T.s, (char*)T.buf, true, cudaMemcpyDeviceToDevice);
  };
  ops.restore = [](void* c) -> upf_status {
    SysTune& T = *static_cast<SysTune*>(c);
    if (!T.buf) return UPF_OK;
    upf_status rc = state_copy(*T.s, (char*)T.buf, false, cudaMemcpyDeviceToDevice);
    cudaStreamSynchronize(T.s->stream);
    cudaFree(T.buf);
    T.buf = nullptr;
    return rc;
  };
  const bool pcisph = s->prm.method == UPF_METHOD_PCISPH;
  ops.prepare = [](void* c, cudaStream_t st) {
    System& S = *static_cast<SysTune*>(c)->s;
    cudaError_t e = launch_sort_phase(S, st);
    if (e == cudaSuccess) e = launch_neighbor_phase(S, st);
    if (e == cudaSuccess) e = launch_force_phase(S, st);
    if (e == cudaSuccess && S.prm.method == UPF_METHOD_PCISPH) e = launch_loop_init(S, st);
    return e;
  };
  ops.nlist = [](void* c, cudaStream_t st) { return launch_neighbor_phase(*static_cast<SysTune*>(c)->s, st); };
  if (pcisph) {
    ops.stage = [](void* c, cudaStream_t st) { return launch_list_staging(*static_cast<SysTune*>(c)->s, st); };
    // the iterations of the last step weigh the staging kernel against the
    // passes' per-iteration saving
    UPF_CUDA(cudaMemcpy(s->st_host, s->st, sizeof(DevState), cudaMemcpyDeviceToHost));
    ops.loop_iterations = (float)std::max(s->st_host->final_iterations, std::max(s->prm.min_loops, 1));
    ops.external = [](void* c, cudaStream_t st) { return launch_force_phase(*static_cast<SysTune*>(c)->s, st); };
    ops.density = [](void* c, cudaStream_t st) { return launch_loop_density(*static_cast<SysTune*>(c)->s, st); };
    ops.pforce = [](void* c, cudaStream_t st) { return launch_loop_pforce(*static_cast<SysTune*>(c)->s, st); };
  }
  // every mode is timed on the lists of the same step: stage them whatever
  // the shape while tuning
  s->stage_always = pcisph;
  const upf_status rc = autotune_shapes(ops, repeats, chosen);
  s->stage_always = false;
  UPF_TRY(rc);
  UPF_TRY(check_device_errors(*s));
  return build_step_graph(*s);
}

upf_status upf_profile_step(upf_system* s, upf_phase_times* out) {
  NvtxRange nvtx("upf_profile_step");
  UPF_TRY(phase_guard(s));
  s->stepped = true;
  if (!out) {
    set_error("upf_profile_step: null");
    return UPF_ERR_INVALID_ARG;
  }
  std::memset(out, 0, sizeof(*out));
  cudaStream_t st = s->stream;
  cudaEvent_t ev[8];
  for (auto& e : ev) UPF_CUDA(cudaEventCreate(&e));
  auto elapsed = [&](cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
  };
  upf_status rc = UPF_OK;
  do {
    UPF_CUDA(cudaEventRecord(ev[0], st));
    UPF_CUDA(launch_sort_phase(*s, st));
    UPF_CUDA(cudaEventRecord(ev[1], st));
    UPF_CUDA(launch_neighbor_phase(*s, st));
    UPF_CUDA(cudaEventRecord(ev[2], st));
    UPF_CUDA(launch_force_phase(*s, st));
    UPF_CUDA(cudaEventRecord(ev[3], st));
    UPF_CUDA(cudaStreamSynchronize(st));
    out->sort_ms = elapsed(ev[0], ev[1]);
    out->neighbors_ms = elapsed(ev[1], ev[2]);
    out->forces_ms = elapsed(ev[2], ev[3]);
    float loop = 0;
    if (s->prm.method == UPF_METHOD_PCISPH) {
      UPF_CUDA(launch_loop_init(*s, st));
      for (int it = 0; it < s->prm.max_loops + 1; ++it) {
        UPF_CUDA(cudaEventRecord(ev[4], st));
        UPF_CUDA(launch_loop_density(*s, st));
        UPF_CUDA(cudaEventRecord(ev[5], st));
        UPF_CUDA(launch_loop_pforce(*s, st));
        UPF_CUDA(cudaEventRecord(ev[6], st));
        UPF_CUDA(launch_loop_ctl(*s, st, 0, false));
        UPF_CUDA(cudaEventRecord(ev[7], st));
        UPF_CUDA(cudaMemcpyAsync(s->st_host, s->st, sizeof(DevState), cudaMemcpyDeviceToHost, st));
        UPF_CUDA(cudaStreamSynchronize(st));
        out->density_ms_total += elapsed(ev[4], ev[5]);
        out->pforce_ms_total += elapsed(ev[5], ev[6]);
        loop += elapsed(ev[4], ev[7]);
        const DevState& d = *s->st_host;
        int cont = (d.iteration < s->prm.min_loops) || (d.too_large && d.iteration < s->prm.max_loops);
        if (d.error_flags & ERR_NAN) cont = 0;
        out->iterations = d.iteration;
        if (!cont) break;
      }
    }
    out->loop_ms = loop;
    UPF_CUDA(cudaEventRecord(ev[0], st));
    UPF_CUDA(launch_integrate_phase(*s, st));
    UPF_CUDA(cudaEventRecord(ev[1], st));
    UPF_CUDA(cudaStreamSynchronize(st));
    out->integrate_ms = elapsed(ev[0], ev[1]);
    out->launches = pipeline_launches_per_step(*s, out->iterations);
  } while (0);
  for (auto& e : ev) cudaEventDestroy(e);
  if (rc != UPF_OK) return rc;
  return check_device_errors(*s);
}

// ---- readback -------------------------------------------------------------
static upf_status copy_out_f4(void* dst, const float4* src, uint32_t n, cudaStream_t st) {
  if (!dst || !n) return UPF_OK;
  UPF_CUDA(cudaMemcpyAsync(dst, src, sizeof(float4) * n, cudaMemcpyDeviceToHost, st));
  return UPF_OK;
}

upf_status upf_get_particles(upf_system* s, float* pos4, float* vel4, float* density, float* pressure,
                             int32_t* type, uint32_t* id, uint32_t* n_out) {
  UPF_TRY(phase_guard(s));
  const uint32_t n = s->n_dyn;
  cudaStream_t st = s->stream;
  UPF_TRY(copy_out_f4(pos4, s->A.pos, n, st));
  UPF_TRY(copy_out_f4(vel4, s->A.vel, n, st));
  if (density && n) UPF_CUDA(cudaMemcpyAsync(density, s->rho, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
  if (pressure && n) UPF_CUDA(cudaMemcpyAsync(pressure, s->press, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
  if (type && n) UPF_CUDA(cudaMemcpyAsync(type, s->A.type, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
  if (id && n) UPF_CUDA(cudaMemcpyAsync(id, s->A.id, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, st));
  UPF_CUDA(cudaStreamSynchronize(st));
  if (n_out) *n_out = n;
  return UPF_OK;
}

upf_status upf_get_particles_input_order(upf_system* s, float* pos4, float* vel4, float* density, float* pressure,
                                        int32_t* type, uint32_t n) {
  UPF_TRY(phase_guard(s));
  const uint32_t total = s->n_dyn + s->n_static;
  if (n != total) {
    set_error("upf_get_particles_input_order: n = %u, but the last upf_set_particles call had %u particles", n,
              total);
    return UPF_ERR_INVALID_ARG;
  }
  if (n == 0) return UPF_OK;
  cudaStream_t st = s->stream;
  // one stream-ordered block: positions, velocities, density, pressure, type
  const size_t bytes = (size_t)n * (16 + 16 + 4 + 4 + 4);
  char* buf = nullptr;
  UPF_CUDA(cudaMallocAsync((void**)&buf, bytes, st));
  float4* opos = (float4*)buf;
  float4* ovel = opos + n;
  float* orho = (float*)(ovel + n);
  float* opress = orho + n;
  int32_t* otype = (int32_t*)(opress + n);
  k_scatter_input_order<<<(n + 255) / 256, 256, 0, st>>>(s->n_dyn, s->A, s->rho, s->press, s->n_static, s->spos,
                                                         s->sid, s->dp.origin, s->dp.scales, s->prm.rest_density,
                                                         n, opos, ovel, orho, opress, otype);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && pos4) e = cudaMemcpyAsync(pos4, opos, sizeof(float4) * n, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && vel4) e = cudaMemcpyAsync(vel4, ovel, sizeof(float4) * n, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && density) e = cudaMemcpyAsync(density, orho, sizeof(float) * n, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && pressure)
    e = cudaMemcpyAsync(pressure, opress, sizeof(float) * n, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && type) e = cudaMemcpyAsync(type, otype, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st);
  const cudaError_t ef = cudaFreeAsync(buf, st);
  if (e == cudaSuccess) e = ef;
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    set_error("upf_get_particles_input_order: %s", cudaGetErrorString(e));
    return UPF_ERR_CUDA;
  }
  return UPF_OK;
}

upf_status upf_get_lagged_state(upf_system* s, float* lag4, uint32_t n) {
  UPF_TRY(phase_guard(s));
  if (n != s->n_dyn || (n && !lag4)) {
    set_error("upf_get_lagged_state: n = %u, the system has %u dynamic particles", n, s->n_dyn);
    return UPF_ERR_INVALID_ARG;
  }
  if (n) UPF_CUDA(cudaMemcpyAsync(lag4, s->A.lag, sizeof(float4) * n, cudaMemcpyDeviceToHost, s->stream));
  UPF_CUDA(cudaStreamSynchronize(s->stream));
  return UPF_OK;
}

// ---- asynchronous per-frame exchange -----------------------------------------
// A host-driven caller uploads its particles before a step and reads the
// result after it (CopyParticleDataHostToDevice, CopyParticlesCUDA). Done
// in stream order, those copies sit between the steps. Here they run on a
// copy stream of each direction against device staging buffers: an upload
// copies into staging while the previous step still runs, and enters the
// state in stream order before the next step; a readback takes a device
// copy of the result in stream order and copies it to the host while the
// next step runs. With one stream per direction, a readback never holds up
// the next upload. Events order the buffers' reuse.
}  // extern "C"

cudaError_t upf::frame_streams_create(FrameIO& io, cudaStream_t compute) {
  cudaError_t e = cudaStreamCreateWithFlags(&io.up, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&io.down, cudaStreamNonBlocking);
  for (cudaEvent_t* ev : {&io.staged, &io.consumed, &io.snapped, &io.read_done})
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
  for (cudaEvent_t& ev : io.chunk_down)
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  for (cudaEvent_t ev : {io.staged, io.consumed, io.snapped, io.read_done})  // all four start completed
    if (e == cudaSuccess) e = cudaEventRecord(ev, compute);
  return e;
}

void upf::frame_streams_destroy(FrameIO& io) {
  for (cudaStream_t c : {io.up, io.down})
    if (c) cudaStreamSynchronize(c);
  for (cudaEvent_t e : {io.staged, io.consumed, io.snapped, io.read_done})
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : io.chunk_down)
    if (e) cudaEventDestroy(e);
  for (cudaStream_t c : {io.up, io.down})
    if (c) cudaStreamDestroy(c);
  io = FrameIO{};
}

namespace upf {
static upf_status frames_ready(System& s) {
  FrameIO& io = s.io;
  if (io.ready) return UPF_OK;
  const uint32_t c = s.capacity;
  UPF_TRY(dalloc(s, &io.in_pos, c));
  UPF_TRY(dalloc(s, &io.in_vel, c));
  UPF_TRY(dalloc(s, &io.out_pos, c));
  UPF_TRY(dalloc(s, &io.out_vel, c));
  UPF_TRY(dalloc(s, &io.out_rho, c));
  UPF_TRY(dalloc(s, &io.out_press, c));
  UPF_TRY(dalloc(s, &io.out_type, c));
  UPF_TRY(dalloc(s, &io.out_id, c));
  UPF_CUDA(frame_streams_create(io, s.stream));
  io.ready = true;
  return UPF_OK;
}

}  // namespace upf

extern "C" {

upf_status upf_upload_state_async(upf_system* s, const float* pos4, const float* vel4, uint32_t n) {
  UPF_TRY(phase_guard(s));
  if (n != s->n_dyn || (n && (!pos4 || !vel4))) {
    set_error("upf_upload_state_async: need %u dynamic particles and non-null arrays", s->n_dyn);
    return UPF_ERR_INVALID_ARG;
  }
  if (!n) return UPF_OK;
  UPF_TRY(frames_ready(*s));
  FrameIO& io = s->io;
  UPF_CUDA(cudaStreamWaitEvent(io.up, io.consumed, 0));  // the last upload has left the staging buffers
  UPF_CUDA(cudaMemcpyAsync(io.in_pos, pos4, sizeof(float4) * n, cudaMemcpyHostToDevice, io.up));
  UPF_CUDA(cudaMemcpyAsync(io.in_vel, vel4, sizeof(float4) * n, cudaMemcpyHostToDevice, io.up));
  UPF_CUDA(cudaEventRecord(io.staged, io.up));
  UPF_CUDA(cudaStreamWaitEvent(s->stream, io.staged, 0));
  UPF_CUDA(cudaMemcpyAsync(s->A.pos, io.in_pos, sizeof(float4) * n, cudaMemcpyDeviceToDevice, s->stream));
  UPF_CUDA(cudaMemcpyAsync(s->A.vel, io.in_vel, sizeof(float4) * n, cudaMemcpyDeviceToDevice, s->stream));
  UPF_CUDA(launch_upload_keys(*s, s->stream));
  UPF_CUDA(cudaEventRecord(io.consumed, s->stream));
  return UPF_OK;
}

upf_status upf_get_particles_async(upf_system* s, float* pos4, float* vel4, float* density, float* pressure,
                                   int32_t* type, uint32_t* id, uint32_t* n_out) {
  UPF_TRY(phase_guard(s));
  const uint32_t n = s->n_dyn;
  if (n_out) *n_out = n;
  if (!n) return UPF_OK;
  UPF_TRY(frames_ready(*s));
  FrameIO& io = s->io;
  cudaStream_t st = s->stream;
  UPF_CUDA(cudaStreamWaitEvent(st, io.read_done, 0));  // the last readback has left the snapshot
  struct Item {
    void* host;
    void* snap;
    const void* src;
    size_t bytes;
  } items[] = {{pos4, io.out_pos, s->A.pos, sizeof(float4) * n},   {vel4, io.out_vel, s->A.vel, sizeof(float4) * n},
               {density, io.out_rho, s->rho, sizeof(float) * n},   {pressure, io.out_press, s->press, sizeof(float) * n},
               {type, io.out_type, s->A.type, sizeof(int32_t) * n}, {id, io.out_id, s->A.id, sizeof(uint32_t) * n}};
  for (const Item& it : items)
    if (it.host) UPF_CUDA(cudaMemcpyAsync(it.snap, it.src, it.bytes, cudaMemcpyDeviceToDevice, st));
  UPF_CUDA(cudaEventRecord(io.snapped, st));
  UPF_CUDA(cudaStreamWaitEvent(io.down, io.snapped, 0));
  for (const Item& it : items)
    if (it.host) UPF_CUDA(cudaMemcpyAsync(it.host, it.snap, it.bytes, cudaMemcpyDeviceToHost, io.down));
  UPF_CUDA(cudaEventRecord(io.read_done, io.down));
  return UPF_OK;
}

upf_status upf_exchange_frame_async(upf_system* s, float* pos4, float* vel4, float* density, float* pressure,
                                    int32_t* type, uint32_t* id, uint32_t chunks, uint32_t* n_out) {
  UPF_TRY(phase_guard(s));
  const uint32_t n = s->n_dyn;
  if (n_out) *n_out = n;
  if (!pos4 || !vel4 || chunks < 1 || chunks > (uint32_t)FrameIO::kMaxChunks) {
    set_error("upf_exchange_frame_async: positions and velocities are required, chunks in 1..%d",
              FrameIO::kMaxChunks);
    return UPF_ERR_INVALID_ARG;
  }
  if (!n) return UPF_OK;
  UPF_TRY(frames_ready(*s));
  FrameIO& io = s->io;
  cudaStream_t st = s->stream;
  // the frame, as upf_get_particles_async takes it
  UPF_CUDA(cudaStreamWaitEvent(st, io.read_done, 0));  // the last readback has left the snapshot
  struct Item {
    char* host;
    char* snap;
    const void* src;
    size_t elem;
  } items[] = {{(char*)pos4, (char*)io.out_pos, s->A.pos, sizeof(float4)},
               {(char*)vel4, (char*)io.out_vel, s->A.vel, sizeof(float4)},
               {(char*)density, (char*)io.out_rho, s->rho, sizeof(float)},
               {(char*)pressure, (char*)io.out_press, s->press, sizeof(float)},
               {(char*)type, (char*)io.out_type, s->A.type, sizeof(int32_t)},
               {(char*)id, (char*)io.out_id, s->A.id, sizeof(uint32_t)}};
  for (const Item& it : items)
    if (it.host) UPF_CUDA(cudaMemcpyAsync(it.snap, it.src, it.elem * n, cudaMemcpyDeviceToDevice, st));
  UPF_CUDA(cudaEventRecord(io.snapped, st));
  // chunk by chunk: the down stream copies the chunk's positions and
  // velocities to the host; once they have landed, the up stream copies them
  // back from those host arrays into the staging buffers. The other fields
  // follow all the chunks, so the upload's last chunk waits for no more than
  // its own positions and velocities.
  UPF_CUDA(cudaStreamWaitEvent(io.down, io.snapped, 0));
  UPF_CUDA(cudaStreamWaitEvent(io.up, io.consumed, 0));  // the last upload has left the staging buffers
  const uint32_t per = (n + chunks - 1) / chunks;
  for (uint32_t c = 0; c < chunks; ++c) {
    const uint32_t b = c * per, e = std::min(n, b + per);
    if (b >= e) break;
    for (int k = 0; k < 2; ++k)
      UPF_CUDA(cudaMemcpyAsync(items[k].host + items[k].elem * b, items[k].snap + items[k].elem * b,
                               items[k].elem * (e - b), cudaMemcpyDeviceToHost, io.down));
    UPF_CUDA(cudaEventRecord(io.chunk_down[c], io.down));
    UPF_CUDA(cudaStreamWaitEvent(io.up, io.chunk_down[c], 0));
    UPF_CUDA(cudaMemcpyAsync(io.in_pos + b, pos4 + 4 * (size_t)b, sizeof(float4) * (e - b), cudaMemcpyHostToDevice,
                             io.up));
    UPF_CUDA(cudaMemcpyAsync(io.in_vel + b, vel4 + 4 * (size_t)b, sizeof(float4) * (e - b), cudaMemcpyHostToDevice,
                             io.up));
  }
  for (int k = 2; k < 6; ++k)
    if (items[k].host)
      UPF_CUDA(cudaMemcpyAsync(items[k].host, items[k].snap, items[k].elem * n, cudaMemcpyDeviceToHost, io.down));
  UPF_CUDA(cudaEventRecord(io.read_done, io.down));
  UPF_CUDA(cudaEventRecord(io.staged, io.up));
  // the upload enters the state before the next step, as in upf_upload_state_async
  UPF_CUDA(cudaStreamWaitEvent(st, io.staged, 0));
  UPF_CUDA(cudaMemcpyAsync(s->A.pos, io.in_pos, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st));
  UPF_CUDA(cudaMemcpyAsync(s->A.vel, io.in_vel, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st));
  UPF_CUDA(launch_upload_keys(*s, st));
  UPF_CUDA(cudaEventRecord(io.consumed, st));
  return UPF_OK;
}

upf_status upf_wait_frames(upf_system* s) {
  if (!s) {
    set_error("upf_wait_frames: null");
    return UPF_ERR_INVALID_ARG;
  }
  if (!s->io.ready) return UPF_OK;
  UPF_CUDA(cudaStreamWaitEvent(s->stream, s->io.read_done, 0));  // later work on the stream comes after
  UPF_CUDA(cudaEventSynchronize(s->io.staged));
  UPF_CUDA(cudaEventSynchronize(s->io.read_done));
  return UPF_OK;
}

upf_status upf_get_step_fields(upf_system* s, float* force4, float* pforce4, float* predicted_density,
                               uint32_t* id, uint32_t* n_out) {
  UPF_TRY(phase_guard(s));
  const uint32_t n = s->n_dyn;
  cudaStream_t st = s->stream;
  UPF_TRY(copy_out_f4(force4, s->force, n, st));
  UPF_TRY(copy_out_f4(pforce4, s->pforce, n, st));
  if (predicted_density && n)
    UPF_CUDA(cudaMemcpyAsync(predicted_density, s->rho, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
  if (id && n) UPF_CUDA(cudaMemcpyAsync(id, s->B.id, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, st));
  UPF_CUDA(cudaStreamSynchronize(st));
  if (n_out) *n_out = n;
  return UPF_OK;
}

upf_status upf_get_neighbors(upf_system* s, uint32_t* counts, uint32_t* lists, uint32_t cap, uint32_t* n_out) {
  UPF_TRY(phase_guard(s));
  const uint32_t n = s->n_dyn;
  if (n_out) *n_out = n;
  if (!n) return UPF_OK;
  cudaStream_t st = s->stream;
  std::vector<uint32_t> cnt(n), bid(n), sid(s->n_static);
  UPF_CUDA(cudaMemcpyAsync(cnt.data(), s->ncnt, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, st));
  UPF_CUDA(cudaMemcpyAsync(bid.data(), s->B.id, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, st));
  if (s->n_static)
    UPF_CUDA(cudaMemcpyAsync(sid.data(), s->sid, sizeof(uint32_t) * s->n_static, cudaMemcpyDeviceToHost, st));
  const uint32_t maxn = s->prm.max_neighbors;
  std::vector<uint32_t> nb((size_t)s->nstride * maxn);
  UPF_CUDA(cudaMemcpyAsync(nb.data(), s->nbr, sizeof(uint32_t) * nb.size(), cudaMemcpyDeviceToHost, st));
  UPF_CUDA(cudaStreamSynchronize(st));
  for (uint32_t i = 0; i < n; ++i) {
    if (counts) counts[i] = cnt[i];
    if (!lists) continue;
    for (uint32_t k = 0; k < cnt[i] && k < cap; ++k) {
      uint32_t code = nb[(size_t)k * s->nstride + i];
      const uint32_t base = s->dp.static_base;
      lists[(size_t)i * cap + k] = (code >= base) ? sid[code - base] : bid[code];
    }
  }
  return UPF_OK;
}

upf_status upf_get_sorted_keys(upf_system* s, uint32_t* keys, uint32_t* ids, uint32_t* n_out) {
  UPF_TRY(phase_guard(s));
  const uint32_t n = s->n_dyn;
  if (keys && n) UPF_CUDA(cudaMemcpyAsync(keys, s->keysA, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s->stream));
  if (ids && n) UPF_CUDA(cudaMemcpyAsync(ids, s->B.id, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s->stream));
  UPF_CUDA(cudaStreamSynchronize(s->stream));
  if (n_out) *n_out = n;
  return UPF_OK;
}

upf_status upf_get_cell_ranges(upf_system* s, uint32_t* start, uint32_t* end, uint32_t* ncells_out) {
  UPF_TRY(phase_guard(s));
  if (start) UPF_CUDA(cudaMemcpyAsync(start, s->cstart, sizeof(uint32_t) * s->ncells, cudaMemcpyDeviceToHost, s->stream));
  if (end) UPF_CUDA(cudaMemcpyAsync(end, s->cend, sizeof(uint32_t) * s->ncells, cudaMemcpyDeviceToHost, s->stream));
  UPF_CUDA(cudaStreamSynchronize(s->stream));
  if (ncells_out) *ncells_out = s->ncells;
  return UPF_OK;
}

// ---- stateless building blocks ---------------------------------------------
upf_status upf_morton_keys(const float* pos4, uint32_t n, const float origin[3], const float scales[3],
                           uint32_t* keys, void* stream) {
  if (n && (!pos4 || !keys || !origin || !scales)) {
    set_error("upf_morton_keys: null argument");
    return UPF_ERR_INVALID_ARG;
  }
  UPF_CUDA(morton_keys((const float4*)pos4, n, make_float3(origin[0], origin[1], origin[2]),
                       make_float3(scales[0], scales[1], scales[2]), keys, (cudaStream_t)stream));
  return UPF_OK;
}

size_t upf_radix_sort_temp_bytes(uint32_t n) { return radix_temp_bytes(n); }

upf_status upf_radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t n, int32_t key_bits, void* temp,
                                size_t temp_bytes, void* stream) {
  if (n == 0) return UPF_OK;
  if (!keys || !vals || !temp || key_bits < 1 || key_bits > 32) {
    set_error("upf_radix_sort_pairs: bad arguments");
    return UPF_ERR_INVALID_ARG;
  }
  if (temp_bytes < radix_temp_bytes(n)) {
    set_error("upf_radix_sort_pairs: temp_bytes %zu < required %zu", temp_bytes, radix_temp_bytes(n));
    return UPF_ERR_INVALID_ARG;
  }
  uint32_t* kalt = (uint32_t*)temp;
  uint32_t* valt = kalt + ((n + 63) & ~63u);
  uint32_t* counts = valt + ((n + 63) & ~63u);
  UPF_CUDA(radix_init());  // once per device
  UPF_CUDA(radix_sort_pairs(keys, vals, kalt, valt, counts, n, key_bits, false, (cudaStream_t)stream));
  return UPF_OK;
}

upf_status upf_cell_ranges(const uint32_t* keys, uint32_t n, int32_t shift, uint32_t ncells, uint32_t* start,
                           uint32_t* end, void* stream) {
  if ((n && !keys) || !start || !end || shift < 0 || shift > 31 || ncells == 0) {
    set_error("upf_cell_ranges: bad arguments");
    return UPF_ERR_INVALID_ARG;
  }
  UPF_CUDA(cell_ranges(keys, n, shift, ncells, start, end, (cudaStream_t)stream));
  return UPF_OK;
}

}  // extern "C"
