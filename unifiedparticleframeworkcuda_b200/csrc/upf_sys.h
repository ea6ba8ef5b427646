// upf_sys.h — the state behind one upf_system handle (library-internal).
//
// Device layout (structure of arrays, float4 for 3-vectors so each gather is
// one 16-byte transaction):
//   dynamic set (liquid, rigid, granular particles), two copies:
//     A = state after integration, in the order of the last sort, with the
//         Morton keys of the new positions (input to the next sort);
//     B = the sorted working copy a step reads (gathered from A by the sort
//         permutation).
//   boundary set (FROZEN particles): sorted once at upload; static.
//   per-step fields (indexed like B): external force, correction pressure
//   force, predicted position, predicted density, correction pressure.
//   neighbour lists: column-major nbr[k * stride + i] (coalesced reads when
//   consecutive threads take consecutive particles). Neighbour index j < stride
//   is dynamic particle j; stride + b is boundary particle b. The arrays a
//   neighbour loop gathers from (B.pos/vel/type, xs, pq, wvol) are allocated
//   with stride + capacity entries and hold the boundary particles' data in
//   that tail, so a gather needs no branch on the particle's set.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <vector>

#include "upf_common.cuh"
#include "upf_internal.h"

namespace upf {

struct DynArrays {
  float4* pos = nullptr;
  float4* vel = nullptr;
  float4* lag = nullptr;   // (previous correction pressure, last final correction pressure, last predicted density, -)
  uint32_t* id = nullptr;
  int32_t* type = nullptr;
};

// Rigid bodies. The rigid particles form a list grouped by body (body b owns
// entries [start[b], start[b+1]), in input-id order); what is fixed per
// particle is indexed by input id or by list entry, so nothing but the
// entry -> sorted-index map changes when the particles are re-sorted.
struct RigidArrays {
  uint32_t n_bodies = 0, n_rigid = 0, n_ids = 0;
  DevBody* bodies = nullptr;
  uint32_t* start = nullptr;    // [n_bodies + 1]
  int32_t* id_body = nullptr;   // input id -> body index, -1 for particles of no body
  uint32_t* id_entry = nullptr; // input id -> list entry, 0xffffffff for particles of no body
  float4* entry_r0 = nullptr;   // list entry -> position relative to the centre of mass, body frame
  int32_t* entry_body = nullptr;
  uint32_t* entry_slot = nullptr; // list entry -> current sorted index (set after each sort)
};

// Launch shapes of the tunable passes (upf_launch_config): CTA sizes, and
// the list rows each TMA stage carries in the loop passes. The loop passes
// are instantiated for the (threads, rows) pairs below, whose ring buffers
// fit the 48 KB of static shared memory per CTA.
struct LaunchShape {
  int nlist_threads = 256;     // 64, 128, 256
  int external_threads = 256;  // 128, 256
  int density_threads = 256;   // with density_rows: see kLoopShapes
  int density_rows = 8;
  int pforce_threads = 256;    // with pforce_rows: the same pairs, where the ring fits
  int pforce_rows = 4;
  int density_mode = 0;        // list entries by 0: the TMA ring, 1: direct loads (rows = entries per batch),
                               // 2: staged neighbourhoods (256 threads; rows = entries per batch)
  int pforce_mode = 0;
  int nlist_mode = 0;          // 0: each lane its own query box; 1: the warp's union of boxes
};
bool shape_valid(const LaunchShape& s, bool batched, const char** why);
// (mode, threads, rows) triples of the loop passes: TMA ring (mode 0),
// direct loads (mode 1) and staged neighbourhoods (mode 2, single scenes)
constexpr int kLoopShapes[][3] = {{0, 128, 4}, {0, 128, 8}, {0, 128, 16}, {0, 256, 2}, {0, 256, 4},
                                  {0, 256, 8}, {0, 512, 2}, {0, 512, 4},  {0, 1024, 2}, {1, 128, 4},
                                  {1, 128, 8}, {1, 256, 4}, {1, 256, 8},  {1, 512, 4},  {1, 512, 8},
                                  {2, 256, 4}, {2, 256, 8}};
constexpr int kNumLoopShapes = sizeof(kLoopShapes) / sizeof(kLoopShapes[0]);
// The pressure-force pass's TMA ring carries a 32-bit value per list entry
// beside its code: shapes whose rings (three stages a warp) leave no room
// within the 48 KB of static shared memory are not built for that pass.
constexpr bool pforce_ring_fits(int mode, int threads, int rows) {
  return mode != 0 || (threads / 32) * ((3 * rows * 32 * 8 + 3 * 8 + 127) / 128 * 128) + 1024 <= 48 * 1024;
}
static_assert(pforce_ring_fits(LaunchShape{}.pforce_mode, LaunchShape{}.pforce_threads, LaunchShape{}.pforce_rows),
              "the default pressure-force shape must be one that is built");
// Staged neighbourhoods (loop-pass mode 2). The lists of each chunk of
// kStageChunk consecutive sorted particles (one CTA of a staged pass) are
// rewritten once per step against the chunk's union of neighbours: ucodes
// holds the union's neighbour indices (at most kUnionMax a chunk), ucount its
// size (kUnionOverflow: the union did not fit, the chunk's passes read the
// plain lists), and lloc the list entries as 16-bit positions in the union,
// four to a 64-bit word, lloc[(k / 4) * stride + i]. A staged pass copies the
// union's data into shared memory once and reads each neighbour from there.
constexpr int kStageChunk = 256;
constexpr uint32_t kUnionMax = 2048;
constexpr uint32_t kUnionOverflow = 0xffffffffu;
constexpr bool loop_mode_staged(int mode) { return mode == 2; }

constexpr int kListRowVariants = 4;  // tensor maps for 2, 4, 8 and 16 rows per box
inline int rows_index(int rows) { return rows == 2 ? 0 : (rows == 4 ? 1 : (rows == 8 ? 2 : 3)); }

// Batched scenes (upf_batch_*): independent scenes in one index space, each
// in its own segment that starts on a kSegAlign boundary, so every CTA of a
// kernel over that space (CTA sizes dividing kSegAlign) belongs to one scene.
// A CTA finds its scene in `group_scene`, and takes the scene's parameters,
// tables, device state and particle range from the tables below.
constexpr uint32_t kSegAlign = 256;
constexpr uint32_t kLutFloats = 5 * UPF_LUT_ENTRIES + kThresholds;

struct BatchView {
  const DevParams* params = nullptr;     // [scenes]
  const float* luts = nullptr;           // [scenes][kLutFloats]
  DevState* st = nullptr;                // [scenes]
  const uint32_t* group_scene = nullptr; // [slots / kSegAlign]
  const uint32_t* seg_end = nullptr;     // [scenes] exclusive end of the scene's particles
  const uint32_t* cell_base = nullptr;   // [scenes] offset of the scene's cell table
};

// Asynchronous per-frame exchange of a system or a batch: host copies run on
// `up` (host to device) and `down` (device to host) against device staging
// buffers, so that they overlap the steps on the compute stream and each
// other. Created on first use.
struct FrameIO {
  cudaStream_t up = nullptr;
  cudaStream_t down = nullptr;
  cudaEvent_t staged = nullptr;     // upload copied into in_*
  cudaEvent_t consumed = nullptr;   // in_* entered into the state
  cudaEvent_t snapped = nullptr;    // result copied into out_*
  cudaEvent_t read_done = nullptr;  // out_* copied to the host
  static constexpr int kMaxChunks = 16;
  cudaEvent_t chunk_down[kMaxChunks] = {};  // upf_exchange_frame_async: chunk c has reached the host
  float4* in_pos = nullptr;
  float4* in_vel = nullptr;
  float4* out_pos = nullptr;
  float4* out_vel = nullptr;
  float* out_rho = nullptr;
  float* out_press = nullptr;
  int32_t* out_type = nullptr;
  uint32_t* out_id = nullptr;
  bool ready = false;
};
// streams and events, all four events recorded once on `compute` (upf_api.cu)
cudaError_t frame_streams_create(FrameIO& io, cudaStream_t compute);
void frame_streams_destroy(FrameIO& io);  // waits for the copies; buffers stay with their owner

struct System {
  upf_params prm{};
  DevParams dp{};
  int device = 0;
  uint32_t capacity = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;

  uint32_t n_dyn = 0, n_static = 0;
  bool have_particles = false;
  bool stepped = false;          // a step or phase ran since the last upf_set_particles
  bool graph_stale = false;      // the dynamic count changed (upf_set_dynamic_device): rebuild the step graph

  DynArrays A, B;
  uint32_t* keysA = nullptr;   // keys of A (sorted in place by the sort)
  uint32_t* perm = nullptr;    // sort values (permutation into A)
  uint32_t* sort_tmp = nullptr;
  size_t sort_tmp_bytes = 0;

  // per-step fields (B order)
  float4* force = nullptr;
  float4* pforce = nullptr;
  float4* xs = nullptr;
  float* rho = nullptr;
  float* press = nullptr;
  float4* pq = nullptr;        // (position, press / rest_density^2): the pressure-force pass's one gather
  float* wvol = nullptr;       // Akinci volume per neighbour index (dynamic, then boundary tail)

  // neighbour lists
  uint32_t* nbr = nullptr;
  // per list entry, at the step's positions: the kernel-table bin (WCSPH),
  // or the bits of the pressure-gradient table value at that bin (PCISPH,
  // the one table the pressure-force pass reads)
  uint32_t* lval = nullptr;
  uint32_t* ncnt = nullptr;
  CUtensorMap nbr_maps[kListRowVariants];   // 2D [max_neighbors][nstride] uint32 views of nbr for TMA, box 32 x {4, 8, 16}
  CUtensorMap lval_maps[kListRowVariants];  // same views of lval (uint32)
  uint32_t nstride = 0;
  LaunchShape shape;
  // staged neighbourhoods (PCISPH systems; see kStageChunk)
  uint32_t* ucodes = nullptr;            // [chunks][kUnionMax]
  uint32_t* ucount = nullptr;            // [chunks]
  unsigned long long* lloc = nullptr;    // [ceil(max_neighbors / 4)][nstride]
  uint32_t stage_cap = kUnionMax;        // union capacity used (tests lower it to reach the fallback)
  bool stage_always = false;             // stage the lists whatever the shape (set while autotuning)
  bool lists_staged = false;             // the last list build was staged (host-side, in launch order)
  bool graph_stages = false;             // a step of the captured step graph stages its lists

  // cells
  uint32_t ncells = 0;
  uint32_t* cstart = nullptr;
  uint32_t* cend = nullptr;
  uint32_t* sstart = nullptr;
  uint32_t* send = nullptr;

  // boundary set
  float4* spos = nullptr;
  uint32_t* skeys = nullptr;
  uint32_t* sid = nullptr;
  float* swvol = nullptr;

  // lookup tables (5 x 301 floats)
  float* luts = nullptr;

  DevState* st = nullptr;      // device scalars
  DevState* st_host = nullptr; // pinned mirror

  // CUDA graph of one full step
  cudaGraphExec_t step_exec = nullptr;
  cudaGraph_t step_graph = nullptr;
  int key_bits = 30;

  RigidArrays rb;
  std::vector<void*> rigid_allocations;   // freed when bodies are set again
  // host copy of the last upload (input order), for body assembly
  std::vector<float4> host_pos, host_vel;
  std::vector<int32_t> host_type;

  std::vector<void*> allocations;
  std::vector<void*> checkpoint_slots;  // device copies of the dynamic state (upf_checkpoint);
                                        // dropped when particles or bodies are set

  FrameIO io;  // asynchronous per-frame exchange (upf_upload_state_async, ...)
};

// The state behind one upf_batch handle: every array spans the batch's slot
// space (scene s owns slots [seg_begin[s], seg_begin[s] + padded count), its
// particles in [seg_begin[s], seg_end[s]), the rest padding that sorts last).
struct BatchSystem {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  uint32_t n_scenes = 0, n_slots = 0, n_particles = 0;
  std::vector<upf_params> prm;
  std::vector<uint32_t> count, seg_begin, seg_end, cell_base;
  uint32_t n_cells = 0;       // sum of the scenes' cell tables
  uint32_t list_rows = 0;     // neighbour-list capacity (max over scenes)
  int scene_bits = 1;         // key bits of the scene index (second sort stage)
  bool have_particles = false;

  DynArrays A, B;
  uint32_t* keysA = nullptr;
  uint32_t* perm = nullptr;
  uint32_t* digits = nullptr;  // second sort stage keys (scene of each element)
  uint32_t* sort_tmp = nullptr;
  float4* force = nullptr;
  float4* pforce = nullptr;
  float4* xs = nullptr;
  float* rho = nullptr;
  float* press = nullptr;
  float4* pq = nullptr;
  uint32_t* nbr = nullptr;
  uint32_t* lval = nullptr;     // pressure-gradient table value bits per list entry
  uint32_t* ncnt = nullptr;
  CUtensorMap nbr_maps[kListRowVariants];
  CUtensorMap lval_maps[kListRowVariants];
  uint32_t* cstart = nullptr;
  uint32_t* cend = nullptr;
  LaunchShape shape;

  DevParams* params_d = nullptr;
  float* luts_d = nullptr;
  DevState* st_d = nullptr;
  DevState* st_h = nullptr;        // pinned mirror [n_scenes]
  uint32_t* group_scene_d = nullptr;
  uint32_t* seg_begin_d = nullptr;
  uint32_t* seg_end_d = nullptr;
  uint32_t* cell_base_d = nullptr;
  int32_t* any_active_d = nullptr; // host-driven loop: any scene still iterating
  uint32_t* active_groups_d = nullptr;  // [n_slots / kSegAlign] groups of the scenes still iterating
  uint32_t* n_active_groups_d = nullptr;
  uint32_t active_grid = 0;             // resident CTAs of the active-group passes
  BatchView view;

  cudaGraphExec_t step_exec = nullptr;
  cudaGraph_t step_graph = nullptr;
  FrameIO io;  // asynchronous per-frame exchange (upf_batch_upload_state_async, ...)
  std::vector<void*> allocations;
  std::vector<void*> checkpoint_slots;
};

// upf_pipeline.cu: neighbour lists of one sorted set without boundary set
cudaError_t launch_nlist_plain(const DevParams& P, uint32_t n, const float4* pos, const uint32_t* keys,
                               const uint32_t* cstart, const uint32_t* cend, uint32_t* nbr, uint32_t* lval,
                               uint32_t* ncnt, const float* luts, DevState* st, cudaStream_t stream);

// upf_pipeline.cu: batched phase launchers (asynchronous on `st`)
cudaError_t batch_launch_init(BatchSystem& b, cudaStream_t st);   // keys and lagged state after upload
cudaError_t batch_launch_keys(BatchSystem& b, cudaStream_t st);   // keys only
cudaError_t batch_launch_sort(BatchSystem& b, cudaStream_t st);
cudaError_t batch_launch_neighbors(BatchSystem& b, cudaStream_t st);
cudaError_t batch_launch_forces(BatchSystem& b, cudaStream_t st);
cudaError_t batch_launch_loop_init(BatchSystem& b, cudaStream_t st);
cudaError_t batch_launch_loop_body(BatchSystem& b, cudaStream_t st, cudaGraphConditionalHandle h, bool use_handle);
cudaError_t batch_launch_loop_density(BatchSystem& b, cudaStream_t st);
cudaError_t batch_launch_loop_pforce(BatchSystem& b, cudaStream_t st);
// the same passes on a resident grid over the groups the last loop control
// listed (n_active_groups_d)
cudaError_t batch_launch_loop_density_active(BatchSystem& b, cudaStream_t st);
cudaError_t batch_launch_loop_pforce_active(BatchSystem& b, cudaStream_t st);
// the graph's loop body: [if most groups iterate: full-grid passes] [else:
// resident passes over the active groups] loop control (sets all three)
cudaError_t batch_capture_loop_body(BatchSystem& b, cudaStream_t st, cudaGraphConditionalHandle h);
cudaError_t batch_launch_loop_ctl(BatchSystem& b, cudaStream_t st, cudaGraphConditionalHandle h = 0,
                                  bool use_handle = false);
cudaError_t batch_launch_integrate(BatchSystem& b, cudaStream_t st);

// upf_api.cu: one step as a CUDA graph, `loop` (if given) under a
// conditional while-node between `pre` and `post`
struct GraphParts {
  cudaError_t (*pre)(void* ctx, cudaStream_t st) = nullptr;
  cudaError_t (*loop)(void* ctx, cudaStream_t st, cudaGraphConditionalHandle h) = nullptr;
  cudaError_t (*post)(void* ctx, cudaStream_t st) = nullptr;
  void* ctx = nullptr;
};
upf_status capture_step_graph(const GraphParts& parts, cudaGraph_t* graph_out, cudaGraphExec_t* exec_out);
DevParams make_dev_params(const upf_params& p, uint32_t nstride);
upf_status encode_list_map(CUtensorMap* map, void* base, CUtensorMapDataType dt, uint32_t elem_bytes,
                           uint64_t cols, uint64_t rows, uint32_t box_rows);
// the box heights of each list (codes, list values)
upf_status encode_list_maps(CUtensorMap* cmaps, CUtensorMap* vmaps, uint32_t* nbr, uint32_t* lval, uint64_t cols,
                            uint64_t rows);

// upf_api.cu: the launch-shape autotuner, over callbacks so that one
// routine serves systems and batches. `prepare` runs a step's passes up to
// the loop (lists, external forces, loop state); each pass callback launches
// that pass once at the current *shape; save/restore bracket the tuning so
// the simulation state is left unchanged. Null callbacks are not tuned.
struct TuneOps {
  void* ctx = nullptr;
  LaunchShape* shape = nullptr;
  bool batched = false;
  cudaStream_t stream = nullptr;
  cudaError_t (*prepare)(void* ctx, cudaStream_t st) = nullptr;
  cudaError_t (*nlist)(void* ctx, cudaStream_t st) = nullptr;
  cudaError_t (*external)(void* ctx, cudaStream_t st) = nullptr;
  cudaError_t (*density)(void* ctx, cudaStream_t st) = nullptr;
  cudaError_t (*pforce)(void* ctx, cudaStream_t st) = nullptr;
  // staging of the lists for the staged loop-pass modes (null: those modes
  // are not tried), and the loop iterations a step is expected to take
  cudaError_t (*stage)(void* ctx, cudaStream_t st) = nullptr;
  float loop_iterations = 0.0f;
  upf_status (*save)(void* ctx) = nullptr;
  upf_status (*restore)(void* ctx) = nullptr;
};
upf_status autotune_shapes(const TuneOps& ops, int repeats, upf_launch_config* out);
void shape_to_config(const LaunchShape& s, upf_launch_config* c);
LaunchShape config_to_shape(const upf_launch_config& c);

// upf_rigid.cu: list entry -> sorted index after a sort; body force/torque,
// body integration and rigid particle sync after integration
cudaError_t launch_rigid_slots(System& s, cudaStream_t st);
// body mass, centre, momenta and inverse inertia, and the particles' relative
// positions, from the bodies' particles in entry order (upf_rigid.cu)
cudaError_t launch_rigid_assemble(float mass, DevBody* bodies, uint32_t n_bodies, const uint32_t* start,
                                  const float4* epos, const float4* evel, float4* entry_r0, cudaStream_t st);
cudaError_t launch_rigid_phase(System& s, cudaStream_t st);
int rigid_launches_per_step(const System& s);

// upf_pipeline.cu: phase launchers (all asynchronous on s.stream)
cudaError_t launch_sort_phase(System& s, cudaStream_t st);
cudaError_t launch_neighbor_phase(System& s, cudaStream_t st);
cudaError_t launch_force_phase(System& s, cudaStream_t st);
cudaError_t launch_loop_init(System& s, cudaStream_t st);
cudaError_t launch_loop_body(System& s, cudaStream_t st, cudaGraphConditionalHandle h, bool use_handle);
cudaError_t launch_loop_density(System& s, cudaStream_t st);
cudaError_t launch_loop_pforce(System& s, cudaStream_t st);
cudaError_t launch_loop_ctl(System& s, cudaStream_t st, cudaGraphConditionalHandle h, bool use_handle);
cudaError_t launch_list_staging(System& s, cudaStream_t st);  // k_stage_lists over the current lists
cudaError_t launch_upload_keys(System& s, cudaStream_t st);
cudaError_t launch_integrate_phase(System& s, cudaStream_t st);
cudaError_t launch_static_setup(System& s, cudaStream_t st);
int pipeline_launches_per_step(const System& s, int iterations);

}  // namespace upf
