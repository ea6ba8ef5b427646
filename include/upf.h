/*
 * upf.h — C ABI of the B200-native per-step particle pipeline.
 *
 * Plain C: opaque handles, POD structs, pointers and sizes; no C++ or torch
 * types cross this boundary. Every function returns a upf_status (0 = OK) and
 * records a message retrievable through upf_last_error().
 *
 * The reference drives its GPU path through an `extern "C"` block that takes
 * a C++ `dataPointers&` (src/gpu/particles.cuh:430-586). Here the handle
 * `upf_system*` owns everything that struct held (device arrays, parameters,
 * lookup tables, ping-pong state), so several independent simulations may
 * live in one process. Each declaration below names the reference entry
 * point it replaces (file:line); the reference's host facade calls these in
 * place of its `dataPointers&` functions.
 */
#ifndef UPF_H_
#define UPF_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UPF_ABI_VERSION 1
#define UPF_LUT_SIZE 300           /* bins per kernel table, src/gpu/particles.cuh:187 */
#define UPF_LUT_ENTRIES (UPF_LUT_SIZE + 1) /* +1: the zero sentinel at index 300 */
#define UPF_GRID_RESOLUTION 1024   /* virtual z-index grid, src/sceneConfigure/global.h:26 */

/* Particle types: same numbering as ParticleObjectType
 * (src/cpu/UnifiedParticle.h:14-23). */
enum {
  UPF_RIGID = 0,
  UPF_SOFT = 1,
  UPF_LIQUID = 2,
  UPF_GRANULAR = 3,
  UPF_CLOTH = 4,
  UPF_SMOKE = 5,
  UPF_FROZEN = 6
};

typedef enum upf_status {
  UPF_OK = 0,
  UPF_ERR_INVALID_ARG = 1,
  UPF_ERR_CUDA = 2,
  UPF_ERR_ALLOC = 3,
  UPF_ERR_NEIGHBOR_OVERFLOW = 4, /* a particle has more neighbours than max_neighbors */
  UPF_ERR_NAN = 5,               /* a predicted or integrated position became NaN */
  UPF_ERR_TIMEOUT = 6,           /* a bounded device-side wait ran out */
  UPF_ERR_STATE = 7,             /* call out of order (e.g. step before set_particles) */
  UPF_ERR_UNSUPPORTED = 8,
  UPF_ERR_NO_DEVICE = 9,
  UPF_ERR_IO = 10                /* a file could not be opened, written, or parsed */
} upf_status;

/* Solver method, UnifiedConstants::setSimulationMethod
 * (src/sceneConfigure/UnifiedConstants.cpp:193-231). */
enum {
  UPF_METHOD_WCSPH = 1,  /* CPU path 'w': UnifiedPhysics::CpuParticlePhysicsPureFluidsSPH */
  UPF_METHOD_PCISPH = 2  /* CPU path 'i': CpuParticlePhysicsVersatileCouplingPCISPH */
};

/* Optional terms. */
enum {
  /* Wall-weight density term of Harada et al. (UnifiedPhysics.cpp:2433-2448,
   * 6034-6060); only used by WCSPH density. */
  UPF_FLAG_WALL_WEIGHT = 1u << 0,
  /* Liquid-liquid cohesion (surface tension spline, UnifiedPhysics.cpp:5283-5287)
   * in the PCISPH external force; also the optional WCSPH surface tension
   * (UnifiedPhysics.cpp:3055-3060, useSurfaceTension). */
  UPF_FLAG_SURFACE_TENSION = 1u << 1,
  /* Penalty wall force on liquid particles (CalculateBoundaryForcePerLiquidParticleHost,
   * UnifiedPhysics.cpp:2032-2069); always on in the reference's PCISPH path. */
  UPF_FLAG_PENALTY_WALLS = 1u << 2,
  /* Akinci boundary pressure force from boundary/rigid particles with the
   * lagged pressure and predicted density (CalculateBoundaryFluidPressureForceHost,
   * UnifiedPhysics.cpp:4240-4250), LUT indexed by distance. */
  UPF_FLAG_BOUNDARY_PRESSURE = 1u << 3,
  /* Adhesion between liquid and boundary/rigid particles
   * (CalculateSurfaceCohesionForcePCISPHHost, UnifiedPhysics.cpp:2000-2008). */
  UPF_FLAG_ADHESION = 1u << 4,
  /* Record per-iteration max predicted density into the step statistics. */
  UPF_FLAG_RECORD_ITERATIONS = 1u << 5
};

/*
 * Scene/solver parameters. Mirrors the scalar block the reference pushes to
 * the device with ~40 setters (src/gpu/particles.cuh:461-503,
 * SetDeviceConstants src/gpu/particles.cu:177-229) and the fields of
 * UnifiedConstants (src/sceneConfigure/UnifiedConstants.h:37-222).
 * upf_default_params() fills the reference's constructor values;
 * upf_params_derive() fills the derived fields (mass, scales, block size,
 * density error factor) exactly as the reference computes them.
 */
typedef struct upf_params {
  int32_t method;            /* UPF_METHOD_* */
  uint32_t flags;            /* UPF_FLAG_* */

  float particle_spacing;    /* particleSpacing */
  float particle_radius;     /* particleRadius = 0.5 * spacing */
  float support_radius;      /* globalSupportRadius h */
  float mass;                /* initialMass = spacing^3 * rest_density */
  float rest_density;        /* fluidRestDensity */
  float gas_constant;        /* fluidGasConstantWCSPH (WCSPH stiffness k) */
  float gamma;               /* Tait exponent (7) */
  float viscosity;           /* fluidViscConst */
  float gravity;             /* gravityConst, applied along -y */
  float dt;                  /* deltaT */

  /* PCISPH */
  float density_error_factor;   /* delta; 0 => computed by upf_params_derive */
  float density_error_fudge;    /* densityErrorFactorParameter; <0 => 0.05*(dt/2e-4)^2 */
  float max_density_error;      /* maxDensityErrorAllowed, percent */
  int32_t min_loops;            /* minLoops (3) */
  int32_t max_loops;            /* maxLoops (50) */

  /* Surface tension / adhesion (Akinci 2013) */
  float surface_tension_gamma;  /* 0.3 */
  float surface_adhesion_beta;  /* 0.0 */

  /* Penalty walls */
  float force_distance;         /* 0.25 * h */
  float max_boundary_force;     /* 64 * spacing^2 */

  /* Rigid bodies (GPU Gems 3 contact model) */
  float spring_coefficient;          /* 300 */
  float spring_coefficient_boundary; /* 300 */
  float damping_coefficient;         /* 0.5 */
  float terminal_speed;              /* 20 */

  /* Granular contact (Bell et al. 2005), UnifiedConstants.cpp:57-60 */
  float granular_kr;
  float granular_kd;
  float granular_kt;
  float granular_mu;

  /* Virtual z-index box: key = Morton(uint16(scales * (x - zindex_origin))) */
  float zindex_origin[3];
  float zindex_extent[3];
  float scales[3];              /* derived: 1024 / extent */
  uint32_t block_size;          /* power-of-two Morton block edge (grid units); 0 => derived */

  /* Collision box (clamp) and real container (wall-weight distance) */
  float collision_min[3];
  float collision_max[3];
  float container_min[3];
  float container_max[3];

  /* Capacity */
  uint32_t max_neighbors;       /* per-particle neighbour list capacity (0 => 128) */
  /* Neighbour search cell edge (grid units, power of two, >= 4). The lists
   * hold exactly the particles within h, in ascending sorted order, whatever
   * the cell size; a cell finer than block_size visits fewer candidates at a
   * higher cost per cell. A query box may span at most 4 cells per axis.
   * 0 => derived: block_size. */
  uint32_t search_cell;
  uint32_t reserved[6];
} upf_params;

/* Per-step statistics (the reference prints these; here they are returned). */
typedef struct upf_step_stats {
  int32_t iterations;        /* PCISPH predict-correct iterations of the last step */
  int32_t hit_max_loops;     /* 1 if iterations == max_loops */
  float max_predicted_density;  /* after the final iteration */
  float density_error_percent;  /* max(0.1*rho*_max - 100, 0) scaled by rest density */
  uint32_t max_neighbor_count;
  uint32_t error_flags;      /* bit0 neighbour overflow, bit1 NaN, bit2 timeout */
  double kinetic_energy;     /* of liquid particles after integration */
  double momentum[3];
  float iteration_max_density[64]; /* per iteration of the last step (first 64) */
  /* cumulative since creation or upf_reset_counters */
  int32_t total_steps;
  int32_t total_iterations;
  int32_t steps_at_max_loops;
  float max_step_density_error_percent;  /* largest density_error_percent of those steps (PCISPH) */
} upf_step_stats;

typedef struct upf_system upf_system;

/* ---- parameters -------------------------------------------------------- */

/* Reference defaults: UnifiedConstants::UnifiedConstants
 * (src/sceneConfigure/UnifiedConstants.cpp:7-159). */
upf_status upf_default_params(upf_params* p);

/* Derived values: mass (UnifiedConstants.cpp:168-191), scales
 * (UnifiedConstants.cpp:308-320), Morton block size (UnifiedPhysics.cpp:2149-2159
 * with ZIndex::SetBlockSize zIndex.cpp:27-39), density error factor
 * (UnifiedPhysics.cpp:5525-5689, accumulated in FP64). Fields already set
 * (non-zero) are kept. */
upf_status upf_params_derive(upf_params* p);

/* PCISPH delta from the prototype block (ComputeDensityErrorFactor,
 * UnifiedPhysics.cpp:5525-5689), FP64 accumulation. */
upf_status upf_density_error_factor(const upf_params* p, double* delta_out);

/* The five 301-entry lookup tables (WeightingKernel::initLookupTables,
 * src/cpu/WeightingKernel.cpp:303-320), row-major [5][301]:
 * M4, pressure-gradient, viscosity-laplacian, surface-tension, adhesion.
 * Replaces CreateLut*Texture (src/gpu/particles.cuh:444-448). */
upf_status upf_build_luts(const upf_params* p, float* out_5x301);

/* Exact squared-distance thresholds of the table bins: out[b] (b = 1..300) is
 * the smallest float r2 with (int)(sqrtf(r2) * (float)(1/h) * 300) >= b,
 * out[0] = 0, out[301] the smallest r2 with sqrtf(r2) >= h. The device picks
 * table bins (WeightingKernel::kernel*Lut, WeightingKernel.cpp:122-128) and
 * the support test (UnifiedPhysics.cpp:2270) from these, bit-identically to
 * the square-root form. No counterpart in the reference. */
upf_status upf_build_bin_thresholds(const upf_params* p, float* out_302);

/* ---- system lifetime (MallocDeviceArrays / FreeDeviceArrays) ------------ */

/* Replaces MallocDeviceArraysParticles + SetDeviceConstants +
 * CreateLut*Texture (src/gpu/particles.cuh:432-448). capacity = maximum
 * number of particles (dynamic + boundary). */
upf_status upf_create(const upf_params* p, int device, uint32_t capacity, upf_system** out);
upf_status upf_destroy(upf_system* s);
upf_status upf_get_params(const upf_system* s, upf_params* out);
/* cudaStream_t passed as void*; NULL = the library's own stream. */
upf_status upf_set_stream(upf_system* s, void* stream);

/* Host arrays, replaces CopyZIndicesKVPairHostToDevice +
 * CopyParticleDataHostToDevice (src/gpu/particles.cuh:436-437).
 * pos/vel: n x 4 floats (w ignored); type: UPF_* per particle.
 * FROZEN particles become the static boundary set (sorted once);
 * all others are dynamic. ids are 0..n-1 in input order. */
upf_status upf_set_particles(upf_system* s, const float* pos4, const float* vel4,
                             const int32_t* type, uint32_t n);

/* Rigid bodies (MallocDeviceArraysRigidBody + CopyRigidBodyDataHostToDevice,
 * src/gpu/particles.cuh:433,438). body_of_particle[i] = body index for every
 * RIGID particle i of the last upf_set_particles call (-1 otherwise); n is
 * that call's particle count. Body mass, centre of mass, momenta and inverse
 * local inertia are computed from the uploaded positions and velocities
 * (AddToRigidBody UnifiedPhysics.cpp:825-885, summed in FP64). PCISPH only;
 * call after upf_set_particles and before the first step (UPF_ERR_STATE
 * otherwise). num_bodies = 0 removes all bodies. Every body needs at least
 * one particle. Setting particles again removes the bodies. */
upf_status upf_set_rigid_bodies(upf_system* s, const int32_t* body_of_particle,
                                uint32_t n, uint32_t num_bodies);

/* ---- stepping ------------------------------------------------------------ */

/* Advance nsteps full steps (ParticlePhysicsOnDevicePCISPH / ...SPH /
 * ...FluidRigidCouplingPCISPH, src/gpu/particles.cuh:534-586). Runs as a CUDA
 * graph; the PCISPH loop is a device-side conditional while-node (no host
 * round trip per iteration). Asynchronous w.r.t. the host unless an error
 * check is requested by upf_synchronize. */
upf_status upf_step(upf_system* s, int32_t nsteps);
upf_status upf_synchronize(upf_system* s);
upf_status upf_get_step_stats(upf_system* s, upf_step_stats* out);
/* Zero the cumulative counters of upf_step_stats (asynchronous, in stream order). */
upf_status upf_reset_counters(upf_system* s);

/* ---- phases (the reference's lower-level entry points) ------------------ */
/* ZindexSorting (particles.cuh:513): sort by key, reorder, cell ranges. */
upf_status upf_phase_sort(upf_system* s);
/* BlockGeneration analogue (particles.cuh:515): build neighbour lists. */
upf_status upf_phase_neighbors(upf_system* s);
/* External forces (CalculateExternalForces*PcisphCUDA) or WCSPH density. */
upf_status upf_phase_forces(upf_system* s);
/* PredictionCorrectionStepPcisphCUDA (particles.cuh:537). */
upf_status upf_phase_predict_correct(upf_system* s);
/* Time integration + clamp + next key (UpdateLiquidParticlePosVel*, CalculateZindex). */
upf_status upf_phase_integrate(upf_system* s);

/* The predict-correct loop pass by pass (PCISPH), for a caller that
 * exchanges fields between the passes, e.g. the halos of a scene split into
 * slabs over several GPUs. After upf_phase_forces: upf_phase_loop_begin, then
 * per iteration upf_phase_density (predicted density, pressure update, the
 * running maximum for the loop test), upf_phase_pressure_force (pressure
 * force, next prediction) and upf_phase_loop_control, which runs the loop
 * test of PredictionCorrectionStep (UnifiedPhysics.cpp:5376-5420) on the
 * maximum found in loop_max_density_bits (which the caller may replace, e.g.
 * by a maximum over all slabs) and returns in *cont whether to iterate again;
 * then upf_phase_integrate. The reference reads its maximum back every
 * iteration as well (GetMaxPredictedDensityCUDA, particles.cu:2139-2154). */
upf_status upf_phase_loop_begin(upf_system* s);
upf_status upf_phase_density(upf_system* s);
upf_status upf_phase_pressure_force(upf_system* s);
upf_status upf_phase_loop_control(upf_system* s, int32_t* cont);

/* Device arrays of a system (no copies), for callers that move particles
 * between systems on the device. The dynamic state (after integration, or
 * as set): pos4/vel4/lag4 n x 4 floats (lag4: previous correction pressure,
 * last correction pressure, last predicted density, -), type, id. The
 * current step's sorted working set (valid after upf_phase_sort): positions,
 * ids, predicted positions, correction pressure, pq4 (position, pressure /
 * rest_density^2: what the pressure-force pass gathers), predicted density.
 * loop_max_density_bits: the loop test's running maximum (float bits).
 * stream: the system's stream; work on these arrays belongs on it. */
typedef struct upf_device_state {
  float* pos4;
  float* vel4;
  float* lag4;
  int32_t* type;
  uint32_t* id;
  uint32_t n;
  uint32_t capacity_dynamic;
  float* sorted_pos4;
  uint32_t* sorted_id;
  float* predicted_pos4;
  float* pressure;
  float* pq4;
  float* density;
  uint32_t* loop_max_density_bits;
  void* stream;
} upf_device_state;
upf_status upf_get_device_state(upf_system* s, upf_device_state* out);
/* Replace the dynamic particles (device arrays, n of them; the boundary set
 * stays) in stream order on the system's stream; the inputs may be the
 * system's own arrays. Ids are the caller's (carried through every step).
 * Not for systems with rigid bodies. */
upf_status upf_set_dynamic_device(upf_system* s, const float* pos4, const float* vel4, const float* lag4,
                                  const int32_t* type, const uint32_t* id, uint32_t n);
/* dst[k] = src[idx[k]] (gather) and dst[idx[k]] = src[k] (scatter) for k < n,
 * rows of row_bytes = 4 or 16, device pointers: the pack and unpack of a
 * halo exchange. */
upf_status upf_gather_rows(const void* src, uint32_t row_bytes, const uint32_t* idx, uint32_t n, void* dst,
                           void* stream);
upf_status upf_scatter_rows(const void* src, uint32_t row_bytes, const uint32_t* idx, uint32_t n, void* dst,
                            void* stream);

/* Replace the dynamic particles' positions and velocities from host arrays in
 * the current device order (the order upf_get_particles returns), keeping the
 * rest of the state; the next step re-sorts them. n must equal the dynamic
 * particle count. This is the per-frame CopyParticleDataHostToDevice of a
 * host-driven caller (src/gpu/particles.cuh:437). */
upf_status upf_upload_state(upf_system* s, const float* pos4, const float* vel4, uint32_t n);

/* Asynchronous counterparts of the per-frame upload and readback, for a
 * host-driven loop (upload, step, read back, every frame). No counterpart in
 * the reference, which copies synchronously between steps. The host copies
 * run on copy streams of the system's own (one per direction), against
 * device staging buffers, so they overlap the steps and each other: an upload is copied while the previous step
 * runs and enters the state in stream order before the next step; a
 * readback is taken in stream order after the step and copied to the host
 * while the next step runs. Each call returns at once; upf_wait_frames waits
 * for the copies issued so far (after it, the upload's host arrays may be
 * rewritten and the readback's host arrays hold their data). Until then
 * neither may be touched. Use pinned host memory for the copies to overlap.
 * The staging buffers (about 72 bytes per particle of capacity) are
 * allocated on the first call. */
upf_status upf_upload_state_async(upf_system* s, const float* pos4, const float* vel4, uint32_t n);
upf_status upf_get_particles_async(upf_system* s, float* pos4, float* vel4, float* density, float* pressure,
                                   int32_t* type, uint32_t* id, uint32_t* n_out);
upf_status upf_wait_frames(upf_system* s);
/* A host round trip of the current frame: reads it back into the host arrays
 * (as upf_get_particles_async; density, pressure, type and id may be NULL)
 * and uploads pos4 and vel4 from those same host arrays as the next step's
 * input (as upf_upload_state_async), in `chunks` pieces (1..16): each piece's
 * upload starts as soon as its positions and velocities have reached host
 * memory, so the two copy directions overlap; the other fields are read back
 * after the last piece's positions and velocities. Returns at once; upf_wait_frames waits for the
 * copies, and until then the host arrays may not be touched (the data a
 * caller would change before uploading needs upf_get_particles_async, a wait
 * and upf_upload_state_async instead). Pinned host memory. */
upf_status upf_exchange_frame_async(upf_system* s, float* pos4, float* vel4, float* density, float* pressure,
                                    int32_t* type, uint32_t* id, uint32_t chunks, uint32_t* n_out);

/* ---- checkpoint / resume ------------------------------------------------- */
/* The reference only has text dumps and readers (src/cpu/UnifiedIO.cpp:14-220).
 * Here the dynamic state (positions, velocities, lagged PCISPH state, ids,
 * types, keys, counters) can be copied to a device-side slot and back (step
 * checkpointing), or to/from a host buffer of upf_state_bytes() bytes (a
 * binary snapshot to resume from). Slots are allocated on first use; all
 * copies are stream-ordered on the system's stream. */
upf_status upf_checkpoint(upf_system* s, int32_t slot);
upf_status upf_restore(upf_system* s, int32_t slot);
size_t upf_state_bytes(const upf_system* s);
upf_status upf_state_save(upf_system* s, void* host, size_t bytes);
upf_status upf_state_load(upf_system* s, const void* host, size_t bytes);

/* Snapshot files: the upf_state_save bytes behind a header (format version,
 * the saving system's upf_params, dynamic-particle and rigid-body counts,
 * method, FNV-1a checksum). To resume in another process: create a system
 * with the stored parameters (upf_state_file_info), set the same scene's
 * particles, then upf_state_read_file; stepping on continues bit for bit.
 * A file from a system of other counts, method or parameters (any
 * upf_params field but the reserved words) is refused (UPF_ERR_INVALID_ARG,
 * the message names the first differing field); a damaged file gives
 * UPF_ERR_IO. */
upf_status upf_state_write_file(upf_system* s, const char* path);
upf_status upf_state_read_file(upf_system* s, const char* path);
upf_status upf_state_file_info(const char* path, upf_params* params, uint32_t* n_dynamic, uint32_t* num_bodies,
                               uint64_t* state_bytes);

/* ---- the reference's text formats (src/cpu/UnifiedIO.cpp,
 * src/sceneConfigure/Scene.cpp) --------------------------------------------
 * Host arrays in, files out (and back), byte for byte as the reference's
 * stream formatting writes them; the reference writes to fixed paths with a
 * per-function file counter, here the caller names the file. pos4: 4 floats
 * per particle (x, y, z, unused), as the reference's device copies. Records
 * are formatted on several host threads; the output does not depend on
 * their number. Errors: UPF_ERR_IO (open/write/parse; upf_last_error says
 * which record), UPF_ERR_INVALID_ARG. */
/* UnifiedIO::SaveLiquidParticleInfoFull (UnifiedIO.cpp:60-105): the header
 * count, then the liquid (type 2) particles among the first
 * num_rounded_particles. */
upf_status upf_io_save_liquid_info_full(const char* path, const float* pos4, const int32_t* type,
                                        int32_t num_rounded_particles, int32_t num_liquid_particles);
/* UnifiedIO::SaveRigidParticleInfoFull (UnifiedIO.cpp:107-152): rigid and
 * frozen (types 0 and 6) particles; header_count is written as given (the
 * reference's caller passes its rigid particle count). */
upf_status upf_io_save_rigid_info_full(const char* path, const float* pos4, const int32_t* type,
                                       int32_t num_rounded_particles, int32_t header_count);
/* UnifiedIO::SaveParticlePositions (UnifiedIO.cpp:14-58). */
upf_status upf_io_save_particle_positions(const char* path, const float* pos4, uint32_t n);
/* Scene::saveParticles (Scene.cpp:247-279): position, rest density, mass,
 * type; rest_density / mass may be NULL, then *_all is written for every
 * particle. */
upf_status upf_io_save_scene_particles(const char* path, const float* pos4, const float* rest_density,
                                       const float* mass, const int32_t* type, uint32_t n, float rest_density_all,
                                       float mass_all);
/* The file UnifiedIO::ReadInFluidParticlesPCISPH reads: the count, then per
 * particle position, type, velocity, correction pressure, predicted density
 * (9 significant digits: floats read back exactly). corr_pressure /
 * predicted_density may be NULL (written as 0). */
upf_status upf_io_save_fluid_particles_pcisph(const char* path, const float* pos4, const float* vel4,
                                              const int32_t* type, const float* corr_pressure,
                                              const float* predicted_density, uint32_t n);
/* UnifiedIO::ReadInFluidParticleNum (UnifiedIO.cpp:154-177). */
upf_status upf_io_read_fluid_particle_num(const char* path, int32_t* count);
/* UnifiedIO::ReadInFluidParticlesPCISPH (UnifiedIO.cpp:179-220); pos3 / vel3
 * hold 3 floats per particle, as the reference's. *n_read: complete records
 * read; a record that does not parse fully is an error (the reference keeps
 * it half-read). More records than capacity: UPF_ERR_INVALID_ARG. */
upf_status upf_io_read_fluid_particles_pcisph(const char* path, float* pos3, float* vel3, int32_t* type,
                                              float* corr_pressure, float* predicted_density, int32_t capacity,
                                              int32_t* n_read);
/* Scene::readInParticles (Scene.cpp:218-243): position, density, mass, type
 * records to the end of the file, granular (type 3) records skipped. All four
 * arrays NULL: *n_out = the number of records kept. pos4 gets (x, y, z, 0).
 * The reference repeats the last record at the end of the file; here it is
 * read once. */
upf_status upf_io_read_scene_particles(const char* path, float* pos4, float* density, float* mass, int32_t* type,
                                       uint32_t capacity, uint32_t* n_out);

/* ---- scene construction --------------------------------------------------
 * ObjLoader::Load + LoadFaces (src/cpu/ObjLoader.cpp:17-233): the triangles
 * of a Wavefront OBJ file, 9 floats each (three corners x, y, z). tri9 NULL:
 * *n_out = the number of triangles. "v" and "f" lines are read (faces as
 * v/vt/vn corners like the reference, also a, a/b, a//c); a corner index
 * outside the file's vertices is UPF_ERR_IO. As in the reference, a file
 * that ends with a newline-terminated "f" line lists its last triangle
 * twice (the reference's read loop handles its last line twice), which
 * takes that face out of the filling's crossing count. */
upf_status upf_obj_read_triangles(const char* path, float* tri9, uint32_t capacity, uint32_t* n_out);
/* ObjectLoader::LoadParticles (src/cpu/ObjectLoader.cpp:8-97) on GPU `device`:
 * the particles that fill the closed triangle mesh tri9 (n_tri triangles),
 * scaled by scale_x/y/z, on the reference's staggered lattice of the given
 * spacing, in the reference's order and bit for bit its positions
 * ((p - box minimum) * scale, as the reference returns them; the caller
 * adds an offset as Scene::CreateFullParticleObject does). pos4: x, y, z, 0
 * per particle; pos4 NULL: *n_out = the count only. More particles than
 * capacity: UPF_ERR_INVALID_ARG with *n_out = the count. The lattice may
 * hold at most 2^31 points. Synchronous; allocates its working buffers. */
upf_status upf_mesh_particles(int device, const float* tri9, uint32_t n_tri, float scale_x, float scale_y,
                              float scale_z, float spacing, float* pos4, uint32_t capacity, uint32_t* n_out);

/* A rigid body's surface particles on GPU `device`, for the coupling
 * scenes' procedural bodies (in place of voxelising an OBJ model with
 * ObjectLoader::LoadParticles, src/cpu/ObjectLoader.cpp:8-97): shape 0 a
 * Fibonacci lattice of n_target points on a sphere of the given radius;
 * 1 a k x k grid of cell centres on each face of a cube of half-edge radius,
 * k = max(2, round(sqrt(n_target / 6))); 2 an nu x nv grid on a torus of
 * major radius `radius` and minor radius radius / 3, nu = max(8,
 * round(sqrt(3 n_target))), nv = max(4, round(n_target / nu)). Each point p
 * becomes rot9 (row-major) p + center, computed in double and stored as
 * float (w = 0). pos4 NULL: *n_out = the count only. Feed the result to
 * upf_set_particles as RIGID particles of one body. */
upf_status upf_scene_rigid_surface(int device, int32_t shape, float radius, uint32_t n_target, const float rot9[9],
                                   const float center[3], float* pos4, uint32_t capacity, uint32_t* n_out);

/* Scene::createFluidObject (src/sceneConfigure/Scene.cpp:597-646) on GPU
 * `device`: a lattice block filling [box_min, box_max) at `spacing`, in the
 * reference's order (y, then x, then z) and bit for bit its positions
 * (jitter + i * spacing, shifted by -0.5 * jitter and by offset in double:
 * the reference's drand48() macro is an integer division that gives 0).
 * pos4 NULL: *n_out = the count only. */
upf_status upf_scene_fluid_block(int device, const float box_min[3], const float box_max[3], float spacing,
                                 float jitter, const float offset[3], float* pos4, uint32_t capacity,
                                 uint32_t* n_out);
/* Scene::createBoxBoundaryFrozenParticles (layers = 1, Scene.cpp:890-1043)
 * and ...MultiLayers (layers = 2, Scene.cpp:1045-1212; 1..8 allowed) on GPU
 * `device`: wall particles around the container (widened by
 * distance_frozen_to_boundary on each side), placed from zindex_start +
 * (support_radius - distance_frozen_to_boundary), with each wall's inward
 * normal in normal4, in the reference's order and bit for bit its
 * positions. A particle at or below zindex_start in some coordinate is an
 * error (the reference aborts). pos4 NULL: *n_out = the count only. */
upf_status upf_scene_box_boundary(int device, const float container_min[3], const float container_max[3],
                                  const float zindex_start[3], float spacing, float support_radius,
                                  float distance_frozen_to_boundary, int32_t layers, float* pos4, float* normal4,
                                  uint32_t capacity, uint32_t* n_out);

/* Per-phase device timings of one step (the reference's SPH_PROFILING_VERBOSE
 * per-phase event timers, src/gpu/particles.cu:1460-1690). Runs one full
 * step through the phase entry points with CUDA events around each phase,
 * and times each predicted-density and pressure-force launch. */
typedef struct upf_phase_times {
  float sort_ms;            /* radix sort + reorder + cell ranges */
  float neighbors_ms;       /* neighbour lists */
  float forces_ms;          /* external forces (PCISPH) / density (WCSPH) */
  float loop_ms;            /* whole predict-correct loop, host-driven */
  float integrate_ms;       /* integration (+ WCSPH force) */
  float density_ms_total;   /* sum over the loop's predicted-density launches */
  float pforce_ms_total;    /* sum over the loop's pressure-force launches */
  int32_t iterations;
  int32_t launches;         /* device kernels launched by the step */
} upf_phase_times;
upf_status upf_profile_step(upf_system* s, upf_phase_times* out);

/* ---- launch shapes and the autotuner (no counterpart in the reference,
 * whose kernels run at fixed block sizes) --------------------------------
 * CTA sizes of the neighbour-list and external-force passes, and CTA size x
 * list rows per stage of the two predict-correct passes, whose list entries
 * come either through a TMA ring in shared memory (mode 0; pairs (128,4)
 * (128,8) (128,16) (256,2) (256,4) (256,8) (512,2) (512,4) (1024,2)) or by
 * direct coalesced loads, rows entries at a time (mode 1; (128,4) (128,8)
 * (256,4) (256,8) (512,4) (512,8)), or from staged neighbourhoods (mode 2;
 * (256,4) (256,8); single PCISPH systems): each 256-particle CTA copies the
 * distinct neighbours of its particles into shared memory once per pass and
 * walks lists rewritten as 16-bit positions in that set (the rewrite runs
 * once per step, after the list build). Batches allow up to 256 threads and
 * modes 0 and 1. Shapes change timing only: every shape gives the same
 * results. */
typedef struct upf_launch_config {
  int32_t nlist_threads;      /* 64, 128, 256 */
  int32_t external_threads;   /* 128, 256 */
  int32_t density_threads;
  int32_t density_rows;
  int32_t pforce_threads;
  int32_t pforce_rows;
  int32_t density_mode;       /* list entries by 0: the TMA ring; 1: direct loads; 2: staged neighbourhoods */
  int32_t pforce_mode;
  int32_t nlist_mode;         /* 0: each thread its own query box; 1: a warp walks the union of its boxes */
  float measured_ms[4];       /* autotune: per-launch ms of the chosen shapes
                                 (neighbour lists, external forces, predicted
                                 density, pressure force); 0 otherwise */
} upf_launch_config;
upf_status upf_get_launch_config(upf_system* s, upf_launch_config* out);
upf_status upf_set_launch_config(upf_system* s, const upf_launch_config* cfg);
/* Times every shape of each tunable pass on the system's current state
 * (repeats launches per shape, CUDA events), keeps the fastest of each, and
 * leaves the simulation state as it found it. */
upf_status upf_autotune(upf_system* s, int32_t repeats, upf_launch_config* chosen);

/* ---- readback (CopyParticlesCUDA, src/gpu/particles.cuh:505) ------------ */

/* Dynamic particles in current device order. Any pointer may be NULL.
 * pos4/vel4/force4/pforce4: n x 4 floats. Returns count in *n_out. */
upf_status upf_get_particles(upf_system* s, float* pos4, float* vel4, float* density,
                             float* pressure, int32_t* type, uint32_t* id, uint32_t* n_out);
/* Every particle of the last upf_set_particles call (n = its count), at its
 * input index: dynamic particles from the current state, boundary (FROZEN)
 * particles at their fixed positions with zero velocity, rest density and
 * zero pressure. pos4.w holds the particle's Morton key as a float (the
 * reference keeps the z-index in pos.w). The permutation back to input order
 * runs on the device. The readback of CopyParticlesCUDA
 * (src/gpu/particles.cu:62-72) for a caller that indexes particles by the
 * order it uploaded them in; any pointer may be NULL. */
upf_status upf_get_particles_input_order(upf_system* s, float* pos4, float* vel4, float* density,
                                        float* pressure, int32_t* type, uint32_t n);
/* The dynamic particles' lagged PCISPH state in current device order (the
 * order of upf_get_particles), n x 4 floats: the final correction pressure
 * of the step before last (what the next step's external forces read as
 * previous_correction_pressure_, UnifiedPhysics.cpp:5360-5363), that of the
 * last step, the last step's predicted density, 0. n = the dynamic count. */
upf_status upf_get_lagged_state(upf_system* s, float* lag4, uint32_t n);
/* Per-particle step fields of the last step, in the sorted order of that step:
 * external force, correction pressure force, predicted density. */
upf_status upf_get_step_fields(upf_system* s, float* force4, float* pforce4,
                               float* predicted_density, uint32_t* id, uint32_t* n_out);
/* Neighbour lists of the dynamic particles (after upf_phase_neighbors), as
 * ids: counts[n], lists[n * cap] (row-major, first counts[i] valid). */
upf_status upf_get_neighbors(upf_system* s, uint32_t* counts, uint32_t* lists_ids,
                             uint32_t cap, uint32_t* n_out);
/* Sorted keys and cell ranges of the dynamic set (after upf_phase_sort).
 * The cell table has one entry per search cell, (1024 / search_cell)^3;
 * start/end must hold that many entries: call with NULL arrays to get the
 * count in *ncells_out first. */
upf_status upf_get_sorted_keys(upf_system* s, uint32_t* keys, uint32_t* ids, uint32_t* n_out);
upf_status upf_get_cell_ranges(upf_system* s, uint32_t* start, uint32_t* end, uint32_t* ncells_out);
/* Rigid body state (RigidBody::rigidbody_pos / velocity / angular_velocity /
 * quaternion, src/cpu/RigidBody.h:105-134): pos3/vel3/omega3 num_bodies x 3
 * floats, quat4 num_bodies x 4 (s, x, y, z). Any pointer may be NULL. */
upf_status upf_get_rigid_bodies(upf_system* s, float* pos3, float* vel3, float* omega3,
                                float* quat4, uint32_t* num_bodies_out);

/* ---- stateless device building blocks ----------------------------------- */
/* Device pointers; stream as void* (NULL = default stream). */

/* 30-bit Morton key per particle (ZIndex::CalcIndex, src/cpu/zIndex.h:40-45,
 * called as zIndex.CalcIndex(fc_->scales * p.position_), UnifiedPhysics.cpp:4005). */
upf_status upf_morton_keys(const float* pos4_dev, uint32_t n, const float origin[3],
                           const float scales[3], uint32_t* keys_dev, void* stream);

/* Stable LSD radix sort of (key, value) pairs on the low key_bits bits.
 * Replaces RadixSort (src/gpu/radixsort.cuh:115-117). keys/vals are sorted in
 * place; temp is caller-provided scratch of upf_radix_sort_temp_bytes(n). */
size_t upf_radix_sort_temp_bytes(uint32_t n);
upf_status upf_radix_sort_pairs(uint32_t* keys_dev, uint32_t* vals_dev, uint32_t n,
                                int32_t key_bits, void* temp_dev, size_t temp_bytes,
                                void* stream);

/* The same sort without caller scratch and without any allocation. No
 * counterpart in the reference. For callers that cannot call cudaMalloc: hosts
 * that own all device memory through their own pool or arena, and per-frame
 * loops that must not pay cudaMalloc's implicit device synchronisation. The
 * scratch is a fixed file-scope device array in the library, sized for at most
 * UPF_NOALLOC_MAX_PAIRS pairs (17 MB); every GPU that loads the library holds it
 * until the process exits. Larger n is rejected with UPF_ERR_INVALID_ARG.
 * The first call on a device looks up that array's device address (once per
 * device, with the device current); make that first call before any stream
 * capture. All calls share the one array and it keeps the last call's
 * contents: calls that overlap on the GPU (different streams or host threads
 * without ordering between them) race on it. The looked-up address is kept
 * for the life of the process: do not call this after a cudaDeviceReset (or
 * any teardown of the device's primary context) in the same process, since the
 * array then lives at a new address the library does not know. */
#define UPF_NOALLOC_MAX_PAIRS (1u << 21)
upf_status upf_radix_sort_pairs_noalloc(uint32_t* keys_dev, uint32_t* vals_dev, uint32_t n,
                                        int32_t key_bits, void* stream);

/* Cell start/end for sorted keys at cell = key >> shift (empty cells start=end=0).
 * Replaces ClearIndexArrays + CalculateBlocksKernel (particles_kernel.cu:656-726). */
upf_status upf_cell_ranges(const uint32_t* sorted_keys_dev, uint32_t n, int32_t shift,
                           uint32_t ncells, uint32_t* start_dev, uint32_t* end_dev,
                           void* stream);

/* ---- batched scenes -------------------------------------------------------
 * No counterpart in the reference (one simulation per process, global device
 * state). Many independent PCISPH scenes of uneven sizes advance together:
 * every pass of a step is one launch over all scenes, the step is one CUDA
 * graph whose predict-correct loop (a device-side while-node) runs until the
 * last scene has converged, each scene keeping its own iteration count. Every
 * scene's result is the one a upf_system with the same parameters and
 * particles computes (same sort order, neighbour lists and sums).
 * Scenes hold LIQUID particles only (walls by the collision box and
 * UPF_FLAG_PENALTY_WALLS); params[s].method must be UPF_METHOD_PCISPH. */
typedef struct upf_batch upf_batch;

/* params: num_scenes parameter sets (derived like upf_params_derive),
 * counts: particles per scene. */
upf_status upf_batch_create(const upf_params* params, const uint32_t* counts, uint32_t num_scenes,
                            int device, upf_batch** out);
upf_status upf_batch_destroy(upf_batch* b);
upf_status upf_batch_set_stream(upf_batch* b, void* stream);
/* Host arrays of all scenes' particles, concatenated in scene order
 * (pos4/vel4: sum(counts) x 4 floats). Particle ids are 0..counts[s]-1 per
 * scene in input order. */
upf_status upf_batch_set_particles(upf_batch* b, const float* pos4, const float* vel4);
upf_status upf_batch_step(upf_batch* b, int32_t nsteps);
/* Waits for the batch's stream; reports the first scene's device error. */
upf_status upf_batch_synchronize(upf_batch* b);
/* Per-scene statistics of the last step: out[num_scenes]. */
upf_status upf_batch_get_stats(upf_batch* b, upf_step_stats* out);
upf_status upf_batch_reset_counters(upf_batch* b);
/* One scene's particles in current device order (any pointer may be NULL). */
upf_status upf_batch_get_particles(upf_batch* b, uint32_t scene, float* pos4, float* vel4,
                                   float* density, float* pressure, uint32_t* id, uint32_t* n_out);
/* Device copies of the whole batch state, as upf_checkpoint / upf_restore. */
upf_status upf_batch_checkpoint(upf_batch* b, int32_t slot);
upf_status upf_batch_restore(upf_batch* b, int32_t slot);
/* Same layout as upf_batch_set_particles: all scenes' positions and
 * velocities replace the current state (H2D), or are read back (D2H), in the
 * batch's current device order per scene. */
upf_status upf_batch_upload_state(upf_batch* b, const float* pos4, const float* vel4);
upf_status upf_batch_download_state(upf_batch* b, float* pos4, float* vel4);
/* Asynchronous counterparts (no counterpart in the reference; the scheme of
 * upf_upload_state_async): the copies overlap the batch's steps;
 * upf_batch_wait_frames waits for the copies issued so far, and until then
 * the host arrays may not be touched. Pinned host memory; staging buffers
 * (64 bytes per particle) are allocated on the first call. */
upf_status upf_batch_upload_state_async(upf_batch* b, const float* pos4, const float* vel4);
upf_status upf_batch_download_state_async(upf_batch* b, float* pos4, float* vel4);
upf_status upf_batch_wait_frames(upf_batch* b);
/* One batch step through its passes with CUDA events (as upf_profile_step);
 * iterations = the largest scene's count; *active_particle_iterations (may be
 * NULL) = the sum over loop iterations of the particles of the scenes still
 * iterating, i.e. the particles the loop passes processed. */
upf_status upf_batch_profile_step(upf_batch* b, upf_phase_times* out, uint64_t* active_particle_iterations);
/* Launch shapes of a batch (as upf_*_launch_config; at most 256 threads). */
upf_status upf_batch_get_launch_config(upf_batch* b, upf_launch_config* out);
upf_status upf_batch_set_launch_config(upf_batch* b, const upf_launch_config* cfg);
upf_status upf_batch_autotune(upf_batch* b, int32_t repeats, upf_launch_config* chosen);

/* ---- differentiation (adjoint) -------------------------------------------
 * No counterpart in the reference. A differentiable PCISPH trajectory and its
 * hand-written adjoint: LIQUID particles, the reference's kernel functions
 * evaluated analytically (the 300-bin tables are piecewise constant, their
 * derivative zero), a fixed number of predict-correct iterations per step (a
 * data-dependent count would make the loss discontinuous), the pressure
 * update's max(rho - rho0, 0) smoothed to 0.5 (d + sqrt(d^2 + eps^2)) with
 * eps = density_smoothing * rho0 (at a hard kink the gradient of a 20-step
 * trajectory changes by percent under float-rounding-sized perturbations of
 * the input; smoothed over +-1% of rho0, the PCISPH tolerance's own scale, an
 * FP32 adjoint of 20 steps agrees with FP64 to 1e-4), viscosity +
 * gravity + PCISPH pressure, no surface tension or wall forces (collision-box
 * clamping is applied forward and treated as inactive by the adjoint: keep
 * the particles clear of the walls). Loss:
 *   L = com_weight * |x_com(T) - target|^2
 *     + density_weight * mean_i (rho_i(T) - rho0)^2,
 * rho_i(T) the SPH density at the final positions. upf_adjoint_backward
 * returns dL/dv(0) per particle and dL/d viscosity, recomputing each
 * checkpoint interval forward from its checkpoint. */
typedef struct upf_adjoint upf_adjoint;
typedef struct upf_adjoint_options {
  int32_t steps;                /* T */
  int32_t checkpoint_interval;  /* steps between stored states (>= 1) */
  int32_t loop_iterations;      /* predict-correct iterations per step (>= 1) */
  float target[3];
  float com_weight;
  float density_weight;
  float density_smoothing;      /* eps / rho0 of the smooth maximum (> 0; 1e-2: the 1% error scale) */
} upf_adjoint_options;

upf_status upf_adjoint_create(const upf_params* p, const upf_adjoint_options* opt, const float* pos4,
                              const float* vel4, uint32_t n, int device, upf_adjoint** out);
upf_status upf_adjoint_destroy(upf_adjoint* a);
upf_status upf_adjoint_set_stream(upf_adjoint* a, void* stream);
/* Runs the T steps from the initial positions with initial velocities vel4
 * (n x 4 host floats; NULL keeps the last ones) and the given viscosity;
 * *loss (may be NULL) receives L. */
upf_status upf_adjoint_forward(upf_adjoint* a, const float* vel4, float viscosity, double* loss);
/* Gradients of the last forward's loss: grad_vel4 (n x 4 host floats, w = 0)
 * and *grad_viscosity (either may be NULL). */
upf_status upf_adjoint_backward(upf_adjoint* a, float* grad_vel4, double* grad_viscosity);
/* Final positions and velocities of the last forward (n x 4 host floats). */
upf_status upf_adjoint_get_state(upf_adjoint* a, float* pos4, float* vel4);
/* Device times of the last forward and backward (CUDA events). */
upf_status upf_adjoint_times(upf_adjoint* a, float* forward_ms, float* backward_ms);

/* ---- failure-detection self-tests (no counterpart in the reference, which
 * exits on API errors and only prints kernel errors) -----------------------
 * upf_test_fail_allocation(nth): the nth library device allocation from now
 * on (0 = the next) fails with UPF_ERR_ALLOC without calling cudaMalloc;
 * nth < 0 disarms. Process-wide; for exercising error paths.
 * upf_selftest_bounded_wait: one warp waits, with the bounded wait the list
 * stream uses, on a barrier that never completes; the wait gives up after
 * limit_us and the call returns UPF_ERR_TIMEOUT, with the context intact.
 * upf_selftest_support_bins: the kernel-table bin the PCISPH density pass
 * takes for each squared distance r2[k] at p's support radius, computed on
 * the device (300 = outside the support: the pair adds nothing); for checking
 * the device's r2 -> bin rule against (int)(sqrtf(r2) * (1/h) * 300) and
 * sqrtf(r2) < h, UnifiedPhysics.cpp:5468-5476. The neighbour-list build's
 * table rule is computed beside it: -2 marks an r2 where the two differ.
 * n <= 2^26.
 * upf_test_stage_union_cap(s, cap): lowers the number of distinct neighbours
 * a chunk of the staged loop passes (mode 2) may stage (at most 2048, the
 * default); chunks whose union is larger read the plain lists. For reaching
 * that fallback on small scenes. */
upf_status upf_test_fail_allocation(int32_t nth);
upf_status upf_test_stage_union_cap(upf_system* s, uint32_t cap);
upf_status upf_selftest_bounded_wait(int device, uint32_t limit_us);
upf_status upf_selftest_support_bins(int device, const upf_params* p, const float* r2, uint32_t n, int32_t* bins);

/* ---- errors ------------------------------------------------------------- */
const char* upf_last_error(void);
const char* upf_status_string(upf_status st);
int32_t upf_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* UPF_H_ */
