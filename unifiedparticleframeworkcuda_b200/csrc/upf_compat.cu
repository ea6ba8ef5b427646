// upf_compat.cu — the reference's GPU entry points (src/gpu/particles.cuh:430-586,
// src/gpu/radixsort.cuh:115-117) over the C ABI of upf.h. Built into
// libupf_compat.so; declarations and conventions in include/upf_compat.h.
//
// The reference keeps its simulation in file-scope device state set by the
// Set* calls (__constant__ memory, particles_kernel.cu:36-165) and in the
// caller's dataPointers. Here the Set* calls fill one process-wide record of
// those constants; MallocDeviceArraysParticles attaches a context to the
// caller's dataPointers; the upload keeps a host copy of the particles; and
// the first step (or phase) call creates the library system from the
// constants, the upload and the method its name implies.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "upf_compat.h"

namespace {

// The device constants of the reference, as its Set* calls leave them.
struct Constants {
  unsigned particle_count = 0, num_rigid_bodies = 0;
  float support_radius = 0, particle_radius = 0, terminal_speed = 0;
  float rb_spring = 0, rb_spring_boundary = 0, rb_damping = 0;
  float surface_tension_gamma = 0, surface_adhesion_beta = 0;
  unsigned grid_resolution = 0, block_size = 0, lut_size = 0;
  float kernel_self = 0, mass = 0, rest_density = 0;
  float3 zindex_origin{0, 0, 0};
  float gamma = 0, gas_constant = 0, gas_constant_wcsph = 0, density_error_factor = 0;
  float force_distance = 0, max_boundary_force = 0;
  float3 collision_min{0, 0, 0}, collision_max{0, 0, 0};
  bool add_boundary_force = false;
  float3 bounding_min{0, 0, 0}, bounding_max{0, 0, 0};
  float3 container_min{0, 0, 0}, container_max{0, 0, 0};
  float dt = 0, dt_wcsph = 0;
  float3 scales{0, 0, 0};
  float gravity = 0, viscosity = 0, spacing = 0;
  float max_density_error = 0;
  int min_loops = 0, max_loops = 0;
  bool set = false;  // SetDeviceConstants or a Set* call ran
};

std::mutex g_mutex;
Constants g_const;
int g_device = 0;
upf_status g_status = UPF_OK;  // process-wide failure (no simulation to attach it to)
std::string g_message;

enum Pipeline { kNone, kPcisph, kPcisphStatic, kPcisphRigid, kSph, kSphRigid };

// rows of upf_build_luts: M4, pressure gradient, viscosity laplacian,
// surface tension, adhesion
enum Table { kM4 = 0, kPressureGrad = 1, kViscosityLap = 2, kSurfaceTension = 3, kAdhesion = 4 };

bool device_present(int device) {
  int count = 0;
  return cudaGetDeviceCount(&count) == cudaSuccess && device >= 0 && device < count;
}

}  // namespace

struct upf_compat_context {
  upf_status status = UPF_OK;
  std::string message;
  upf_system* sys = nullptr;
  Pipeline pipeline = kNone;
  upf_params prm{};
  unsigned num_bodies = 0;
  std::vector<float> pos, vel;
  std::vector<int> type, body;
  bool uploaded = false;
};

namespace {

void fail_ctx(upf_compat_context* c, upf_status st, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) {
    if (c->status != UPF_OK) return;  // the first failure is the one reported
    c->status = st;
    c->message = buf;
  } else {
    if (g_status != UPF_OK) return;
    g_status = st;
    g_message = buf;
  }
  std::fprintf(stderr, "upf_compat: %s\n", buf);
}

// A library call's status; false (and the context failed) if not UPF_OK.
bool ok_call(upf_compat_context* c, upf_status st, const char* what) {
  if (st == UPF_OK) return true;
  fail_ctx(c, st, "%s: %s (%s)", what, upf_status_string(st), upf_last_error());
  return false;
}

upf_compat_context* ctx_of(dataPointers& d, const char* who) {
  if (!d.upf) {
    fail_ctx(nullptr, UPF_ERR_STATE, "%s: call MallocDeviceArraysParticles first", who);
    return nullptr;
  }
  return d.upf->status == UPF_OK ? d.upf : nullptr;
}

uint32_t flags_for(Pipeline p, bool add_boundary_force) {
  uint32_t f = UPF_FLAG_SURFACE_TENSION | (add_boundary_force ? UPF_FLAG_PENALTY_WALLS : 0u);
  if (p == kPcisphStatic || p == kPcisphRigid || p == kSphRigid) f |= UPF_FLAG_BOUNDARY_PRESSURE;
  return f;
}

bool is_pcisph(Pipeline p) { return p == kPcisph || p == kPcisphStatic || p == kPcisphRigid; }

// upf_params from the device constants, for one pipeline.
upf_params params_from_constants(const Constants& k, Pipeline p) {
  upf_params q;
  upf_default_params(&q);
  q.method = is_pcisph(p) ? UPF_METHOD_PCISPH : UPF_METHOD_WCSPH;
  q.flags = flags_for(p, k.add_boundary_force);
  q.particle_spacing = k.spacing;
  q.particle_radius = k.particle_radius;
  q.support_radius = k.support_radius;
  q.mass = k.mass;
  q.rest_density = k.rest_density;
  q.gas_constant = k.gas_constant_wcsph;
  q.gamma = k.gamma;
  q.viscosity = k.viscosity;
  q.gravity = k.gravity;
  q.dt = is_pcisph(p) ? k.dt : k.dt_wcsph;
  q.density_error_factor = k.density_error_factor;
  q.max_density_error = k.max_density_error;
  q.min_loops = k.min_loops;
  q.max_loops = k.max_loops;
  q.surface_tension_gamma = k.surface_tension_gamma;
  q.surface_adhesion_beta = k.surface_adhesion_beta;
  q.force_distance = k.force_distance;
  q.max_boundary_force = k.max_boundary_force;
  q.spring_coefficient = k.rb_spring;
  q.spring_coefficient_boundary = k.rb_spring_boundary;
  q.damping_coefficient = k.rb_damping;
  q.terminal_speed = k.terminal_speed;
  const float o[3] = {k.zindex_origin.x, k.zindex_origin.y, k.zindex_origin.z};
  const float sc[3] = {k.scales.x, k.scales.y, k.scales.z};
  const float cmin[3] = {k.collision_min.x, k.collision_min.y, k.collision_min.z};
  const float cmax[3] = {k.collision_max.x, k.collision_max.y, k.collision_max.z};
  const float rmin[3] = {k.container_min.x, k.container_min.y, k.container_min.z};
  const float rmax[3] = {k.container_max.x, k.container_max.y, k.container_max.z};
  for (int a = 0; a < 3; ++a) {
    q.zindex_origin[a] = o[a];
    q.scales[a] = sc[a];
    q.zindex_extent[a] = sc[a] > 0 ? (float)k.grid_resolution / sc[a] : 0.0f;
    q.collision_min[a] = cmin[a];
    q.collision_max[a] = cmax[a];
    q.container_min[a] = rmin[a];
    q.container_max[a] = rmax[a];
  }
  q.block_size = k.block_size;
  return q;
}

// The simulation of `d`, created at the first call that needs it, for the
// pipeline the call implies. Null (and the context failed) on error.
upf_system* system_for(dataPointers& d, Pipeline p, const char* who) {
  upf_compat_context* c = ctx_of(d, who);
  if (!c) return nullptr;
  if (c->sys) {
    if (is_pcisph(c->pipeline) != is_pcisph(p)) {
      fail_ctx(c, UPF_ERR_INVALID_ARG, "%s: the simulation runs %s; this call needs %s", who,
               is_pcisph(c->pipeline) ? "PCISPH" : "WCSPH", is_pcisph(p) ? "PCISPH" : "WCSPH");
      return nullptr;
    }
    return c->sys;
  }
  if (!c->uploaded) {
    fail_ctx(c, UPF_ERR_STATE, "%s: call CopyParticleDataHostToDevice first", who);
    return nullptr;
  }
  Constants k;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    k = g_const;
  }
  if (!k.set) {
    fail_ctx(c, UPF_ERR_STATE, "%s: call SetDeviceConstants first", who);
    return nullptr;
  }
  upf_params q = params_from_constants(k, p);
  if (!ok_call(c, upf_params_derive(&q), who)) return nullptr;
  const uint32_t n = (uint32_t)c->type.size();
  upf_system* s = nullptr;
  if (!ok_call(c, upf_create(&q, g_device, n ? n : 1u, &s), who)) return nullptr;
  if (!ok_call(c, upf_set_particles(s, c->pos.data(), c->vel.data(), c->type.data(), n), who)) {
    upf_destroy(s);
    return nullptr;
  }
  unsigned nb = 0;
  for (uint32_t i = 0; i < n; ++i)
    if (c->type[i] == UPF_RIGID && c->body[i] >= 0) nb = std::max<unsigned>(nb, (unsigned)c->body[i] + 1);
  if (nb && is_pcisph(p)) {
    std::vector<int32_t> b(n, -1);
    for (uint32_t i = 0; i < n; ++i)
      if (c->type[i] == UPF_RIGID) b[i] = c->body[i];
    if (!ok_call(c, upf_set_rigid_bodies(s, b.data(), n, nb), who)) {
      upf_destroy(s);
      return nullptr;
    }
  }
  c->sys = s;
  c->pipeline = p;
  c->prm = q;
  return s;
}

void step(dataPointers& d, Pipeline p, const char* who) {
  upf_system* s = system_for(d, p, who);
  if (!s) return;
  upf_compat_context* c = d.upf;
  if (ok_call(c, upf_step(s, 1), who)) ok_call(c, upf_synchronize(s), who);
}

void phase(dataPointers& d, Pipeline p, upf_status (*fn)(upf_system*), const char* who) {
  upf_system* s = system_for(d, p, who);
  if (!s) return;
  ok_call(d.upf, fn(s), who);
}

// Pipeline of a phase-level call that does not name one: the existing
// simulation's, else PCISPH with the Akinci boundary when the upload holds
// boundary particles.
Pipeline default_pipeline(dataPointers& d) {
  if (d.upf && d.upf->sys) return d.upf->pipeline;
  if (d.upf)
    for (int t : d.upf->type)
      if (t == UPF_FROZEN) return kPcisphStatic;
  return kPcisph;
}

void unsupported(dataPointers* d, const char* who) {
  fail_ctx(d ? d->upf : nullptr, UPF_ERR_UNSUPPORTED,
           "%s is not available: this library does not build that variant", who);
}

template <class F>
void set_const(F&& f) {
  std::lock_guard<std::mutex> lock(g_mutex);
  f(g_const);
  g_const.set = true;
}

// Kernel-table check of Create*Texture: the caller's table against the
// library's own for the current support radius.
void check_lut(int which, const float* A, int lut_size, const char* who) {
  Constants k;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    k = g_const;
  }
  if (!A || lut_size <= 0) {
    fail_ctx(nullptr, UPF_ERR_INVALID_ARG, "%s: null table or size %d", who, lut_size);
    return;
  }
  upf_params q = params_from_constants(k, kPcisph);
  if (upf_params_derive(&q) != UPF_OK) {
    fail_ctx(nullptr, UPF_ERR_STATE, "%s: call SetDeviceConstants first", who);
    return;
  }
  std::vector<float> luts(5 * UPF_LUT_ENTRIES);
  if (upf_build_luts(&q, luts.data()) != UPF_OK) {
    fail_ctx(nullptr, UPF_ERR_INVALID_ARG, "%s: %s", who, upf_last_error());
    return;
  }
  const int n = std::min(lut_size, (int)UPF_LUT_ENTRIES);
  if (std::memcmp(A, luts.data() + which * UPF_LUT_ENTRIES, sizeof(float) * n) != 0)
    fail_ctx(nullptr, UPF_ERR_INVALID_ARG,
             "%s: the caller's table differs from the library's for h = %g (the library computes its own)", who,
             (double)q.support_radius);
}

__global__ void k_split_pairs(uint32_t n, const KeyValuePair* __restrict__ in, uint32_t* __restrict__ keys,
                              uint32_t* __restrict__ vals) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const KeyValuePair p = in[i];
  keys[i] = p.key;
  vals[i] = p.value;
}

__global__ void k_join_pairs(uint32_t n, const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                             KeyValuePair* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  KeyValuePair p;
  p.key = keys[i];
  p.value = vals[i];
  out[i] = p;
}

void* g_sort_tmp = nullptr;
size_t g_sort_tmp_bytes = 0;

}  // namespace

extern "C" {

void upf_compat_set_device(int device) { g_device = device; }

upf_status upf_compat_status(const dataPointers& d) {
  if (g_status != UPF_OK) return g_status;
  return d.upf ? d.upf->status : UPF_ERR_STATE;
}

const char* upf_compat_message(const dataPointers& d) {
  if (g_status != UPF_OK) return g_message.c_str();
  return d.upf ? d.upf->message.c_str() : "MallocDeviceArraysParticles has not run";
}

upf_status upf_compat_params(const dataPointers& d, upf_params* out) {
  if (!out || !d.upf || !d.upf->sys) return UPF_ERR_STATE;
  *out = d.upf->prm;
  return UPF_OK;
}

upf_system* upf_compat_system(const dataPointers& d) { return d.upf ? d.upf->sys : nullptr; }

void upf_compat_upload(dataPointers& d, const float* pos4, const float* vel4, const int* type,
                       const int* parent_body, uint n) {
  upf_compat_context* c = ctx_of(d, "CopyParticleDataHostToDevice");
  if (!c) return;
  if (c->sys) {
    // a new upload to a running simulation: replace its particles
    upf_destroy(c->sys);
    c->sys = nullptr;
    c->pipeline = kNone;
  }
  c->pos.assign(pos4, pos4 + 4 * (size_t)n);
  c->vel.assign(vel4, vel4 + 4 * (size_t)n);
  c->type.assign(type, type + n);
  c->body.assign(parent_body, parent_body + n);
  c->uploaded = true;
  if (!device_present(g_device))
    fail_ctx(c, UPF_ERR_NO_DEVICE, "CopyParticleDataHostToDevice: no CUDA device %d", g_device);
}

// ---- init -----------------------------------------------------------------
// MallocDeviceArraysParticles (particles.cu:100-175): the rounded counts as
// the reference computes them; the device arrays are the library's.
void MallocDeviceArraysParticles(dataPointers& d) {
  const unsigned block = 64;  // MAX_THREADS_PER_BLOCK_SPH (particles.cuh:184)
  auto round_up = [&](unsigned c) { return (c % block) ? c + (block - c % block) : c; };
  d.finalParticleCountRounded = round_up(d.finalParticleCount);
  d.particleCountRounded = round_up(d.particleCount);
  for (int k = 0; k < 2; ++k) {
    d.d_pos_zindex[k] = nullptr;
    d.d_vel[k] = nullptr;
    d.d_type[k] = nullptr;
    d.d_active_type[k] = nullptr;
    d.particlesKVPair_d[k] = nullptr;
  }
  d.upf = new upf_compat_context();
  if (!device_present(g_device))
    fail_ctx(d.upf, UPF_ERR_NO_DEVICE, "MallocDeviceArraysParticles: no CUDA device %d", g_device);
}

void MallocDeviceArraysRigidBody(dataPointers& d, std::vector<RigidBody*>& rigidbodies_h) {
  upf_compat_context* c = ctx_of(d, "MallocDeviceArraysRigidBody");
  if (c) c->num_bodies = (unsigned)rigidbodies_h.size();
}

// SetDeviceConstants (particles.cu:177-229): the same Set* calls in the same
// order; the loop controls come from the PCISPH parameters of dataPointers.
void SetDeviceConstants(dataPointers& d) {
  SetParticleCount(d.particleCount);
  SetRigidBodyCount(d.num_rigid_bodies);
  SetGlobalSupportRadius(d.globalSupportRadius);
  SetDistToCenterMassCutoffApproximate(d.distToCenterMassCutoff);
  SetVelCutoffApproximate(d.gradientVelCutoff);
  SetParticleRadius(d.particleRadius);
  SetTerminalSpeed(d.rb_terminalSpeed);
  SetRigidBodyCoefficients(d.rb_spring, d.rb_spring_boundary, d.rb_damping);
  SetSurfaceTensionAdhesionCoefficients(d.surface_tension_gamma, d.surface_adhesion_beta);
  SetGridResolution(d.grid_resolution);
  SetBlockSize(d.block_size);
  SetGridDimensions(d.dimX, d.dimY, d.dimZ);
  SetLutSize(d.lutSize);
  SetKernelSelf(d.kernelSelf);
  SetInitialMass(d.initialMass);
  SetFluidRestDensity(d.fluidRestDensity);
  SetFluidRestVolume(d.initialMass, d.fluidRestDensity);
  SetZindexStartingVec(d.zindexStartingVec);
  SetGamma(d.gamma);
  SetFluidGasConstant(d.fluidGasConstant, d.fluidGasConstantWCSPH);
  SetDensityErrorFactorPCISPH(d.param_density_error_factor);
  SetBoundaryConstants(d.forceDistance, d.maxBoundaryForce, d.minCollisionBox, d.maxCollisionBox,
                       d.addBoundaryForce);
  SetBoundingBox(d.minBoundingBox, d.maxBoundingBox);
  SetRealContainerValues(d.boxLength, d.boxHeigth, d.boxWidth, d.minContainerBox, d.maxContainerBox);
  SetDeltaT(d.deltaT, d.deltaTWCSPH);
  SetScales(d.scales);
  SetGravityConstant(d.gravityConstant);
  SetInitialMassIntoGravityRatio(d.initialMass, d.gravityConstant);
  SetFluidViscosityConstant(d.fluidViscosityConstant);
  SetSpacing(d.spacing);
  SetParticleRenderingSize(d.particleRenderingSize);
  SetMaximumArrayLength(d.maxLength);
  set_const([&](Constants& k) {
    k.max_density_error = d.param_max_density_error_allowed;
    k.min_loops = d.param_min_loops;
    k.max_loops = d.param_max_loops;
  });
  SetOtherConstants();
}

// FreeDeviceArrays (particles.cu:263-346): releases the simulation.
void FreeDeviceArrays(dataPointers& d) {
  if (!d.upf) return;
  if (d.upf->sys) upf_destroy(d.upf->sys);
  delete d.upf;
  d.upf = nullptr;
}

// CopyIndicesDeviceToHost (particles.cu:381-385): (key, index) pairs of the
// particles in their current sorted order.
void CopyIndicesDeviceToHost(dataPointers& d, uint*& indices) {
  upf_system* s = system_for(d, default_pipeline(d), "CopyIndicesDeviceToHost");
  if (!s || !indices) return;
  const uint32_t n = d.upf->type.size();
  std::vector<uint32_t> keys(n), ids(n);
  uint32_t got = 0;
  if (!ok_call(d.upf, upf_get_sorted_keys(s, keys.data(), ids.data(), &got), "CopyIndicesDeviceToHost")) return;
  for (uint32_t i = 0; i < got && i < d.particleCount; ++i) {
    indices[2 * i] = keys[i];
    indices[2 * i + 1] = ids[i];
  }
}

// CopyZIndicesKVPairHostToDevice (particles.cu:349-379): the library keys the
// particles itself from their positions, so the caller's keys are not needed.
void CopyZIndicesKVPairHostToDevice(dataPointers& d, std::vector<UnifiedParticle>&) {
  ctx_of(d, "CopyZIndicesKVPairHostToDevice");
}

// CopyRigidBodyDataHostToDevice (particles.cu:651-700): body mass, centre of
// mass, inertia and momenta come from the uploaded rigid particles (grouped
// by parent_rigid_body_index_) when the simulation is created.
void CopyRigidBodyDataHostToDevice(const std::vector<RigidBody*>& rigidbodies_h, dataPointers& d) {
  upf_compat_context* c = ctx_of(d, "CopyRigidBodyDataHostToDevice");
  if (c) c->num_bodies = (unsigned)rigidbodies_h.size();
}

// CopyParticlesDeviceToHost (particles.cu:808-812): particleCount positions
// (float4) into p, in upload order.
void CopyParticlesDeviceToHost(dataPointers& d, std::vector<UnifiedParticle>&, float*& p) {
  upf_system* s = system_for(d, default_pipeline(d), "CopyParticlesDeviceToHost");
  if (!s || !p) return;
  const uint32_t n = d.upf->type.size();
  std::vector<float> pos(4 * (size_t)n);
  if (!ok_call(d.upf, upf_get_particles_input_order(s, pos.data(), nullptr, nullptr, nullptr, nullptr, n),
               "CopyParticlesDeviceToHost"))
    return;
  std::memcpy(p, pos.data(), sizeof(float) * 4 * std::min<size_t>(n, d.particleCount));
}

// ---- tables ---------------------------------------------------------------
void CreateZIndexTexture(unsigned int* A) {
  if (!A) {
    fail_ctx(nullptr, UPF_ERR_INVALID_ARG, "CreateZIndexTexture: null table");
    return;
  }
  // ZIndex::z_table_ (zIndex.cpp:10-24): entry [i][a] spreads the 10 bits of
  // i to every third bit from bit a; the library interleaves the same way
  for (unsigned i = 0; i < 1024; ++i) {
    unsigned v = 0;
    for (int b = 0; b < 10; ++b) v |= ((i >> b) & 1u) << (3 * b);
    for (unsigned a = 0; a < 3; ++a)
      if (A[3 * i + a] != (v << a)) {
        fail_ctx(nullptr, UPF_ERR_INVALID_ARG,
                 "CreateZIndexTexture: entry [%u][%u] = %u differs from the Morton interleave the library uses (%u)",
                 i, a, A[3 * i + a], v << a);
        return;
      }
  }
}
void CreateLutKernelM4Texture(float* A, const int lutSize) { check_lut(kM4, A, lutSize, "CreateLutKernelM4Texture"); }
void CreateLutKernelPressureGradientTexture(float* A, const int lutSize) {
  check_lut(kPressureGrad, A, lutSize, "CreateLutKernelPressureGradientTexture");
}
void CreateLutKernelViscosityLapTexture(float* A, const int lutSize) {
  check_lut(kViscosityLap, A, lutSize, "CreateLutKernelViscosityLapTexture");
}
void CreateLutSplineSurfaceTensionTexture(float* A, const int lutSize) {
  check_lut(kSurfaceTension, A, lutSize, "CreateLutSplineSurfaceTensionTexture");
}
void CreateLutSplineSurfaceAdhesionTexture(float* A, const int lutSize) {
  check_lut(kAdhesion, A, lutSize, "CreateLutSplineSurfaceAdhesionTexture");
}
void CreateLutKernelM4(float* A, const int& lutSize) { CreateLutKernelM4Texture(A, lutSize); }
void CreateLutKernelPressureGradient(float* A, const int& lutSize) { CreateLutKernelPressureGradientTexture(A, lutSize); }
void CreateLutKernelViscosityLap(float* A, const int& lutSize) { CreateLutKernelViscosityLapTexture(A, lutSize); }
void CreateLutSplineSurfaceTension(float* A, const int& lutSize) { CreateLutSplineSurfaceTensionTexture(A, lutSize); }
void CreateLutSplineSurfaceAdhesion(float* A, const int& lutSize) { CreateLutSplineSurfaceAdhesionTexture(A, lutSize); }

// ---- device constants -------------------------------------------------------
void SetParticleCount(const unsigned int& count) { set_const([&](Constants& k) { k.particle_count = count; }); }
void SetRigidBodyCount(const unsigned int& n) { set_const([&](Constants& k) { k.num_rigid_bodies = n; }); }
void SetGlobalSupportRadius(const float& rad) { set_const([&](Constants& k) { k.support_radius = rad; }); }
void SetDistToCenterMassCutoffApproximate(const float&) {}  // approximate SPH only
void SetVelCutoffApproximate(const float&) {}               // approximate SPH only
void SetParticleRadius(const float& r) { set_const([&](Constants& k) { k.particle_radius = r; }); }
void SetTerminalSpeed(const float& v) { set_const([&](Constants& k) { k.terminal_speed = v; }); }
void SetRigidBodyCoefficients(const float& spring, const float& spring_boundary, const float& damp) {
  set_const([&](Constants& k) {
    k.rb_spring = spring;
    k.rb_spring_boundary = spring_boundary;
    k.rb_damping = damp;
  });
}
void SetSurfaceTensionAdhesionCoefficients(const float& g, const float& b) {
  set_const([&](Constants& k) {
    k.surface_tension_gamma = g;
    k.surface_adhesion_beta = b;
  });
}
void SetGridResolution(const unsigned int& r) { set_const([&](Constants& k) { k.grid_resolution = r; }); }
void SetBlockSize(const unsigned int& b) { set_const([&](Constants& k) { k.block_size = b; }); }
void SetLutSize(const unsigned int& n) { set_const([&](Constants& k) { k.lut_size = n; }); }
void SetKernelSelf(const float& v) { set_const([&](Constants& k) { k.kernel_self = v; }); }
void SetInitialMass(const float& m) { set_const([&](Constants& k) { k.mass = m; }); }
void SetFluidRestDensity(const float& r) { set_const([&](Constants& k) { k.rest_density = r; }); }
void SetFluidRestVolume(const float&, const float&) {}  // derived: mass / rest density
void SetZindexStartingVec(const float3& o) { set_const([&](Constants& k) { k.zindex_origin = o; }); }
void SetGamma(const float& g) { set_const([&](Constants& k) { k.gamma = g; }); }
void SetFluidGasConstant(const float& c, const float& c_wcsph) {
  set_const([&](Constants& k) {
    k.gas_constant = c;
    k.gas_constant_wcsph = c_wcsph;
  });
}
void SetDensityErrorFactorPCISPH(const float& f) { set_const([&](Constants& k) { k.density_error_factor = f; }); }
void SetBoundaryConstants(const float& force_distance, const float& max_force, const float3& minB, const float3& maxB,
                          bool& add) {
  set_const([&](Constants& k) {
    k.force_distance = force_distance;
    k.max_boundary_force = max_force;
    k.collision_min = minB;
    k.collision_max = maxB;
    k.add_boundary_force = add;
  });
}
void SetBoundingBox(const float3& minB, const float3& maxB) {
  set_const([&](Constants& k) {
    k.bounding_min = minB;
    k.bounding_max = maxB;
  });
}
void SetRealContainerValues(const float&, const float&, const float&, const float3& minB, const float3& maxB) {
  set_const([&](Constants& k) {
    k.container_min = minB;
    k.container_max = maxB;
  });
}
void SetDeltaT(const float& dt, const float& dt_wcsph) {
  set_const([&](Constants& k) {
    k.dt = dt;
    k.dt_wcsph = dt_wcsph;
  });
}
void SetScales(const float3& s) { set_const([&](Constants& k) { k.scales = s; }); }
void SetGravityConstant(const float& g) { set_const([&](Constants& k) { k.gravity = g; }); }
void SetInitialMassIntoGravityRatio(const float&, const float&) {}  // derived
void SetFluidViscosityConstant(const float& v) { set_const([&](Constants& k) { k.viscosity = v; }); }
void SetFluidViscosityConstantTube(float&) {}  // demo scene 2 (pipe) only
void SetSpacing(const float& s) { set_const([&](Constants& k) { k.spacing = s; }); }
void SetParticleRenderingSize(const float&) {}  // rendering
void SetOtherConstants() {}
void SetPipePoints(const float3&, const float3&) {}  // demo scene 2 (pipe) only
void SetPipeRadius(float&) {}
void SetWallConstant(const float&) {}
void SetGridDimensions(uint&, uint&, uint&) {}  // the library sizes its own cell tables
void SetMaximumArrayLength(uint&) {}

// ---- readback ---------------------------------------------------------------
uint CopyParticlesCUDA(float* pos_zindex, float* vel, float* corr_pressure, float* predicted_density,
                       int* particleType, int* activeType, dataPointers& d) {
  upf_system* s = system_for(d, default_pipeline(d), "CopyParticlesCUDA");
  if (!s) return 0;
  upf_compat_context* c = d.upf;
  const uint32_t n = (uint32_t)c->type.size();
  if (n > d.particleCountRounded) {
    // the caller's arrays hold particleCountRounded entries
    fail_ctx(c, UPF_ERR_INVALID_ARG, "CopyParticlesCUDA: %u particles uploaded, but particleCountRounded is %u", n,
             d.particleCountRounded);
    return 0;
  }
  if (!ok_call(c, upf_get_particles_input_order(s, pos_zindex, vel, predicted_density, corr_pressure, particleType,
                                                n),
               "CopyParticlesCUDA"))
    return 0;
  // activeType belongs to the approximate SPH variant; its upload value is
  // 100 (CopyParticleDataHostToDevice, particles.cu:431) and stays so
  if (activeType)
    for (uint32_t i = 0; i < n; ++i) activeType[i] = 100;
  // the padding of the rounded arrays, as the reference fills it
  // (particles.cu:460-497)
  for (uint32_t i = n; i < d.particleCountRounded; ++i) {
    if (pos_zindex) {
      pos_zindex[4 * i] = d.maxCollisionBox.x * 4.0f;
      pos_zindex[4 * i + 1] = d.maxCollisionBox.y * 4.0f;
      pos_zindex[4 * i + 2] = d.maxCollisionBox.z * 4.0f;
      pos_zindex[4 * i + 3] = (float)UINT_MAX;
    }
    if (vel)
      for (int a = 0; a < 4; ++a) vel[4 * i + a] = 0.0f;
    if (corr_pressure) corr_pressure[i] = 0.0f;
    if (predicted_density) predicted_density[i] = 0.0f;
    if (particleType) particleType[i] = 100;
    if (activeType) activeType[i] = 100;
  }
  return d.particleCount;
}

// ---- GL interop: headless -------------------------------------------------
void RegisterGLBufferObject(uint, struct cudaGraphicsResource** r) {
  if (r) *r = nullptr;
}
void UnregisterGLBufferObject(struct cudaGraphicsResource*) {}
void* MapGLBufferObject(struct cudaGraphicsResource**) { return nullptr; }
void UnmapGLBufferObject(struct cudaGraphicsResource*) {}

// ---- SPH / WCSPH --------------------------------------------------------------
void ZindexSorting(int, int, dataPointers& d) { phase(d, default_pipeline(d), upf_phase_sort, "ZindexSorting"); }
void BlockGeneration(dataPointers& d, int&, int&) {
  phase(d, default_pipeline(d), upf_phase_neighbors, "BlockGeneration");
}
void DensityPressureComputation(int, dataPointers& d, int&) {
  phase(d, kSph, upf_phase_forces, "DensityPressureComputation");
}
void ForceComputation(int, dataPointers& d, int&) { phase(d, kSph, upf_phase_integrate, "ForceComputation"); }
void CalculateZindex(int, dataPointers& d) { ctx_of(d, "CalculateZindex"); }  // keyed in the integration
void UnbindTexturesSPH() {}
void UnbindTexturesPCISPH() {}
void UnbindTextureRigidFluidSPH() {}
void UnbindTextureRigidFluidPCISPH() {}
void PingPongScheme(dataPointers&) {}  // the library's buffers need no swap
void PingPongSchemeRigidBody(dataPointers&) {}
void ParticlePhysicsOnDeviceSPH(dataPointers& d) { step(d, kSph, "ParticlePhysicsOnDeviceSPH"); }
void ZindexSortingApproximate(int, int, dataPointers& d) { unsupported(&d, "ZindexSortingApproximate"); }
void DensityPressureComputationApproximate(int, dataPointers& d, int&) {
  unsupported(&d, "DensityPressureComputationApproximate");
}
void ForceComputationApproximate(int, dataPointers& d, int&) { unsupported(&d, "ForceComputationApproximate"); }
void ExtractSurface(dataPointers& d, int&) { unsupported(&d, "ExtractSurface"); }
void ParticlePhysicsOnDeviceSPHApproximate(dataPointers& d) {
  unsupported(&d, "ParticlePhysicsOnDeviceSPHApproximate");
}

// ---- PCISPH -------------------------------------------------------------------
void ParticlePhysicsOnDevicePCISPH(dataPointers& d) { step(d, kPcisph, "ParticlePhysicsOnDevicePCISPH"); }
void CalculateExternalForcesPcisphCUDA(int, dataPointers& d, int&) {
  phase(d, default_pipeline(d), upf_phase_forces, "CalculateExternalForcesPcisphCUDA");
}
void PredictionCorrectionStepPcisphCUDA(dataPointers& d, int&) {
  phase(d, default_pipeline(d), upf_phase_predict_correct, "PredictionCorrectionStepPcisphCUDA");
}
void TimeIntegrationPcisphCUDAPureFluid(int, dataPointers& d, int&) {
  phase(d, default_pipeline(d), upf_phase_integrate, "TimeIntegrationPcisphCUDAPureFluid");
}
void GetMaxPredictedDensityCUDA(dataPointers& d, float& max_predicted_density) {
  upf_system* s = system_for(d, default_pipeline(d), "GetMaxPredictedDensityCUDA");
  if (!s) return;
  upf_step_stats st;
  if (ok_call(d.upf, upf_get_step_stats(s, &st), "GetMaxPredictedDensityCUDA"))
    max_predicted_density = st.max_predicted_density;
}
void ParticlePhysicsOnDevicePCISPHIhmsen2010(dataPointers& d) {
  unsupported(&d, "ParticlePhysicsOnDevicePCISPHIhmsen2010");
}

// ---- static boundaries, rigid coupling ------------------------------------------
void CalculateExternalForcesStaticBoundariesPcisphCUDA(int, dataPointers& d, int&) {
  phase(d, kPcisphStatic, upf_phase_forces, "CalculateExternalForcesStaticBoundariesPcisphCUDA");
}
void TimeIntegrationStaticBoundariesPcisphCUDA(int, dataPointers& d, int&) {
  phase(d, kPcisphStatic, upf_phase_integrate, "TimeIntegrationStaticBoundariesPcisphCUDA");
}
void ZindexSortingStaticBoundariesPCISPH(int, int, dataPointers& d) {
  phase(d, kPcisphStatic, upf_phase_sort, "ZindexSortingStaticBoundariesPCISPH");
}
void ParticlePhysicsOnDeviceFluidStaticBoundariesPCISPH(dataPointers& d) {
  step(d, kPcisphStatic, "ParticlePhysicsOnDeviceFluidStaticBoundariesPCISPH");
}
void ZindexSortingRigidBodySPH(int, dataPointers& d) { phase(d, kSphRigid, upf_phase_sort, "ZindexSortingRigidBodySPH"); }
void ZindexSortingRigidBodyPCISPH(int, dataPointers& d) {
  phase(d, kPcisphRigid, upf_phase_sort, "ZindexSortingRigidBodyPCISPH");
}
void ParticlePhysicsOnDeviceFluidRigidCouplingSPH(dataPointers& d) {
  step(d, kSphRigid, "ParticlePhysicsOnDeviceFluidRigidCouplingSPH");
}
// rigid body integration and particle sync run inside the library's
// integration phase (TimeIntegration*), which is also where these belong in
// the reference's step sequence
void RigidBodyIntegration(int, dataPointers& d) { ctx_of(d, "RigidBodyIntegration"); }
void SynRigidParticlesDevice(int, dataPointers& d) { ctx_of(d, "SynRigidParticlesDevice"); }
void ParticlePhysicsOnDeviceFluidRigidCouplingPCISPH(dataPointers& d) {
  step(d, kPcisphRigid, "ParticlePhysicsOnDeviceFluidRigidCouplingPCISPH");
}
void CalculateExternalForcesFluidRigidCouplingPcisphCUDA(int, dataPointers& d, int&) {
  phase(d, kPcisphRigid, upf_phase_forces, "CalculateExternalForcesFluidRigidCouplingPcisphCUDA");
}
void RigidBodyIntegrationTwoWayCoupling(int, dataPointers& d) { ctx_of(d, "RigidBodyIntegrationTwoWayCoupling"); }

// ---- radix sort -----------------------------------------------------------------
// RadixSort (particles.cu:31-60) on interleaved pairs: split into key and
// value arrays inside pData1, sort them with the library's sort, join back
// into pData0. The library's scratch is kept between calls.
void RadixSort(KeyValuePair* pData0, KeyValuePair* pData1, uint elements, uint bits) {
  if (elements == 0) return;
  if (!pData0 || !pData1 || bits == 0 || bits > 32) {
    fail_ctx(nullptr, UPF_ERR_INVALID_ARG, "RadixSort: null arrays or bits = %u", bits);
    return;
  }
  std::lock_guard<std::mutex> lock(g_mutex);
  uint32_t* keys = reinterpret_cast<uint32_t*>(pData1);
  uint32_t* vals = keys + elements;
  const size_t need = upf_radix_sort_temp_bytes(elements);
  cudaError_t e = cudaSuccess;
  if (need > g_sort_tmp_bytes) {
    if (g_sort_tmp) cudaFree(g_sort_tmp);
    g_sort_tmp = nullptr;
    g_sort_tmp_bytes = 0;
    e = cudaMalloc(&g_sort_tmp, need);
    if (e == cudaSuccess) g_sort_tmp_bytes = need;
  }
  if (e == cudaSuccess) {
    k_split_pairs<<<(elements + 255) / 256, 256>>>(elements, pData0, keys, vals);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    fail_ctx(nullptr, UPF_ERR_CUDA, "RadixSort: %s", cudaGetErrorString(e));
    return;
  }
  const upf_status st = upf_radix_sort_pairs(keys, vals, elements, (int32_t)bits, g_sort_tmp, g_sort_tmp_bytes,
                                             nullptr);
  if (st != UPF_OK) {
    fail_ctx(nullptr, st, "RadixSort: %s", upf_last_error());
    return;
  }
  k_join_pairs<<<(elements + 255) / 256, 256>>>(elements, keys, vals, pData0);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) fail_ctx(nullptr, UPF_ERR_CUDA, "RadixSort: %s", cudaGetErrorString(e));
}

}  // extern "C"
