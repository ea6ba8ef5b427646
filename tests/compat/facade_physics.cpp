// A host program shaped like the reference's facade (UnifiedPhysics,
// src/cpu/UnifiedPhysics.cpp): InitDptr (:478-600) fills dataPointers from
// the scene constants, InitCudaVariables (:615-643) makes the reference's
// init calls in its order, CudaParticlePhysics (:4051-4141) steps through
// the chosen ParticlePhysicsOnDevice* entry point and reads the particles
// back with CopyParticlesCUDA (CopyGPUParticles, :404-407), and the
// teardown calls FreeDeviceArrays. Built against include/upf_compat.h and
// linked with libupf_compat.so. Test infrastructure only.
//
//   facade_physics <input file> <output file>
//
// input: "UPFC", upf_params, uint32 n, uint32 steps, char[64] entry point,
//        float pos4[4n], float vel4[4n], int32 type[n], int32 body[n]
// output: int32 status, uint32 count, uint32 rounded, float pos4[4 rounded],
//         float vel4[4 rounded], float pressure[rounded], float density[rounded],
//         int32 type[rounded], int32 active[rounded], upf_params used,
//         char message[256]
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <vector_functions.h>

#include "UnifiedParticle.h"
#include "upf_compat.h"

namespace {

struct ParticleInfoForRendering {
  std::vector<float> pos, vel, corr_pressure, predicted_density;
  std::vector<int> type, active;
};

class Facade {
 public:
  upf_params fc_;  // the scene constants (the reference's UnifiedConstants)
  std::vector<UnifiedParticle> particles_;
  std::vector<RigidBody*> rigid_bodies_;
  dataPointers dptr_;
  ParticleInfoForRendering info_;
  std::string entry_;

  void InitDptr(uint32_t count) {
    std::memset(&dptr_, 0, sizeof dptr_);
    dptr_.demoScene = 1;
    dptr_.particleCount = count;
    dptr_.finalParticleCount = count;
    dptr_.globalSupportRadius = fc_.support_radius;
    dptr_.particleRadius = fc_.particle_radius;
    dptr_.rb_spring = fc_.spring_coefficient;
    dptr_.rb_spring_boundary = fc_.spring_coefficient_boundary;
    dptr_.rb_damping = fc_.damping_coefficient;
    dptr_.surface_tension_gamma = fc_.surface_tension_gamma;
    dptr_.surface_adhesion_beta = fc_.surface_adhesion_beta;
    dptr_.rb_terminalSpeed = fc_.terminal_speed;
    dptr_.grid_resolution = UPF_GRID_RESOLUTION;
    dptr_.block_size = fc_.block_size;
    dptr_.lutSize = UPF_LUT_SIZE;
    dptr_.initialMass = fc_.mass;
    dptr_.fluidRestDensity = fc_.rest_density;
    dptr_.gamma = fc_.gamma;
    dptr_.fluidGasConstantWCSPH = fc_.gas_constant;
    dptr_.fluidGasConstant = fc_.gas_constant;
    dptr_.addBoundaryForce = (fc_.flags & UPF_FLAG_PENALTY_WALLS) != 0;
    dptr_.forceDistance = fc_.force_distance;
    dptr_.maxBoundaryForce = fc_.max_boundary_force;
    dptr_.minCollisionBox = make_float3(fc_.collision_min[0], fc_.collision_min[1], fc_.collision_min[2]);
    dptr_.maxCollisionBox = make_float3(fc_.collision_max[0], fc_.collision_max[1], fc_.collision_max[2]);
    dptr_.minContainerBox = make_float3(fc_.container_min[0], fc_.container_min[1], fc_.container_min[2]);
    dptr_.maxContainerBox = make_float3(fc_.container_max[0], fc_.container_max[1], fc_.container_max[2]);
    dptr_.zindexStartingVec = make_float3(fc_.zindex_origin[0], fc_.zindex_origin[1], fc_.zindex_origin[2]);
    dptr_.scales = make_float3(fc_.scales[0], fc_.scales[1], fc_.scales[2]);
    dptr_.deltaT = fc_.dt;
    dptr_.deltaTWCSPH = fc_.dt;
    dptr_.gravityConstant = fc_.gravity;
    dptr_.fluidViscosityConstant = fc_.viscosity;
    dptr_.spacing = fc_.particle_spacing;
    dptr_.num_rigid_bodies = (unsigned)rigid_bodies_.size();
    dptr_.param_density_error_factor = fc_.density_error_factor;
    dptr_.param_max_density_error_allowed = fc_.max_density_error;
    dptr_.param_min_loops = fc_.min_loops;
    dptr_.param_max_loops = fc_.max_loops;
  }

  void InitCudaVariables(uint32_t count) {
    InitDptr(count);
    // the reference's order (UnifiedPhysics.cpp:619-641)
    MallocDeviceArraysParticles(dptr_);
    MallocDeviceArraysRigidBody(dptr_, rigid_bodies_);
    SetDeviceConstants(dptr_);
    std::vector<unsigned> z(3 * 1024);
    for (unsigned i = 0; i < 1024; ++i) {
      unsigned v = 0;
      for (int b = 0; b < 10; ++b) v |= ((i >> b) & 1u) << (3 * b);
      for (unsigned a = 0; a < 3; ++a) z[3 * i + a] = v << a;
    }
    CreateZIndexTexture(z.data());
    std::vector<float> luts(5 * UPF_LUT_ENTRIES);
    upf_build_luts(&fc_, luts.data());
    CreateLutKernelM4Texture(&luts[0], UPF_LUT_SIZE);
    CreateLutKernelPressureGradientTexture(&luts[UPF_LUT_ENTRIES], UPF_LUT_SIZE);
    CreateLutKernelViscosityLapTexture(&luts[2 * UPF_LUT_ENTRIES], UPF_LUT_SIZE);
    CreateLutSplineSurfaceTensionTexture(&luts[3 * UPF_LUT_ENTRIES], UPF_LUT_SIZE);
    CreateLutSplineSurfaceAdhesionTexture(&luts[4 * UPF_LUT_ENTRIES], UPF_LUT_SIZE);
    CopyZIndicesKVPairHostToDevice(dptr_, particles_);
    CopyParticleDataHostToDevice(dptr_, particles_);
    CopyRigidBodyDataHostToDevice(rigid_bodies_, dptr_);
    const size_t r = dptr_.particleCountRounded;
    info_.pos.resize(4 * r);
    info_.vel.resize(4 * r);
    info_.corr_pressure.resize(r);
    info_.predicted_density.resize(r);
    info_.type.resize(r);
    info_.active.resize(r);
  }

  void CopyGPUParticles() {
    CopyParticlesCUDA(info_.pos.data(), info_.vel.data(), info_.corr_pressure.data(), info_.predicted_density.data(),
                      info_.type.data(), info_.active.data(), dptr_);
  }

  void CudaParticlePhysics() {
    if (dptr_.particleCount > 0) {
      if (entry_ == "ParticlePhysicsOnDevicePCISPH") ParticlePhysicsOnDevicePCISPH(dptr_);
      else if (entry_ == "ParticlePhysicsOnDeviceFluidStaticBoundariesPCISPH")
        ParticlePhysicsOnDeviceFluidStaticBoundariesPCISPH(dptr_);
      else if (entry_ == "ParticlePhysicsOnDeviceFluidRigidCouplingPCISPH")
        ParticlePhysicsOnDeviceFluidRigidCouplingPCISPH(dptr_);
      else if (entry_ == "ParticlePhysicsOnDeviceSPH") ParticlePhysicsOnDeviceSPH(dptr_);
      else ParticlePhysicsOnDeviceFluidRigidCouplingSPH(dptr_);
      const size_t r = dptr_.particleCountRounded;
      std::memset(info_.pos.data(), 0, r * 4 * sizeof(float));
      std::memset(info_.vel.data(), 0, r * 4 * sizeof(float));
      std::memset(info_.corr_pressure.data(), 0, r * sizeof(float));
      std::memset(info_.predicted_density.data(), 0, r * sizeof(float));
      std::memset(info_.type.data(), 0, r * sizeof(int));
      std::memset(info_.active.data(), 0, r * sizeof(int));
      CopyGPUParticles();
    }
  }
};

template <class T>
bool rd(FILE* f, T* p, size_t n) {
  return std::fread(p, sizeof(T), n, f) == n;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s <input> <output>\n", argv[0]);
    return 2;
  }
  FILE* in = std::fopen(argv[1], "rb");
  if (!in) return 2;
  Facade fa;
  char magic[4];
  uint32_t n = 0, steps = 0;
  char entry[64];
  bool ok = rd(in, magic, 4) && std::memcmp(magic, "UPFC", 4) == 0 && rd(in, &fa.fc_, 1) && rd(in, &n, 1) &&
            rd(in, &steps, 1) && rd(in, entry, 64);
  std::vector<float> pos(4 * (size_t)n), vel(4 * (size_t)n);
  std::vector<int32_t> type(n), body(n);
  ok = ok && rd(in, pos.data(), pos.size()) && rd(in, vel.data(), vel.size()) && rd(in, type.data(), n) &&
       rd(in, body.data(), n);
  std::fclose(in);
  if (!ok) return 2;
  entry[63] = 0;
  fa.entry_ = entry;
  int32_t nbodies = 0;
  fa.particles_.resize(n);
  for (uint32_t i = 0; i < n; ++i) {
    UnifiedParticle& q = fa.particles_[i];
    q.position_ = {pos[4 * i], pos[4 * i + 1], pos[4 * i + 2]};
    q.velocity_ = {vel[4 * i], vel[4 * i + 1], vel[4 * i + 2]};
    q.type_ = type[i];
    q.parent_rigid_body_index_ = body[i];
    if (body[i] + 1 > nbodies) nbodies = body[i] + 1;
  }
  std::vector<RigidBody> bodies(nbodies);
  for (auto& b : bodies) fa.rigid_bodies_.push_back(&b);

  fa.InitCudaVariables(n);
  for (uint32_t k = 0; k < steps; ++k) fa.CudaParticlePhysics();

  FILE* out = std::fopen(argv[2], "wb");
  if (!out) return 2;
  const int32_t status = upf_compat_status(fa.dptr_);
  const uint32_t rounded = fa.dptr_.particleCountRounded;
  upf_params used{};
  upf_compat_params(fa.dptr_, &used);
  char msg[256] = {0};
  std::strncpy(msg, upf_compat_message(fa.dptr_), sizeof msg - 1);
  std::fwrite(&status, 4, 1, out);
  std::fwrite(&n, 4, 1, out);
  std::fwrite(&rounded, 4, 1, out);
  std::fwrite(fa.info_.pos.data(), sizeof(float), fa.info_.pos.size(), out);
  std::fwrite(fa.info_.vel.data(), sizeof(float), fa.info_.vel.size(), out);
  std::fwrite(fa.info_.corr_pressure.data(), sizeof(float), fa.info_.corr_pressure.size(), out);
  std::fwrite(fa.info_.predicted_density.data(), sizeof(float), fa.info_.predicted_density.size(), out);
  std::fwrite(fa.info_.type.data(), sizeof(int), fa.info_.type.size(), out);
  std::fwrite(fa.info_.active.data(), sizeof(int), fa.info_.active.size(), out);
  std::fwrite(&used, sizeof used, 1, out);
  std::fwrite(msg, 1, sizeof msg, out);
  std::fclose(out);
  FreeDeviceArrays(fa.dptr_);
  std::printf("status %d (%s) steps %u particles %u\n", status, upf_status_string((upf_status)status), steps, n);
  return 0;
}
