// ref_pins_physics.cpp — TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's own CPU step — CpuParticlePhysicsVersatileCouplingPCISPH
// (src/cpu/UnifiedPhysics.cpp:4991-5024) and the member functions it calls,
// copied unchanged by extract_reference_physics.py and compiled beside
// ref_physics_harness.h into oracle/_ref/libupfref_physics.so — on a scene
// of liquid, frozen boundary and rigid particles, so that the oracle's
// restatement of the step (density, pressure, forces, the predict-correct
// loop, integration, the rigid bodies) can be pinned to the reference
// itself; and the WCSPH step CpuParticlePhysicsPureFluidsSPH the same way.
//
// What the harness sets up, since the reference's own set-up (Scene.cpp and
// the UnifiedPhysics constructor) does not compile here:
//  * UnifiedConstants from the scene's derived parameters (the same values
//    the oracle and the library use), WeightingKernel from them, kernel_self_
//    as the constructor computes it (UnifiedPhysics.cpp:113), the Morton
//    block size as CreatePartilcesCPU does (UnifiedPhysics.cpp:2152-2159);
//  * particles with the 7-argument UnifiedParticle constructor (correction
//    pressure 0, predicted density = rest density), the fields that
//    constructor leaves unset and the step reads set to what the oracle
//    assumes (previous correction pressure 0, no parent rigid body), and the
//    particle's input index kept in color_ (which the step never touches);
//  * optionally the boundary volumes by the reference's CalculateWeightedVolume
//    at set-up (the CPU coupling step has that call commented out,
//    UnifiedPhysics.cpp:4997; the oracle and the GPU path compute them when
//    adhesion is on);
//  * one OpenMP thread: the loop's maximum predicted density is a shared
//    member updated without a reduction (UnifiedPhysics.cpp:5488), which races
//    with several threads.
// Function-local statics in the reference (collision box, time step, particle
// count, lookup factor) take the first scene's values: one scene per process.
#include <cstdio>
#include <cstdlib>
#include <sstream>
#include <string>

#include "../include/upf.h"
#include "ref_physics_harness.h"

ZIndex zIndex;  // the reference's file-scope index (UnifiedPhysics.cpp:36)

namespace {
struct Quiet {
  std::streambuf* old;
  std::ostringstream sink;
  Quiet() : old(std::cout.rdbuf(sink.rdbuf())) {}
  ~Quiet() { std::cout.rdbuf(old); }
};
}  // namespace

// UnifiedConstants from the derived parameters: the fields the extracted
// functions read.
static void set_constants(UnifiedConstants& fc, const upf_params* prm, char physics) {
  fc.globalSupportRadius = prm->support_radius;
  fc.initialMass = prm->mass;
  fc.fluidRestDensity = prm->rest_density;
  fc.fluidViscConst = prm->viscosity;
  fc.gravityConst = prm->gravity;
  fc.deltaT = prm->dt;
  fc.densityErrorFactor = prm->density_error_factor;
  fc.maxDensityErrorAllowed = prm->max_density_error;
  fc.minLoops = prm->min_loops;
  fc.maxLoops = prm->max_loops;
  fc.scales = vmml::Vector3f(prm->scales[0], prm->scales[1], prm->scales[2]);
  fc.collisionBox.set(vmml::Vector3f(prm->collision_min[0], prm->collision_min[1], prm->collision_min[2]),
                      vmml::Vector3f(prm->collision_max[0], prm->collision_max[1], prm->collision_max[2]));
  fc.realBoxContainer.set(vmml::Vector3f(prm->container_min[0], prm->container_min[1], prm->container_min[2]),
                          vmml::Vector3f(prm->container_max[0], prm->container_max[1], prm->container_max[2]));
  fc.boxLength = prm->container_max[0] - prm->container_min[0];
  fc.boxHeight = prm->container_max[1] - prm->container_min[1];
  fc.boxWidth = prm->container_max[2] - prm->container_min[2];
  fc.physicsType = physics;
  fc.particleSpacing = prm->particle_spacing;
  fc.fluidGasConstantWCSPH = prm->gas_constant;
  fc.surface_tension_gamma = prm->surface_tension_gamma;
  fc.surface_adhesion_beta = prm->surface_adhesion_beta;
  fc.particleRadius = prm->particle_radius;
  fc.forceDistance = prm->force_distance;
  fc.maxBoundaryForce = prm->max_boundary_force;
  fc.springCoefficient = prm->spring_coefficient;
  fc.springCoefficientBoundary = prm->spring_coefficient_boundary;
  fc.dampingCoefficient = prm->damping_coefficient;
  fc.terminalSpeed = prm->terminal_speed;
  fc.useSurfaceTension = (prm->flags & UPF_FLAG_SURFACE_TENSION) != 0;
  fc.addWallWeightFunction = (prm->flags & UPF_FLAG_WALL_WEIGHT) != 0;
  fc.addBoundaryForce = false;
  fc.printDebuggingInfo = 0;
}

// The physics object over the particles, as the reference's constructor and
// CreatePartilcesCPU leave it; lag_* (nullable) set the lagged PCISPH state of
// a run resumed mid-trajectory, per input particle: the final correction
// pressure of the step before last (previous_correction_pressure_) and of the
// last step (correction_pressure_), and the last predicted density.
static UnifiedConstants g_fc;
static void set_up(UnifiedPhysics& up, char physics, const upf_params* prm, const float* pos4, const float* vel4,
                   const int32_t* type, uint32_t n, const float* lag_prev, const float* lag_p,
                   const float* lag_rho) {
  set_constants(g_fc, prm, physics);
  static WeightingKernel kernel(&g_fc);
  up.fc_ = &g_fc;
  up.my_kernel_ = &kernel;
  up.kernel_self_ = kernel.KernelM4(0.0f, g_fc.globalSupportRadius);
  up.density_error_too_large_ = true;
  up.max_loops_sim_ = 0;
  up.avg_loops_sim_ = 0.0f;
  up.max_predicted_density_ = 0.0f;
  up.num_nonfrozen_particles_ = 0;
  up.iteration_counter_ = 0;
  up.min_dens_ = std::numeric_limits<float>::max();
  up.max_dens_ = 0.0f;
  up.dens_avg_timestep_ = 0.0f;
  float block = g_fc.scales.x * g_fc.globalSupportRadius;
  block = MAX(block, g_fc.scales.y * g_fc.globalSupportRadius);
  block = MAX(block, g_fc.scales.z * g_fc.globalSupportRadius);
  zIndex.SetBlockSize(block);

  up.particles_.reserve(n);
  for (uint32_t i = 0; i < n; ++i) {
    UnifiedParticle q(vmml::Vector3f(pos4[4 * i], pos4[4 * i + 1], pos4[4 * i + 2]), type[i],
                      vmml::Vector3f(vel4[4 * i], vel4[4 * i + 1], vel4[4 * i + 2]), 0.0f, prm->rest_density,
                      prm->rest_density, prm->mass);
    q.previous_correction_pressure_ = lag_prev ? lag_prev[i] : 0.0f;
    if (lag_p) q.correction_pressure_ = lag_p[i];
    if (lag_rho) q.predicted_density_ = lag_rho[i];
    q.correction_pressure_force_ = vmml::Vector3f(0.0f, 0.0f, 0.0f);
    q.density_error_ = 0.0f;
    q.parent_rigidbody_ = nullptr;
    q.color_ = vmml::Vector3f((float)i, 0.0f, 0.0f);
    q.index_ = zIndex.CalcIndex(g_fc.scales * q.position_);
    if (type[i] != FROZEN_PARTICLE) up.num_nonfrozen_particles_++;
    up.particles_.push_back(q);
  }
  up.SortParticles();
  up.neighbor_indices_.resize(n);
}

static int run_steps(char physics, const upf_params* prm, const float* pos4, const float* vel4,
                     const int32_t* type, const float* const* lag, const int32_t* body_of, uint32_t n_bodies,
                     uint32_t n, int32_t steps, int32_t weighted_volumes, float* out_pos4, float* out_vel4,
                     float* out_density, float* out_pressure, int32_t* out_type, uint32_t* out_id,
                     float* out_body) {
  if (!prm || !pos4 || !vel4 || !type || steps < 0 || (n_bodies && !body_of)) return 3;
  for (uint32_t i = 0; body_of && i < n; ++i)
    if (body_of[i] >= (int32_t)n_bodies || (body_of[i] >= 0) != (type[i] == RIGID_PARTICLE)) return 3;
  Quiet quiet;
  omp_set_num_threads(1);
  UnifiedPhysics up;
  set_up(up, physics, prm, pos4, vel4, type, n, lag ? lag[0] : nullptr, lag ? lag[1] : nullptr,
         lag ? lag[2] : nullptr);
  auto keys_unique = [&]() {
    for (size_t k = 1; k < up.particles_.size(); ++k)
      if (up.particles_[k].index_ == up.particles_[k - 1].index_) return false;
    return true;
  };
  if (!keys_unique()) return 1;
  // Rigid bodies: each particle added to its body by the reference's
  // AddToRigidBody, in array order. The reference's scene construction
  // (SolidifyParticle, UnifiedPhysics.cpp:810-850) adds particles with the
  // same function, in an order its solid-neighbour lists decide, which this
  // set-up does not build. Then the constructor's loop over the bodies
  // (UnifiedPhysics.cpp:144-160): parent index, order in the body, initial
  // relative position. That loop's
  // Matrix3x3::CalculateInverse(rb->inertia(), rb->inverted_inertia_local())
  // writes into the temporary the getter returns, so the body's local
  // inverse inertia keeps its zero initial value; it is left out here with
  // the same effect.
  std::vector<RigidBody> bodies(n_bodies);
  for (uint32_t b = 0; b < n_bodies; ++b) up.rigid_bodies_.push_back(&bodies[b]);
  for (uint32_t k = 0; k < n && n_bodies; ++k) {
    const int b = body_of[(uint32_t)up.particles_[k].color_.x];
    if (b >= 0) up.AddToRigidBody(up.rigid_bodies_[b], (int)k);
  }
  for (uint32_t b = 0; b < n_bodies; ++b) {
    RigidBody* rb = up.rigid_bodies_[b];
    const size_t count = rb->rigid_particle_indices().size();
    for (size_t j = 0; j < count; ++j) {
      UnifiedParticle& p = up.particles_[rb->rigid_particle_indices()[j]];
      p.parent_rigid_body_index_ = (int)b;
      p.order_in_child_particles_array_ = (int)j;
      p.init_relative_pos_ = p.position_ - rb->rigidbody_pos();
    }
  }
  if (weighted_volumes) {
    up.NeighborSearchOMP();
    up.CalculateWeightedVolumeOMP();
  }
  for (int32_t s = 0; s < steps; ++s) {
    if (physics == 'i')
      up.CpuParticlePhysicsVersatileCouplingPCISPH();
    else
      up.CpuParticlePhysicsPureFluidsSPH();
    if (!keys_unique()) return 1;
  }
  for (uint32_t b = 0; b < n_bodies && out_body; ++b) {
    const RigidBody* rb = up.rigid_bodies_[b];
    float* o = out_body + 16 * b;
    for (int a = 0; a < 3; ++a) {
      o[a] = rb->rigidbody_pos()[a];
      o[3 + a] = rb->velocity()[a];
      o[6 + a] = rb->angular_velocity()[a];
    }
    o[9] = rb->mass();
    for (int a = 0; a < 4; ++a) o[10 + a] = rb->quaternion()[a];
    o[14] = o[15] = 0.0f;
  }
  for (uint32_t k = 0; k < n; ++k) {
    const UnifiedParticle& q = up.particles_[k];
    for (int a = 0; a < 3; ++a) {
      out_pos4[4 * k + a] = q.position_[a];
      out_vel4[4 * k + a] = q.velocity_[a];
    }
    out_pos4[4 * k + 3] = 0.0f;
    out_vel4[4 * k + 3] = 0.0f;
    out_density[k] = physics == 'i' ? q.predicted_density_ : q.density_;
    out_pressure[k] = physics == 'i' ? q.correction_pressure_ : q.pressure_;
    out_type[k] = q.type_;
    out_id[k] = (uint32_t)q.color_.x;
  }
  return 0;
}

extern "C" {

// The PCISPH coupling step (CpuParticlePhysicsVersatileCouplingPCISPH).
// body_of[i] is input particle i's body (-1 for none; rigid particles and
// only they have one), n_bodies the number of bodies (body_of may be null
// when it is 0). Returns 0 on success; 1 if two particles share a Morton key
// (the reference's std::sort leaves their order unspecified, so no
// comparison is possible); 3 on bad arguments. Outputs are in the
// reference's final particle order (ascending key); density and pressure are
// the predicted density and correction pressure; out_body (16 floats a body,
// may be null) holds position, velocity, angular velocity, mass, quaternion.
// lag_prev, lag_p, lag_rho (all null for a run from rest) resume a run as in
// set_up.
int ref_physics_pcisph_steps(const upf_params* prm, const float* pos4, const float* vel4, const int32_t* type,
                             const float* lag_prev, const float* lag_p, const float* lag_rho,
                             const int32_t* body_of, uint32_t n_bodies, uint32_t n, int32_t steps,
                             int32_t weighted_volumes, float* out_pos4, float* out_vel4, float* out_density,
                             float* out_pressure, int32_t* out_type, uint32_t* out_id, float* out_body) {
  const float* lag[3] = {lag_prev, lag_p, lag_rho};
  return run_steps('i', prm, pos4, vel4, type, lag_prev ? lag : nullptr, body_of, n_bodies, n, steps,
                   weighted_volumes, out_pos4, out_vel4, out_density, out_pressure, out_type, out_id, out_body);
}

// The WCSPH step (CpuParticlePhysicsPureFluidsSPH), the same way, without
// rigid bodies; density and pressure are the step's density_ and pressure_.
int ref_physics_wcsph_steps(const upf_params* prm, const float* pos4, const float* vel4, const int32_t* type,
                            uint32_t n, int32_t steps, float* out_pos4, float* out_vel4, float* out_density,
                            float* out_pressure, int32_t* out_type, uint32_t* out_id) {
  return run_steps('w', prm, pos4, vel4, type, nullptr, nullptr, 0, n, steps, 0, out_pos4, out_vel4, out_density,
                   out_pressure, out_type, out_id, nullptr);
}

// Times the reference's step on the host cores: the PCISPH coupling step
// ('i') or the WCSPH step ('w') on a scene of liquid and frozen boundary
// particles (lag_* as in set_up, nullable), `threads` OpenMP threads (the
// reference's own parallel loops; with more than one the loop's maximum
// predicted density is the reference's unsynchronised one), `warmup`
// untimed steps, then timed steps until `steps` have run, or until at least
// `min_steps` have run and `max_seconds` have passed. Per timed step: wall seconds, and for PCISPH
// the predict-correct iterations and the last iteration's density error in
// percent, read from the loop's own report (printDebuggingInfo = 1 prints
// "ERROR: <percent>%" once per iteration, UnifiedPhysics.cpp:5390-5391).
// Returns the number of timed steps, or -3 on bad arguments.
int ref_physics_time(int32_t wcsph, const upf_params* prm, const float* pos4, const float* vel4,
                     const int32_t* type, uint32_t n, const float* lag_prev, const float* lag_p, const float* lag_rho,
                     int32_t threads, int32_t warmup, int32_t steps, int32_t min_steps, double max_seconds,
                     double* seconds, int32_t* iterations, float* error_percent) {
  if (!prm || !pos4 || !vel4 || !type || threads < 1 || warmup < 0 || steps < 1 || min_steps < 1 || !seconds)
    return -3;
  Quiet quiet;
  omp_set_num_threads(threads);
  const char physics = wcsph ? 'w' : 'i';
  UnifiedPhysics up;
  set_up(up, physics, prm, pos4, vel4, type, n, lag_prev, lag_p, lag_rho);
  g_fc.printDebuggingInfo = 1;
  auto one = [&]() {
    if (physics == 'i')
      up.CpuParticlePhysicsVersatileCouplingPCISPH();
    else
      up.CpuParticlePhysicsPureFluidsSPH();
  };
  for (int32_t k = 0; k < warmup; ++k) one();
  int32_t done = 0;
  double total = 0.0;
  while (done < steps && (done < min_steps || total < max_seconds)) {
    quiet.sink.str("");
    const double t0 = omp_get_wtime();
    one();
    const double dt = omp_get_wtime() - t0;
    seconds[done] = dt;
    total += dt;
    // the loop's per-iteration reports
    const std::string log = quiet.sink.str();
    int32_t its = 0;
    float err = 0.0f;
    for (size_t at = log.find("ERROR: "); at != std::string::npos; at = log.find("ERROR: ", at + 7)) {
      ++its;
      err = std::strtof(log.c_str() + at + 7, nullptr);
    }
    if (iterations) iterations[done] = its;
    if (error_percent) error_percent[done] = err;
    ++done;
  }
  return done;
}

}  // extern "C"
