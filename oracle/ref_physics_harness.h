// ref_physics_harness.h — TEST INFRASTRUCTURE ONLY.
//
// The reference's CPU step lives in src/cpu/UnifiedPhysics.cpp, whose
// includes (windows.h, GL, render_particles.h, the CUDA interop header) need
// a graphics stack this build does not have. oracle/extract_reference_physics.py
// copies, unchanged and into oracle/_ref/ only, the member functions of the
// PCISPH step with static boundaries and rigid bodies; this header gives them
// the class they are members of: the data members and member functions they
// use, declared with the reference's own names and types
// (src/cpu/UnifiedPhysics.h:40-500), and nothing of its rendering, CUDA or
// file state. ref_pins_physics.cpp drives the result.
#pragma once

#include <math.h>  // float overloads of sqrt and pow, as MSVC's math header gives them
#include <omp.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <iostream>
#include <limits>
#include <vector>

#include "Matrix3x3.h"
#include "RigidBody.h"
#include "UnifiedConstants.h"
#include "UnifiedParticle.h"
#include "WeightingKernel.h"
#include "global.h"
#include "sort.h"
#include "vmmlib/vector3.h"
#include "zIndex.h"

class UnifiedPhysics {
 public:
  // data members the step reads and writes (UnifiedPhysics.h:413-500)
  std::vector<UnifiedParticle> particles_;
  std::vector<std::vector<int> > neighbor_indices_;
  std::vector<RigidBody*> rigid_bodies_;
  UnifiedConstants* fc_;
  WeightingKernel* my_kernel_;
  float kernel_self_;
  bool density_error_too_large_;
  int max_loops_sim_;
  float avg_loops_sim_;
  float max_predicted_density_;
  size_t num_nonfrozen_particles_;
  int iteration_counter_;
  float min_dens_;
  float max_dens_;
  float dens_avg_timestep_;

  // the step (UnifiedPhysics.cpp:4991-5024) and what it calls
  void CpuParticlePhysicsVersatileCouplingPCISPH();
  void NeighborSearchOMP();
  void GetNeighbors(const int i);
  void CalculateWeightedVolumeOMP();
  void CalculateWeightedVolume(const int i);
  void CalculateExternalForcesVersatilCouplingPCISPHOMP();
  void CalculateExternalForcesVersatilCouplingPCISPH(const int i);
  vmml::Vector3f CalculateBoundaryFluidPressureForceHost(uint dist_lut, vmml::Vector3f p_pos, vmml::Vector3f neigh_pos,
                                                         float p_density, float p_corr_pressure, float weighted_vol);
  vmml::Vector3f CalculateSurfaceTensionForcePCISPHHost(const uint dist_lut, const float dist,
                                                        const vmml::Vector3f p_pos, const vmml::Vector3f neigh_pos);
  vmml::Vector3f CalculateSurfaceCohesionForcePCISPHHost(const uint dist_lut, const float dist,
                                                         const vmml::Vector3f p_pos, const vmml::Vector3f neigh_pos,
                                                         float neigh_weighted_vol);
  vmml::Vector3f CalculateSpringForceHost(const float& dist, const float& overlap, const vmml::Vector3f& r_ij);
  vmml::Vector3f CalculateDampingForceHost(const vmml::Vector3f& v_ij);
  vmml::Vector3f CalculateBoundaryForcePerLiquidParticleHost(const vmml::Vector3f& position);
  vmml::Vector3f CalculateBoundaryForcePerRigidParticleHost(const vmml::Vector3f& position, const vmml::Vector3f& vel);
  void PredictionCorrectionStep();
  void PredictPositionAndVelocity(const int i);
  void CollisionHandling(vmml::Vector3f& pos, vmml::Vector3f& vel);
  void ComputePredictedDensityAndPressure(const int i);
  void ComputeCorrectivePressureForce(const int i);
  void UpdateLiquidParticlePosVelSphCPUOMP();
  void UpdateLiquidParticlePosVelSphCPU(const int i);
  void BoundaryHandlingPureFluidOMP();
  void BoundaryHandlingBoxPerNonRigidParticle(const vmml::Vector3f& minBox, const vmml::Vector3f& maxBox,
                                              const float damping, vmml::Vector3f& pos, vmml::Vector3f& vel);
  void SortParticles();
  void RigidBodyIntegrationOMP();
  void UpdateRigidBodyParticleInformationOMP();
  void SynRigidParticlesOMP();
  vmml::Vector3f BoxBoundaryForce(const int i);
  // the WCSPH step (UnifiedPhysics.cpp:4200-4260) and what it calls
  void CpuParticlePhysicsPureFluidsSPH();
  void CalculateDensityPressurePureFluidSPH(const int i);
  float CalculatePressureSPH(const float density);
  float CalculatePressureWCSPH(const float density);
  vmml::Vector3f CalculateLiquidParticleForces(UnifiedParticle& p, const int i);
  vmml::Vector3f CalculateSurfaceTensionForcePCISPH(const float dist, const vmml::Vector3f p_pos,
                                                    const vmml::Vector3f neigh_pos, const float splineCoefficient);
  // the reference's default argument binds a temporary to the non-const
  // reference (an MSVC extension); a scratch vector stands in for it
  static vmml::Vector3f& scratch_normal() {
    static vmml::Vector3f n;
    n.set(0.0f, 0.0f, 0.0f);
    return n;
  }
  float DistanceToWall(const float& x, const float& y, const float& z, vmml::Vector3f& norm = scratch_normal());
  float WallWeight(float distToWall, float effectiveDist);
  // inline in the reference's class (UnifiedPhysics.h:161)
  float PythagoreanDist(float x, float y) { return sqrt(x * x + y * y); }
  // the rigid phase's per-body functions and the assembly of a body
  void CalculateRigidBodyForceTorqueMomenta(const int i);
  void SynRigidParticlesPerRigidBody(RigidBody* body);
  void AddToRigidBody(RigidBody* rigid, const int pIndex);
};

// Matrix3x3::operator*(vmml::Vector3f&) takes a non-const reference
// (Matrix3x3.h:23), and CalculateRigidBodyForceTorqueMomenta passes it the
// temporary that angular_momentum() returns (UnifiedPhysics.cpp:3676), which
// only MSVC accepts. This overload is chosen only where the member cannot
// bind (an rvalue vector); it makes the member call on copies, as MSVC does.
inline vmml::Vector3f operator*(const Matrix3x3& m, const vmml::Vector3f& v) {
  Matrix3x3 mm(m);
  vmml::Vector3f vv(v);
  return mm * vv;
}
