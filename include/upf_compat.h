/* upf_compat.h — the reference's own GPU entry points, over upf.h.
 *
 * Drop-in for the extern "C" block of src/gpu/particles.cuh:430-586 and
 * RadixSort (src/gpu/radixsort.cuh:115-117) of Gfans/UnifiedParticleFrameworkCUDA:
 * the same names, signatures and call order, so that the reference's facade
 * (UnifiedPhysics::InitCudaVariables, UnifiedPhysics.cpp:615-643;
 * CudaParticlePhysics, :4051-4141; CopyGPUParticles, :404-407) compiles
 * against this header in place of particles.cuh and runs on this library.
 *
 * C++ only (the reference's block takes C++ references and std::vector).
 * Link against libupf_compat.so (which links libupf.so), and compile
 * unifiedparticleframeworkcuda_b200/compat/upf_compat_particles.cpp in the
 * caller's build: it reads the caller's UnifiedParticle fields
 * (CopyParticleDataHostToDevice) and is the only part that needs the
 * caller's particle class.
 *
 * Conventions, where this layer differs from the reference:
 *  - Errors: the legacy calls return void (or a count) as before. A failure
 *    prints one line "upf_compat: ..." to stderr and sets a sticky status
 *    (upf_compat_status); later calls on a failed simulation do nothing. The
 *    reference exits the process (CUDA_SAFE_CALL, cutil.h:761-769).
 *  - Device memory: the library owns every device array; the pointer
 *    members below stay null. GL interop is headless: MapGLBufferObject
 *    returns null, positions live in library buffers and come back through
 *    CopyParticlesCUDA.
 *  - Order: CopyParticlesCUDA and CopyParticlesDeviceToHost return the
 *    particles in the order the caller uploaded them
 *    (CopyParticleDataHostToDevice), permuted back on the device; the
 *    reference returns its own current sorted order.
 *  - Kernel tables and the z-index table: the library computes its own. The
 *    Create*Texture calls compare the caller's tables with them and flag a
 *    difference (UPF_ERR_INVALID_ARG) instead of uploading.
 *  - The simulation is created at the first step call, when the method is
 *    known: ParticlePhysicsOnDevice*PCISPH runs PCISPH, ...SPH the WCSPH
 *    step. The optional GPU terms follow the entry point:
 *      ParticlePhysicsOnDevicePCISPH / ...SPH: surface tension, and the
 *        penalty walls when addBoundaryForce;
 *      ...FluidStaticBoundariesPCISPH, ...FluidRigidCouplingPCISPH,
 *      ...FluidRigidCouplingSPH: the same plus the Akinci boundary pressure
 *        (UPF_FLAG_BOUNDARY_PRESSURE); rigid bodies are grouped by each
 *        RIGID particle's parent_rigid_body_index_.
 *  - Not available (sticky UPF_ERR_UNSUPPORTED): the approximate SPH variant,
 *    surface extraction, the Ihmsen-2010 boundary variant and the wall-weight
 *    and versatile-coupling phase calls, which this library does not build.
 */
#ifndef UPF_COMPAT_H_
#define UPF_COMPAT_H_

#ifndef __cplusplus
#error "upf_compat.h is C++ (the reference's entry points take C++ references)"
#endif

#include <vector_types.h>  /* float3, float4, as the reference's dataPointers */

#include <vector>

#include "upf.h"

class UnifiedParticle;  /* the caller's particle class (src/cpu/UnifiedParticle.h) */
class RigidBody;        /* the caller's rigid body class (src/cpu/RigidBody.h) */
struct cudaGraphicsResource;
struct upf_compat_context;

typedef unsigned int uint;

/* KeyValuePair of src/gpu/radixsort.cuh:52-60: a 32-bit key and its value. */
typedef struct {
  uint key;
  uint value;
} KeyValuePair;

/* The scalar block of dataPointers (src/gpu/particles.cuh:49-121) under the
 * reference's member names, which its facade sets (InitDptr,
 * UnifiedPhysics.cpp:478-600) and SetDeviceConstants reads; the device
 * pointer members the facade names are kept (null: the library owns the
 * arrays); `upf` is this layer's state for the simulation, set by
 * MallocDeviceArraysParticles and released by FreeDeviceArrays. */
struct dataPointers {
  uint demoScene;
  uint particleCount;
  uint particleCountRounded;
  uint finalParticleCount;
  uint finalParticleCountRounded;
  uint filledBlocks;
  uint dimX;
  uint dimY;
  uint dimZ;
  uint maxLength;
  uint filteredParticleCount;

  float globalSupportRadius;
  float distToCenterMassCutoff;
  float gradientVelCutoff;
  float particleRadius;
  float3 scales;
  uint grid_resolution;
  uint block_size;
  uint currIndex;
  uint currType;
  uint currActiveType;

  float rb_spring;
  float rb_spring_boundary;
  float rb_damping;
  float rb_terminalSpeed;
  float surface_tension_gamma;
  float surface_adhesion_beta;

  uint lutSize;
  float kernelSelf;
  float initialMass;
  float fluidRestDensity;
  float gamma;
  float fluidGasConstant;
  float fluidGasConstantWCSPH;
  float fluidViscosityConstant;
  float fluidViscosityConstant_tube;
  float gravityConstant;
  bool addBoundaryForce;
  float3 minCollisionBox;
  float3 maxCollisionBox;
  float3 minBoundingBox;
  float3 maxBoundingBox;
  float3 minContainerBox;
  float3 maxContainerBox;
  float3 zindexStartingVec;
  float boxLength;
  float boxHeigth;
  float boxWidth;
  float wallX;
  float3 pipePoint1;
  float3 pipePoint2;
  float pipeRadius;
  float forceDistance;
  float maxBoundaryForce;
  float deltaT;
  float deltaTWCSPH;
  float spacing;
  float particleRenderingSize;
  unsigned int num_rigid_bodies;

  float4* d_pos_zindex[2];
  float4* d_vel[2];
  int* d_type[2];
  int* d_active_type[2];

  float param_density_error_factor;
  float param_max_density_error_allowed;
  uint param_num_threads_custom_reduction;
  uint param_num_blocks_custom_reduction;
  int param_min_loops;
  int param_max_loops;

  uint* particlesKVPair_d[2];
  uint m_posVbo[2];

  upf_compat_context* upf;
};

extern "C" {

/* ---- this layer's own calls (no counterpart in the reference) ------------ */
/* The GPU the legacy calls use (default 0); before MallocDeviceArraysParticles. */
void upf_compat_set_device(int device);
/* Sticky status of the simulation (UPF_OK while nothing failed), and the
 * message of its first failure ("" if none). Also valid on a dataPointers
 * whose MallocDeviceArraysParticles failed; process-wide failures (a
 * Set* call before any simulation) are reported for every simulation. */
upf_status upf_compat_status(const dataPointers& dptr);
const char* upf_compat_message(const dataPointers& dptr);
/* The upf_params the simulation runs with (after its first step call). */
upf_status upf_compat_params(const dataPointers& dptr, upf_params* out);
/* The simulation's library handle (null before the first step call), for
 * calls of upf.h on the same simulation. */
upf_system* upf_compat_system(const dataPointers& dptr);
/* Particle upload used by CopyParticleDataHostToDevice
 * (compat/upf_compat_particles.cpp): n particles, pos4/vel4 n x 4 floats
 * (w ignored), reference type codes, parent rigid body index (-1: none). */
void upf_compat_upload(dataPointers& dptr, const float* pos4, const float* vel4, const int* type,
                       const int* parent_body, uint n);

/* ---- init (particles.cuh:432-440) ---------------------------------------- */
void MallocDeviceArraysParticles(dataPointers& dptr);
void MallocDeviceArraysRigidBody(dataPointers& dptr, std::vector<RigidBody*>& rigidbodies_h);
void SetDeviceConstants(dataPointers& dptr);
void FreeDeviceArrays(dataPointers& dptr);
void CopyIndicesDeviceToHost(dataPointers& dptr, uint*& indices);
void CopyZIndicesKVPairHostToDevice(dataPointers& dptr, std::vector<UnifiedParticle>& particles_h);
void CopyParticleDataHostToDevice(dataPointers& dptr, std::vector<UnifiedParticle>& particles_h);
void CopyRigidBodyDataHostToDevice(const std::vector<RigidBody*>& rigidbodies_h, dataPointers& dptr);
void CopyParticlesDeviceToHost(dataPointers& dptr, std::vector<UnifiedParticle>& particles_h, float*& p);

/* ---- tables (particles.cuh:450-455) -------------------------------------- */
void CreateZIndexTexture(unsigned int* A);
void CreateLutKernelM4Texture(float* A, const int lutSize);
void CreateLutKernelPressureGradientTexture(float* A, const int lutSize);
void CreateLutKernelViscosityLapTexture(float* A, const int lutSize);
void CreateLutSplineSurfaceTensionTexture(float* A, const int lutSize);
void CreateLutSplineSurfaceAdhesionTexture(float* A, const int lutSize);

/* ---- device constants (particles.cuh:459-503) ---------------------------- */
void SetParticleCount(const unsigned int& count);
void SetRigidBodyCount(const unsigned int& num_rigids);
void SetGlobalSupportRadius(const float& rad);
void SetDistToCenterMassCutoffApproximate(const float& cutoff);
void SetVelCutoffApproximate(const float& cutoff);
void SetParticleRadius(const float& radius);
void SetTerminalSpeed(const float& terminal);
void SetRigidBodyCoefficients(const float& spring, const float& spring_boundary, const float& damp);
void SetSurfaceTensionAdhesionCoefficients(const float& surface_tension_gamma, const float& surface_adhesion_beta);
void SetGridResolution(const unsigned int& grid_resolution);
void SetBlockSize(const unsigned int& block_Size);
void SetLutSize(const unsigned int& lut_size);
void SetKernelSelf(const float& kernelSelf);
void SetInitialMass(const float& initialMass);
void SetFluidRestDensity(const float& fluidRestDensity);
void SetFluidRestVolume(const float& initialMass, const float& fluidRestDensity);
void SetZindexStartingVec(const float3& zindexStartingVec_);
void SetGamma(const float& gamme);
void SetFluidGasConstant(const float& fluidGasConstant, const float& fluidGasConstantWCSPH);
void SetDensityErrorFactorPCISPH(const float& denErrorFactor_);
void SetBoundaryConstants(const float& forceDistance, const float& maxBoundaryForce, const float3& minB,
                          const float3& maxB, bool& add_boundary_force_);
void SetBoundingBox(const float3& minB, const float3& maxB);
void SetRealContainerValues(const float& length, const float& height, const float& width, const float3& minB,
                            const float3& maxB);
void SetDeltaT(const float& deltaT, const float& deltaTWCSPH);
void SetScales(const float3& scale);
void SetGravityConstant(const float& gravityConstant);
void SetInitialMassIntoGravityRatio(const float& initialMass, const float& gravityConstant);
void SetFluidViscosityConstant(const float& fluidViscosityConstant);
void SetFluidViscosityConstantTube(float& fluidViscosityConstant_tube);
void SetSpacing(const float& spacing);
void SetParticleRenderingSize(const float& pradius);
void SetOtherConstants();
void CreateLutKernelM4(float* A, const int& lutSize);
void CreateLutKernelPressureGradient(float* A, const int& lutSize);
void CreateLutKernelViscosityLap(float* A, const int& lutSize);
void CreateLutSplineSurfaceTension(float* A, const int& lutSize);
void CreateLutSplineSurfaceAdhesion(float* A, const int& lutSize);
void SetPipePoints(const float3& p1, const float3& p2);
void SetPipeRadius(float& pipeRadius);
void SetWallConstant(const float& wallX_);
void SetGridDimensions(uint& dimX_, uint& dimY_, uint& dimZ_);
void SetMaximumArrayLength(uint& arrL_);

/* ---- readback (particles.cuh:505) ---------------------------------------- */
/* Every particle in upload order (see above); arrays of particleCountRounded
 * entries, the tail filled as the reference pads (pos 4 x maxCollisionBox,
 * w = UINT_MAX, type and activeType 100). Returns particleCount. */
uint CopyParticlesCUDA(float* pos_zindex, float* vel, float* corr_pressure, float* predicted_density,
                       int* particleType, int* activeType, dataPointers& dptr);

/* ---- GL interop (particles.cuh:508-511): headless ------------------------ */
void RegisterGLBufferObject(uint vbo, struct cudaGraphicsResource** cuda_vbo_resource);
void UnregisterGLBufferObject(struct cudaGraphicsResource* cuda_vbo_resource);
void* MapGLBufferObject(struct cudaGraphicsResource** cuda_vbo_resource);
void UnmapGLBufferObject(struct cudaGraphicsResource* cuda_vbo_resource);

/* ---- SPH / WCSPH (particles.cuh:513-534) --------------------------------- */
void ZindexSorting(int currIndex, int currType, dataPointers& dptr);
void BlockGeneration(dataPointers& dptr, int& x, int& y);
void DensityPressureComputation(int currIndex, dataPointers& dptr, int& y);
void ForceComputation(int currIndex, dataPointers& dptr, int& y);
void CalculateZindex(int currIndex, dataPointers& dptr);
void UnbindTexturesSPH();
void UnbindTexturesPCISPH();
void UnbindTextureRigidFluidSPH();
void UnbindTextureRigidFluidPCISPH();
void PingPongScheme(dataPointers& dptr);
void PingPongSchemeRigidBody(dataPointers& dptr);
void ParticlePhysicsOnDeviceSPH(dataPointers& dptr);
void ZindexSortingApproximate(int currIndex, int currActiveType, dataPointers& dptr);
void DensityPressureComputationApproximate(int currIndex, dataPointers& dptr, int& y);
void ForceComputationApproximate(int currIndex, dataPointers& dptr, int& y);
void ExtractSurface(dataPointers& dptr, int& x);
void ParticlePhysicsOnDeviceSPHApproximate(dataPointers& dptr);

/* ---- PCISPH (particles.cuh:537-546) -------------------------------------- */
void ParticlePhysicsOnDevicePCISPH(dataPointers& dptr);
void CalculateExternalForcesPcisphCUDA(int currIndex, dataPointers& dptr, int& y);
void PredictionCorrectionStepPcisphCUDA(dataPointers& dptr, int& y);
void TimeIntegrationPcisphCUDAPureFluid(int currIndex, dataPointers& dptr, int& y);
void GetMaxPredictedDensityCUDA(dataPointers& dptr, float& max_predicted_density);
void ParticlePhysicsOnDevicePCISPHIhmsen2010(dataPointers& dptr);

/* ---- static boundaries, rigid coupling (particles.cuh:553-585) ----------- */
void CalculateExternalForcesStaticBoundariesPcisphCUDA(int currIndex, dataPointers& dptr, int& y);
void TimeIntegrationStaticBoundariesPcisphCUDA(int currIndex, dataPointers& dptr, int& y);
void ZindexSortingStaticBoundariesPCISPH(int currIndex, int currType, dataPointers& dptr);
void ParticlePhysicsOnDeviceFluidStaticBoundariesPCISPH(dataPointers& dptr);
void ZindexSortingRigidBodySPH(int currIndex, dataPointers& dptr);
void ZindexSortingRigidBodyPCISPH(int currIndex, dataPointers& dptr);
void ParticlePhysicsOnDeviceFluidRigidCouplingSPH(dataPointers& dptr);
void RigidBodyIntegration(int currIndex, dataPointers& dptr);
void SynRigidParticlesDevice(int currIndex, dataPointers& dptr);
void ParticlePhysicsOnDeviceFluidRigidCouplingPCISPH(dataPointers& dptr);
void CalculateExternalForcesFluidRigidCouplingPcisphCUDA(int currIndex, dataPointers& dptr, int& y);
void RigidBodyIntegrationTwoWayCoupling(int currIndex, dataPointers& dptr);

/* ---- radix sort (radixsort.cuh:115-117) ---------------------------------- */
/* Stable LSD sort of `elements` device pairs in pData0 by the low `bits`
 * bits of the key (whole 8-bit digits, as the reference); pData1 is the
 * same-sized device scratch. The result is in pData0 for every bit count
 * (the reference leaves it in pData1 after an odd number of passes). */
void RadixSort(KeyValuePair* pData0, KeyValuePair* pData1, uint elements, uint bits);

}  /* extern "C" */

#endif /* UPF_COMPAT_H_ */
