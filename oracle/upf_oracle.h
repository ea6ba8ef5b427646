/*
 * upf_oracle.h — TEST INFRASTRUCTURE. CPU restatement of the reference's CPU
 * particle path (src/cpu/UnifiedPhysics.cpp, zIndex.cpp, WeightingKernel.cpp,
 * RigidBody.cpp, UnifiedConstants.cpp). Used only by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg, as the checker.
 * Never linked into, or called by, the product library.
 *
 * Two twins: FP32 (operation-for-operation restatement, compiled with
 * -ffp-contract=off so every float op rounds like the reference) and FP64
 * (same algorithm in double, for error reporting).
 */
#ifndef UPF_ORACLE_H_
#define UPF_ORACLE_H_

#include <stdint.h>
#include "../include/upf.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sim orc_sim;

typedef struct orc_step_info {
  int32_t iterations;
  float max_predicted_density;
  float density_error_percent;
  uint32_t max_neighbor_count;
  double kinetic_energy;
  double momentum[3];
  float iteration_max_density[64];
} orc_step_info;

/* parameters (restatement of UnifiedConstants + derived values) */
void orc_default_params(upf_params* p);
int orc_params_derive(upf_params* p);              /* FP32 delta, reference order */
double orc_density_error_factor(const upf_params* p, int fp64);

/* tables */
void orc_build_luts(const upf_params* p, float* out_5x301);
uint32_t orc_morton(const upf_params* p, float x, float y, float z);
void orc_morton_table(uint32_t* out_1024x3);
/* BoxQuery ranges for a query box in grid coordinates (already converted to
 * unsigned short); returns number of ranges written (<= cap). */
int orc_box_query(uint32_t block_size, const uint16_t mn[3], const uint16_t mx[3],
                  uint32_t* first, uint32_t* last, int cap);

/* simulation (n particles, all types, input order = ids 0..n-1) */
orc_sim* orc_create(const upf_params* p, const float* pos4, const float* vel4,
                    const int32_t* type, uint32_t n, int fp64, int threads);
void orc_destroy(orc_sim* s);
int orc_set_rigid_bodies(orc_sim* s, const int32_t* body_of_particle, uint32_t n,
                         uint32_t num_bodies);
int orc_step(orc_sim* s, orc_step_info* info);
uint32_t orc_count(const orc_sim* s);
/* keep a copy of the step-start fields of every step (for orc_get_step_fields) */
void orc_keep_fields(orc_sim* s, int on);
/* The reference's own rule where the restatement deviates on purpose, one
 * bit per deviation (set before orc_set_rigid_bodies for the inertia bit):
 *   GRANULAR_TANGENTIAL_ONLY  grains add only F_t, friction bound mu * f_n
 *                             with the signed f_n (UnifiedPhysics.cpp:3276-3287)
 *   OWN_BODY_SPRING           the rigid spring-damper acts between particles
 *                             of the same body too (UnifiedPhysics.cpp:5300-5311)
 *   ZERO_INVERSE_INERTIA      the local inverse inertia stays zero, as the
 *                             reference's inverse lands in a temporary
 *                             (UnifiedPhysics.cpp:150)
 *   WCSPH_CLAMP_ALL           the WCSPH step clamps every particle to the
 *                             collision box, frozen ones included
 *                             (UnifiedPhysics.cpp:4296-4326)
 *   FLOAT_RIGID_ASSEMBLY      bodies assembled one particle at a time in
 *                             float, in array order (AddToRigidBody,
 *                             UnifiedPhysics.cpp:825-885), with the linear
 *                             momentum left at the constructor's zero
 *   FLOAT_BODY_SUMS           per-body force and torque summed in float in
 *                             array order, gravity after each particle's
 *                             force (UnifiedPhysics.cpp:3631-3643)
 *   STALE_RIGID_KEYS          rigid particles keep the key of their position
 *                             before the rigid sync (UnifiedPhysics.cpp:3995,
 *                             5011-5023)
 *   STALE_RIGID_PREDICTED     rigid particles keep the predicted position
 *                             they were created with (nothing in the coupling
 *                             step writes it; UnifiedParticle.cpp:17)
 * Set before orc_set_rigid_bodies for the inertia and assembly bits. */
#define ORC_LITERAL_GRANULAR_TANGENTIAL_ONLY 1u
#define ORC_LITERAL_OWN_BODY_SPRING 2u
#define ORC_LITERAL_ZERO_INVERSE_INERTIA 4u
#define ORC_LITERAL_WCSPH_CLAMP_ALL 8u
#define ORC_LITERAL_FLOAT_RIGID_ASSEMBLY 16u
#define ORC_LITERAL_FLOAT_BODY_SUMS 32u
#define ORC_LITERAL_STALE_RIGID_KEYS 64u
#define ORC_LITERAL_STALE_RIGID_PREDICTED 128u
void orc_set_reference_literal(orc_sim* s, uint32_t mask);
/* continue from another run's state, per particle in creation order: the
 * final correction pressure of the step before last and of the last step,
 * and the last step's predicted density */
void orc_set_lagged(orc_sim* s, const float* pressure_prev, const float* pressure, const float* density);
/* the same three arrays of the current state, per particle in creation order */
void orc_get_lagged(const orc_sim* s, float* pressure_prev, float* pressure, float* density);
/* current array order (sorted by key at the end of the last step) */
void orc_get(const orc_sim* s, float* pos4, float* vel4, float* density, float* pressure,
             int32_t* type, uint32_t* id, uint32_t* key);
/* fields of the last step in that step's start order: external force,
 * correction pressure force, predicted density, correction pressure,
 * WCSPH density/pressure */
void orc_get_step_fields(const orc_sim* s, float* force4, float* pforce4,
                         float* predicted_density, float* corr_pressure, float* density,
                         float* pressure, uint32_t* id);
/* neighbour lists of the current order, as ids, CSR (offsets n+1) */
uint32_t orc_neighbors(orc_sim* s, uint32_t* offsets, uint32_t* ids, uint32_t cap);
/* rigid body state: per body pos[3], vel[3], omega[3], quat[4] */
int orc_get_rigid(const orc_sim* s, float* pos3, float* vel3, float* omega3, float* quat4);
/* one FP32 body update (momenta, inverse world inertia, linear and angular
 * step, rotation matrix) in place on ORC_BODY_FLOATS floats: mass, pos[3],
 * vel[3], P[3], L[3], omega[3], q[4] (s,x,y,z), rot[9], inv_inertia_local[9],
 * inv_inertia_world[9] (row-major) */
#define ORC_BODY_FLOATS 47
/* FP64 adjugate inverse of a row-major 3x3 (rounded to float); 0 if singular */
int orc_inverse3(const float* in9, float* out9);
void orc_rigid_body_step(float* state, const float* force3, const float* torque3, float dt,
                         float terminal_speed);

#ifdef __cplusplus
}
#endif
#endif
