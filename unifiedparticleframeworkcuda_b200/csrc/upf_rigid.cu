// upf_rigid.cu — rigid bodies: per-body force/torque reduction, body
// integration and particle sync.
//
// The reference integrates each body on one thread that loops serially over
// up to 15,000 particles in FP32 (RigidBodyIntegrationTwoWayCouplingKernel,
// particles_kernel.cu:8321-8381; CalculateForceTorque*_d, particles_kernel.cuh:972-1012),
// after a pass that rewrites every body's particle index list once the
// particles are re-sorted (UpdateRigidParticleIndicesKernel,
// particles_kernel.cu:7692-7703). Here the body-grouped rigid list maps to the
// particles' current sorted positions (k_rigid_slots), one CTA per body reduces
// force and torque in FP64 in a fixed order (deterministic), one thread per
// body integrates in float exactly as RigidBody.cpp does, and the sync pass
// places the rigid particles and re-keys them for the next sort.
#include <cuda_runtime.h>

#include "upf_sys.h"

namespace upf {

namespace {

constexpr int kReduceThreads = 256;

// list entry -> sorted index, after each sort
__global__ void k_rigid_slots(uint32_t n, const uint32_t* __restrict__ id, const uint32_t* __restrict__ id_entry,
                              uint32_t* __restrict__ slot) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t r = id_entry[id[i]];
  if (r != 0xffffffffu) slot[r] = i;
}

// CalculateRigidBodyForceTorqueMomenta step 1 (UnifiedPhysics.cpp:3627-3643):
// F = sum(f_p + m g), tau = sum((x_p - x_cm) x f_p), in FP64.
__global__ void __launch_bounds__(kReduceThreads) k_rigid_reduce(DevParams P, DevBody* __restrict__ bodies,
                                                                 const uint32_t* __restrict__ body_start,
                                                                 const uint32_t* __restrict__ slot,
                                                                 const float4* __restrict__ pos,
                                                                 const float4* __restrict__ force) {
  __shared__ double red[6][kReduceThreads];
  const int b = blockIdx.x;
  const float3 c = bodies[b].pos;
  const double g = (double)(-P.mass * P.gravity);
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (uint32_t k = body_start[b] + threadIdx.x; k < body_start[b + 1]; k += kReduceThreads) {
    const uint32_t i = slot[k];
    const float4 f = force[i], x = pos[i];
    const double fx = f.x, fy = f.y, fz = f.z;
    const double rx = (double)x.x - (double)c.x, ry = (double)x.y - (double)c.y, rz = (double)x.z - (double)c.z;
    acc[0] += fx;
    acc[1] += fy + g;
    acc[2] += fz;
    acc[3] += ry * fz - rz * fy;
    acc[4] += rz * fx - rx * fz;
    acc[5] += rx * fy - ry * fx;
  }
  for (int a = 0; a < 6; ++a) red[a][threadIdx.x] = acc[a];
  __syncthreads();
  for (int w = kReduceThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int a = 0; a < 6; ++a) red[a][threadIdx.x] += red[a][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int a = 0; a < 3; ++a) {
      bodies[b].force[a] = red[a][0];
      bodies[b].torque[a] = red[3 + a][0];
    }
  }
}

// AddToRigidBody (UnifiedPhysics.cpp:825-885) and
// ComputeLocalInertiaTensorRigidBody (:1143-1176), one CTA per body: mass,
// centre of mass and momentum, then the inertia tensor and angular momentum
// about the centre, each an FP64 tree sum over the body's particles (entries
// in the body's input order); the FP64 adjugate inverse of the inertia
// (Matrix3x3::CalculateInverse, Matrix3x3.cpp:121-156); the body at rest
// orientation; and every particle's position relative to the centre, in
// float as the reference stores it.
__device__ __forceinline__ void tree_sum(double (*red)[kReduceThreads], int nvals) {
  __syncthreads();
  for (int w = kReduceThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int a = 0; a < nvals; ++a) red[a][threadIdx.x] += red[a][threadIdx.x + w];
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kReduceThreads) k_rigid_assemble(float mass, DevBody* __restrict__ bodies,
                                                                   const uint32_t* __restrict__ body_start,
                                                                   const float4* __restrict__ epos,
                                                                   const float4* __restrict__ evel,
                                                                   float4* __restrict__ entry_r0) {
  __shared__ double red[9][kReduceThreads];
  __shared__ double centre[3];
  const int b = blockIdx.x;
  const uint32_t k0 = body_start[b], k1 = body_start[b + 1];
  const double m = mass;
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (uint32_t k = k0 + threadIdx.x; k < k1; k += kReduceThreads) {
    const float4 x = epos[k], v = evel[k];
    acc[0] += m * (double)x.x;
    acc[1] += m * (double)x.y;
    acc[2] += m * (double)x.z;
    acc[3] += m * (double)v.x;
    acc[4] += m * (double)v.y;
    acc[5] += m * (double)v.z;
  }
  for (int a = 0; a < 6; ++a) red[a][threadIdx.x] = acc[a];
  tree_sum(red, 6);
  const double M = m * (double)(k1 - k0);
  double P[3];
  for (int a = 0; a < 3; ++a) P[a] = red[3 + a][0];
  if (threadIdx.x < 3) centre[threadIdx.x] = red[threadIdx.x][0] / M;
  __syncthreads();
  const double c[3] = {centre[0], centre[1], centre[2]};
  for (int a = 0; a < 9; ++a) acc[a] = 0.0;
  for (uint32_t k = k0 + threadIdx.x; k < k1; k += kReduceThreads) {
    const float4 x = epos[k], v4 = evel[k];
    const double r[3] = {(double)x.x - c[0], (double)x.y - c[1], (double)x.z - c[2]};
    const double v[3] = {m * (double)v4.x, m * (double)v4.y, m * (double)v4.z};
    const double rr = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    acc[0] += m * (rr - r[0] * r[0]);  // xx
    acc[1] += m * (-r[0] * r[1]);      // xy
    acc[2] += m * (-r[0] * r[2]);      // xz
    acc[3] += m * (rr - r[1] * r[1]);  // yy
    acc[4] += m * (-r[1] * r[2]);      // yz
    acc[5] += m * (rr - r[2] * r[2]);  // zz
    acc[6] += r[1] * v[2] - r[2] * v[1];
    acc[7] += r[2] * v[0] - r[0] * v[2];
    acc[8] += r[0] * v[1] - r[1] * v[0];
  }
  for (int a = 0; a < 9; ++a) red[a][threadIdx.x] = acc[a];
  tree_sum(red, 9);
  const float3 cf = make_float3((float)c[0], (float)c[1], (float)c[2]);
  if (threadIdx.x == 0) {
    const double A[9] = {red[0][0], red[1][0], red[2][0], red[1][0], red[3][0], red[4][0],
                         red[2][0], red[4][0], red[5][0]};
    double inv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const double det = A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
                       A[2] * (A[3] * A[7] - A[4] * A[6]);
    if (det != 0.0) {
      inv[0] = (A[4] * A[8] - A[5] * A[7]) / det;
      inv[1] = (A[2] * A[7] - A[1] * A[8]) / det;
      inv[2] = (A[1] * A[5] - A[2] * A[4]) / det;
      inv[3] = (A[5] * A[6] - A[3] * A[8]) / det;
      inv[4] = (A[0] * A[8] - A[2] * A[6]) / det;
      inv[5] = (A[2] * A[3] - A[0] * A[5]) / det;
      inv[6] = (A[3] * A[7] - A[4] * A[6]) / det;
      inv[7] = (A[1] * A[6] - A[0] * A[7]) / det;
      inv[8] = (A[0] * A[4] - A[1] * A[3]) / det;
    }
    DevBody B;
    memset(&B, 0, sizeof(B));
    B.mass = (float)M;
    B.pos = cf;
    B.P = make_float3((float)P[0], (float)P[1], (float)P[2]);
    B.vel = make_float3((float)(P[0] / M), (float)(P[1] / M), (float)(P[2] / M));
    B.L = make_float3((float)red[6][0], (float)red[7][0], (float)red[8][0]);
    B.q[0] = 1.0f;
    for (int i = 0; i < 3; ++i) {
      B.rot[i][i] = 1.0f;
      for (int j = 0; j < 3; ++j) B.iinv_local[i][j] = (float)inv[3 * i + j];
    }
    bodies[b] = B;
  }
  for (uint32_t k = k0 + threadIdx.x; k < k1; k += kReduceThreads) {
    const float4 x = epos[k];
    entry_r0[k] = make_float4(x.x - cf.x, x.y - cf.y, x.z - cf.z, 0.0f);
  }
}

// the reference's MIN / MAX macros (global.h:4-5)
__device__ __forceinline__ float min_ref(float a, float b) { return (a <= b) ? a : b; }
__device__ __forceinline__ float max_ref(float a, float b) { return (a >= b) ? a : b; }

__device__ __forceinline__ void mat_mul(const float a[3][3], const float b[3][3], float out[3][3]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      float s = 0.0f;
      for (int k = 0; k < 3; ++k) s += a[i][k] * b[k][j];
      out[i][j] = s;
    }
}

__device__ __forceinline__ float3 mat_vec(const float a[3][3], float3 v) {
  const float x[3] = {v.x, v.y, v.z};
  float r[3];
  for (int i = 0; i < 3; ++i) {
    r[i] = 0.0f;
    for (int j = 0; j < 3; ++j) r[i] += a[i][j] * x[j];
  }
  return make_float3(r[0], r[1], r[2]);
}

// UpdateMomenta, PerformStep and UpdateRotationMatrix (RigidBody.cpp:15-161),
// float as in the reference. The reference's cos/sin calls take the float
// half-angle promoted to double, and `axis * sin(...)` multiplies in double
// before rounding to float; the same here.
__global__ void k_rigid_integrate(DevParams P, DevBody* __restrict__ bodies, uint32_t nb) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  DevBody B = bodies[b];
  const float dt = P.dt;
  const float3 F = make_float3((float)B.force[0], (float)B.force[1], (float)B.force[2]);
  const float3 T = make_float3((float)B.torque[0], (float)B.torque[1], (float)B.torque[2]);
  const float terminal = B.mass * P.terminal_speed;
  B.P.x = B.P.x + F.x * dt;
  B.P.y = B.P.y + F.y * dt;
  B.P.z = B.P.z + F.z * dt;
  float* Pv = &B.P.x;
  for (int a = 0; a < 3; ++a) Pv[a] = (Pv[a] > 0.0f) ? min_ref(Pv[a], terminal) : max_ref(Pv[a], -terminal);
  B.L.x = B.L.x + T.x * dt;
  B.L.y = B.L.y + T.y * dt;
  B.L.z = B.L.z + T.z * dt;
  float rt[3][3], tmp[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) rt[j][i] = B.rot[i][j];
  mat_mul(B.rot, B.iinv_local, tmp);
  mat_mul(tmp, rt, B.iinv_world);
  const float inv = 1.0f / B.mass;  // vmml vector / scalar
  B.vel = make_float3(B.P.x * inv, B.P.y * inv, B.P.z * inv);
  B.pos = make_float3(B.pos.x + B.vel.x * dt, B.pos.y + B.vel.y * dt, B.pos.z + B.vel.z * dt);
  B.omega = mat_vec(B.iinv_world, B.L);
  const float speed = sqrtf(B.omega.x * B.omega.x + B.omega.y * B.omega.y + B.omega.z * B.omega.z);
  if (speed > 0.0f) {
    const float ll = (float)(1.0 / (double)speed);
    const float ax = B.omega.x * ll, ay = B.omega.y * ll, az = B.omega.z * ll;
    const float angle = speed * dt;
    const double half = (double)(angle / 2.0f);
    const float ds = (float)cos(half);
    const double sn = sin(half);
    const float dvx = (float)((double)ax * sn), dvy = (float)((double)ay * sn), dvz = (float)((double)az * sn);
    const float s = B.q[0], vx = B.q[1], vy = B.q[2], vz = B.q[3];
    B.q[0] = s * ds - vx * dvx - vy * dvy - vz * dvz;
    B.q[1] = ds * vx + s * dvx + dvy * vz - dvz * vy;
    B.q[2] = ds * vy + s * dvy + dvz * vx - dvx * vz;
    B.q[3] = ds * vz + s * dvz + dvx * vy - dvy * vx;
  }
  const float w = B.q[0], x = B.q[1], y = B.q[2], z = B.q[3];
  const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z, wx = w * x, wy = w * y,
              wz = w * z;
  B.rot[0][0] = 1.0f - 2.0f * (yy + zz);
  B.rot[0][1] = 2.0f * (xy - wz);
  B.rot[0][2] = 2.0f * (xz + wy);
  B.rot[1][0] = 2.0f * (xy + wz);
  B.rot[1][1] = 1.0f - 2.0f * (xx + zz);
  B.rot[1][2] = 2.0f * (yz - wx);
  B.rot[2][0] = 2.0f * (xz - wy);
  B.rot[2][1] = 2.0f * (yz + wx);
  B.rot[2][2] = 1.0f - 2.0f * (xx + yy);
  bodies[b] = B;
}

// SynRigidParticlesPerRigidBody (UnifiedPhysics.cpp:3766-3782): x = x_cm + R r0,
// v = v_cm + omega x (R r0); the particle's key is taken at its new position.
__global__ void k_rigid_sync(DevParams P, uint32_t n_rigid, const uint32_t* __restrict__ slot,
                             const int32_t* __restrict__ entry_body, const float4* __restrict__ entry_r0,
                             const DevBody* __restrict__ bodies, DynArrays A, uint32_t* __restrict__ keysA) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_rigid) return;
  const uint32_t i = slot[k];
  const DevBody& b = bodies[entry_body[k]];
  const float4 r0 = entry_r0[k];
  const float3 rel = mat_vec(b.rot, make_float3(r0.x, r0.y, r0.z));
  const float3 w = b.omega;
  const float3 c = make_float3(w.y * rel.z - w.z * rel.y, w.z * rel.x - w.x * rel.z, w.x * rel.y - w.y * rel.x);
  const float4 v = make_float4(b.vel.x + c.x, b.vel.y + c.y, b.vel.z + c.z, 0.0f);
  const float4 x = make_float4(b.pos.x + rel.x, b.pos.y + rel.y, b.pos.z + rel.z, 0.0f);
  A.pos[i] = x;
  A.vel[i] = v;
  keysA[i] = morton_key(x, P.origin, P.scales);
}

}  // namespace

cudaError_t launch_rigid_slots(System& s, cudaStream_t st) {
  const RigidArrays& r = s.rb;
  if (!r.n_rigid || !s.n_dyn) return cudaSuccess;
  k_rigid_slots<<<(s.n_dyn + 255) / 256, 256, 0, st>>>(s.n_dyn, s.B.id, r.id_entry, r.entry_slot);
  return cudaGetLastError();
}

cudaError_t launch_rigid_assemble(float mass, DevBody* bodies, uint32_t n_bodies, const uint32_t* start,
                                  const float4* epos, const float4* evel, float4* entry_r0, cudaStream_t st) {
  if (!n_bodies) return cudaSuccess;
  k_rigid_assemble<<<n_bodies, kReduceThreads, 0, st>>>(mass, bodies, start, epos, evel, entry_r0);
  return cudaGetLastError();
}

cudaError_t launch_rigid_phase(System& s, cudaStream_t st) {
  const RigidArrays& r = s.rb;
  if (!r.n_bodies) return cudaSuccess;
  k_rigid_reduce<<<r.n_bodies, kReduceThreads, 0, st>>>(s.dp, r.bodies, r.start, r.entry_slot, s.B.pos, s.force);
  k_rigid_integrate<<<(r.n_bodies + 31) / 32, 32, 0, st>>>(s.dp, r.bodies, r.n_bodies);
  if (r.n_rigid)
    k_rigid_sync<<<(r.n_rigid + 255) / 256, 256, 0, st>>>(s.dp, r.n_rigid, r.entry_slot, r.entry_body, r.entry_r0,
                                                          r.bodies, s.A, s.keysA);
  return cudaGetLastError();
}

int rigid_launches_per_step(const System& s) {
  if (!s.rb.n_bodies) return 0;
  return 2 + (s.rb.n_rigid ? 1 : 0);  // reduce, integrate, sync (the slot pass runs with the sort)
}

}  // namespace upf
