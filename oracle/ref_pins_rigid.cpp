// ref_pins_rigid.cpp — TEST INFRASTRUCTURE ONLY.
//
// C wrappers over the reference's own RigidBody (src/cpu/RigidBody.cpp) and
// Matrix3x3 (src/cpu/Matrix3x3.cpp), compiled where they lie into
// oracle/_ref/libupfref.so by oracle/Makefile, so that the oracle's body
// update and 3x3 inverse can be pinned to the reference itself.
//
// RigidBody keeps its local inverse inertia private with no setter (the
// reference's only assignment goes to a temporary, UnifiedPhysics.cpp:150);
// the wrapper opens the class's private members to set it. The standard and
// vector headers are included first so that only the reference's class
// definitions see the redefinition.
#include <cmath>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "vmmlib/vector3.h"
#include "vmmlib/vector4.h"
#define private public
#include "RigidBody.h"
#undef private

extern "C" {

// RigidBody::UpdateMomenta + PerformStep + UpdateRotationMatrix
// (RigidBody.cpp:96-161), the sequence of
// CalculateRigidBodyForceTorqueMomenta's quaternion method
// (UnifiedPhysics.cpp:3682-3696), with the step's force and torque given.
// state (47 floats, in place): mass, pos[3], vel[3], P[3], L[3], omega[3],
// q[4] (s,x,y,z), rot[9], inv_inertia_local[9], inv_inertia_world[9].
void ref_rigid_body_step(float* st, const float* force3, const float* torque3, float dt, float terminal_speed) {
  RigidBody b;
  const float* q = st;
  auto v3 = [&]() {
    vmml::Vector3f v(q[0], q[1], q[2]);
    q += 3;
    return v;
  };
  auto m3 = [&](Matrix3x3& m) {
    for (int i = 0; i < 9; ++i) m.elements[i / 3][i % 3] = q[i];
    q += 9;
  };
  b.mass_ = *q++;
  b.rigidbody_pos_ = v3();
  b.velocity_ = v3();
  b.linear_momentum_ = v3();
  b.angular_momentum_ = v3();
  b.angular_velocity_ = v3();
  b.quaternion_ = vmml::Vector4f(q[0], q[1], q[2], q[3]);
  q += 4;
  m3(b.rotation_matrix_);
  m3(b.inverted_inertia_local_);
  m3(b.inverted_inertia_world_);
  b.force_ = vmml::Vector3f(force3[0], force3[1], force3[2]);
  b.torque_ = vmml::Vector3f(torque3[0], torque3[1], torque3[2]);
  const float terminal = b.mass_ * terminal_speed;
  b.UpdateMomenta(dt, terminal);
  b.PerformStep(dt);
  b.UpdateRotationMatrix();
  float* o = st;
  auto w3 = [&](const vmml::Vector3f& v) {
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
    o += 3;
  };
  auto n3 = [&](const Matrix3x3& m) {
    for (int i = 0; i < 9; ++i) o[i] = m.elements[i / 3][i % 3];
    o += 9;
  };
  *o++ = b.mass_;
  w3(b.rigidbody_pos_);
  w3(b.velocity_);
  w3(b.linear_momentum_);
  w3(b.angular_momentum_);
  w3(b.angular_velocity_);
  for (int k = 0; k < 4; ++k) *o++ = b.quaternion_[k];
  n3(b.rotation_matrix_);
  n3(b.inverted_inertia_local_);
  n3(b.inverted_inertia_world_);
}

// Matrix3x3::CalculateInverse (Matrix3x3.cpp:121-156); returns its success flag
int ref_inverse3(const float* in9, float* out9) {
  Matrix3x3 a, r;
  for (int i = 0; i < 9; ++i) {
    a.elements[i / 3][i % 3] = in9[i];
    r.elements[i / 3][i % 3] = 0.0f;
  }
  const bool ok = Matrix3x3::CalculateInverse(a, r);
  for (int i = 0; i < 9; ++i) out9[i] = r.elements[i / 3][i % 3];
  return ok ? 1 : 0;
}

}  // extern "C"
