// A stand-in for the reference's particle class (src/cpu/UnifiedParticle.h)
// for the compatibility test: the members CopyParticleDataHostToDevice
// reads, under the same names and with the same member access (the
// reference's vmml::Vector3f exposes x, y, z). Test infrastructure only.
#pragma once

struct TestVector3f {
  float x, y, z;
};

class UnifiedParticle {
 public:
  TestVector3f position_{0, 0, 0};
  TestVector3f velocity_{0, 0, 0};
  int type_ = 2;
  int parent_rigid_body_index_ = -1;
};

class RigidBody {};
