// upf_compat_particles.cpp — the one entry point of include/upf_compat.h that
// reads the caller's particle class: compile this file in the caller's build,
// next to the reference's UnifiedParticle.h (src/cpu/UnifiedParticle.h), and
// link libupf_compat.so.
//
// CopyParticleDataHostToDevice (src/gpu/particles.cu:391-520) uploads each
// particle's position, velocity, type and parent rigid body index; the
// library derives everything else (keys, weighted volumes, lagged PCISPH
// state, rigid body mass and inertia) on the device.
#include <vector>

#include "UnifiedParticle.h"
#include "upf_compat.h"

void CopyParticleDataHostToDevice(dataPointers& dptr, std::vector<UnifiedParticle>& particles_h) {
  const size_t n = particles_h.size();
  std::vector<float> pos(4 * n), vel(4 * n);
  std::vector<int> type(n), body(n);
  for (size_t i = 0; i < n; ++i) {
    const UnifiedParticle& q = particles_h[i];
    pos[4 * i] = q.position_.x;
    pos[4 * i + 1] = q.position_.y;
    pos[4 * i + 2] = q.position_.z;
    pos[4 * i + 3] = 0.0f;
    vel[4 * i] = q.velocity_.x;
    vel[4 * i + 1] = q.velocity_.y;
    vel[4 * i + 2] = q.velocity_.z;
    vel[4 * i + 3] = 0.0f;
    type[i] = q.type_;
    body[i] = q.parent_rigid_body_index_;
  }
  upf_compat_upload(dptr, pos.data(), vel.data(), type.data(), body.data(), (uint)n);
}
