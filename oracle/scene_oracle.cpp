// scene_oracle.cpp — TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the reference's scene generators in
// src/sceneConfigure/Scene.cpp, which does not compile here (it includes the
// GL application headers): Scene::createFluidObject (Scene.cpp:597-646) and
// Scene::createBoxBoundaryFrozenParticles / ...MultiLayers
// (Scene.cpp:890-1212), loop by loop, with the reference's float and double
// expressions. The device generators (upf_scene_fluid_block,
// upf_scene_box_boundary) are checked against these.
#include <cstdint>
#include <cstdlib>

extern "C" {

// createFluidObject: returns the particle count; writes at most cap
// positions (x, y, z, 0). drand48() is the macro rand() / RAND_MAX
// (src/sceneConfigure/global.h:12), integer division: 0 (it is 1 only when
// rand() returns RAND_MAX), so each coordinate is x + (0 - 0.5) * jitter +
// offset in double, stored as float.
int64_t orc_scene_fluid_block(const float box_min[3], const float box_max[3], float spacing, float jitter,
                              const float offset[3], float* pos4, int64_t cap) {
  float delta[3];
  int num[3];
  for (int a = 0; a < 3; ++a) {
    delta[a] = box_max[a] - box_min[a];
    num[a] = (int)(delta[a] / spacing);  // Vector3i(delta / Vector3f(spacing)): static_cast<int>
  }
  const int drand = 0;
  int64_t k = 0;
  for (int iy = 0; iy < num[1]; iy++) {
    float y = jitter + iy * spacing;
    for (int ix = 0; ix < num[0]; ix++) {
      float x = jitter + ix * spacing;
      for (int iz = 0; iz < num[2]; iz++) {
        float z = jitter + iz * spacing;
        if (k < cap) {
          pos4[4 * k] = (float)(x + (drand - 0.5) * jitter + offset[0]);
          pos4[4 * k + 1] = (float)(y + (drand - 0.5) * jitter + offset[1]);
          pos4[4 * k + 2] = (float)(z + (drand - 0.5) * jitter + offset[2]);
          pos4[4 * k + 3] = 0.0f;
        }
        ++k;
      }
    }
  }
  return k;
}

// createBoxBoundaryFrozenParticlesMultiLayers with `layers` layers (the
// reference's numLayers = 2; one layer is createBoxBoundaryFrozenParticles):
// positions and normals (x, y, z, 0) in the reference's order. Returns the
// count, or -1 where the reference aborts (a particle at or below the
// z-index origin in some coordinate).
int64_t orc_scene_box_boundary(const float container_min[3], const float container_max[3], const float zstart[3],
                               float spacing, float support_radius, float dist_frozen, int layers, float* pos4,
                               float* nrm4, int64_t cap) {
  const float distance = support_radius - dist_frozen;
  float delta[3];
  int num[3];
  for (int a = 0; a < 3; ++a) {
    const float mn = container_min[a] - dist_frozen, mx = container_max[a] + dist_frozen;
    delta[a] = mx - mn;
    num[a] = (int)(delta[a] / spacing);
  }
  int64_t k = 0;
  bool bad = false;
  auto add = [&](float px, float py, float pz, float nx, float ny, float nz) {
    if (!(px - zstart[0] > 0.0 && py - zstart[1] > 0.0 && pz - zstart[2] > 0.0)) bad = true;
    if (k < cap) {
      pos4[4 * k] = px, pos4[4 * k + 1] = py, pos4[4 * k + 2] = pz, pos4[4 * k + 3] = 0.0f;
      nrm4[4 * k] = nx, nrm4[4 * k + 1] = ny, nrm4[4 * k + 2] = nz, nrm4[4 * k + 3] = 0.0f;
    }
    ++k;
  };
  const float sx = zstart[0], sy = zstart[1], sz = zstart[2];
  for (int x = 0; x < num[0] + 2; ++x)  // ground & ceiling (xz planes)
    for (int z = 0; z < num[2] + 2; ++z)
      for (int y = 0; y < layers; ++y) {
        add(sx + distance + x * spacing, sy + distance - y * spacing, sz + distance + z * spacing, 0, 1, 0);
        add(sx + distance + x * spacing, sy + distance + delta[1] + y * spacing, sz + distance + z * spacing, 0, -1,
            0);
      }
  for (int x = 0; x < num[0] + 2; ++x)  // back & front (xy planes)
    for (int y = 1; y < num[1] + 1; ++y)
      for (int z = 0; z < layers; ++z) {
        add(sx + distance + x * spacing, sy + distance + y * spacing, sz + distance - z * spacing, 0, 0, 1);
        add(sx + distance + x * spacing, sy + distance + y * spacing, sz + distance + delta[2] + z * spacing, 0, 0,
            -1);
      }
  for (int y = 1; y < num[1] + 1; ++y)  // left & right (yz planes)
    for (int z = 1; z < num[2] + 1; ++z)
      for (int x = 0; x < layers; ++x) {
        add(sx + distance - x * spacing, sy + distance + y * spacing, sz + distance + z * spacing, 1, 0, 0);
        add(sx + distance + delta[0] + x * spacing, sy + distance + y * spacing, sz + distance + z * spacing, -1, 0,
            0);
      }
  return bad ? -1 : k;
}

}  // extern "C"
