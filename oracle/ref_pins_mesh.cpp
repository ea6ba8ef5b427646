// ref_pins_mesh.cpp — TEST INFRASTRUCTURE ONLY.
//
// A C wrapper around the reference's own OBJ voxeliser
// (ObjectLoader::LoadParticles, src/cpu/ObjectLoader.cpp, with the OBJ parser
// src/cpu/ObjLoader.cpp and the face tests src/cpu/Polygon.cpp, compiled
// where they lie by oracle/Makefile into oracle/_ref/libupfref.so), so the
// library's device voxeliser can be compared with it particle for particle.
#include <iostream>
#include <sstream>
#include <vector>

#include "ObjLoader.h"
#include "UnifiedParticle.h"

namespace {
struct Quiet {  // the loader prints face and particle counts to std::cout
  std::streambuf* old;
  std::ostringstream sink;
  Quiet() : old(std::cout.rdbuf(sink.rdbuf())) {}
  ~Quiet() { std::cout.rdbuf(old); }
};
}  // namespace

extern "C" {

// ObjLoader::GetInstance().LoadParticles(path, sx, sy, sz, spacing, template):
// the particle positions in the order the reference makes them (3 floats
// each, at most cap particles stored); returns the particle count.
int ref_obj_particles(const char* path, float sx, float sy, float sz, float spacing, float* pos3, int cap) {
  Quiet q;
  UnifiedParticle templ(0.0f, 0.0f, 0.0f, 1000.0, 1.0, 0);
  std::vector<UnifiedParticle>* ps = ObjLoader::GetInstance().LoadParticles(path, sx, sy, sz, spacing, templ);
  const int n = (int)ps->size();
  for (int i = 0; i < n && i < cap; ++i)
    for (int a = 0; a < 3; ++a) pos3[3 * i + a] = (*ps)[i].position_[a];
  delete ps;
  return n;
}

}  // extern "C"
