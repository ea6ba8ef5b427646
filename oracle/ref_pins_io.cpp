// ref_pins_io.cpp — TEST INFRASTRUCTURE ONLY.
//
// C wrappers around the reference's own particle file writers and readers
// (src/cpu/UnifiedIO.cpp, compiled where it lies with src/cpu/UnifiedParticle.cpp
// by oracle/Makefile into oracle/_ref/libupfref.so), so the library's text
// formats can be compared with the reference's output byte for byte.
//
// The reference writers open fixed relative paths ("K:/SimulationData/output/
// ..." with a per-function file counter); each wrapper changes into the
// caller's scratch directory, creates those folders, calls the writer, and
// returns the file name it wrote (relative to that directory).
#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "UnifiedIO.h"
#include "UnifiedParticle.h"

namespace {
struct Quiet {  // the writers print file names and counts to std::cout
  std::streambuf* old;
  std::ostringstream sink;
  Quiet() : old(std::cout.rdbuf(sink.rdbuf())) {}
  ~Quiet() { std::cout.rdbuf(old); }
};

// Runs fn inside dir with the reference's output folders present.
template <class F>
int in_dir(const char* dir, F&& fn) {
  char cwd[4096];
  if (!getcwd(cwd, sizeof cwd)) return -1;
  if (chdir(dir) != 0) return -1;
  for (const char* d : {"K:", "K:/SimulationData", "K:/SimulationData/output", "K:/SimulationData/output/FluidParticles",
                        "K:/SimulationData/output/RigidParticles"})
    mkdir(d, 0755);
  fn();
  return chdir(cwd) == 0 ? 0 : -1;
}

int g_liquid = 0, g_rigid = 0, g_positions = 0;  // mirror the writers' static counters

int name_out(char* out, int cap, const char* fmt, int counter) {
  return std::snprintf(out, (size_t)cap, fmt, counter) < cap ? 0 : -1;
}
}  // namespace

extern "C" {

// UnifiedIO::SaveLiquidParticleInfoFull (src/cpu/UnifiedIO.cpp:60-105)
int ref_io_save_liquid(const char* dir, float* pos4, int* type, int num_rounded, int num_liquid, char* out, int cap) {
  Quiet q;
  UnifiedIO io;
  if (in_dir(dir, [&] { io.SaveLiquidParticleInfoFull(pos4, type, num_rounded, num_liquid); }) != 0) return -1;
  return name_out(out, cap, "K:/SimulationData/output/FluidParticles/particles%04d.txt", g_liquid++);
}

// UnifiedIO::SaveRigidParticleInfoFull (src/cpu/UnifiedIO.cpp:107-152)
int ref_io_save_rigid(const char* dir, float* pos4, int* type, int num_rounded, int count, char* out, int cap) {
  Quiet q;
  UnifiedIO io;
  if (in_dir(dir, [&] { io.SaveRigidParticleInfoFull(pos4, type, num_rounded, count); }) != 0) return -1;
  return name_out(out, cap, "K:/SimulationData/output/RigidParticles/rigid1Particles%04d.txt", g_rigid++);
}

// UnifiedIO::SaveParticlePositions (src/cpu/UnifiedIO.cpp:14-58), on
// particles built with the reference's UnifiedParticle(x, y, z, ...) constructor
int ref_io_save_positions(const char* dir, const float* pos4, int n, char* out, int cap) {
  Quiet q;
  std::vector<UnifiedParticle> ps;
  ps.reserve((size_t)n);
  for (int i = 0; i < n; ++i) ps.emplace_back(pos4[4 * i], pos4[4 * i + 1], pos4[4 * i + 2], 1000.0, 1.0, 2);
  UnifiedIO io;
  if (in_dir(dir, [&] { io.SaveParticlePositions(ps); }) != 0) return -1;
  return name_out(out, cap, "K:/SimulationData/output/particles%04d.txt", g_positions++);
}

// UnifiedIO::ReadInFluidParticleNum (src/cpu/UnifiedIO.cpp:154-177); the
// file must exist (the reference exits the process otherwise)
int ref_io_read_num(const char* path) {
  Quiet q;
  UnifiedIO io;
  return io.ReadInFluidParticleNum(path);
}

// UnifiedIO::ReadInFluidParticlesPCISPH (src/cpu/UnifiedIO.cpp:179-220)
void ref_io_read_pcisph(const char* path, float* pos3, float* vel3, int* type, float* p, float* rho) {
  Quiet q;
  UnifiedIO io;
  io.ReadInFluidParticlesPCISPH(path, pos3, vel3, type, p, rho);
}

}  // extern "C"
