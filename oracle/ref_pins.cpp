// ref_pins.cpp — TEST INFRASTRUCTURE ONLY.
//
// A thin C wrapper, compiled together with the reference's own CPU sources
// (src/cpu/zIndex.cpp, src/cpu/WeightingKernel.cpp,
// src/sceneConfigure/UnifiedConstants.cpp, built where they lie by
// oracle/Makefile into oracle/_ref/libupfref.so), that exposes the tables and
// constants the reference computes, so the oracle restatement and the golden
// fixtures can be pinned to the reference itself.
#include <cstring>
#include <iostream>
#include <sstream>

#include "UnifiedConstants.h"
#include "WeightingKernel.h"
#include "zIndex.h"

namespace {
// The reference constructors print to std::cout; keep test output clean.
struct Quiet {
  std::streambuf* old;
  std::ostringstream sink;
  Quiet() : old(std::cout.rdbuf(sink.rdbuf())) {}
  ~Quiet() { std::cout.rdbuf(old); }
};
}  // namespace

extern "C" {

// ZIndex::ZIndex table, z_table_[1024][3] (src/cpu/zIndex.cpp:10-24)
void ref_morton_table(unsigned int* out) {
  ZIndex z;
  std::memcpy(out, z.z_table(), sizeof(unsigned int) * 1024 * 3);
}

// ZIndex::BoxQuery (src/cpu/zIndex.cpp:43-73) for a grid-coordinate box
int ref_box_query(unsigned int block_size, const unsigned short mn[3], const unsigned short mx[3],
                  unsigned int* first, unsigned int* last, int cap) {
  Quiet q;
  ZIndex z;
  z.SetBlockSize((int)block_size);
  ZRanges r;
  z.BoxQuery(Vector3ui(mn[0], mn[1], mn[2]), Vector3ui(mx[0], mx[1], mx[2]), r);
  int n = (int)r.size();
  for (int i = 0; i < n && i < cap; ++i) {
    first[i] = r[i].first;
    last[i] = r[i].second;
  }
  return n;
}

// ZIndex::SetBlockSize rounding (src/cpu/zIndex.cpp:27-39)
unsigned int ref_block_size(int size) {
  Quiet q;
  ZIndex z;
  z.SetBlockSize(size);
  return z.block_size();
}

// WeightingKernel::initLookupTables (src/cpu/WeightingKernel.cpp:303-320) for
// support radius h: out[5][301] = m4, pressure grad, visc lap, surface
// tension, adhesion.
void ref_luts(float h, float* out) {
  Quiet q;
  UnifiedConstants fc;
  fc.globalSupportRadius = h;
  WeightingKernel k(&fc);
  std::memcpy(out + 0 * 301, k.lut_kernel_m4(), sizeof(float) * 301);
  std::memcpy(out + 1 * 301, k.lut_kernel_pressure_grad(), sizeof(float) * 301);
  std::memcpy(out + 2 * 301, k.lut_kernel_viscosity_lap(), sizeof(float) * 301);
  std::memcpy(out + 3 * 301, k.lut_spline_surface_tension(), sizeof(float) * 301);
  std::memcpy(out + 4 * 301, k.lut_spline_surface_adhesion(), sizeof(float) * 301);
}

// Analytic kernels at a distance (src/cpu/WeightingKernel.cpp:75-263)
void ref_kernels(float dist, float h, float* out5) {
  Quiet q;
  UnifiedConstants fc;
  fc.globalSupportRadius = h;
  WeightingKernel k(&fc);
  out5[0] = k.KernelM4(dist, h);
  out5[1] = k.kernelPressureGrad(dist, h);
  out5[2] = k.kernelViscosityLaplacian(dist, h);
  out5[3] = k.kernelSplineSurfaceTension(dist, h);
  out5[4] = k.kernelSplineSurfaceAdhesion(dist, h);
}

// LUT lookups with the reference's function-static factor
// (WeightingKernel::kernelM4Lut etc., src/cpu/WeightingKernel.cpp:122-128).
// The factor is initialised on the first call in the process, so every
// lookup here uses the support radius of the first call.
void ref_lut_lookup(float h, const float* dists, int n, float* out3) {
  Quiet q;
  UnifiedConstants fc;
  fc.globalSupportRadius = h;
  WeightingKernel k(&fc);
  for (int i = 0; i < n; ++i) {
    out3[3 * i + 0] = k.kernelM4Lut(dists[i]);
    out3[3 * i + 1] = k.kernelPressureGradLut(dists[i]);
    out3[3 * i + 2] = k.kernelViscosityLaplacianLut(dists[i]);
  }
}

// Constants after UnifiedConstants::UnifiedConstants
// (src/sceneConfigure/UnifiedConstants.cpp:7-159).
void ref_default_constants(float* out) {
  Quiet q;
  UnifiedConstants fc;
  int i = 0;
  out[i++] = fc.particleSpacing;
  out[i++] = fc.particleRadius;
  out[i++] = fc.globalSupportRadius;
  out[i++] = fc.initialMass;
  out[i++] = fc.fluidRestDensity;
  out[i++] = fc.fluidGasConstantWCSPH;
  out[i++] = fc.gamma;
  out[i++] = fc.fluidViscConst;
  out[i++] = fc.gravityConst;
  out[i++] = fc.deltaT_pcisph;
  out[i++] = fc.densityErrorFactorParameter;
  out[i++] = fc.maxDensityErrorAllowed;
  out[i++] = (float)fc.minLoops;
  out[i++] = (float)fc.maxLoops;
  out[i++] = fc.surface_tension_gamma;
  out[i++] = fc.surface_adhesion_beta;
  out[i++] = fc.forceDistance;
  out[i++] = fc.maxBoundaryForce;
  out[i++] = fc.springCoefficient;
  out[i++] = fc.springCoefficientBoundary;
  out[i++] = fc.dampingCoefficient;
  out[i++] = fc.terminalSpeed;
  out[i++] = fc.k_r;
  out[i++] = fc.k_d;
  out[i++] = fc.k_t;
  out[i++] = fc.mu;
  out[i++] = fc.scales.x;
  out[i++] = fc.scales.y;
  out[i++] = fc.scales.z;
  out[i++] = fc.collisionBox.getMin().x;
  out[i++] = fc.collisionBox.getMin().y;
  out[i++] = fc.collisionBox.getMin().z;
  out[i++] = fc.collisionBox.getMax().x;
  out[i++] = fc.collisionBox.getMax().y;
  out[i++] = fc.collisionBox.getMax().z;
  out[i++] = fc.realBoxContainer.getMin().x;
  out[i++] = fc.realBoxContainer.getMin().y;
  out[i++] = fc.realBoxContainer.getMin().z;
  out[i++] = fc.realBoxContainer.getMax().x;
  out[i++] = fc.realBoxContainer.getMax().y;
  out[i++] = fc.realBoxContainer.getMax().z;
}

}  // extern "C"
