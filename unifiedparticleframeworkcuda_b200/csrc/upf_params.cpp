// upf_params.cpp — host-side parameter defaults, derived values, kernel
// lookup tables and the PCISPH density error factor.
//
// Compiled with -ffp-contract=off: the lookup tables must be bit-identical to
// the ones WeightingKernel::initLookupTables builds
// (src/cpu/WeightingKernel.cpp:303-320), so the kernel formulas keep the
// reference's float expressions, including the double literals that promote
// parts of them.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "upf_internal.h"

namespace upf {

namespace {

const double kPi = 3.1415926535897932384626;

// Cubic spline M4, WeightingKernel::KernelM4 (WeightingKernel.cpp:75-96)
float m4(float dist, float sr) {
  float s = dist / sr;
  float factor = 2.546479089470325472f / (sr * sr * sr);
  if (dist < 0.0f || dist >= sr) return 0.0f;
  float result;
  if (s < 0.5f)
    result = 1.0f - 6.0 * s * s + 6.0f * s * s * s;
  else {
    float t = 1.0f - s;
    result = 2.0 * t * t * t;
  }
  return factor * result;
}

// Spiky gradient factor, WeightingKernel::kernelPressureGrad (WeightingKernel.cpp:165-180)
float spiky_grad(float dist, float sr) {
  if (dist == 0) return 0.0f;
  if (dist > sr) return 0.0f;
  float c = -45.f / ((float(kPi) * sr * sr * sr * sr * sr * sr));
  return c / dist * (sr - dist) * (sr - dist);
}

// Viscosity Laplacian, WeightingKernel::kernelViscosityLaplacian (WeightingKernel.cpp:190-200)
float visc_lap(float dist, float sr) {
  if (dist > sr) return 0.0f;
  float c = 45.f / ((float(kPi) * sr * sr * sr * sr * sr * sr));
  return c * (sr - dist);
}

// Akinci cohesion spline, WeightingKernel::kernelSplineSurfaceTension (WeightingKernel.cpp:210-231)
float cohesion_spline(float dist, float sr) {
  const float c = 32.0f / ((float(kPi) * sr * sr * sr * sr * sr * sr * sr * sr * sr));
  if (dist > 0.5 * sr && dist <= sr) return c * (sr - dist) * (sr - dist) * (sr - dist) * dist * dist * dist;
  if (dist > 0 && dist <= 0.5 * sr)
    return c * (2.0f * (sr - dist) * (sr - dist) * (sr - dist) * dist * dist * dist -
                sr * sr * sr * sr * sr * sr / 64.0f);
  return 0.0f;
}

// Akinci adhesion spline, WeightingKernel::kernelSplineSurfaceAdhesion (WeightingKernel.cpp:241-256)
float adhesion_spline(float dist, float sr) {
  const float c = 0.007f / (powf(sr, 3.25));
  if (dist > 0.5 * sr && dist <= sr) {
    const float base = -4.0f * dist * dist / sr + 6.0f * dist - 2.0f * sr;
    return c * powf(base, 1.0 / 4.0);
  }
  return 0.0f;
}

uint32_t spread(uint32_t v) {
  v &= 0x3FFu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

uint32_t host_key(const upf_params& p, const float x[3]) {
  uint32_t k = 0;
  for (int a = 0; a < 3; ++a) {
    float c = p.scales[a] * (x[a] - p.zindex_origin[a]);
    uint32_t u = (!(c > 0.0f)) ? 0u : (c >= 1023.0f ? 1023u : (uint32_t)c);
    k |= spread(u) << a;
  }
  return k;
}

// PCISPH delta (UnifiedPhysics::ComputeDensityErrorFactor, UnifiedPhysics.cpp:5525-5689):
// the prototype block of CreatePreParticlesISPH (UnifiedPhysics.cpp:5577-5606)
// is laid out in float as the reference does (positions, counts, neighbour
// test), and the gradient sums are accumulated in double. Pair terms are
// added from both ends, as ComputeGradWValues does (UnifiedPhysics.cpp:5560-5572).
double density_error_factor_fp64(const upf_params& p) {
  const float spacing = p.particle_spacing;
  const float h = p.support_radius;
  float mn[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
  if ((double)spacing != 0.0125) {  // float vs double literal, as in the reference
    float scale = spacing / 0.0125;
    mn[0] = -0.1f * scale; mn[1] = 0.0f * scale; mn[2] = -0.1f * scale;
    mx[0] = 0.1f * scale; mx[1] = 0.2f * scale; mx[2] = 0.1f * scale;
  }
  int num[3];
  for (int a = 0; a < 3; ++a) num[a] = int((mx[a] - mn[a]) / spacing);
  struct Proto {
    float x[3];
    uint32_t key;
  };
  std::vector<Proto> v;
  v.reserve((size_t)std::max(0, num[0] * num[1] * num[2]));
  for (int iy = 0; iy < num[1]; iy++)
    for (int ix = 0; ix < num[0]; ix++)
      for (int iz = 0; iz < num[2]; iz++) {
        Proto q;
        q.x[0] = 0.0f + ix * spacing;
        q.x[1] = 0.0f + iy * spacing;
        q.x[2] = 0.0f + iz * spacing;
        q.key = host_key(p, q.x);
        v.push_back(q);
      }
  std::stable_sort(v.begin(), v.end(), [](const Proto& a, const Proto& b) { return a.key < b.key; });
  const int n = (int)v.size();
  if (n == 0) return 0.0;
  std::vector<double> sx(n, 0), sy(n, 0), sz(n, 0), sd(n, 0);
  std::vector<int> cnt(n, 0);
  const double c = -45.0 / (kPi * std::pow((double)h, 6));
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      float dx = v[i].x[0] - v[j].x[0], dy = v[i].x[1] - v[j].x[1], dz = v[i].x[2] - v[j].x[2];
      float d = sqrtf(dx * dx + dy * dy + dz * dz);
      if (!(d < h)) continue;
      cnt[i]++;
      double g = (d == 0.0f) ? 0.0 : c / (double)d * ((double)h - d) * ((double)h - d);
      double gx = (double)dx * g, gy = (double)dy * g, gz = (double)dz * g;
      double gg = gx * gx + gy * gy + gz * gz;
      sx[i] += gx; sy[i] += gy; sz[i] += gz;
      sx[j] -= gx; sy[j] -= gy; sz[j] -= gz;
      sd[i] += gg;
      sd[j] += gg;
    }
  }
  int best = 0, maxn = 0;
  for (int i = 0; i < n; ++i)
    if (cnt[i] > maxn) { maxn = cnt[i]; best = i; }
  const double rest_vol = (double)p.mass / (double)p.rest_density;
  const double pre = rest_vol * rest_vol * (double)p.dt * (double)p.dt;
  const double term = -(sx[best] * sx[best] + sy[best] * sy[best] + sz[best] * sz[best]) - sd[best];
  const double divisor = pre * term;
  if (divisor == 0.0) return 0.0;
  return (-1.0 / divisor) * (double)p.density_error_fudge;
}

}  // namespace

float kernel_self(float h) { return m4(0.0f, h); }

namespace {
// bin of WeightingKernel::kernel*Lut for a squared distance: (int)(sqrtf(r2) * factor * 300)
int bin_exact(float r2, float factor) { return (int)(sqrtf(r2) * factor * (float)UPF_LUT_SIZE); }

uint32_t fbits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}
float bitsf(uint32_t u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}
// smallest non-negative float r2 with pred(r2) true (pred monotone, true at hi)
template <class Pred>
float first_true(uint32_t hi_bits, Pred pred) {
  uint32_t lo = 0, hi = hi_bits;  // pred(bitsf(hi)) is true
  if (pred(0.0f)) return 0.0f;
  while (hi - lo > 1) {
    uint32_t mid = lo + (hi - lo) / 2;
    if (pred(bitsf(mid)))
      hi = mid;
    else
      lo = mid;
  }
  return bitsf(hi);
}
}  // namespace

// Exact squared-distance thresholds of the table bins (the device picks the
// bin of r2 from these instead of a correctly rounded square root; sqrt,
// the two products and the truncation are all monotone in r2).
void build_bin_thresholds(const upf_params& p, float* out) {
  const float h = p.support_radius;
  const float factor = (float)(1.0 / (double)h);
  const uint32_t top = fbits(h * h * 4.0f);
  out[0] = 0.0f;
  for (int b = 1; b <= UPF_LUT_SIZE; ++b)
    out[b] = first_true(top, [&](float r2) { return bin_exact(r2, factor) >= b; });
  out[UPF_LUT_SIZE + 1] = first_true(top, [&](float r2) { return sqrtf(r2) >= h; });
  // Outside the support the reference adds nothing (it tests dist < h before
  // the table, e.g. ComputePredictedDensityAndPressure, UnifiedPhysics.cpp:
  // 5470). For some h, (int)(h * factor * 300) is 299, so the first r2 of
  // bin 300 lies above h^2 and a pair just outside the support would still
  // take bin 299. Starting bin 300 no later than the support's edge sends
  // those pairs to the tables' zero entry; r2 inside the support is below
  // both thresholds and keeps its bin. (bin_of_r2's guess near h^2 is 299,
  // never lower, so the device then compares against this entry.)
  if (out[UPF_LUT_SIZE] > out[UPF_LUT_SIZE + 1]) out[UPF_LUT_SIZE] = out[UPF_LUT_SIZE + 1];
}

void build_luts(const upf_params& p, float* out) {
  const float sr = p.support_radius;
  for (int i = 0; i < UPF_LUT_SIZE; i++) {
    float dist = sr * i / UPF_LUT_SIZE;
    out[0 * UPF_LUT_ENTRIES + i] = m4(dist, sr);
    out[1 * UPF_LUT_ENTRIES + i] = spiky_grad(dist, sr);
    out[2 * UPF_LUT_ENTRIES + i] = visc_lap(dist, sr);
    out[3 * UPF_LUT_ENTRIES + i] = cohesion_spline(dist, sr);
    out[4 * UPF_LUT_ENTRIES + i] = adhesion_spline(dist, sr);
  }
  for (int k = 0; k < 5; ++k) out[k * UPF_LUT_ENTRIES + UPF_LUT_SIZE] = 0.0f;
}

void default_params(upf_params* p) {
  // UnifiedConstants::UnifiedConstants (UnifiedConstants.cpp:7-159)
  std::memset(p, 0, sizeof(*p));
  p->method = UPF_METHOD_PCISPH;
  p->flags = UPF_FLAG_SURFACE_TENSION | UPF_FLAG_PENALTY_WALLS;
  p->particle_spacing = 1.0 / 40.0;
  p->rest_density = 1000;
  p->gas_constant = 2000;
  p->gamma = 7.0f;
  p->viscosity = 1.0f;
  p->gravity = 9.81f;
  p->dt = 0.0012f;
  p->density_error_fudge = -1.0f;
  p->max_density_error = 1.0f;
  p->min_loops = 3;
  p->max_loops = 50;
  p->surface_tension_gamma = 0.3f;
  p->surface_adhesion_beta = 0.0f;
  p->spring_coefficient = 300.0f;
  p->spring_coefficient_boundary = 300.0f;
  p->damping_coefficient = 0.5f;
  p->terminal_speed = 20.0f;
  p->granular_kr = 1.0f;
  p->granular_kd = 0.1f;
  p->granular_kt = 100.0f;
  p->granular_mu = 0.4f;
  p->zindex_extent[0] = 2.0f;
  p->zindex_extent[1] = 2.0f;
  p->zindex_extent[2] = 1.5f;
  p->max_neighbors = 128;
}

int derive_params(upf_params* p, double* delta_fp64) {
  if (!(p->particle_spacing > 0)) return -1;
  // UnifiedConstants::setParticleSpacing (UnifiedConstants.cpp:162-191)
  if (p->particle_radius == 0) p->particle_radius = p->particle_spacing * 0.5f;
  if (p->support_radius == 0) p->support_radius = p->particle_spacing * 2.0 * 1.00001;
  if (p->mass == 0) p->mass = p->particle_spacing * p->particle_spacing * p->particle_spacing * p->rest_density;
  if (p->force_distance == 0) p->force_distance = 0.25 * p->support_radius;
  if (p->max_boundary_force == 0) p->max_boundary_force = 1.0f * 64 * p->particle_spacing * p->particle_spacing;
  // UnifiedConstants::setBoundingBoxValues (UnifiedConstants.cpp:308-320)
  for (int a = 0; a < 3; ++a) {
    if (!(p->zindex_extent[a] > 0)) return -1;
    if (p->scales[a] == 0) p->scales[a] = float(UPF_GRID_RESOLUTION) / p->zindex_extent[a];
  }
  if (p->block_size == 0) {
    // UnifiedPhysics.cpp:2149-2156 + ZIndex::SetBlockSize (zIndex.cpp:27-39)
    float mb = p->scales[0] * p->support_radius;
    mb = std::max(mb, p->scales[1] * p->support_radius);
    mb = std::max(mb, p->scales[2] * p->support_radius);
    int size = (int)mb;
    uint32_t bs;
    for (bs = 1; (int)bs < size; bs *= 2) {
    }
    p->block_size = bs;
  }
  if (p->density_error_fudge < 0) {
    const float factor = p->dt / 0.0002f;  // UnifiedConstants.cpp:101-103
    p->density_error_fudge = 0.05 * factor * factor;
  }
  if (p->max_neighbors == 0) p->max_neighbors = 128;
  if (p->search_cell == 0) p->search_cell = default_search_cell(*p);
  double d = 0.0;
  if (p->method == UPF_METHOD_PCISPH && p->density_error_factor == 0) {
    d = density_error_factor_fp64(*p);
    p->density_error_factor = (float)d;
  }
  if (delta_fp64) *delta_fp64 = d;
  return 0;
}

double density_error_factor(const upf_params& p) { return density_error_factor_fp64(p); }

// Cells a query box [x - h - 1, x + h + 1] (grid units) can span per axis,
// for a cell edge c: floor((2r + 3) / c) + 2, r = max(scales) * h.
static int query_cells_per_axis(const upf_params& p, uint32_t c) {
  const double r = (double)std::max(p.scales[0], std::max(p.scales[1], p.scales[2])) * (double)p.support_radius;
  return (int)std::floor((2.0 * r + 3.0) / (double)c) + 2;
}

// The reference's block size: finer cells visit fewer candidates but pay
// more per cell (table lookups, ordering the cells, divergent short ranges);
// measured on B200 the block size is the faster of the two at h = 2 spacing.
uint32_t default_search_cell(const upf_params& p) {
  uint32_t c = std::max<uint32_t>(p.block_size, 4);
  while (c < 1024 && query_cells_per_axis(p, c) > 4) c *= 2;
  return c;
}

uint32_t effective_search_cell(const upf_params& p) {
  return p.search_cell ? p.search_cell : default_search_cell(p);
}

int validate_params(const upf_params& p, const char** why) {
  auto bad = [&](const char* w) {
    if (why) *why = w;
    return -1;
  };
  if (p.method != UPF_METHOD_WCSPH && p.method != UPF_METHOD_PCISPH) return bad("unknown method");
  if (!(p.support_radius > 0)) return bad("support_radius must be > 0");
  if (!(p.mass > 0)) return bad("mass must be > 0");
  if (!(p.rest_density > 0)) return bad("rest_density must be > 0");
  if (!(p.dt > 0)) return bad("dt must be > 0");
  if (p.block_size == 0 || (p.block_size & (p.block_size - 1)) || p.block_size > 1024)
    return bad("block_size must be a power of two <= 1024");
  if (p.block_size < 4) return bad("block_size must be >= 4 (cell table size)");
  for (int a = 0; a < 3; ++a)
    if (!(p.scales[a] > 0)) return bad("scales must be > 0");
  {
    // the neighbour search visits (2R+1)^3 blocks around a cell, R <= 2
    float r = std::max(p.scales[0], std::max(p.scales[1], p.scales[2])) * p.support_radius;
    if (std::ceil((double)(r + 1.0f) / (double)p.block_size) > 2.0)
      return bad("block_size too small for the support radius (need block_size >= (scales*h + 1) / 2)");
  }
  if (p.max_neighbors == 0 || p.max_neighbors > 1024) return bad("max_neighbors must be in 1..1024");
  {
    const uint32_t c = effective_search_cell(p);
    if (c < 4 || c > 1024 || (c & (c - 1))) return bad("search_cell must be a power of two in 4..1024");
    if (query_cells_per_axis(p, c) > 4)
      return bad("search_cell too small for the support radius (a query box may span at most 4 cells per axis)");
  }
  if (p.method == UPF_METHOD_PCISPH) {
    if (p.min_loops < 1 || p.max_loops < p.min_loops) return bad("need 1 <= min_loops <= max_loops");
    if (p.max_loops > 1000) return bad("max_loops must be <= 1000");
  }
  return 0;
}

}  // namespace upf
