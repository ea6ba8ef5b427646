// upf_oracle.cpp — TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// CPU restatement of the reference's CPU particle path. Each function cites
// the reference function it follows (paths relative to the reference's
// project root). The FP32 twin keeps the reference's operation order and its
// float/double promotions so that, compiled with -ffp-contract=off, every
// float operation rounds exactly as the reference's does. The FP64 twin runs
// the same algorithm in double precision and serves as the error yardstick.
//
// Deliberate deviations from the reference (each one documented where it is
// made): stable sort with input-order tie-break, lifted function-static
// constants, the boundary pressure lookup indexed by distance, lagged
// boundary-pressure state initialised to (p=0, rho=rest density), boundary
// particles excluded from the final clamp, and no data race on the max
// predicted density.
#include "upf_oracle.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

namespace {

constexpr int kLut = UPF_LUT_SIZE;
const double kPi = 3.1415926535897932384626;  // WeightingKernel.cpp:5

// ---------------------------------------------------------------------------
// Kernel functions (src/cpu/WeightingKernel.cpp), FP32 exactly as written,
// including the double-precision literals that promote parts of the
// expressions.
// ---------------------------------------------------------------------------
float KernelM4(float dist, float sr) {  // WeightingKernel.cpp:75-96
  float s = dist / sr;
  float result;
  float factor = 2.546479089470325472f / (sr * sr * sr);
  if (dist < 0.0f || dist >= sr) return 0.0f;
  if (s < 0.5f) {
    result = 1.0f - 6.0 * s * s + 6.0f * s * s * s;
  } else {
    float tmp = 1.0f - s;
    result = 2.0 * tmp * tmp * tmp;
  }
  return factor * result;
}

float KernelPressureGrad(float dist, float sr) {  // WeightingKernel.cpp:165-180
  if (dist == 0) return 0.0f;
  if (dist > sr) return 0.0f;
  float c = -45.f / ((float(kPi) * sr * sr * sr * sr * sr * sr));
  return c / dist * (sr - dist) * (sr - dist);
}

float KernelViscosityLaplacian(float dist, float sr) {  // WeightingKernel.cpp:190-200
  if (dist > sr) return 0.0f;
  float c = 45.f / ((float(kPi) * sr * sr * sr * sr * sr * sr));
  return c * (sr - dist);
}

float KernelSplineSurfaceTension(float dist, float sr) {  // WeightingKernel.cpp:210-231
  const float c = 32.0f / ((float(kPi) * sr * sr * sr * sr * sr * sr * sr * sr * sr));
  if (dist > 0.5 * sr && dist <= sr) {
    return c * (sr - dist) * (sr - dist) * (sr - dist) * dist * dist * dist;
  } else if (dist > 0 && dist <= 0.5 * sr) {
    return c * (2.0f * (sr - dist) * (sr - dist) * (sr - dist) * dist * dist * dist -
                sr * sr * sr * sr * sr * sr / 64.0f);
  }
  return 0.0f;
}

float KernelSplineSurfaceAdhesion(float dist, float sr) {  // WeightingKernel.cpp:241-256
  const float c = 0.007f / (powf(sr, 3.25));
  if (dist > 0.5 * sr && dist <= sr) {
    const float base = -4.0f * dist * dist / sr + 6.0f * dist - 2.0f * sr;
    return c * powf(base, 1.0 / 4.0);
  }
  return 0.0f;
}

struct Tables {
  float lut[5][kLut + 1];  // M4, pressure grad, visc lap, surface tension, adhesion
  uint32_t ztab[1024][3];
  float kernel_self;
};

enum { L_M4 = 0, L_PGRAD = 1, L_VISC = 2, L_ST = 3, L_ADH = 4 };

void BuildTables(const upf_params& p, Tables& t) {
  // WeightingKernel::initLookupTables, WeightingKernel.cpp:303-320
  float sr = p.support_radius;
  for (int i = 0; i < kLut; i++) {
    float dist = sr * i / kLut;
    t.lut[L_M4][i] = KernelM4(dist, sr);
    t.lut[L_PGRAD][i] = KernelPressureGrad(dist, sr);
    t.lut[L_VISC][i] = KernelViscosityLaplacian(dist, sr);
    t.lut[L_ST][i] = KernelSplineSurfaceTension(dist, sr);
    t.lut[L_ADH][i] = KernelSplineSurfaceAdhesion(dist, sr);
  }
  for (int k = 0; k < 5; ++k) t.lut[k][kLut] = 0.0f;
  // ZIndex::ZIndex, zIndex.cpp:10-24
  for (unsigned k = 0; k < 1024; k++) {
    t.ztab[k][0] = t.ztab[k][1] = t.ztab[k][2] = 0;
    for (unsigned i = 0; i < 10; i++) {
      t.ztab[k][0] |= ((k >> i) & 1u) << (3 * i);
      t.ztab[k][1] |= ((k >> i) & 1u) << (3 * i + 1);
      t.ztab[k][2] |= ((k >> i) & 1u) << (3 * i + 2);
    }
  }
  t.kernel_self = KernelM4(0.0f, sr);  // UnifiedPhysics.cpp:113
}

// ---------------------------------------------------------------------------
// 3-vectors with vmml's operation order (src/vmmlib/vector3.h): binary ops
// are component-wise, vector/scalar multiplies by the reciprocal
// (vector3.h:599-605), length = sqrt(x*x + y*y + z*z) (vector3.h:459-476).
// ---------------------------------------------------------------------------
template <class R>
struct V3 {
  R x, y, z;
};
template <class R> inline V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> operator*(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> inline V3<R> divs(V3<R> a, R s) {
  R inv = R(1) / s;  // vmml float specialisation
  return {a.x * inv, a.y * inv, a.z * inv};
}
template <class R> inline R lensq(V3<R> a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
inline float vsqrt(float v) { return sqrtf(v); }
inline double vsqrt(double v) { return std::sqrt(v); }
template <class R> inline R dist(V3<R> a, V3<R> b) { return vsqrt(lensq(a - b)); }
template <class R> inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline V3<R> cross(V3<R> a, V3<R> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

template <class R>
struct Particle {
  V3<R> x, v;          // position_, velocity_
  V3<R> F, Fp;         // force_, correction_pressure_force_
  V3<R> xs, vs;        // predicted_position_, predicted_velocity_
  R density, pressure; // WCSPH density_, pressure_
  R rho_star;          // predicted_density_
  R p_corr;            // correction_pressure_
  R p_prev;            // previous_correction_pressure_
  R rho_prev;          // predicted density of the previous step (lagged)
  R err;               // density_error_
  R wvol;              // weighted_volume_
  int type;
  uint32_t id;
  uint32_t key;        // index_
  int body;
  V3<R> r0;            // init_relative_pos_
};

// RigidBody (src/cpu/RigidBody.h:105-134): the state is float as in the
// reference; the per-body sums (force, torque, mass, inertia) are FP64.
template <class R>
struct Body {
  R mass;
  V3<R> pos, vel, P, L, omega;
  R q[4];              // quaternion_ (s, x, y, z)
  R rot[3][3];
  R inv_inertia_local[3][3];
  R inv_inertia_world[3][3];
};

// Matrix3x3::operator* (Matrix3x3.cpp:15-31, 34-47): sums from zero in k order
template <class R>
void mat_mul(const R a[3][3], const R b[3][3], R out[3][3]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      R s = 0;
      for (int k = 0; k < 3; ++k) s += a[i][k] * b[k][j];
      out[i][j] = s;
    }
}
template <class R>
V3<R> mat_vec(const R a[3][3], V3<R> v) {
  const R* x = &v.x;
  R r[3];
  for (int i = 0; i < 3; ++i) {
    r[i] = 0;
    for (int j = 0; j < 3; ++j) r[i] += a[i][j] * x[j];
  }
  return {r[0], r[1], r[2]};
}
// Vector3::normalize (vmmlib/vector3.h:516-528): returns the length
template <class R>
R normalize(V3<R>& v) {
  const R l = vsqrt(lensq(v));
  if (l == 0) return 0;
  const R ll = R(1.0 / l);
  v.x *= ll;
  v.y *= ll;
  v.z *= ll;
  return l;
}
// Matrix3x3::CalculateInverse (Matrix3x3.cpp:121-156) in FP64: adjugate over
// determinant, row-major; a singular matrix leaves `inv` unchanged and
// returns false.
inline bool inverse3_fp64(const double* A, double* inv) {
  const double det = A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
                     A[2] * (A[3] * A[7] - A[4] * A[6]);
  if (det == 0.0) return false;
  inv[0] = (A[4] * A[8] - A[5] * A[7]) / det;
  inv[1] = (A[2] * A[7] - A[1] * A[8]) / det;
  inv[2] = (A[1] * A[5] - A[2] * A[4]) / det;
  inv[3] = (A[5] * A[6] - A[3] * A[8]) / det;
  inv[4] = (A[0] * A[8] - A[2] * A[6]) / det;
  inv[5] = (A[2] * A[3] - A[0] * A[5]) / det;
  inv[6] = (A[3] * A[7] - A[4] * A[6]) / det;
  inv[7] = (A[1] * A[6] - A[0] * A[7]) / det;
  inv[8] = (A[0] * A[4] - A[1] * A[3]) / det;
  return true;
}

// RigidBody::UpdateMomenta, PerformStep (UpdateInverseInertiaTensor,
// PerformLinearStep, PerformAngularStep) and UpdateRotationMatrix
// (RigidBody.cpp:15-161, 96-128) for one body, given the step's force and
// torque. Float as the reference; its cos/sin calls take and return double
// (the float angle is promoted), and `axis * sin(...)` multiplies in double
// before rounding. The quaternion is not renormalised (RigidBody.cpp:99
// discards getNormalized()'s result). MIN/MAX are the reference's macros
// (global.h:4-5).
template <class R>
void body_update(Body<R>& b, V3<R> force, V3<R> torque, R dt, R terminal_speed) {
  const R terminal = b.mass * terminal_speed;
  b.P = b.P + force * dt;
  R* P = &b.P.x;
  for (int a = 0; a < 3; ++a) {
    if (P[a] > R(0.0f))
      P[a] = (P[a] <= terminal) ? P[a] : terminal;
    else
      P[a] = (P[a] >= -terminal) ? P[a] : -terminal;
  }
  b.L = b.L + torque * dt;
  R rt[3][3], tmp[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) rt[j][i] = b.rot[i][j];
  mat_mul(b.rot, b.inv_inertia_local, tmp);
  mat_mul(tmp, rt, b.inv_inertia_world);
  b.vel = divs(b.P, b.mass);
  b.pos = b.pos + b.vel * dt;
  b.omega = mat_vec(b.inv_inertia_world, b.L);
  const R speed = vsqrt(lensq(b.omega));
  if (speed > R(0.0f)) {
    V3<R> axis = b.omega;
    normalize(axis);
    const R angle = speed * dt;
    const double half = (double)(angle / R(2.0f));
    const R ds = R(std::cos(half));
    const double sn = std::sin(half);
    const R dvx = R((double)axis.x * sn);
    const R dvy = R((double)axis.y * sn);
    const R dvz = R((double)axis.z * sn);
    const R s = b.q[0], vx = b.q[1], vy = b.q[2], vz = b.q[3];
    b.q[0] = s * ds - vx * dvx - vy * dvy - vz * dvz;
    b.q[1] = ds * vx + s * dvx + dvy * vz - dvz * vy;
    b.q[2] = ds * vy + s * dvy + dvz * vx - dvx * vz;
    b.q[3] = ds * vz + s * dvz + dvx * vy - dvy * vx;
  }
  const R w = b.q[0], x = b.q[1], y = b.q[2], z = b.q[3];
  const R xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z, wx = w * x, wy = w * y,
          wz = w * z;
  b.rot[0][0] = R(1.0f) - R(2.0f) * (yy + zz);
  b.rot[0][1] = R(2.0f) * (xy - wz);
  b.rot[0][2] = R(2.0f) * (xz + wy);
  b.rot[1][0] = R(2.0f) * (xy + wz);
  b.rot[1][1] = R(1.0f) - R(2.0f) * (xx + zz);
  b.rot[1][2] = R(2.0f) * (yz - wx);
  b.rot[2][0] = R(2.0f) * (xz - wy);
  b.rot[2][1] = R(2.0f) * (yz + wx);
  b.rot[2][2] = R(1.0f) - R(2.0f) * (xx + yy);
}

// ---------------------------------------------------------------------------
// The simulation: one particle array for every type, as in the reference.
// ---------------------------------------------------------------------------
struct SimBase {
  virtual ~SimBase() {}
  virtual int step(orc_step_info* info) = 0;
  virtual uint32_t count() const = 0;
  virtual void get(float*, float*, float*, float*, int32_t*, uint32_t*, uint32_t*) const = 0;
  virtual void get_fields(float*, float*, float*, float*, float*, float*, uint32_t*) const = 0;
  virtual uint32_t neighbors(uint32_t*, uint32_t*, uint32_t) = 0;
  virtual int set_bodies(const int32_t*, uint32_t, uint32_t) = 0;
  virtual int get_rigid(float*, float*, float*, float*) const = 0;
  virtual void set_keep_fields(bool on) = 0;
  virtual void set_lagged(const float*, const float*, const float*) = 0;
  virtual void get_lagged(float*, float*, float*) const = 0;
  virtual void set_literal(uint32_t mask) = 0;
};

template <class R>
struct Sim : SimBase {
  upf_params prm;
  Tables tab;
  std::vector<Particle<R>> ps;
  std::vector<std::vector<int>> nbr;
  std::vector<Body<R>> bodies;
  std::vector<Particle<R>> snapshot;  // step-start order fields
  R lut_factor;                       // static float factor = 1.0 / h (WeightingKernel.cpp:124)
  int threads;
  bool keep_fields = false;           // snapshot step-start fields for parity tests
  uint32_t literal = 0;               // ORC_LITERAL_*: the reference's own rule where this build deviates

  // ---- lookup tables (WeightingKernel::kernel*Lut, WeightingKernel.cpp:122-128 etc.)
  inline R lut(int k, R d) const {
    int index = d * lut_factor * kLut;
    return (index >= kLut) ? R(0) : R(tab.lut[k][index]);
  }
  // dist_lut of the PCISPH external force (UnifiedPhysics.cpp:5266-5268)
  inline unsigned dist_lut(R d) const {
    unsigned dl = d * (kLut) / R(prm.support_radius);
    if (dl > (unsigned)kLut) dl = kLut;
    return dl;
  }

  // ---- z-index key (ZIndex::CalcIndex via zIndex.CalcIndex(fc_->scales * p.position_),
  // UnifiedPhysics.cpp:4005). The float -> unsigned short conversion truncates;
  // coordinates are clamped to the 1024 grid (the reference indexes its table
  // out of bounds otherwise).
  inline uint32_t key_of(V3<R> x) const {
    R c[3] = {R(prm.scales[0]) * (x.x - R(prm.zindex_origin[0])),
              R(prm.scales[1]) * (x.y - R(prm.zindex_origin[1])),
              R(prm.scales[2]) * (x.z - R(prm.zindex_origin[2]))};
    uint32_t k = 0;
    for (int a = 0; a < 3; ++a) {
      int u = (c[a] <= R(0)) ? 0 : (c[a] >= R(1023) ? 1023 : (int)(unsigned short)c[a]);
      k |= tab.ztab[u][a];
    }
    return k;
  }

  Sim(const upf_params& p, const float* pos4, const float* vel4, const int32_t* type, uint32_t n,
      int nthreads)
      : prm(p), threads(nthreads) {
    BuildTables(prm, tab);
    lut_factor = R(1.0 / prm.support_radius);
    ps.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
      Particle<R>& q = ps[i];
      std::memset(&q, 0, sizeof(q));
      q.x = {R(pos4[4 * i]), R(pos4[4 * i + 1]), R(pos4[4 * i + 2])};
      q.v = {R(vel4[4 * i]), R(vel4[4 * i + 1]), R(vel4[4 * i + 2])};
      q.xs = q.x;  // UnifiedParticle ctor: predicted_position_ = position_
      q.vs = q.v;
      q.type = type[i];
      q.id = i;
      q.body = -1;
      q.wvol = R(prm.mass) / R(prm.rest_density);  // UnifiedParticle.cpp:24
      q.rho_prev = R(prm.rest_density);
      q.key = key_of(q.x);
    }
    sort_particles();
    nbr.resize(n);
    // boundary particle volumes for the Akinci terms (CalculateWeightedVolume,
    // UnifiedPhysics.cpp:2703-2746), once for the static boundary.
    if (needs_wvol()) {
      find_neighbors();
      compute_weighted_volume(true);
    }
  }

  bool needs_wvol() const {
    return (prm.method == UPF_METHOD_PCISPH) && (prm.flags & UPF_FLAG_ADHESION);
  }

  // SortParticles (UnifiedPhysics.cpp:353-358). std::sort there is not stable;
  // the restatement sorts stably so that equal keys keep their previous order.
  void sort_particles() {
    std::stable_sort(ps.begin(), ps.end(),
                     [](const Particle<R>& a, const Particle<R>& b) { return a.key < b.key; });
  }

  // ZIndex::BoxQuery (zIndex.cpp:43-73) + GetNeighbors (UnifiedPhysics.cpp:2242-2280).
  void get_neighbors(int i, std::vector<std::pair<uint32_t, uint32_t>>& ranges) {
    const Particle<R>& p = ps[i];
    const R h = R(prm.support_radius);
    R mn[3] = {R(prm.scales[0]) * (p.x.x - h), R(prm.scales[1]) * (p.x.y - h), R(prm.scales[2]) * (p.x.z - h)};
    R mx[3] = {R(prm.scales[0]) * (p.x.x + h), R(prm.scales[1]) * (p.x.y + h), R(prm.scales[2]) * (p.x.z + h)};
    // Both corners are clamped into [0, 1024]. The reference clamps only the
    // lower one from below and the upper one from above. A particle outside
    // the grid then converts a negative float (or one above 65535) to
    // unsigned short, which is undefined, and an upper corner below the lower
    // one makes an empty box of negative size. Particles inside the grid are
    // unaffected.
    uint16_t a[3], b[3];
    for (int k = 0; k < 3; ++k) {
      mn[k] = std::min(std::max(mn[k], R(0)), R(UPF_GRID_RESOLUTION));
      mx[k] = std::min(std::max(mx[k], R(0)), R(UPF_GRID_RESOLUTION));
      a[k] = (unsigned short)mn[k];
      b[k] = (unsigned short)mx[k];
    }
    box_query(prm.block_size, a, b, ranges);
    std::sort(ranges.begin(), ranges.end());
    std::vector<int>& out = nbr[i];
    out.clear();
    for (size_t k = 0; k < ranges.size(); ++k) {
      auto it = std::lower_bound(ps.begin(), ps.end(), ranges[k].first,
                                 [](const Particle<R>& q, uint32_t key) { return q.key < key; });
      for (; it != ps.end() && it->key <= ranges[k].second; ++it) {
        int j = int(it - ps.begin());
        if (j == i) continue;
        R d = dist(p.x, it->x);
        if (d < h) out.push_back(j);
      }
    }
  }

  static void box_query(uint32_t bs, const uint16_t mn[3], const uint16_t mx[3],
                        std::vector<std::pair<uint32_t, uint32_t>>& ranges) {
    static const unsigned XMASK = 0xB6DB6DB6, YMASK = 0x6DB6DB6D, ZMASK = 0xDB6DB6DB;  // zIndex.h:12-14
    auto xinc = [](unsigned i) { return (((i | XMASK) + 1) & ~XMASK) | (i & XMASK); };
    auto yinc = [](unsigned i) { return (((i | YMASK) + 1) & ~YMASK) | (i & YMASK); };
    auto zinc = [](unsigned i) { return (((i | ZMASK) + 1) & ~ZMASK) | (i & ZMASK); };
    const unsigned offset = bs * bs * bs;
    unsigned s[3], e[3];
    for (int k = 0; k < 3; ++k) {
      s[k] = (unsigned short)(mn[k] / bs);
      e[k] = (unsigned short)(mx[k] / bs);
    }
    ranges.resize(size_t(1 + e[0] - s[0]) * (1 + e[1] - s[1]) * (1 + e[2] - s[2]));
    auto morton = [](unsigned x, unsigned y, unsigned z) {
      unsigned k = 0;
      for (unsigned i = 0; i < 10; i++)
        k |= ((x >> i) & 1u) << (3 * i) | ((y >> i) & 1u) << (3 * i + 1) | ((z >> i) & 1u) << (3 * i + 2);
      return k;
    };
    int cnt = 0;
    unsigned xind = morton(s[0], s[1], s[2]);
    for (unsigned i = s[0]; i <= e[0]; i++) {
      unsigned yind = xind;
      for (unsigned j = s[1]; j <= e[1]; j++) {
        unsigned zind = yind;
        for (unsigned k = s[2]; k <= e[2]; k++) {
          ranges[cnt++] = {offset * zind, offset * (zind + 1) - 1};
          zind = zinc(zind);
        }
        yind = yinc(yind);
      }
      xind = xinc(xind);
    }
  }

  void find_neighbors() {
#pragma omp parallel num_threads(threads)
    {
      std::vector<std::pair<uint32_t, uint32_t>> ranges;
#pragma omp for schedule(dynamic, 100)
      for (int i = 0; i < (int)ps.size(); i++) get_neighbors(i, ranges);
    }
  }

  // CalculateWeightedVolume (UnifiedPhysics.cpp:2703-2746): V_b = 1 / sum of
  // W over boundary/rigid neighbours. The reference aborts when the sum is
  // zero; here the particle keeps its rest volume.
  void compute_weighted_volume(bool static_only) {
#pragma omp parallel for num_threads(threads) schedule(dynamic, 100)
    for (int i = 0; i < (int)ps.size(); i++) {
      Particle<R>& p = ps[i];
      bool is_b = (p.type == UPF_FROZEN || p.type == UPF_RIGID);
      if (!is_b) continue;
      if (static_only && p.type != UPF_FROZEN) continue;
      R inv = 0;
      for (int j : nbr[i]) {
        const Particle<R>& q = ps[j];
        R d = dist(p.x, q.x);
        if (d < R(prm.support_radius)) {
          R kv = lut(L_M4, d);
          if (q.type == UPF_FROZEN || q.type == UPF_RIGID) inv += kv;
        }
      }
      if (inv != 0) p.wvol = R(1.0 / inv);
    }
  }

  // ---------------- WCSPH (CpuParticlePhysicsPureFluidsSPH, UnifiedPhysics.cpp:4252-4329)
  // DistanceToWall (UnifiedPhysics.cpp:5926-5990) against the real container.
  R distance_to_wall(V3<R> x) const {
    R L = R(prm.container_max[0]) - R(prm.container_min[0]);
    R H = R(prm.container_max[1]) - R(prm.container_min[1]);
    R W = R(prm.container_max[2]) - R(prm.container_min[2]);
    R result = std::max(L, std::max(H, W));
    R d;
    d = std::max(x.y - R(prm.container_min[1]), R(0)); result = std::min(result, d);
    d = std::max(R(prm.container_max[1]) - x.y, R(0)); result = std::min(result, d);
    d = std::max(x.x - R(prm.container_min[0]), R(0)); result = std::min(result, d);
    d = std::max(R(prm.container_max[0]) - x.x, R(0)); result = std::min(result, d);
    d = std::max(x.z - R(prm.container_min[2]), R(0)); result = std::min(result, d);
    d = std::max(R(prm.container_max[2]) - x.z, R(0)); result = std::min(result, d);
    return result;
  }
  // WallWeight (UnifiedPhysics.cpp:6032-6060)
  R wall_weight(R dw) const {
    const R eff = R(prm.support_radius) - R(prm.particle_radius);
    if (dw >= eff) return 0;
    const R s = R(prm.particle_spacing);
    R d1 = dw + R(prm.particle_radius);
    R d2 = d1 + s;
    R d3 = vsqrt(d1 * d1 + s * s);
    R d4 = vsqrt(d1 * d1 + (s * 2) * (s * 2));
    R d5 = vsqrt(d2 * d2 + s * s);
    R d6 = vsqrt(d2 * d2 + (s * 2) * (s * 2));
    R k1 = lut(L_M4, d1), k2 = lut(L_M4, d2), k3 = lut(L_M4, d3), k4 = lut(L_M4, d4),
      k5 = lut(L_M4, d5), k6 = lut(L_M4, d6);
    return R(prm.mass) * (k1 + k2 + 2 * (k3 + k4 + k5 + k6));
  }

  void wcsph_density(int i) {  // CalculateDensityPressurePureFluidSPH, UnifiedPhysics.cpp:2408-2477
    Particle<R>& p = ps[i];
    const R m = R(prm.mass);
    p.density = R(tab.kernel_self) * m;
    for (int j : nbr[i]) {
      R d = dist(p.x, ps[j].x);
      if (d < R(prm.support_radius)) {
        R kv = lut(L_M4, d);
        p.density += kv * m;
      }
    }
    if (prm.flags & UPF_FLAG_WALL_WEIGHT) p.density += wall_weight(distance_to_wall(p.x));
    // CalculatePressureWCSPH, UnifiedPhysics.cpp:2491-2501
    const R gamma = R(prm.gamma);
    const R b_i = R(prm.rest_density) * R(prm.gas_constant) / gamma;
    const R frac = p.density / R(prm.rest_density);
    const R powg = std::pow(frac, gamma);
    p.pressure = std::max(R(0), b_i * (powg - R(1)));
  }

  V3<R> wcsph_force(int i) {  // CalculateLiquidParticleForces, UnifiedPhysics.cpp:3009-3083
    Particle<R>& p = ps[i];
    const R m = R(prm.mass), h = R(prm.support_radius);
    const R invDensity = R(1.0 / p.density);
    const R pVol = m * invDensity;
    V3<R> force = {0, 0, 0};
    for (int j : nbr[i]) {
      const Particle<R>& q = ps[j];
      R d = dist(p.x, q.x);
      if (d < h) {
        R kernelVisc = lut(L_VISC, d);
        R nVol = m / q.density;
        const V3<R> distVec = p.x - q.x;
        if (q.type == UPF_LIQUID) {
          V3<R> kg = distVec * lut(L_PGRAD, d);
          R grad = p.pressure * invDensity * invDensity + q.pressure / (q.density * q.density);
          V3<R> tpf = kg * grad * m * m;
          force = force - tpf;
          V3<R> vij = p.v - q.v;
          force = force - vij * pVol * nVol * R(prm.viscosity) * kernelVisc;
          if ((prm.flags & UPF_FLAG_SURFACE_TENSION) && d >= h * R(0.25f)) {
            // CalculateSurfaceTensionForcePCISPH, UnifiedPhysics.cpp:4180-4185
            R spline = R(KernelSplineSurfaceTension(float(d), float(h)));
            force = force - (p.x - q.x) * R(prm.surface_tension_gamma) * m * m * spline * (R(1) / d);
          }
        }
      }
    }
    return force;
  }

  // UpdateLiquidParticlePosVelSphCPU (UnifiedPhysics.cpp:3705-3742); granular
  // grains take the same symplectic Euler step with their contact force
  void integrate(Particle<R>& p) {
    if (p.type != UPF_LIQUID && p.type != UPF_GRANULAR) return;
    if (prm.method == UPF_METHOD_PCISPH && p.type == UPF_LIQUID) p.F = p.F + p.Fp;
    const R invMass = R(1.0 / prm.mass);
    const R dt = R(prm.dt);
    p.v = p.v + p.F * invMass * dt;
    p.x = p.x + p.v * dt;
  }

  // BoundaryHandlingBoxPerNonRigidParticle (UnifiedPhysics.cpp:4000-4044)
  void clamp_box(V3<R>& pos, V3<R>& vel, R damping) {
    R* x = &pos.x;
    R* v = &vel.x;
    const int order[3] = {1, 0, 2};
    for (int o = 0; o < 3; ++o) {
      int a = order[o];
      if (x[a] < R(prm.collision_min[a])) { x[a] = R(prm.collision_min[a]); v[a] *= damping; }
      if (x[a] > R(prm.collision_max[a])) { x[a] = R(prm.collision_max[a]); v[a] *= damping; }
    }
  }

  void finish_step_stats(orc_step_info* info) {
    double ke = 0, mom[3] = {0, 0, 0};
    const double m = prm.mass;
    for (auto& p : ps) {
      if (p.type != UPF_LIQUID) continue;
      double vx = p.v.x, vy = p.v.y, vz = p.v.z;
      ke += 0.5 * m * (vx * vx + vy * vy + vz * vz);
      mom[0] += m * vx; mom[1] += m * vy; mom[2] += m * vz;
    }
    uint32_t mx = 0;
    for (auto& l : nbr) mx = std::max<uint32_t>(mx, (uint32_t)l.size());
    if (info) {
      info->kinetic_energy = ke;
      for (int k = 0; k < 3; ++k) info->momentum[k] = mom[k];
      info->max_neighbor_count = mx;
    }
  }

  int step_wcsph(orc_step_info* info) {
    const int n = (int)ps.size();
    find_neighbors();
#pragma omp parallel for num_threads(threads) schedule(dynamic, 100)
    for (int i = 0; i < n; i++) wcsph_density(i);
#pragma omp parallel for num_threads(threads) schedule(dynamic, 100)
    for (int i = 0; i < n; i++) {
      Particle<R>& p = ps[i];
      if (p.type == UPF_LIQUID) {
        p.F = wcsph_force(i);
        p.F.y -= R(prm.mass) * R(prm.gravity);  // UnifiedPhysics.cpp:4287
      }
    }
    if (keep_fields) snapshot = ps;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 100)
    for (int i = 0; i < n; i++) integrate(ps[i]);
    // Boundary handling (UnifiedPhysics.cpp:4296-4326). The reference clamps
    // every particle here; static boundary particles may sit outside the
    // collision box, so only liquid particles are clamped (as in
    // BoundaryHandlingPureFluidOMP, UnifiedPhysics.cpp:3972-3998), unless
    // the reference's literal rule is asked for.
    const R damping = R(-0.5);
    const bool all = (literal & ORC_LITERAL_WCSPH_CLAMP_ALL) != 0;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 100)
    for (int i = 0; i < n; i++) {
      Particle<R>& p = ps[i];
      if (p.type == UPF_LIQUID || all) clamp_box(p.x, p.v, damping);
      p.key = key_of(p.x);
    }
    finish_step_stats(info);
    sort_particles();
    if (info) info->iterations = 0;
    return 0;
  }

  // ---------------- PCISPH (CpuParticlePhysicsVersatileCouplingPCISPH, UnifiedPhysics.cpp:4991-5024)

  // CalculateBoundaryForcePerLiquidParticleHost (UnifiedPhysics.cpp:2032-2069);
  // note the double-precision 2.0 literal.
  V3<R> penalty_walls(V3<R> x) const {
    V3<R> f = {0, 0, 0};
    const R fd = R(prm.force_distance);
    const R inv = R(1.0f / prm.force_distance);
    const double mbf = prm.max_boundary_force;
    const R* pos = &x.x;
    R* fv = &f.x;
    for (int a = 0; a < 3; ++a) {
      const R mn = R(prm.collision_min[a]), mx = R(prm.collision_max[a]);
      if (pos[a] < mn + fd) fv[a] += R(R((mn + fd - pos[a]) * inv) * 2.0 * mbf);
      if (pos[a] > mx - fd) fv[a] += R(-1) * R(R((pos[a] + fd - mx) * inv) * 2.0 * mbf);
    }
    return f;
  }

  // CalculateBoundaryFluidPressureForceHost (UnifiedPhysics.cpp:4240-4250). The
  // reference passes the bin index where the distance belongs, which makes
  // the lookup return 0 for every pair; here the table is indexed by the
  // distance, as the function intends.
  V3<R> boundary_pressure(R d, V3<R> ppos, V3<R> npos, R p_density, R p_press, R wvol) const {
    R inv_den = R(1.0f) / p_density;
    V3<R> kg = (ppos - npos) * lut(L_PGRAD, d);
    R press_grad = p_press * inv_den * inv_den;
    return kg * press_grad * R(prm.mass) * R(prm.rest_density) * wvol * R(-1.0f);
  }

  void pcisph_external(int i) {  // CalculateExternalForcesVersatilCouplingPCISPH, UnifiedPhysics.cpp:5252-5365
    Particle<R>& p = ps[i];
    const R m = R(prm.mass), h = R(prm.support_radius), rho0 = R(prm.rest_density);
    if (p.type == UPF_LIQUID) {
      p.F = {0, 0, 0};
      const R restVolume = m / rho0;
      for (int j : nbr[i]) {
        const Particle<R>& q = ps[j];
        R d = dist(p.x, q.x);
        if (!(d < h)) continue;
        unsigned dl = dist_lut(d);
        if (q.type == UPF_LIQUID) {
          R kernelVisc = lut(L_VISC, d);
          V3<R> vij = p.v - q.v;
          p.F = p.F - vij * restVolume * restVolume * R(prm.viscosity) * kernelVisc;
          if ((prm.flags & UPF_FLAG_SURFACE_TENSION) && d >= h * R(0.25f)) {
            // CalculateSurfaceTensionForcePCISPHHost, UnifiedPhysics.cpp:1990-1998
            R spline = R(tab.lut[L_ST][dl]);
            p.F = p.F - (p.x - q.x) * R(prm.surface_tension_gamma) * m * m * spline * (R(1.0f) / d);
          }
        } else if (q.type == UPF_FROZEN || q.type == UPF_RIGID || q.type == UPF_GRANULAR) {
          // boundary-like neighbours (granular grains are treated as the
          // reference treats rigid particles); the liquid particle's own
          // weighted volume, as UnifiedPhysics.cpp:5292 passes
          if (prm.flags & UPF_FLAG_BOUNDARY_PRESSURE)
            p.F = p.F + boundary_pressure(d, p.x, q.x, p.rho_prev, p.p_prev, p.wvol);
          if ((prm.flags & UPF_FLAG_ADHESION) && d >= h * R(0.25f)) {
            // CalculateSurfaceCohesionForcePCISPHHost, UnifiedPhysics.cpp:2000-2008
            R spline = R(tab.lut[L_ADH][dl]);
            p.F = p.F - (p.x - q.x) * R(prm.surface_adhesion_beta) * m * rho0 * q.wvol * spline * (R(1.0f) / d);
          }
        }
      }
      p.F.y -= m * R(prm.gravity);
      if (prm.flags & UPF_FLAG_PENALTY_WALLS) p.F = p.F + penalty_walls(p.x);
    } else {
      // predicted position of a non-liquid particle: its current position.
      // Literal: nothing in the reference's coupling step writes a rigid
      // particle's predicted_position_, so it keeps the position it was
      // created with (UnifiedParticle.cpp:17), and the liquid's predicted
      // density sees the body where it started.
      if (!(p.type == UPF_RIGID && (literal & ORC_LITERAL_STALE_RIGID_PREDICTED))) p.xs = p.x;
      if (p.type == UPF_RIGID) rigid_external(i);
      else if (p.type == UPF_GRANULAR) granular_external(i);
    }
  }

  // CalculateBoundaryForcePerRigidParticleHost (UnifiedPhysics.cpp:2071-2131)
  V3<R> rigid_box_force(V3<R> x, V3<R> v) const {
    V3<R> f = {0, 0, 0};
    bool hit = false;
    const R r = R(prm.particle_radius), ks = R(prm.spring_coefficient_boundary), kd = R(prm.damping_coefficient);
    const R* xv = &x.x;
    R* fv = &f.x;
    for (int a = 0; a < 3; ++a) {
      const R mn = R(prm.collision_min[a]), mx = R(prm.collision_max[a]);
      if (xv[a] - r < mn) {
        hit = true;
        fv[a] += (mn + r - xv[a]) * ks;
      }
      if (xv[a] + r > mx) {
        hit = true;
        fv[a] += (R(-1.0f) * (xv[a] + r - mx)) * ks;
      }
    }
    if (hit) {
      f.x -= kd * v.x;
      f.y -= kd * v.y;
      f.z -= kd * v.z;
    }
    return f;
  }

  // Rigid branch of CalculateExternalForcesVersatilCouplingPCISPH
  // (UnifiedPhysics.cpp:5300-5326, 5344-5348). Deviations: spring-damper
  // contacts only between different bodies, as the reference's comment
  // intends (UnifiedPhysics.cpp:5307); the reaction of the boundary pressure
  // uses the liquid particle's lagged values, so the pair force is exactly
  // antisymmetric (the reference reads a value that other threads reset
  // concurrently).
  void rigid_external(int i) {
    Particle<R>& p = ps[i];
    const R m = R(prm.mass), h = R(prm.support_radius), rho0 = R(prm.rest_density);
    p.F = {0, 0, 0};
    for (int j : nbr[i]) {
      const Particle<R>& q = ps[j];
      R d = dist(p.x, q.x);
      if (!(d < h)) continue;
      unsigned dl = dist_lut(d);
      if (q.type == UPF_RIGID) {
        // literal: every rigid neighbour, the particle's own body included
        // (UnifiedPhysics.cpp:5300-5311)
        if (q.body == p.body && !(literal & ORC_LITERAL_OWN_BODY_SPRING)) continue;
        const R overlap = R(2.0f) * R(prm.particle_radius) - d;
        if (overlap > R(0.00001f)) {
          // CalculateSpringForceHost / CalculateDampingForceHost (UnifiedPhysics.cpp:2010-2030)
          const V3<R> rij = q.x - p.x;
          const R ks = R(prm.spring_coefficient), kd = R(prm.damping_coefficient);
          const V3<R> spring = {R(-1.0f) * ks * overlap * rij.x / d, R(-1.0f) * ks * overlap * rij.y / d,
                                R(-1.0f) * ks * overlap * rij.z / d};
          const V3<R> vij = q.v - p.v;
          const V3<R> damp = {kd * vij.x, kd * vij.y, kd * vij.z};
          p.F = p.F + (spring + damp);
        }
      } else if (q.type == UPF_LIQUID) {
        if (prm.flags & UPF_FLAG_BOUNDARY_PRESSURE)
          p.F = p.F - boundary_pressure(d, q.x, p.x, q.rho_prev, q.p_prev, q.wvol);
        if ((prm.flags & UPF_FLAG_ADHESION) && d >= h * R(0.25f)) {
          R spline = R(tab.lut[L_ADH][dl]);
          p.F = p.F + (q.x - p.x) * R(prm.surface_adhesion_beta) * m * rho0 * q.wvol * spline * (R(1.0f) / d);
        }
      }
    }
    p.F = p.F + rigid_box_force(p.x, p.v);
  }

  // Granular grains: the contact model of CalculateForcesWithContactForces
  // (UnifiedPhysics.cpp:3219-3338, Bell et al. 2005) against grains, rigid and
  // boundary particles closer than collisionDistThreshold = 2 r. Deviations:
  // the normal force is applied (the reference adds only the tangential one,
  // UnifiedPhysics.cpp:3287) and the friction bound uses |f_n| so friction
  // opposes slip. Liquid neighbours act on grains as on rigid particles;
  // gravity and the rigid box penalty act as on rigid particles.
  void granular_external(int i) {
    Particle<R>& p = ps[i];
    const R m = R(prm.mass), h = R(prm.support_radius), rho0 = R(prm.rest_density);
    const R dc = R(2.0f) * R(prm.particle_radius);
    p.F = {0, 0, 0};
    for (int j : nbr[i]) {
      const Particle<R>& q = ps[j];
      R d = dist(p.x, q.x);
      if (!(d < h)) continue;
      unsigned dl = dist_lut(d);
      if ((q.type == UPF_GRANULAR || q.type == UPF_RIGID || q.type == UPF_FROZEN) && d < dc) {
        const R ksi = std::max(dc - d, R(0.0f));
        V3<R> N = (p.x - q.x) * R(-1.0f);
        normalize(N);
        const V3<R> V = p.v - q.v;
        const R ksiDot = dot(V, N);
        V3<R> Vt = V - N * ksiDot;
        const R fn = -R(prm.granular_kd) * ksiDot - R(prm.granular_kr) * ksi;
        const V3<R> Fn = N * fn;
        const R vtl = normalize(Vt);
        if (literal & ORC_LITERAL_GRANULAR_TANGENTIAL_ONLY) {
          // literal (UnifiedPhysics.cpp:3276-3287): the friction bound uses
          // the signed f_n and only F_t is added
          const R t = std::min(R(prm.granular_mu) * fn, R(prm.granular_kt) * vtl);
          p.F = p.F + Vt * (-t);
        } else {
          const R t = std::min(R(prm.granular_mu) * std::fabs(fn), R(prm.granular_kt) * vtl);
          const V3<R> Ft = Vt * (-t);
          p.F = p.F + (Fn + Ft);
        }
      } else if (q.type == UPF_LIQUID) {
        if (prm.flags & UPF_FLAG_BOUNDARY_PRESSURE)
          p.F = p.F - boundary_pressure(d, q.x, p.x, q.rho_prev, q.p_prev, q.wvol);
        if ((prm.flags & UPF_FLAG_ADHESION) && d >= h * R(0.25f)) {
          R spline = R(tab.lut[L_ADH][dl]);
          p.F = p.F + (q.x - p.x) * R(prm.surface_adhesion_beta) * m * rho0 * q.wvol * spline * (R(1.0f) / d);
        }
      }
    }
    p.F.y -= m * R(prm.gravity);
    p.F = p.F + rigid_box_force(p.x, p.v);
  }

  // RigidBodyIntegrationOMP -> CalculateRigidBodyForceTorqueMomenta
  // (UnifiedPhysics.cpp:3620-3703) with RigidBody::UpdateMomenta, PerformStep,
  // UpdateRotationMatrix (RigidBody.cpp:15-161). Force and torque are summed
  // in FP64 (particles in array order, gravity after each particle's force);
  // the body update is float as in the reference. The quaternion is not
  // renormalised (RigidBody.cpp:99 discards getNormalized()'s result).
  void rigid_step() {
    const int nb = (int)bodies.size();
    if (!nb) return;
    if (literal & ORC_LITERAL_FLOAT_BODY_SUMS) {
      // literal: RigidBody::ApplyForce / ApplyTorque (RigidBody.cpp:16-19)
      // add each particle's force, its torque about the body's position, then
      // the particle's weight, in the precision of the state
      std::vector<V3<R>> F(nb, V3<R>{0, 0, 0}), T(nb, V3<R>{0, 0, 0});
      for (const Particle<R>& p : ps) {
        if (p.type != UPF_RIGID || p.body < 0) continue;
        F[p.body] = F[p.body] + p.F;
        T[p.body] = T[p.body] + cross(p.x - bodies[p.body].pos, p.F);
        F[p.body] = F[p.body] + V3<R>{R(0), -R(prm.mass) * R(prm.gravity), R(0)};
      }
      for (int k = 0; k < nb; ++k) body_update(bodies[k], F[k], T[k], R(prm.dt), R(prm.terminal_speed));
      return;
    }
    std::vector<double> F(3 * nb, 0.0), T(3 * nb, 0.0);
    for (const Particle<R>& p : ps) {
      if (p.type != UPF_RIGID || p.body < 0) continue;
      const Body<R>& b = bodies[p.body];
      double* f = &F[3 * p.body];
      double* t = &T[3 * p.body];
      const double fx = p.F.x, fy = p.F.y, fz = p.F.z;
      const double rx = (double)p.x.x - (double)b.pos.x, ry = (double)p.x.y - (double)b.pos.y,
                   rz = (double)p.x.z - (double)b.pos.z;
      f[0] += fx;
      f[1] += fy;
      f[2] += fz;
      t[0] += ry * fz - rz * fy;
      t[1] += rz * fx - rx * fz;
      t[2] += rx * fy - ry * fx;
      f[1] += (double)(-R(prm.mass) * R(prm.gravity));
    }
    for (int k = 0; k < nb; ++k) {
      const V3<R> force = {R(F[3 * k]), R(F[3 * k + 1]), R(F[3 * k + 2])};
      const V3<R> torque = {R(T[3 * k]), R(T[3 * k + 1]), R(T[3 * k + 2])};
      body_update(bodies[k], force, torque, R(prm.dt), R(prm.terminal_speed));
    }
  }

  // SynRigidParticlesPerRigidBody, new method (UnifiedPhysics.cpp:3766-3782)
  void rigid_sync() {
    if (bodies.empty()) return;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 100)
    for (int i = 0; i < (int)ps.size(); i++) {
      Particle<R>& p = ps[i];
      if (p.type != UPF_RIGID || p.body < 0) continue;
      const Body<R>& b = bodies[p.body];
      const V3<R> rel = mat_vec(b.rot, p.r0);
      p.v = b.vel + cross(b.omega, rel);
      p.x = b.pos + rel;
    }
  }

  void predict(Particle<R>& p) {  // PredictPositionAndVelocity, UnifiedPhysics.cpp:5426-5454
    if (p.type != UPF_LIQUID) return;
    p.vs = p.v + divs((p.F + p.Fp) * R(prm.dt), R(prm.mass));
    p.xs = p.x + p.vs * R(prm.dt);
    // CollisionHandling (UnifiedPhysics.cpp:5739-5757), damping 0
    R* x = &p.xs.x;
    R* v = &p.vs.x;
    for (int a = 0; a < 3; a++) {
      if (x[a] < R(prm.collision_min[a])) { x[a] = R(prm.collision_min[a]); v[a] *= R(0.0); }
      if (x[a] > R(prm.collision_max[a])) { x[a] = R(prm.collision_max[a]); v[a] *= R(0.0); }
    }
    p.rho_star = 0;
  }

  R predicted_density(int i) {  // ComputePredictedDensityAndPressure, UnifiedPhysics.cpp:5456-5491
    Particle<R>& p = ps[i];
    const R m = R(prm.mass);
    p.rho_star = R(tab.kernel_self) * m;
    for (int j : nbr[i]) {
      R d = dist(p.xs, ps[j].xs);
      if (d < R(prm.support_radius)) {
        R kv = lut(L_M4, d);
        p.rho_star += kv * m;
      }
    }
    p.err = std::max(p.rho_star - R(prm.rest_density), R(0));
    p.p_corr += std::max(p.err * R(prm.density_error_factor), R(0));
    return p.rho_star;
  }

  void pressure_force(int i) {  // ComputeCorrectivePressureForce, UnifiedPhysics.cpp:5493-5522
    Particle<R>& p = ps[i];
    const R m = R(prm.mass), rho0 = R(prm.rest_density);
    p.Fp = {0, 0, 0};
    R densSq = rho0 * rho0;
    R pi = p.p_corr;
    for (int j : nbr[i]) {
      const Particle<R>& q = ps[j];
      R d = dist(p.x, q.x);
      if (d < R(prm.support_radius)) {
        R pj = q.p_corr;
        R kgv = lut(L_PGRAD, d);
        V3<R> kg = (p.x - q.x) * kgv;
        R grad = pi / densSq + pj / (rho0 * rho0);
        p.Fp = p.Fp - kg * grad * m * m;
      }
    }
  }

  int step_pcisph(orc_step_info* info) {
    const int n = (int)ps.size();
    find_neighbors();
#pragma omp parallel for num_threads(threads) schedule(dynamic, 100)
    for (int i = 0; i < n; i++) pcisph_external(i);
    // lagged state (UnifiedPhysics.cpp:5360-5363)
    for (int i = 0; i < n; i++) {
      Particle<R>& p = ps[i];
      p.p_prev = p.p_corr;
      p.p_corr = 0;
      p.Fp = {0, 0, 0};
    }
    // PredictionCorrectionStep (UnifiedPhysics.cpp:5367-5424). The maximum is
    // a proper reduction (the reference races on max_predicted_density_).
    bool too_large = true;
    int it = 0;
    R maxd = 0;
    R errpct = 0;
    while (it < prm.min_loops || (too_large && it < prm.max_loops)) {
#pragma omp parallel for num_threads(threads) schedule(dynamic, 100)
      for (int i = 0; i < n; i++) predict(ps[i]);
      maxd = 0;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 100) reduction(max : maxd)
      for (int i = 0; i < n; i++) {
        if (ps[i].type != UPF_LIQUID) continue;
        R d = predicted_density(i);
        maxd = std::max(maxd, d);
      }
      // MAX(0.1f * max - 100.0f, 0) with rest density 1000; 100/rho0 in general
      const R scale = R(100.0f / prm.rest_density);
      errpct = std::max(scale * maxd - R(100.0f), R(0.0f));
      if (info && it < 64) info->iteration_max_density[it] = float(maxd);
      if (errpct < R(prm.max_density_error)) too_large = false;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 100)
      for (int i = 0; i < n; i++)
        if (ps[i].type == UPF_LIQUID) pressure_force(i);
      it++;
    }
    for (int i = 0; i < n; i++) ps[i].rho_prev = ps[i].rho_star;
    if (keep_fields) snapshot = ps;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 100)
    for (int i = 0; i < n; i++) integrate(ps[i]);
    // BoundaryHandlingPureFluidOMP (UnifiedPhysics.cpp:3972-3998)
    const R damping = R(-0.5);
#pragma omp parallel for num_threads(threads) schedule(dynamic, 100)
    for (int i = 0; i < n; i++) {
      Particle<R>& p = ps[i];
      if (p.type == UPF_LIQUID || p.type == UPF_GRANULAR) clamp_box(p.x, p.v, damping);
    }
    // RigidBodyIntegrationOMP + SynRigidParticlesOMP (UnifiedPhysics.cpp:5011-5023).
    // Keys are taken after the rigid particles move. Literal: the reference
    // keys every particle in BoundaryHandlingPureFluidOMP
    // (UnifiedPhysics.cpp:3995), before the rigid phase, so its sort and next
    // neighbour search use the rigid particles' keys from before the sync.
    const bool stale_keys = (literal & ORC_LITERAL_STALE_RIGID_KEYS) != 0;
    if (stale_keys) {
#pragma omp parallel for num_threads(threads) schedule(dynamic, 100)
      for (int i = 0; i < n; i++) ps[i].key = key_of(ps[i].x);
    }
    rigid_step();
    rigid_sync();
    if (!stale_keys) {
#pragma omp parallel for num_threads(threads) schedule(dynamic, 100)
      for (int i = 0; i < n; i++) ps[i].key = key_of(ps[i].x);
    }
    finish_step_stats(info);
    sort_particles();
    if (info) {
      info->iterations = it;
      info->max_predicted_density = float(maxd);
      info->density_error_percent = float(errpct);
    }
    return 0;
  }

  int step(orc_step_info* info) override {
    if (prm.method == UPF_METHOD_WCSPH) return step_wcsph(info);
    if (prm.method == UPF_METHOD_PCISPH) return step_pcisph(info);
    return -1;
  }

  uint32_t count() const override { return (uint32_t)ps.size(); }

  // Resume a PCISPH run from another run's state, per particle in creation
  // order: the final correction pressure of the step before last (what the
  // next step's external forces read as previous_correction_pressure_), of
  // the last step (which becomes it after them, UnifiedPhysics.cpp:5360-5363),
  // and the last step's predicted density.
  void set_lagged(const float* pressure_prev, const float* pressure, const float* density) override {
    for (Particle<R>& p : ps) {
      p.p_prev = R(pressure_prev[p.id]);
      p.p_corr = R(pressure[p.id]);
      p.rho_star = p.rho_prev = R(density[p.id]);
    }
  }

  void get_lagged(float* pressure_prev, float* pressure, float* density) const override {
    for (const Particle<R>& p : ps) {
      pressure_prev[p.id] = float(p.p_prev);
      pressure[p.id] = float(p.p_corr);
      density[p.id] = float(p.rho_prev);
    }
  }

  void get(float* pos4, float* vel4, float* density, float* pressure, int32_t* type, uint32_t* id,
           uint32_t* key) const override {
    for (size_t i = 0; i < ps.size(); ++i) {
      const Particle<R>& p = ps[i];
      if (pos4) { pos4[4 * i] = float(p.x.x); pos4[4 * i + 1] = float(p.x.y); pos4[4 * i + 2] = float(p.x.z); pos4[4 * i + 3] = 0; }
      if (vel4) { vel4[4 * i] = float(p.v.x); vel4[4 * i + 1] = float(p.v.y); vel4[4 * i + 2] = float(p.v.z); vel4[4 * i + 3] = 0; }
      if (density) density[i] = float(prm.method == UPF_METHOD_PCISPH ? p.rho_star : p.density);
      if (pressure) pressure[i] = float(prm.method == UPF_METHOD_PCISPH ? p.p_corr : p.pressure);
      if (type) type[i] = p.type;
      if (id) id[i] = p.id;
      if (key) key[i] = p.key;
    }
  }

  void get_fields(float* f4, float* fp4, float* rs, float* pc, float* den, float* pr,
                  uint32_t* id) const override {
    for (size_t i = 0; i < snapshot.size(); ++i) {
      const Particle<R>& p = snapshot[i];
      if (f4) { f4[4 * i] = float(p.F.x); f4[4 * i + 1] = float(p.F.y); f4[4 * i + 2] = float(p.F.z); f4[4 * i + 3] = 0; }
      if (fp4) { fp4[4 * i] = float(p.Fp.x); fp4[4 * i + 1] = float(p.Fp.y); fp4[4 * i + 2] = float(p.Fp.z); fp4[4 * i + 3] = 0; }
      if (rs) rs[i] = float(p.rho_star);
      if (pc) pc[i] = float(p.p_corr);
      if (den) den[i] = float(p.density);
      if (pr) pr[i] = float(p.pressure);
      if (id) id[i] = p.id;
    }
  }

  uint32_t neighbors(uint32_t* offsets, uint32_t* ids, uint32_t cap) override {
    find_neighbors();
    uint32_t off = 0;
    for (size_t i = 0; i < ps.size(); ++i) {
      if (offsets) offsets[i] = off;
      for (int j : nbr[i]) {
        if (ids && off < cap) ids[off] = ps[j].id;
        off++;
      }
    }
    if (offsets) offsets[ps.size()] = off;
    return off;
  }

  void set_keep_fields(bool on) override { keep_fields = on; }
  void set_literal(uint32_t mask) override { literal = mask; }
  // Rigid body assembly (AddToRigidBody UnifiedPhysics.cpp:825-885, inverse
  // Matrix3x3::CalculateInverse Matrix3x3.cpp:121-156, relative positions
  // UnifiedPhysics.cpp:150-158): mass, centre of mass, momenta and inertia are
  // summed in FP64 over the body's particles in input order and the inertia
  // is inverted in FP64 (the reference sums incrementally in float and its
  // ComputeLocalInertiaTensorRigidBody indexes particles_[i] for indices[i]).
  // The inverse is stored as the body's local inverse inertia: the reference
  // writes it into the temporary that inverted_inertia_local() returns
  // (UnifiedPhysics.cpp:150), so its bodies keep a zero inverse inertia and
  // never rotate.
  int set_bodies(const int32_t* bop, uint32_t n, uint32_t nb) override {
    if (n != ps.size()) return -1;
    std::vector<int> where(n);
    for (size_t k = 0; k < ps.size(); ++k) where[ps[k].id] = (int)k;
    const double m = prm.mass;
    std::vector<double> M(nb, 0.0), C(3 * nb, 0.0), Pm(3 * nb, 0.0), I(9 * nb, 0.0), L(3 * nb, 0.0);
    for (uint32_t id = 0; id < n; ++id) {
      const int b = bop[id];
      if (b < 0) continue;
      if (b >= (int)nb || ps[where[id]].type != UPF_RIGID) return -2;
      const Particle<R>& p = ps[where[id]];
      M[b] += m;
      C[3 * b] += m * (double)p.x.x;
      C[3 * b + 1] += m * (double)p.x.y;
      C[3 * b + 2] += m * (double)p.x.z;
      Pm[3 * b] += m * (double)p.v.x;
      Pm[3 * b + 1] += m * (double)p.v.y;
      Pm[3 * b + 2] += m * (double)p.v.z;
    }
    for (uint32_t b = 0; b < nb; ++b)
      if (M[b] > 0)
        for (int a = 0; a < 3; ++a) C[3 * b + a] /= M[b];
    for (uint32_t id = 0; id < n; ++id) {
      const int b = bop[id];
      if (b < 0) continue;
      const Particle<R>& p = ps[where[id]];
      const double r[3] = {(double)p.x.x - C[3 * b], (double)p.x.y - C[3 * b + 1], (double)p.x.z - C[3 * b + 2]};
      const double v[3] = {m * (double)p.v.x, m * (double)p.v.y, m * (double)p.v.z};
      const double rr = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) I[9 * b + 3 * i + j] += m * ((i == j ? rr : 0.0) - r[i] * r[j]);
      L[3 * b] += r[1] * v[2] - r[2] * v[1];
      L[3 * b + 1] += r[2] * v[0] - r[0] * v[2];
      L[3 * b + 2] += r[0] * v[1] - r[1] * v[0];
    }
    bodies.assign(nb, Body<R>());
    for (uint32_t b = 0; b < nb; ++b) {
      Body<R>& B = bodies[b];
      std::memset(&B, 0, sizeof(B));
      double inv[9] = {0};
      inverse3_fp64(&I[9 * b], inv);
      B.mass = R(M[b]);
      B.pos = {R(C[3 * b]), R(C[3 * b + 1]), R(C[3 * b + 2])};
      B.P = {R(Pm[3 * b]), R(Pm[3 * b + 1]), R(Pm[3 * b + 2])};
      B.vel = M[b] > 0 ? V3<R>{R(Pm[3 * b] / M[b]), R(Pm[3 * b + 1] / M[b]), R(Pm[3 * b + 2] / M[b])}
                       : V3<R>{0, 0, 0};
      B.L = {R(L[3 * b]), R(L[3 * b + 1]), R(L[3 * b + 2])};
      B.q[0] = 1;
      for (int i = 0; i < 3; ++i) {
        B.rot[i][i] = 1;
        // literal: CalculateInverse writes into the temporary that
        // inverted_inertia_local() returns (UnifiedPhysics.cpp:150), so the
        // body's local inverse inertia keeps its zero initial value
        for (int j = 0; j < 3; ++j)
          B.inv_inertia_local[i][j] = (literal & ORC_LITERAL_ZERO_INVERSE_INERTIA) ? R(0) : R(inv[3 * i + j]);
      }
    }
    if (literal & ORC_LITERAL_FLOAT_RIGID_ASSEMBLY) {
      // literal: AddToRigidBody (UnifiedPhysics.cpp:825-885) for each rigid
      // particle in array order, in the precision of the state, on a body the
      // RigidBody constructor zeroed (RigidBody.cpp:4-13). The linear momentum
      // is never set there, so it stays zero; the angular momentum update on
      // the temporary angular_momentum() returns (:871) has no effect.
      std::vector<R> In(9 * nb, R(0));
      for (uint32_t b = 0; b < nb; ++b) {
        Body<R>& B = bodies[b];
        B.mass = 0;
        B.pos = B.vel = B.P = B.L = V3<R>{0, 0, 0};
      }
      for (size_t k = 0; k < ps.size(); ++k) {
        const Particle<R>& p = ps[k];
        const int b = bop[p.id];
        if (b < 0) continue;
        Body<R>& B = bodies[b];
        R* I = &In[9 * b];
        const R pm = R(prm.mass);
        const R nm = B.mass + pm;
        const V3<R> c = divs(B.pos * B.mass + p.x * pm, nm);
        const V3<R> dc = B.pos - c, dp = p.x - c;
        const R c0 = dc.x * dc.x, c1 = dc.y * dc.y, c2 = dc.z * dc.z;
        const R q0 = dp.x * dp.x, q1 = dp.y * dp.y, q2 = dp.z * dp.z;
        I[0] += B.mass * (c1 + c2) + pm * (q1 + q2);
        I[4] += B.mass * (c0 + c2) + pm * (q0 + q2);
        I[8] += B.mass * (c1 + c0) + pm * (q1 + q0);
        I[1] -= B.mass * dc.x * dc.y + pm * dp.x * dp.y;
        I[2] -= B.mass * dc.x * dc.z + pm * dp.x * dp.z;
        I[5] -= B.mass * dc.y * dc.z + pm * dp.y * dp.z;
        I[3] = I[1];
        I[6] = I[2];
        I[7] = I[5];
        B.L = B.L + cross(dc, B.vel * B.mass);
        B.vel = divs(B.vel * B.mass + p.v * pm, nm);
        B.pos = c;
        B.mass = nm;
      }
      for (uint32_t b = 0; b < nb; ++b) {
        Body<R>& B = bodies[b];
        double I64[9], inv[9] = {0};
        for (int a = 0; a < 9; ++a) I64[a] = (double)In[9 * b + a];
        inverse3_fp64(I64, inv);
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j)
            B.inv_inertia_local[i][j] = (literal & ORC_LITERAL_ZERO_INVERSE_INERTIA) ? R(0) : R(inv[3 * i + j]);
      }
    }
    for (uint32_t id = 0; id < n; ++id) {
      const int b = bop[id];
      Particle<R>& p = ps[where[id]];
      p.body = b;
      if (b >= 0) p.r0 = p.x - bodies[b].pos;
    }
    return 0;
  }

  int get_rigid(float* pos3, float* vel3, float* omega3, float* quat4) const override {
    for (size_t b = 0; b < bodies.size(); ++b) {
      const Body<R>& B = bodies[b];
      if (pos3) { pos3[3 * b] = float(B.pos.x); pos3[3 * b + 1] = float(B.pos.y); pos3[3 * b + 2] = float(B.pos.z); }
      if (vel3) { vel3[3 * b] = float(B.vel.x); vel3[3 * b + 1] = float(B.vel.y); vel3[3 * b + 2] = float(B.vel.z); }
      if (omega3) { omega3[3 * b] = float(B.omega.x); omega3[3 * b + 1] = float(B.omega.y); omega3[3 * b + 2] = float(B.omega.z); }
      if (quat4) for (int k = 0; k < 4; ++k) quat4[4 * b + k] = float(B.q[k]);
    }
    return (int)bodies.size();
  }
};

// FP32 restatement of ComputeDensityErrorFactor (UnifiedPhysics.cpp:5525-5689)
// on the prototype block of CreatePreParticlesISPH (UnifiedPhysics.cpp:5577-5606).
template <class A>
double density_error_factor_impl(const upf_params& p) {
  const float spacing = p.particle_spacing;
  const float h = p.support_radius;
  // prototype block: [-0.1,0,-0.1]..[0.1,0.2,0.1] scaled by spacing/0.0125
  float mn[3], mx[3];
  if ((double)spacing == 0.0125) {
    // float vs double literal: never true for a float spacing, as in the
    // reference (UnifiedPhysics.cpp:5589-5593)
    mn[0] = mn[1] = mn[2] = 0;
    mx[0] = mx[1] = mx[2] = 0;
  } else {
    float scale = spacing / 0.0125;
    mn[0] = -0.1f * scale; mn[1] = 0.0f * scale; mn[2] = -0.1f * scale;
    mx[0] = 0.1f * scale; mx[1] = 0.2f * scale; mx[2] = 0.1f * scale;
  }
  // CreatePartilcesCPU (UnifiedPhysics.cpp:2134-2199) with jitter 0
  int num[3];
  for (int a = 0; a < 3; ++a) num[a] = int((mx[a] - mn[a]) / spacing);
  struct PP {
    float x[3];
    uint32_t key;
  };
  upf_params q = p;
  Tables tab;
  BuildTables(q, tab);
  std::vector<PP> v;
  for (int iy = 0; iy < num[1]; iy++) {
    float y = 0.0f + iy * spacing;
    for (int ix = 0; ix < num[0]; ix++) {
      float x = 0.0f + ix * spacing;
      for (int iz = 0; iz < num[2]; iz++) {
        float z = 0.0f + iz * spacing;
        PP pp;
        pp.x[0] = x; pp.x[1] = y; pp.x[2] = z;
        uint32_t k = 0;
        for (int a = 0; a < 3; ++a) {
          float c = p.scales[a] * (pp.x[a] - p.zindex_origin[a]);
          int u = (c <= 0) ? 0 : (c >= 1023 ? 1023 : (int)(unsigned short)c);
          k |= tab.ztab[u][a];
        }
        pp.key = k;
        v.push_back(pp);
      }
    }
  }
  std::stable_sort(v.begin(), v.end(), [](const PP& a, const PP& b) { return a.key < b.key; });
  const int n = (int)v.size();
  // neighbour sets: every pair closer than h (the box query is a superset),
  // in ascending sorted index like GetNeighbors
  std::vector<A> sgx(n, 0), sgy(n, 0), sgz(n, 0), sdot(n, 0);
  std::vector<int> ncount(n, 0);
  auto fdist = [&](int i, int j) {
    float dx = v[i].x[0] - v[j].x[0], dy = v[i].x[1] - v[j].x[1], dz = v[i].x[2] - v[j].x[2];
    return sqrtf(dx * dx + dy * dy + dz * dz);
  };
  // ComputeGradWValues (UnifiedPhysics.cpp:5546-5575): each pair is visited
  // from both ends and accumulated into both particles.
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      float d = fdist(i, j);
      if (!(d < h)) continue;
      ncount[i]++;
      A g = A(KernelPressureGrad(d, h));
      A gx = A(v[i].x[0] - v[j].x[0]) * g;
      A gy = A(v[i].x[1] - v[j].x[1]) * g;
      A gz = A(v[i].x[2] - v[j].x[2]) * g;
      sgx[i] += gx; sgy[i] += gy; sgz[i] += gz;
      sgx[j] -= gx; sgy[j] -= gy; sgz[j] -= gz;
      A gg = gx * gx + gy * gy + gz * gz;
      sdot[i] += gg;
      A ngx = gx * A(-1.0), ngy = gy * A(-1.0), ngz = gz * A(-1.0);
      sdot[j] += ngx * ngx + ngy * ngy + ngz * ngz;
    }
  }
  // ComputeFactor (UnifiedPhysics.cpp:5638-5689)
  int best = 0, maxn = 0;
  for (int i = 0; i < n; ++i)
    if (ncount[i] > maxn) { maxn = ncount[i]; best = i; }
  A restVol = A(p.mass) / A(p.rest_density);
  A preFactor = restVol * restVol * A(p.dt) * A(p.dt);
  A gradWTerm = ((sgx[best] * A(-1.0)) * sgx[best] + (sgy[best] * A(-1.0)) * sgy[best] +
                 (sgz[best] * A(-1.0)) * sgz[best]) - sdot[best];
  A divisor = preFactor * gradWTerm;
  if (divisor == 0) return 0.0;
  A fudge = A(p.density_error_fudge);
  A delta = A(-1.0 / divisor);
  delta *= fudge;
  return double(delta);
}

}  // namespace

struct orc_sim {
  SimBase* impl;
};

extern "C" {

void orc_default_params(upf_params* p) {
  // UnifiedConstants::UnifiedConstants (UnifiedConstants.cpp:7-159) with the
  // spacing setter (UnifiedConstants.cpp:162-191) and the virtual box
  // (UnifiedConstants.cpp:308-320).
  std::memset(p, 0, sizeof(*p));
  p->method = UPF_METHOD_PCISPH;
  p->flags = UPF_FLAG_SURFACE_TENSION | UPF_FLAG_PENALTY_WALLS;
  float spacing = 1.0 / 40.0;
  p->particle_spacing = spacing;
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
  p->zindex_extent[0] = 2.0f; p->zindex_extent[1] = 2.0f; p->zindex_extent[2] = 1.5f;
  p->max_neighbors = 128;
}

int orc_params_derive(upf_params* p) {
  if (!(p->particle_spacing > 0)) return -1;
  if (p->particle_radius == 0) p->particle_radius = p->particle_spacing * 0.5f;
  if (p->support_radius == 0) p->support_radius = p->particle_spacing * 2.0 * 1.00001;
  if (p->mass == 0) p->mass = p->particle_spacing * p->particle_spacing * p->particle_spacing * p->rest_density;
  if (p->force_distance == 0) p->force_distance = 0.25 * p->support_radius;
  if (p->max_boundary_force == 0) p->max_boundary_force = 1.0f * 64 * p->particle_spacing * p->particle_spacing;
  for (int a = 0; a < 3; ++a)
    if (p->scales[a] == 0) p->scales[a] = float(UPF_GRID_RESOLUTION) / p->zindex_extent[a];
  if (p->block_size == 0) {
    // UnifiedPhysics.cpp:2149-2156 and ZIndex::SetBlockSize (zIndex.cpp:27-39);
    // the float is passed to an int parameter (truncation).
    float mb = p->scales[0] * p->support_radius;
    mb = std::max(mb, p->scales[1] * p->support_radius);
    mb = std::max(mb, p->scales[2] * p->support_radius);
    int size = (int)mb;
    unsigned bs;
    for (bs = 1; (int)bs < size; bs *= 2) {
    }
    p->block_size = bs;
  }
  if (p->density_error_fudge < 0) {
    // UnifiedConstants.cpp:101-103
    const float factor = p->dt / 0.0002f;
    p->density_error_fudge = 0.05 * factor * factor;
  }
  if (p->max_neighbors == 0) p->max_neighbors = 128;
  if (p->method == UPF_METHOD_PCISPH && p->density_error_factor == 0)
    p->density_error_factor = float(density_error_factor_impl<float>(*p));
  return 0;
}

double orc_density_error_factor(const upf_params* p, int fp64) {
  return fp64 ? density_error_factor_impl<double>(*p) : density_error_factor_impl<float>(*p);
}

void orc_build_luts(const upf_params* p, float* out) {
  Tables t;
  BuildTables(*p, t);
  std::memcpy(out, t.lut, sizeof(t.lut));
}

void orc_morton_table(uint32_t* out) {
  upf_params p;
  orc_default_params(&p);
  p.support_radius = 1.0f;
  Tables t;
  BuildTables(p, t);
  std::memcpy(out, t.ztab, sizeof(t.ztab));
}

uint32_t orc_morton(const upf_params* p, float x, float y, float z) {
  Sim<float> s(*p, nullptr, nullptr, nullptr, 0, 1);
  return s.key_of({x, y, z});
}

int orc_box_query(uint32_t block_size, const uint16_t mn[3], const uint16_t mx[3], uint32_t* first,
                  uint32_t* last, int cap) {
  std::vector<std::pair<uint32_t, uint32_t>> r;
  Sim<float>::box_query(block_size, mn, mx, r);
  int n = (int)r.size();
  for (int i = 0; i < n && i < cap; ++i) {
    first[i] = r[i].first;
    last[i] = r[i].second;
  }
  return n;
}

orc_sim* orc_create(const upf_params* p, const float* pos4, const float* vel4, const int32_t* type,
                    uint32_t n, int fp64, int threads) {
  if (threads <= 0) threads = omp_get_max_threads();
  orc_sim* s = new orc_sim;
  if (fp64)
    s->impl = new Sim<double>(*p, pos4, vel4, type, n, threads);
  else
    s->impl = new Sim<float>(*p, pos4, vel4, type, n, threads);
  return s;
}

void orc_destroy(orc_sim* s) {
  if (!s) return;
  delete s->impl;
  delete s;
}

int orc_set_rigid_bodies(orc_sim* s, const int32_t* b, uint32_t n, uint32_t nb) {
  return s->impl->set_bodies(b, n, nb);
}

int orc_step(orc_sim* s, orc_step_info* info) {
  if (info) std::memset(info, 0, sizeof(*info));
  return s->impl->step(info);
}

uint32_t orc_count(const orc_sim* s) { return s->impl->count(); }

void orc_keep_fields(orc_sim* s, int on) { s->impl->set_keep_fields(on != 0); }

void orc_set_reference_literal(orc_sim* s, uint32_t mask) { s->impl->set_literal(mask); }

void orc_set_lagged(orc_sim* s, const float* pressure_prev, const float* pressure, const float* density) {
  s->impl->set_lagged(pressure_prev, pressure, density);
}

void orc_get_lagged(const orc_sim* s, float* pressure_prev, float* pressure, float* density) {
  s->impl->get_lagged(pressure_prev, pressure, density);
}

void orc_get(const orc_sim* s, float* pos4, float* vel4, float* density, float* pressure,
             int32_t* type, uint32_t* id, uint32_t* key) {
  s->impl->get(pos4, vel4, density, pressure, type, id, key);
}

void orc_get_step_fields(const orc_sim* s, float* force4, float* pforce4, float* rs, float* pc,
                         float* den, float* pr, uint32_t* id) {
  s->impl->get_fields(force4, pforce4, rs, pc, den, pr, id);
}

uint32_t orc_neighbors(orc_sim* s, uint32_t* offsets, uint32_t* ids, uint32_t cap) {
  return s->impl->neighbors(offsets, ids, cap);
}

int orc_get_rigid(const orc_sim* s, float* pos3, float* vel3, float* omega3, float* quat4) {
  return s->impl->get_rigid(pos3, vel3, omega3, quat4);
}

int orc_inverse3(const float* in9, float* out9) {
  double a[9], inv[9] = {0};
  for (int i = 0; i < 9; ++i) a[i] = in9[i];
  const bool ok = inverse3_fp64(a, inv);
  for (int i = 0; i < 9; ++i) out9[i] = (float)inv[i];
  return ok ? 1 : 0;
}

void orc_rigid_body_step(float* st, const float* force3, const float* torque3, float dt, float terminal_speed) {
  Body<float> b;
  const float* q = st;
  auto v3 = [&](V3<float>& v) { v = {q[0], q[1], q[2]}; q += 3; };
  auto m3 = [&](float m[3][3]) { for (int i = 0; i < 9; ++i) m[i / 3][i % 3] = q[i]; q += 9; };
  b.mass = *q++;
  v3(b.pos); v3(b.vel); v3(b.P); v3(b.L); v3(b.omega);
  for (int k = 0; k < 4; ++k) b.q[k] = *q++;
  m3(b.rot); m3(b.inv_inertia_local); m3(b.inv_inertia_world);
  body_update(b, V3<float>{force3[0], force3[1], force3[2]}, V3<float>{torque3[0], torque3[1], torque3[2]}, dt,
              terminal_speed);
  float* o = st;
  auto w3 = [&](const V3<float>& v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; o += 3; };
  auto n3 = [&](const float m[3][3]) { for (int i = 0; i < 9; ++i) o[i] = m[i / 3][i % 3]; o += 9; };
  *o++ = b.mass;
  w3(b.pos); w3(b.vel); w3(b.P); w3(b.L); w3(b.omega);
  for (int k = 0; k < 4; ++k) *o++ = b.q[k];
  n3(b.rot); n3(b.inv_inertia_local); n3(b.inv_inertia_world);
}

}  // extern "C"
