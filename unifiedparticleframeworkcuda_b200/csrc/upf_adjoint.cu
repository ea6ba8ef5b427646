// upf_adjoint.cu — the differentiation form (include/upf.h, upf_adjoint_*):
// a differentiable PCISPH trajectory and its hand-written adjoint.
//
// Forward step (LIQUID particles, in the Morton order of the step):
//   F_i  = -sum_j (v_i - v_j) V0^2 mu L(r_ij) - m g y          (viscosity, gravity)
//   k = 1..K:  v*_i = v_i + (F_i + Fp_i^{k-1}) dt / m,  x*_i = x_i + v*_i dt
//              rho_i^k = m W(0) + sum_j m W(|x*_i - x*_j|)
//              p_i^k = p_i^{k-1} + delta smax(rho_i^k - rho0)
//              (smax(d) = 0.5 (d + sqrt(d^2 + eps^2)): max(d, 0) smoothed)
//              Fp_i^k = -sum_j m^2 (p_i^k + p_j^k) / rho0^2 (x_i - x_j) G(r_ij)
//   v' = v + (F + Fp^K) dt / m,  x' = x + v' dt
// with the reference's kernel functions evaluated analytically (W: M4 cubic
// spline, WeightingKernel::KernelM4; G: the spiky gradient factor,
// kernelPressureGrad; L: the viscosity Laplacian, kernelViscosityLaplacian;
// WeightingKernel.cpp:75-200) and the formulas of
// CalculateExternalForcesPCISPH / PredictionCorrectionStep /
// ComputeCorrectivePressureForce (UnifiedPhysics.cpp:5165-5522).
//
// Every forward pass has an adjoint kernel (k_ab_*). Pair terms are
// symmetric (j in N(i) iff i in N(j)), so each adjoint is a gather over the
// particle's own list with no atomics. The trajectory's state is stored every
// `checkpoint_interval` steps; the backward pass recomputes each interval
// from its checkpoint, keeping that interval's per-step lists and
// intermediates (perm, lists, x, v, F, x*^k, rho^k, p^k) in HBM, then runs the
// interval's adjoint steps in reverse.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "upf_sys.h"

namespace upf {

namespace {

#define UPF_CUDA(call)                                                                       \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) {                                                                 \
      set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
      return UPF_ERR_CUDA;                                                                   \
    }                                                                                        \
  } while (0)

#define UPF_TRY(call)              \
  do {                             \
    upf_status st_ = (call);       \
    if (st_ != UPF_OK) return st_; \
  } while (0)

constexpr int kT = 256;  // threads per CTA of the adjoint kernels

// analytic kernel functions of support h (WeightingKernel.cpp:75-200)
struct AK {
  float h, inv_h;
  float w_norm;  // 8 / (pi h^3): KernelM4's factor 2.546479089470325472 / h^3
  float g_c;     // -45 / (pi h^6)
  float l_c;     // 45 / (pi h^6)
};

__device__ __forceinline__ float kW(const AK& k, float r) {
  const float s = r * k.inv_h;
  if (s >= 1.0f) return 0.0f;
  if (s < 0.5f) return k.w_norm * (1.0f - 6.0f * s * s + 6.0f * s * s * s);
  const float t = 1.0f - s;
  return k.w_norm * 2.0f * t * t * t;
}
__device__ __forceinline__ float kdW(const AK& k, float r) {  // dW/dr
  const float s = r * k.inv_h;
  if (s >= 1.0f) return 0.0f;
  if (s < 0.5f) return k.w_norm * k.inv_h * (-12.0f * s + 18.0f * s * s);
  const float t = 1.0f - s;
  return k.w_norm * k.inv_h * (-6.0f * t * t);
}
__device__ __forceinline__ float kG(const AK& k, float r) {  // spiky gradient factor: grad = r_vec * G(r)
  if (r <= 0.0f || r >= k.h) return 0.0f;
  const float d = k.h - r;
  return k.g_c * d * d / r;
}
__device__ __forceinline__ float kdG(const AK& k, float r) {
  if (r <= 0.0f || r >= k.h) return 0.0f;
  const float d = k.h - r;
  return k.g_c * (-2.0f * d / r - d * d / (r * r));
}
__device__ __forceinline__ float kL(const AK& k, float r) { return r < k.h ? k.l_c * (k.h - r) : 0.0f; }
__device__ __forceinline__ float kdL(const AK& k, float r) { return r < k.h ? -k.l_c : 0.0f; }

__device__ __forceinline__ float3 sub3(float4 a, float4 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float len3(float3 a) { return sqrtf(dot3(a, a)); }

struct Lists {
  const uint32_t* nbr;
  const uint32_t* cnt;
  uint32_t stride;
};

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[kT / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
  __syncthreads();
  return t;
}

// The passes that walk neighbour lists give each particle kLanes lanes of
// one warp: lane r takes list entries r, r + kLanes, ..., and the lanes'
// partial sums are added over the group by xor shuffles, a fixed order, so
// the results are deterministic (a recomputed forward step equals the
// original bit for bit). At a few tens of thousands of particles a thread
// per particle would leave most of the GPU idle.
constexpr uint32_t kLanes = 4;
struct Group {
  uint32_t i;      // particle
  uint32_t r;      // lane within the group
  uint32_t mask;   // the group's lanes
};
__device__ __forceinline__ Group group_index() {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31u;
  return Group{t / kLanes, t % kLanes, ((1u << kLanes) - 1u) << (lane - lane % kLanes)};
}
__device__ __forceinline__ float gsum(const Group& g, float v) {
  for (uint32_t o = kLanes / 2; o > 0; o >>= 1) v += __shfl_xor_sync(g.mask, v, o, kLanes);
  return v;
}
__device__ __forceinline__ float3 gsum(const Group& g, float3 v) {
  return make_float3(gsum(g, v.x), gsum(g, v.y), gsum(g, v.z));
}

// --------------------------------------------------------------- forward
__global__ void k_af_gather(uint32_t n, const uint32_t* __restrict__ perm, const float4* __restrict__ x,
                            const float4* __restrict__ v, float4* __restrict__ xs, float4* __restrict__ vs) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t j = perm[i];
  xs[i] = x[j];
  vs[i] = v[j];
}

__global__ void k_af_external(uint32_t n, AK k, float a_visc, float mg, const float4* __restrict__ xs,
                              const float4* __restrict__ vs, Lists L, float4* __restrict__ F) {
  const Group gr = group_index();
  const uint32_t i = gr.i;
  if (i >= n) return;  // uniform over the group
  const float4 xi = xs[i], vi = vs[i];
  float3 f = make_float3(0, 0, 0);
  const uint32_t c = L.cnt[i];
  for (uint32_t q = gr.r; q < c; q += kLanes) {
    const uint32_t j = L.nbr[(size_t)q * L.stride + i];
    const float r = len3(sub3(xi, xs[j]));
    const float w = a_visc * kL(k, r);
    const float4 vj = vs[j];
    f.x -= (vi.x - vj.x) * w;
    f.y -= (vi.y - vj.y) * w;
    f.z -= (vi.z - vj.z) * w;
  }
  f = gsum(gr, f);
  f.y -= mg;
  if (gr.r == 0) F[i] = make_float4(f.x, f.y, f.z, 0.0f);
}

__device__ __forceinline__ void clamp_pos(float4& x, float4& v, const float3& lo, const float3& hi, float damping) {
  if (x.x < lo.x) { x.x = lo.x; v.x *= damping; }
  if (x.x > hi.x) { x.x = hi.x; v.x *= damping; }
  if (x.y < lo.y) { x.y = lo.y; v.y *= damping; }
  if (x.y > hi.y) { x.y = hi.y; v.y *= damping; }
  if (x.z < lo.z) { x.z = lo.z; v.z *= damping; }
  if (x.z > hi.z) { x.z = hi.z; v.z *= damping; }
}

__global__ void k_af_predict(uint32_t n, float dt, float inv_m, float3 lo, float3 hi, const float4* __restrict__ xs,
                             const float4* __restrict__ vs, const float4* __restrict__ F,
                             const float4* __restrict__ Fp, float4* __restrict__ xstar) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 f = F[i];
  const float4 fp = Fp ? Fp[i] : make_float4(0, 0, 0, 0);
  const float4 v = vs[i], x = xs[i];
  float4 vv = make_float4(v.x + (f.x + fp.x) * dt * inv_m, v.y + (f.y + fp.y) * dt * inv_m,
                          v.z + (f.z + fp.z) * dt * inv_m, 0.0f);
  float4 xx = make_float4(x.x + vv.x * dt, x.y + vv.y * dt, x.z + vv.z * dt, 0.0f);
  clamp_pos(xx, vv, lo, hi, 0.0f);
  xstar[i] = xx;
}

__device__ __forceinline__ float smax(float d, float eps) { return 0.5f * (d + sqrtf(d * d + eps * eps)); }
__device__ __forceinline__ float dsmax(float d, float eps) { return 0.5f * (1.0f + d / sqrtf(d * d + eps * eps)); }

__global__ void k_af_density(uint32_t n, AK k, float m, float rho0, float delta, float eps, const float4* __restrict__ xstar,
                             Lists L, const float* __restrict__ p_prev, float* __restrict__ rho,
                             float* __restrict__ p) {
  const Group gr = group_index();
  const uint32_t i = gr.i;
  if (i >= n) return;  // uniform over the group
  const float4 xi = xstar[i];
  float d = 0.0f;
  const uint32_t c = L.cnt[i];
  for (uint32_t q = gr.r; q < c; q += kLanes) {
    const uint32_t j = L.nbr[(size_t)q * L.stride + i];
    d += m * kW(k, len3(sub3(xi, xstar[j])));
  }
  d = m * kW(k, 0.0f) + gsum(gr, d);
  if (gr.r != 0) return;
  rho[i] = d;
  p[i] = (p_prev ? p_prev[i] : 0.0f) + delta * smax(d - rho0, eps);
}

__global__ void k_af_pforce(uint32_t n, AK k, float c0, const float4* __restrict__ xs, const float* __restrict__ p,
                            Lists L, float4* __restrict__ Fp) {
  const Group gr = group_index();
  const uint32_t i = gr.i;
  if (i >= n) return;  // uniform over the group
  const float4 xi = xs[i];
  const float pi = p[i];
  float3 f = make_float3(0, 0, 0);
  const uint32_t c = L.cnt[i];
  for (uint32_t q = gr.r; q < c; q += kLanes) {
    const uint32_t j = L.nbr[(size_t)q * L.stride + i];
    const float3 r = sub3(xi, xs[j]);
    const float w = -c0 * (pi + p[j]) * kG(k, len3(r));
    f.x += r.x * w;
    f.y += r.y * w;
    f.z += r.z * w;
  }
  f = gsum(gr, f);
  if (gr.r == 0) Fp[i] = make_float4(f.x, f.y, f.z, 0.0f);
}

__global__ void k_af_integrate(uint32_t n, float dt, float inv_m, float3 lo, float3 hi,
                               const uint32_t* __restrict__ perm, const float4* __restrict__ xs,
                               const float4* __restrict__ vs, const float4* __restrict__ F,
                               const float4* __restrict__ Fp, float4* __restrict__ x, float4* __restrict__ v) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 f = F[i], fp = Fp[i], vi = vs[i], xi = xs[i];
  float4 vv = make_float4(vi.x + (f.x + fp.x) * dt * inv_m, vi.y + (f.y + fp.y) * dt * inv_m,
                          vi.z + (f.z + fp.z) * dt * inv_m, 0.0f);
  float4 xx = make_float4(xi.x + vv.x * dt, xi.y + vv.y * dt, xi.z + vv.z * dt, 0.0f);
  clamp_pos(xx, vv, lo, hi, -0.5f);
  const uint32_t j = perm[i];
  x[j] = xx;
  v[j] = vv;
}

// loss: densities at the final positions, sum of positions, sum of (rho - rho0)^2
__global__ void __launch_bounds__(kT) k_af_loss(uint32_t n, AK k, float m, float rho0, const float4* __restrict__ xs,
                                                Lists L, float* __restrict__ rho, double* __restrict__ sums) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  double sx = 0, sy = 0, sz = 0, sd = 0;
  if (i < n) {
    const float4 xi = xs[i];
    float d = m * kW(k, 0.0f);
    const uint32_t c = L.cnt[i];
    for (uint32_t q = 0; q < c; ++q) {
      const uint32_t j = L.nbr[(size_t)q * L.stride + i];
      d += m * kW(k, len3(sub3(xi, xs[j])));
    }
    rho[i] = d;
    sx = xi.x;
    sy = xi.y;
    sz = xi.z;
    sd = ((double)d - rho0) * ((double)d - rho0);
  }
  sx = block_sum(sx);
  sy = block_sum(sy);
  sz = block_sum(sz);
  sd = block_sum(sd);
  if (threadIdx.x == 0) {
    atomicAdd(&sums[0], sx);
    atomicAdd(&sums[1], sy);
    atomicAdd(&sums[2], sz);
    atomicAdd(&sums[3], sd);
  }
}

// --------------------------------------------------------------- backward
// seeds of the loss: xb = dL/dx(T) (sorted order of the final lists)
__global__ void k_ab_loss_seed(uint32_t n, AK k, float m, float g_com_x, float g_com_y, float g_com_z,
                               float g_rho, float rho0, const float4* __restrict__ xs, const float* __restrict__ rho,
                               Lists L, float4* __restrict__ xb) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 xi = xs[i];
  const float bi = g_rho * (rho[i] - rho0);
  float3 g = make_float3(g_com_x, g_com_y, g_com_z);
  const uint32_t c = L.cnt[i];
  for (uint32_t q = 0; q < c; ++q) {
    const uint32_t j = L.nbr[(size_t)q * L.stride + i];
    const float3 r = sub3(xi, xs[j]);
    const float rl = len3(r);
    if (rl <= 0.0f) continue;
    const float w = m * kdW(k, rl) / rl * (bi + g_rho * (rho[j] - rho0));
    g.x += r.x * w;
    g.y += r.y * w;
    g.z += r.z * w;
  }
  xb[i] = make_float4(g.x, g.y, g.z, 0.0f);
}

__global__ void k_ab_gather(uint32_t n, const uint32_t* __restrict__ perm, const float4* __restrict__ xbar,
                            const float4* __restrict__ vbar, float4* __restrict__ xb, float4* __restrict__ vb) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t j = perm[i];
  xb[i] = xbar[j];
  vb[i] = vbar[j];
}

__global__ void k_ab_scatter(uint32_t n, const uint32_t* __restrict__ perm, const float4* __restrict__ xb,
                             const float4* __restrict__ vb, float4* __restrict__ xbar, float4* __restrict__ vbar) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t j = perm[i];
  xbar[j] = xb[i];
  vbar[j] = vb[i];
}

// adjoint of the integration: x' = x + v' dt, v' = v + (F + Fp^K) dt / m
__global__ void k_ab_integrate(uint32_t n, float dt, float inv_m, float4* __restrict__ xb, float4* __restrict__ vb,
                               float4* __restrict__ Fb, float4* __restrict__ Fpb, float* __restrict__ pcarry) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 x = xb[i], v = vb[i];
  const float4 vt = make_float4(v.x + x.x * dt, v.y + x.y * dt, v.z + x.z * dt, 0.0f);
  vb[i] = vt;
  const float s = dt * inv_m;
  Fb[i] = make_float4(vt.x * s, vt.y * s, vt.z * s, 0.0f);
  Fpb[i] = Fb[i];
  pcarry[i] = 0.0f;
}

// adjoint of the pressure force of iteration k: pbar (+ the later
// iterations' carry), the density seed rhob, and the position adjoint
__global__ void k_ab_pforce(uint32_t n, AK k, float c0, float delta, float rho0, float eps, const float4* __restrict__ xs,
                            const float* __restrict__ p, const float* __restrict__ rho, const float4* __restrict__ Fpb,
                            Lists L, float* __restrict__ pcarry, float* __restrict__ rhob, float4* __restrict__ xb) {
  const Group gr = group_index();
  const uint32_t i = gr.i;
  if (i >= n) return;  // uniform over the group
  const float4 xi = xs[i], fi = Fpb[i];
  const float pi = p[i];
  float pb = 0.0f;
  float3 g = make_float3(0, 0, 0);
  const uint32_t c = L.cnt[i];
  for (uint32_t q = gr.r; q < c; q += kLanes) {
    const uint32_t j = L.nbr[(size_t)q * L.stride + i];
    const float3 r = sub3(xi, xs[j]);
    const float rl = len3(r);
    const float G = kG(k, rl);
    const float4 fj = Fpb[j];
    const float3 d = make_float3(fi.x - fj.x, fi.y - fj.y, fi.z - fj.z);
    const float rd = dot3(r, d);
    pb += -c0 * rd * G;
    // c_ij J d, J = G I + (G'/r) r r^T, c_ij = -c0 (p_i + p_j)
    const float cij = -c0 * (pi + p[j]);
    const float t = rl > 0.0f ? kdG(k, rl) / rl * rd : 0.0f;
    g.x += cij * (G * d.x + t * r.x);
    g.y += cij * (G * d.y + t * r.y);
    g.z += cij * (G * d.z + t * r.z);
  }
  pb = gsum(gr, pb);
  g = gsum(gr, g);
  if (gr.r != 0) return;
  const float ptot = pcarry[i] + pb;
  pcarry[i] = ptot;
  rhob[i] = delta * dsmax(rho[i] - rho0, eps) * ptot;
  float4 x = xb[i];
  xb[i] = make_float4(x.x + g.x, x.y + g.y, x.z + g.z, 0.0f);
}

// adjoint of the predicted density of iteration k: dL/dx*
__global__ void k_ab_density(uint32_t n, AK k, float m, const float4* __restrict__ xstar,
                             const float* __restrict__ rhob, Lists L, float4* __restrict__ xstarb) {
  const Group gr = group_index();
  const uint32_t i = gr.i;
  if (i >= n) return;  // uniform over the group
  const float4 xi = xstar[i];
  const float bi = rhob[i];
  float3 g = make_float3(0, 0, 0);
  const uint32_t c = L.cnt[i];
  for (uint32_t q = gr.r; q < c; q += kLanes) {
    const uint32_t j = L.nbr[(size_t)q * L.stride + i];
    const float3 r = sub3(xi, xstar[j]);
    const float rl = len3(r);
    if (rl <= 0.0f) continue;
    const float w = m * kdW(k, rl) / rl * (bi + rhob[j]);
    g.x += r.x * w;
    g.y += r.y * w;
    g.z += r.z * w;
  }
  g = gsum(gr, g);
  if (gr.r == 0) xstarb[i] = make_float4(g.x, g.y, g.z, 0.0f);
}

// adjoint of the prediction of iteration k: x* = x + v* dt,
// v* = v + (F + Fp^{k-1}) dt / m; Fpb receives dL/dFp^{k-1} (k > 1)
__global__ void k_ab_predict(uint32_t n, float dt, float inv_m, const float4* __restrict__ xstarb,
                             float4* __restrict__ xb, float4* __restrict__ vb, float4* __restrict__ Fb,
                             float4* __restrict__ Fpb, int has_prev) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 s = xstarb[i];
  const float4 x = xb[i], v = vb[i], f = Fb[i];
  xb[i] = make_float4(x.x + s.x, x.y + s.y, x.z + s.z, 0.0f);
  const float4 vs = make_float4(s.x * dt, s.y * dt, s.z * dt, 0.0f);
  vb[i] = make_float4(v.x + vs.x, v.y + vs.y, v.z + vs.z, 0.0f);
  const float c = dt * inv_m;
  Fb[i] = make_float4(f.x + vs.x * c, f.y + vs.y * c, f.z + vs.z * c, 0.0f);
  Fpb[i] = has_prev ? make_float4(vs.x * c, vs.y * c, vs.z * c, 0.0f) : make_float4(0, 0, 0, 0);
}

// adjoint of the external force: dL/dv, dL/dx, dL/dmu
__global__ void __launch_bounds__(kT) k_ab_external(uint32_t n, AK k, float vol2, float mu,
                                                    const float4* __restrict__ xs, const float4* __restrict__ vs,
                                                    const float4* __restrict__ Fb, Lists L, float4* __restrict__ xb,
                                                    float4* __restrict__ vb, double* __restrict__ mu_bar) {
  const Group gr = group_index();
  const uint32_t i = gr.i;
  double mb = 0.0;
  if (i < n) {  // uniform over the group; every thread reaches block_sum
    const float4 xi = xs[i], vi = vs[i], fi = Fb[i];
    float3 gx = make_float3(0, 0, 0), gv = make_float3(0, 0, 0);
    float m_acc = 0.0f;
    const uint32_t c = L.cnt[i];
    const float a = vol2 * mu;
    for (uint32_t q = gr.r; q < c; q += kLanes) {
      const uint32_t j = L.nbr[(size_t)q * L.stride + i];
      const float3 r = sub3(xi, xs[j]);
      const float rl = len3(r);
      const float Lr = kL(k, rl), dLr = kdL(k, rl);
      const float4 fj = Fb[j], vj = vs[j];
      const float3 dF = make_float3(fi.x - fj.x, fi.y - fj.y, fi.z - fj.z);
      const float3 dv = make_float3(vi.x - vj.x, vi.y - vj.y, vi.z - vj.z);
      gv.x -= a * Lr * dF.x;
      gv.y -= a * Lr * dF.y;
      gv.z -= a * Lr * dF.z;
      if (rl > 0.0f) {
        const float t = -a * dLr * dot3(dv, dF) / rl;
        gx.x += t * r.x;
        gx.y += t * r.y;
        gx.z += t * r.z;
      }
      m_acc += -vol2 * Lr * (dv.x * fi.x + dv.y * fi.y + dv.z * fi.z);
    }
    gx = gsum(gr, gx);
    gv = gsum(gr, gv);
    m_acc = gsum(gr, m_acc);
    if (gr.r == 0) {
      const float4 x = xb[i], v = vb[i];
      xb[i] = make_float4(x.x + gx.x, x.y + gx.y, x.z + gx.z, 0.0f);
      vb[i] = make_float4(v.x + gv.x, v.y + gv.y, v.z + gv.z, 0.0f);
      mb = m_acc;
    }
  }
  mb = block_sum(mb);
  if (threadIdx.x == 0) atomicAdd(mu_bar, mb);
}

inline uint32_t grid(uint32_t n) { return (n + kT - 1) / kT; }
inline uint32_t grid_lanes(uint32_t n) { return (uint32_t)(((uint64_t)n * kLanes + kT - 1) / kT); }

}  // namespace
}  // namespace upf

using namespace upf;

struct upf_adjoint {
  upf_params prm{};
  DevParams dp{};
  upf_adjoint_options opt{};
  AK k{};
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  uint32_t n = 0, stride = 0, rows = 0, ncells = 0;
  int nseg = 0;  // checkpoints: ceil(T / C) + 1
  float visc = 0.0f;
  bool have_forward = false;
  float fwd_ms = 0.0f, bwd_ms = 0.0f;

  // id-order state
  float4 *x0 = nullptr, *v0 = nullptr, *x = nullptr, *v = nullptr;
  float4 *xf = nullptr, *vf = nullptr;  // final state of the last forward
  float4 *ck_x = nullptr, *ck_v = nullptr;  // [nseg][n]
  float4 *xbar = nullptr, *vbar = nullptr;
  // neighbour machinery (per step)
  uint32_t *keys = nullptr, *sort_tmp = nullptr, *cstart = nullptr, *cend = nullptr;
  uint32_t* lval = nullptr;
  float* luts = nullptr;
  DevState* st = nullptr;
  // per-step storage of one checkpoint interval: [C][...]
  uint32_t *perm = nullptr, *nbr = nullptr, *ncnt = nullptr;
  float4 *xs = nullptr, *vs = nullptr, *F = nullptr, *xstar = nullptr;  // xstar [C][K][n]
  float *rho = nullptr, *p = nullptr;                                   // [C][K][n]
  float4* Fp = nullptr;                                                 // scratch [2][n]
  // backward scratch (sorted order)
  float4 *xb = nullptr, *vb = nullptr, *Fb = nullptr, *Fpb = nullptr, *xstarb = nullptr;
  float *pcarry = nullptr, *rhob = nullptr;
  double* sums = nullptr;  // [4] loss sums, [4] mu_bar
  double loss = 0.0;
  std::vector<void*> allocations;

  template <class T>
  upf_status alloc(T** ptr, size_t count) {
    *ptr = nullptr;
    if (inject_alloc_failure()) {
      set_error("upf_adjoint: cudaMalloc failed: injected by upf_test_fail_allocation");
      return UPF_ERR_ALLOC;
    }
    cudaError_t e = cudaMalloc((void**)ptr, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) {
      *ptr = nullptr;
      set_error("upf_adjoint: cudaMalloc of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
      return UPF_ERR_ALLOC;
    }
    allocations.push_back(*ptr);
    return UPF_OK;
  }

  int C() const { return opt.checkpoint_interval; }
  float eps_rho() const { return opt.density_smoothing * dp.rho0; }
  int K() const { return opt.loop_iterations; }
  size_t slot(int s) const { return (size_t)s * n; }
  Lists lists(int s) const { return Lists{nbr + (size_t)s * rows * stride, ncnt + slot(s), stride}; }

  // sort, gather and neighbour lists of the state (x, v) into step slot s
  upf_status prepare_step(int s) {
    cudaStream_t q = stream;
    UPF_CUDA(morton_keys(x, n, dp.origin, dp.scales, keys, q));
    uint32_t* kalt = sort_tmp;
    uint32_t* valt = kalt + ((n + 63) & ~63u);
    uint32_t* counts = valt + ((n + 63) & ~63u);
    uint32_t* pm = perm + slot(s);
    UPF_CUDA(radix_sort_pairs(keys, pm, kalt, valt, counts, n, 30, true, q));
    k_af_gather<<<grid(n), kT, 0, q>>>(n, pm, x, v, xs + slot(s), vs + slot(s));
    UPF_CUDA(cudaGetLastError());
    UPF_CUDA(cell_ranges(keys, n, 3 * (int)dp.cell_shift, ncells, cstart, cend, q));
    UPF_CUDA(launch_nlist_plain(dp, n, xs + slot(s), keys, cstart, cend, nbr + (size_t)s * rows * stride, lval,
                                ncnt + slot(s), luts, st, q));
    return UPF_OK;
  }

  // one forward step from (x, v) into slot s (x, v advanced in place)
  upf_status forward_step(int s) {
    cudaStream_t q = stream;
    UPF_TRY(prepare_step(s));
    const Lists L = lists(s);
    const float4* X = xs + slot(s);
    const float4* V = vs + slot(s);
    float4* Fs = F + slot(s);
    const float vol2 = dp.rest_volume * dp.rest_volume;
    k_af_external<<<grid_lanes(n), kT, 0, q>>>(n, k, vol2 * visc, dp.mass * dp.gravity, X, V, L, Fs);
    const float3 lo = dp.cmin, hi = dp.cmax;
    const float c0 = dp.mass * dp.mass / (dp.rho0 * dp.rho0);
    for (int it = 0; it < K(); ++it) {
      const size_t sk = ((size_t)s * K() + it) * n;
      const float4* fp_prev = it ? Fp + (size_t)((it - 1) & 1) * n : nullptr;
      float4* fp_out = Fp + (size_t)(it & 1) * n;
      k_af_predict<<<grid(n), kT, 0, q>>>(n, dp.dt, dp.inv_mass, lo, hi, X, V, Fs, fp_prev, xstar + sk);
      k_af_density<<<grid_lanes(n), kT, 0, q>>>(n, k, dp.mass, dp.rho0, dp.delta, eps_rho(), xstar + sk, L,
                                          it ? p + sk - n : nullptr, rho + sk, p + sk);
      k_af_pforce<<<grid_lanes(n), kT, 0, q>>>(n, k, c0, X, p + sk, L, fp_out);
    }
    k_af_integrate<<<grid(n), kT, 0, q>>>(n, dp.dt, dp.inv_mass, lo, hi, perm + slot(s), X, V, Fs,
                                          Fp + (size_t)((K() - 1) & 1) * n, x, v);
    UPF_CUDA(cudaGetLastError());
    return UPF_OK;
  }

  // one adjoint step for slot s: (xbar, vbar) at step end -> at step start
  upf_status backward_step(int s) {
    cudaStream_t q = stream;
    const Lists L = lists(s);
    const uint32_t* pm = perm + slot(s);
    const float4* X = xs + slot(s);
    const float4* V = vs + slot(s);
    const float c0 = dp.mass * dp.mass / (dp.rho0 * dp.rho0);
    k_ab_gather<<<grid(n), kT, 0, q>>>(n, pm, xbar, vbar, xb, vb);
    k_ab_integrate<<<grid(n), kT, 0, q>>>(n, dp.dt, dp.inv_mass, xb, vb, Fb, Fpb, pcarry);
    for (int it = K() - 1; it >= 0; --it) {
      const size_t sk = ((size_t)s * K() + it) * n;
      k_ab_pforce<<<grid_lanes(n), kT, 0, q>>>(n, k, c0, dp.delta, dp.rho0, eps_rho(), X, p + sk, rho + sk, Fpb, L, pcarry, rhob,
                                         xb);
      k_ab_density<<<grid_lanes(n), kT, 0, q>>>(n, k, dp.mass, xstar + sk, rhob, L, xstarb);
      k_ab_predict<<<grid(n), kT, 0, q>>>(n, dp.dt, dp.inv_mass, xstarb, xb, vb, Fb, Fpb, it > 0 ? 1 : 0);
    }
    const float vol2 = dp.rest_volume * dp.rest_volume;
    k_ab_external<<<grid_lanes(n), kT, 0, q>>>(n, k, vol2, visc, X, V, Fb, L, xb, vb, sums + 4);
    k_ab_scatter<<<grid(n), kT, 0, q>>>(n, pm, xb, vb, xbar, vbar);
    UPF_CUDA(cudaGetLastError());
    return UPF_OK;
  }

  upf_status check_flags() {
    DevState h;
    UPF_CUDA(cudaMemcpyAsync(&h, st, sizeof(DevState), cudaMemcpyDeviceToHost, stream));
    UPF_CUDA(cudaStreamSynchronize(stream));
    if (h.error_flags & ERR_OVERFLOW) {
      set_error("upf_adjoint: a particle has %u neighbours, more than max_neighbors=%u", h.max_neighbors,
                prm.max_neighbors);
      return UPF_ERR_NEIGHBOR_OVERFLOW;
    }
    return UPF_OK;
  }
};

extern "C" {

upf_status upf_adjoint_create(const upf_params* p, const upf_adjoint_options* opt, const float* pos4,
                              const float* vel4, uint32_t n, int device, upf_adjoint** out) {
  if (!p || !opt || !out || (n && (!pos4 || !vel4)) || n == 0) {
    set_error("upf_adjoint_create: null argument or no particles");
    return UPF_ERR_INVALID_ARG;
  }
  *out = nullptr;
  const char* why = nullptr;
  if (validate_params(*p, &why) != 0) {
    set_error("upf_adjoint_create: invalid parameters: %s", why);
    return UPF_ERR_INVALID_ARG;
  }
  if (p->method != UPF_METHOD_PCISPH) {
    set_error("upf_adjoint_create: the adjoint differentiates the PCISPH solver");
    return UPF_ERR_UNSUPPORTED;
  }
  if (opt->steps < 1 || opt->checkpoint_interval < 1 || opt->loop_iterations < 1 || opt->loop_iterations > 64 ||
      !(opt->density_smoothing > 0.0f)) {
    set_error("upf_adjoint_create: need steps >= 1, checkpoint_interval >= 1, 1 <= loop_iterations <= 64, "
              "density_smoothing > 0");
    return UPF_ERR_INVALID_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("upf_adjoint_create: no CUDA device");
    return UPF_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) {
    set_error("upf_adjoint_create: device %d out of range", device);
    return UPF_ERR_INVALID_ARG;
  }
  UPF_CUDA(cudaSetDevice(device));
  UPF_CUDA(radix_init());
  upf_adjoint* a = new upf_adjoint();
  a->prm = *p;
  a->opt = *opt;
  a->opt.checkpoint_interval = std::min(opt->checkpoint_interval, opt->steps);
  a->device = device;
  a->n = n;
  a->stride = (n + 31) & ~31u;
  a->rows = p->max_neighbors;
  a->dp = make_dev_params(*p, a->stride);
  a->visc = p->viscosity;
  const float h = p->support_radius;
  const double pi = 3.14159265358979323846;
  a->k.h = h;
  a->k.inv_h = (float)(1.0 / (double)h);
  a->k.w_norm = (float)(2.546479089470325472 / ((double)h * h * h));
  a->k.g_c = (float)(-45.0 / (pi * std::pow((double)h, 6)));
  a->k.l_c = (float)(45.0 / (pi * std::pow((double)h, 6)));
  const uint32_t bpa = UPF_GRID_RESOLUTION / effective_search_cell(*p);
  a->ncells = bpa * bpa * bpa;
  const int C = a->opt.checkpoint_interval, K = a->opt.loop_iterations;
  a->nseg = (opt->steps + C - 1) / C + 1;
  auto bail = [&](upf_status st) {
    upf_adjoint_destroy(a);
    return st;
  };
  cudaError_t e = cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    set_error("cudaStreamCreate: %s", cudaGetErrorString(e));
    return bail(UPF_ERR_CUDA);
  }
  a->own_stream = true;
  upf_status st = UPF_OK;
  const size_t N = n;
#define ALLOC(ptr, cnt) \
  if ((st = a->alloc(&(ptr), (cnt))) != UPF_OK) return bail(st);
  ALLOC(a->x0, N); ALLOC(a->v0, N); ALLOC(a->x, N); ALLOC(a->v, N); ALLOC(a->xf, N); ALLOC(a->vf, N);
  ALLOC(a->ck_x, (size_t)a->nseg * N); ALLOC(a->ck_v, (size_t)a->nseg * N);
  ALLOC(a->xbar, N); ALLOC(a->vbar, N);
  ALLOC(a->keys, N); ALLOC(a->sort_tmp, radix_temp_words(n)); ALLOC(a->cstart, a->ncells); ALLOC(a->cend, a->ncells);
  ALLOC(a->lval, (size_t)a->rows * a->stride); ALLOC(a->luts, kLutFloats); ALLOC(a->st, 1);
  ALLOC(a->perm, (size_t)C * N); ALLOC(a->nbr, (size_t)C * a->rows * a->stride); ALLOC(a->ncnt, (size_t)C * N);
  ALLOC(a->xs, (size_t)C * N); ALLOC(a->vs, (size_t)C * N); ALLOC(a->F, (size_t)C * N);
  ALLOC(a->xstar, (size_t)C * K * N); ALLOC(a->rho, (size_t)C * K * N); ALLOC(a->p, (size_t)C * K * N);
  ALLOC(a->Fp, 2 * N);
  ALLOC(a->xb, N); ALLOC(a->vb, N); ALLOC(a->Fb, N); ALLOC(a->Fpb, N); ALLOC(a->xstarb, N);
  ALLOC(a->pcarry, N); ALLOC(a->rhob, N); ALLOC(a->sums, 8);
#undef ALLOC
  std::vector<float> lut(kLutFloats);
  build_luts(*p, lut.data());
  build_bin_thresholds(*p, lut.data() + 5 * UPF_LUT_ENTRIES);
  std::vector<float4> hp(n), hv(n);
  for (uint32_t i = 0; i < n; ++i) {
    hp[i] = make_float4(pos4[4 * i], pos4[4 * i + 1], pos4[4 * i + 2], 0.0f);
    hv[i] = make_float4(vel4[4 * i], vel4[4 * i + 1], vel4[4 * i + 2], 0.0f);
  }
  e = cudaMemcpy(a->luts, lut.data(), sizeof(float) * kLutFloats, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(a->x0, hp.data(), sizeof(float4) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(a->v0, hv.data(), sizeof(float4) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(a->st, 0, sizeof(DevState));
  if (e != cudaSuccess) {
    set_error("upf_adjoint_create: upload: %s", cudaGetErrorString(e));
    return bail(UPF_ERR_CUDA);
  }
  *out = a;
  return UPF_OK;
}

upf_status upf_adjoint_destroy(upf_adjoint* a) {
  if (!a) return UPF_OK;
  cudaSetDevice(a->device);
  if (a->stream) cudaStreamSynchronize(a->stream);
  for (void* ptr : a->allocations) cudaFree(ptr);
  if (a->stream && a->own_stream) cudaStreamDestroy(a->stream);
  delete a;
  return UPF_OK;
}

upf_status upf_adjoint_set_stream(upf_adjoint* a, void* stream) {
  if (!a) {
    set_error("upf_adjoint_set_stream: null");
    return UPF_ERR_INVALID_ARG;
  }
  UPF_CUDA(cudaStreamSynchronize(a->stream));
  if (a->own_stream) cudaStreamDestroy(a->stream);
  if (stream) {
    a->stream = (cudaStream_t)stream;
    a->own_stream = false;
  } else {
    UPF_CUDA(cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking));
    a->own_stream = true;
  }
  return UPF_OK;
}

upf_status upf_adjoint_forward(upf_adjoint* a, const float* vel4, float viscosity, double* loss) {
  NvtxRange nvtx("upf_adjoint_forward");
  if (!a) {
    set_error("upf_adjoint_forward: null");
    return UPF_ERR_INVALID_ARG;
  }
  UPF_CUDA(cudaSetDevice(a->device));
  cudaStream_t q = a->stream;
  const uint32_t n = a->n;
  if (vel4) {
    std::vector<float4> hv(n);
    for (uint32_t i = 0; i < n; ++i) hv[i] = make_float4(vel4[4 * i], vel4[4 * i + 1], vel4[4 * i + 2], 0.0f);
    UPF_CUDA(cudaMemcpyAsync(a->v0, hv.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, q));
    UPF_CUDA(cudaStreamSynchronize(q));
  }
  a->visc = viscosity;
  cudaEvent_t e0, e1;
  UPF_CUDA(cudaEventCreate(&e0));
  UPF_CUDA(cudaEventCreate(&e1));
  UPF_CUDA(cudaEventRecord(e0, q));
  UPF_CUDA(cudaMemcpyAsync(a->x, a->x0, sizeof(float4) * n, cudaMemcpyDeviceToDevice, q));
  UPF_CUDA(cudaMemcpyAsync(a->v, a->v0, sizeof(float4) * n, cudaMemcpyDeviceToDevice, q));
  UPF_CUDA(cudaMemsetAsync(a->st, 0, sizeof(DevState), q));
  const int T = a->opt.steps, C = a->C();
  for (int t = 0; t < T; ++t) {
    if (t % C == 0) {
      const size_t o = (size_t)(t / C) * n;
      UPF_CUDA(cudaMemcpyAsync(a->ck_x + o, a->x, sizeof(float4) * n, cudaMemcpyDeviceToDevice, q));
      UPF_CUDA(cudaMemcpyAsync(a->ck_v + o, a->v, sizeof(float4) * n, cudaMemcpyDeviceToDevice, q));
    }
    UPF_TRY(a->forward_step(0));
  }
  UPF_CUDA(cudaMemcpyAsync(a->xf, a->x, sizeof(float4) * n, cudaMemcpyDeviceToDevice, q));
  UPF_CUDA(cudaMemcpyAsync(a->vf, a->v, sizeof(float4) * n, cudaMemcpyDeviceToDevice, q));
  // loss at the final positions (lists in slot 0)
  UPF_TRY(a->prepare_step(0));
  UPF_CUDA(cudaMemsetAsync(a->sums, 0, sizeof(double) * 8, q));
  k_af_loss<<<grid(n), kT, 0, q>>>(n, a->k, a->dp.mass, a->dp.rho0, a->xs, a->lists(0), a->rho, a->sums);
  UPF_CUDA(cudaGetLastError());
  UPF_CUDA(cudaEventRecord(e1, q));
  double sums[4];
  UPF_CUDA(cudaMemcpyAsync(sums, a->sums, sizeof(double) * 4, cudaMemcpyDeviceToHost, q));
  UPF_CUDA(cudaStreamSynchronize(q));
  UPF_CUDA(cudaEventElapsedTime(&a->fwd_ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  UPF_TRY(a->check_flags());
  double L = 0.0;
  for (int c = 0; c < 3; ++c) {
    const double com = sums[c] / n - (double)a->opt.target[c];
    L += a->opt.com_weight * com * com;
  }
  L += a->opt.density_weight * sums[3] / n;
  a->loss = L;
  a->have_forward = true;
  if (loss) *loss = L;
  return UPF_OK;
}

upf_status upf_adjoint_backward(upf_adjoint* a, float* grad_vel4, double* grad_viscosity) {
  NvtxRange nvtx("upf_adjoint_backward");
  if (!a || !a->have_forward) {
    set_error("upf_adjoint_backward: run upf_adjoint_forward first");
    return a ? UPF_ERR_STATE : UPF_ERR_INVALID_ARG;
  }
  UPF_CUDA(cudaSetDevice(a->device));
  cudaStream_t q = a->stream;
  const uint32_t n = a->n;
  cudaEvent_t e0, e1;
  UPF_CUDA(cudaEventCreate(&e0));
  UPF_CUDA(cudaEventCreate(&e1));
  UPF_CUDA(cudaEventRecord(e0, q));
  // seeds: the final state's lists and densities are in slot 0 (forward)
  double sums[4];
  UPF_CUDA(cudaMemcpyAsync(sums, a->sums, sizeof(double) * 4, cudaMemcpyDeviceToHost, q));
  UPF_CUDA(cudaStreamSynchronize(q));
  const float gc[3] = {(float)(2.0 * a->opt.com_weight * (sums[0] / n - a->opt.target[0]) / n),
                       (float)(2.0 * a->opt.com_weight * (sums[1] / n - a->opt.target[1]) / n),
                       (float)(2.0 * a->opt.com_weight * (sums[2] / n - a->opt.target[2]) / n)};
  const float gr = (float)(2.0 * a->opt.density_weight / n);
  k_ab_loss_seed<<<grid(n), kT, 0, q>>>(n, a->k, a->dp.mass, gc[0], gc[1], gc[2], gr, a->dp.rho0, a->xs, a->rho,
                                        a->lists(0), a->xb);
  UPF_CUDA(cudaMemsetAsync(a->vb, 0, sizeof(float4) * n, q));
  k_ab_scatter<<<grid(n), kT, 0, q>>>(n, a->perm, a->xb, a->vb, a->xbar, a->vbar);
  UPF_CUDA(cudaGetLastError());
  UPF_CUDA(cudaMemsetAsync(a->sums + 4, 0, sizeof(double), q));
  const int T = a->opt.steps, C = a->C();
  for (int seg = (T - 1) / C; seg >= 0; --seg) {
    const int t0 = seg * C, len = std::min(C, T - t0);
    const size_t o = (size_t)seg * n;
    UPF_CUDA(cudaMemcpyAsync(a->x, a->ck_x + o, sizeof(float4) * n, cudaMemcpyDeviceToDevice, q));
    UPF_CUDA(cudaMemcpyAsync(a->v, a->ck_v + o, sizeof(float4) * n, cudaMemcpyDeviceToDevice, q));
    for (int s = 0; s < len; ++s) UPF_TRY(a->forward_step(s));
    for (int s = len - 1; s >= 0; --s) UPF_TRY(a->backward_step(s));
  }
  UPF_CUDA(cudaEventRecord(e1, q));
  UPF_CUDA(cudaEventSynchronize(e1));
  UPF_CUDA(cudaEventElapsedTime(&a->bwd_ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (grad_vel4) {
    std::vector<float4> h(n);
    UPF_CUDA(cudaMemcpyAsync(h.data(), a->vbar, sizeof(float4) * n, cudaMemcpyDeviceToHost, q));
    UPF_CUDA(cudaStreamSynchronize(q));
    for (uint32_t i = 0; i < n; ++i) {
      grad_vel4[4 * i] = h[i].x;
      grad_vel4[4 * i + 1] = h[i].y;
      grad_vel4[4 * i + 2] = h[i].z;
      grad_vel4[4 * i + 3] = 0.0f;
    }
  }
  if (grad_viscosity) {
    UPF_CUDA(cudaMemcpyAsync(grad_viscosity, a->sums + 4, sizeof(double), cudaMemcpyDeviceToHost, q));
    UPF_CUDA(cudaStreamSynchronize(q));
  }
  return a->check_flags();
}

upf_status upf_adjoint_get_state(upf_adjoint* a, float* pos4, float* vel4) {
  if (!a || !a->have_forward) {
    set_error("upf_adjoint_get_state: run upf_adjoint_forward first");
    return a ? UPF_ERR_STATE : UPF_ERR_INVALID_ARG;
  }
  const uint32_t n = a->n;
  if (pos4) UPF_CUDA(cudaMemcpyAsync(pos4, a->xf, sizeof(float4) * n, cudaMemcpyDeviceToHost, a->stream));
  if (vel4) UPF_CUDA(cudaMemcpyAsync(vel4, a->vf, sizeof(float4) * n, cudaMemcpyDeviceToHost, a->stream));
  UPF_CUDA(cudaStreamSynchronize(a->stream));
  return UPF_OK;
}

upf_status upf_adjoint_times(upf_adjoint* a, float* forward_ms, float* backward_ms) {
  if (!a) {
    set_error("upf_adjoint_times: null");
    return UPF_ERR_INVALID_ARG;
  }
  if (forward_ms) *forward_ms = a->fwd_ms;
  if (backward_ms) *backward_ms = a->bwd_ms;
  return UPF_OK;
}

}  // extern "C"
