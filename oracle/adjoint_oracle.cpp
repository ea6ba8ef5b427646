// adjoint_oracle.cpp — TEST INFRASTRUCTURE ONLY: an FP64 CPU restatement of
// the differentiable PCISPH trajectory of the library's upf_adjoint (the
// reference's kernel functions WeightingKernel::KernelM4 /
// kernelPressureGrad / kernelViscosityLaplacian, WeightingKernel.cpp:75-200,
// evaluated analytically; the step formulas of
// CalculateExternalForcesPCISPH, PredictionCorrectionStep and
// ComputeCorrectivePressureForce, UnifiedPhysics.cpp:5165-5522, with a fixed
// number of predict-correct iterations and the density error's maximum with
// zero smoothed to 0.5 (d + sqrt(d^2 + eps^2))) and of its adjoint, for checking the
// device adjoint and, through central differences of the loss, the adjoint
// itself. Plain loops, all steps kept in memory (small scenes only).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "../include/upf.h"

namespace {

struct V {
  double x, y, z;
};
inline V operator+(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V operator-(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V operator*(V a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double len(V a) { return std::sqrt(dot(a, a)); }

struct Kern {
  double h, wn, gc, lc;
  double W(double r) const {
    const double s = r / h;
    if (s >= 1.0) return 0.0;
    if (s < 0.5) return wn * (1.0 - 6.0 * s * s + 6.0 * s * s * s);
    const double t = 1.0 - s;
    return wn * 2.0 * t * t * t;
  }
  double dW(double r) const {
    const double s = r / h;
    if (s >= 1.0) return 0.0;
    if (s < 0.5) return wn / h * (-12.0 * s + 18.0 * s * s);
    const double t = 1.0 - s;
    return wn / h * (-6.0 * t * t);
  }
  double G(double r) const {
    if (r <= 0.0 || r >= h) return 0.0;
    return gc * (h - r) * (h - r) / r;
  }
  double dG(double r) const {
    if (r <= 0.0 || r >= h) return 0.0;
    const double d = h - r;
    return gc * (-2.0 * d / r - d * d / (r * r));
  }
  double L(double r) const { return r < h ? lc * (h - r) : 0.0; }
  double dL(double r) const { return r < h ? -lc : 0.0; }
};

// pairs within h (uniform grid of cell h)
void neighbors(const std::vector<V>& x, double h, std::vector<std::vector<int>>& nb) {
  const int n = (int)x.size();
  nb.assign(n, {});
  std::unordered_map<int64_t, std::vector<int>> grid;
  auto key = [&](int64_t a, int64_t b, int64_t c) { return (a * 73856093) ^ (b * 19349663) ^ (c * 83492791); };
  auto cell = [&](double v) { return (int64_t)std::floor(v / h); };
  for (int i = 0; i < n; ++i) grid[key(cell(x[i].x), cell(x[i].y), cell(x[i].z))].push_back(i);
  for (int i = 0; i < n; ++i) {
    const int64_t cx = cell(x[i].x), cy = cell(x[i].y), cz = cell(x[i].z);
    for (int64_t a = cx - 1; a <= cx + 1; ++a)
      for (int64_t b = cy - 1; b <= cy + 1; ++b)
        for (int64_t c = cz - 1; c <= cz + 1; ++c) {
          auto it = grid.find(key(a, b, c));
          if (it == grid.end()) continue;
          for (int j : it->second) {
            if (j == i) continue;
            if (cell(x[j].x) != a || cell(x[j].y) != b || cell(x[j].z) != c) continue;  // hash collision
            if (len(x[i] - x[j]) < h) nb[i].push_back(j);
          }
        }
  }
}

struct Model {
  Kern k;
  double m, rho0, dt, delta, vol2, g;
  double eps;  // width of the smooth maximum, eps_rho * rho0
  V lo, hi;
  int K;
};

// the smooth maximum of the density error: 0.5 (d + sqrt(d^2 + eps^2)) and its slope
inline double smax(double d, double eps) { return 0.5 * (d + std::sqrt(d * d + eps * eps)); }
inline double dsmax(double d, double eps) { return 0.5 * (1.0 + d / std::sqrt(d * d + eps * eps)); }

struct StepRec {
  std::vector<V> x, v, F;
  std::vector<std::vector<int>> nb;
  std::vector<std::vector<V>> xs;      // [K][n] predicted positions
  std::vector<std::vector<double>> rho, p;
};

void clamp(V& x, V& v, const Model& M, double damping) {
  double* xp = &x.x;
  double* vp = &v.x;
  const double* lo = &M.lo.x;
  const double* hi = &M.hi.x;
  for (int a = 0; a < 3; ++a) {
    if (xp[a] < lo[a]) { xp[a] = lo[a]; vp[a] *= damping; }
    if (xp[a] > hi[a]) { xp[a] = hi[a]; vp[a] *= damping; }
  }
}

// one step; records what the adjoint needs
void step(const Model& M, double mu, std::vector<V>& x, std::vector<V>& v, StepRec* rec) {
  const int n = (int)x.size();
  std::vector<std::vector<int>> nb;
  neighbors(x, M.k.h, nb);
  std::vector<V> F(n), Fp(n, V{0, 0, 0}), xs(n);
  for (int i = 0; i < n; ++i) {
    V f{0, 0, 0};
    for (int j : nb[i]) f = f - (v[i] - v[j]) * (M.vol2 * mu * M.k.L(len(x[i] - x[j])));
    f.y -= M.m * M.g;
    F[i] = f;
  }
  std::vector<double> p(n, 0.0), rho(n);
  if (rec) {
    rec->x = x;
    rec->v = v;
    rec->F = F;
    rec->nb = nb;
    rec->xs.assign(M.K, {});
    rec->rho.assign(M.K, {});
    rec->p.assign(M.K, {});
  }
  const double c0 = M.m * M.m / (M.rho0 * M.rho0);
  for (int it = 0; it < M.K; ++it) {
    for (int i = 0; i < n; ++i) {
      V vv = v[i] + (F[i] + Fp[i]) * (M.dt / M.m);
      V xx = x[i] + vv * M.dt;
      clamp(xx, vv, M, 0.0);
      xs[i] = xx;
    }
    for (int i = 0; i < n; ++i) {
      double d = M.m * M.k.W(0.0);
      for (int j : nb[i]) d += M.m * M.k.W(len(xs[i] - xs[j]));
      rho[i] = d;
      p[i] += M.delta * smax(d - M.rho0, M.eps);
    }
    for (int i = 0; i < n; ++i) {
      V f{0, 0, 0};
      for (int j : nb[i]) {
        const V r = x[i] - x[j];
        f = f + r * (-c0 * (p[i] + p[j]) * M.k.G(len(r)));
      }
      Fp[i] = f;
    }
    if (rec) {
      rec->xs[it] = xs;
      rec->rho[it] = rho;
      rec->p[it] = p;
    }
  }
  for (int i = 0; i < n; ++i) {
    V vv = v[i] + (F[i] + Fp[i]) * (M.dt / M.m);
    V xx = x[i] + vv * M.dt;
    clamp(xx, vv, M, -0.5);
    x[i] = xx;
    v[i] = vv;
  }
}

// adjoint of one step: (xb, vb) at the step's end -> at its start; mub += dL/dmu
void step_adjoint(const Model& M, double mu, const StepRec& R, std::vector<V>& xb, std::vector<V>& vb, double& mub) {
  const int n = (int)R.x.size();
  const double c0 = M.m * M.m / (M.rho0 * M.rho0);
  const double s = M.dt / M.m;
  std::vector<V> Fb(n), Fpb(n), xsb(n);
  std::vector<double> pc(n, 0.0), rb(n);
  for (int i = 0; i < n; ++i) {
    vb[i] = vb[i] + xb[i] * M.dt;
    Fb[i] = vb[i] * s;
    Fpb[i] = vb[i] * s;
  }
  for (int it = M.K - 1; it >= 0; --it) {
    const std::vector<double>& p = R.p[it];
    const std::vector<double>& rho = R.rho[it];
    const std::vector<V>& xs = R.xs[it];
    for (int i = 0; i < n; ++i) {
      double pb = 0.0;
      V g{0, 0, 0};
      for (int j : R.nb[i]) {
        const V r = R.x[i] - R.x[j];
        const double rl = len(r);
        const double G = M.k.G(rl);
        const V d = Fpb[i] - Fpb[j];
        const double rd = dot(r, d);
        pb += -c0 * rd * G;
        const double cij = -c0 * (p[i] + p[j]);
        const double t = rl > 0.0 ? M.k.dG(rl) / rl * rd : 0.0;
        g = g + (d * G + r * t) * cij;
      }
      pc[i] += pb;
      rb[i] = M.delta * dsmax(rho[i] - M.rho0, M.eps) * pc[i];
      xb[i] = xb[i] + g;
    }
    for (int i = 0; i < n; ++i) {
      V g{0, 0, 0};
      for (int j : R.nb[i]) {
        const V r = xs[i] - xs[j];
        const double rl = len(r);
        if (rl <= 0.0) continue;
        g = g + r * (M.m * M.k.dW(rl) / rl * (rb[i] + rb[j]));
      }
      xsb[i] = g;
    }
    for (int i = 0; i < n; ++i) {
      xb[i] = xb[i] + xsb[i];
      const V vs = xsb[i] * M.dt;
      vb[i] = vb[i] + vs;
      Fb[i] = Fb[i] + vs * s;
      Fpb[i] = it > 0 ? vs * s : V{0, 0, 0};
    }
  }
  std::vector<V> gx(n), gv(n);
  for (int i = 0; i < n; ++i) {
    V ax{0, 0, 0}, av{0, 0, 0};
    for (int j : R.nb[i]) {
      const V r = R.x[i] - R.x[j];
      const double rl = len(r);
      const double Lr = M.k.L(rl), dLr = M.k.dL(rl);
      const V dF = Fb[i] - Fb[j];
      const V dv = R.v[i] - R.v[j];
      av = av - dF * (M.vol2 * mu * Lr);
      if (rl > 0.0) ax = ax + r * (-M.vol2 * mu * dLr * dot(dv, dF) / rl);
      mub += -M.vol2 * Lr * dot(dv, Fb[i]);
    }
    gx[i] = ax;
    gv[i] = av;
  }
  for (int i = 0; i < n; ++i) {
    xb[i] = xb[i] + gx[i];
    vb[i] = vb[i] + gv[i];
  }
}

}  // namespace

extern "C" {

// loss (and, when grad_v3 or grad_mu is non-null, its gradient with respect
// to the initial velocities and the viscosity) of `steps` steps from
// (pos3, vel3), n x 3 doubles each.
int orc_adjoint_run(const upf_params* prm, const double* pos3, const double* vel3, uint32_t n, int32_t steps,
                    int32_t iterations, const double* target3, double com_weight, double density_weight,
                    double viscosity, double eps_rho, double* loss_out, double* grad_v3, double* grad_mu) {
  if (!prm || !pos3 || !vel3 || n == 0 || steps < 1 || iterations < 1) return -1;
  Model M;
  const double h = prm->support_radius;
  const double pi = 3.14159265358979323846;
  M.k.h = h;
  M.k.wn = 2.546479089470325472 / (h * h * h);
  M.k.gc = -45.0 / (pi * std::pow(h, 6));
  M.k.lc = 45.0 / (pi * std::pow(h, 6));
  M.m = prm->mass;
  M.rho0 = prm->rest_density;
  M.dt = prm->dt;
  M.delta = prm->density_error_factor;
  M.vol2 = ((double)prm->mass / prm->rest_density) * ((double)prm->mass / prm->rest_density);
  M.g = prm->gravity;
  M.lo = {prm->collision_min[0], prm->collision_min[1], prm->collision_min[2]};
  M.hi = {prm->collision_max[0], prm->collision_max[1], prm->collision_max[2]};
  M.K = iterations;
  M.eps = eps_rho * M.rho0;
  std::vector<V> x(n), v(n);
  for (uint32_t i = 0; i < n; ++i) {
    x[i] = {pos3[3 * i], pos3[3 * i + 1], pos3[3 * i + 2]};
    v[i] = {vel3[3 * i], vel3[3 * i + 1], vel3[3 * i + 2]};
  }
  const bool grad = grad_v3 || grad_mu;
  std::vector<StepRec> recs(grad ? steps : 0);
  for (int t = 0; t < steps; ++t) step(M, viscosity, x, v, grad ? &recs[t] : nullptr);
  // loss at the final positions
  std::vector<std::vector<int>> nb;
  neighbors(x, h, nb);
  std::vector<double> rho(n);
  V com{0, 0, 0};
  double sd = 0.0;
  for (uint32_t i = 0; i < n; ++i) {
    double d = M.m * M.k.W(0.0);
    for (int j : nb[i]) d += M.m * M.k.W(len(x[i] - x[j]));
    rho[i] = d;
    com = com + x[i];
    sd += (d - M.rho0) * (d - M.rho0);
  }
  com = com * (1.0 / n);
  const V tgt{target3[0], target3[1], target3[2]};
  const V dc = com - tgt;
  if (loss_out) *loss_out = com_weight * dot(dc, dc) + density_weight * sd / n;
  if (!grad) return 0;
  std::vector<V> xb(n), vb(n, V{0, 0, 0});
  const V gcom = dc * (2.0 * com_weight / n);
  const double gr = 2.0 * density_weight / n;
  for (uint32_t i = 0; i < n; ++i) {
    V g = gcom;
    for (int j : nb[i]) {
      const V r = x[i] - x[j];
      const double rl = len(r);
      if (rl <= 0.0) continue;
      g = g + r * (M.m * M.k.dW(rl) / rl * (gr * (rho[i] - M.rho0) + gr * (rho[j] - M.rho0)));
    }
    xb[i] = g;
  }
  double mub = 0.0;
  for (int t = steps - 1; t >= 0; --t) step_adjoint(M, viscosity, recs[t], xb, vb, mub);
  if (grad_v3)
    for (uint32_t i = 0; i < n; ++i) {
      grad_v3[3 * i] = vb[i].x;
      grad_v3[3 * i + 1] = vb[i].y;
      grad_v3[3 * i + 2] = vb[i].z;
    }
  if (grad_mu) *grad_mu = mub;
  return 0;
}

}  // extern "C"
