// akb_fe2_oracle.cc -- CPU restatement of the periodic RVE relaxation.
//
// TEST INFRASTRUCTURE ONLY (checker of akantu_b200/csrc/akb_rve.cu).
//
// The RVE is a cube of n^3 hexahedron_8 voxels with periodic nodes (n^3
// unique nodes). Its displacement is u(X) = H X + w(X), w periodic, so the
// gradient at a Gauss point is H + sum_a w_a (x) grad N_a. Stresses follow the
// reference's laws (small-strain elastic: material_elastic_inline_impl.hh:
// 41-55; neo-Hookean S = mu (I - C^-1) + lambda ln J C^-1:
// material_neohookean_inline_impl.hh:46-65) with P = F S, and the element
// force is the reference's -sum_q P grad N_a detJ w (material.cc:637-722 in
// its P form). The fluctuation w solves sum forces = 0 by dynamic relaxation:
// a leapfrog with mass-proportional damping on a fictitious mass that gives
// every voxel the same P-wave speed. The homogenised stress is the volume
// average of P.
#include "akb_fe2_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace {

constexpr int kOx[8] = {0, 1, 1, 0, 0, 1, 1, 0};
constexpr int kOy[8] = {0, 0, 1, 1, 0, 0, 1, 1};
constexpr int kOz[8] = {0, 0, 0, 0, 1, 1, 1, 1};

// grad N_a at Gauss point q of a cube voxel of side h: B[(q*8 + a)*3 + j]
// (hexahedron_8 shapes, element_class_hexahedron_8_inline_impl.hh:118-215;
// 2 x 2 x 2 Gauss points +-1/sqrt(3), bit k of q = sign along axis k).
void voxel_gradients(double h, double* B) {
  const double g = 1.0 / std::sqrt(3.0);
  for (int q = 0; q < 8; ++q) {
    const double c[3] = {(q & 1) ? g : -g, (q & 2) ? g : -g, (q & 4) ? g : -g};
    for (int a = 0; a < 8; ++a) {
      const double s[3] = {2.0 * kOx[a] - 1, 2.0 * kOy[a] - 1, 2.0 * kOz[a] - 1};
      for (int j = 0; j < 3; ++j) {
        double v = 0.125 * s[j];
        for (int k = 0; k < 3; ++k)
          if (k != j) v *= 1.0 + s[k] * c[k];
        B[(q * 8 + a) * 3 + j] = v * (2.0 / h);
      }
    }
  }
}

double det3(const double* m) {
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
         m[2] * (m[3] * m[7] - m[4] * m[6]);
}

void inv3(const double* m, double* r) {
  const double d = det3(m);
  r[0] = (m[4] * m[8] - m[5] * m[7]) / d;
  r[1] = (m[2] * m[7] - m[1] * m[8]) / d;
  r[2] = (m[1] * m[5] - m[2] * m[4]) / d;
  r[3] = (m[5] * m[6] - m[3] * m[8]) / d;
  r[4] = (m[0] * m[8] - m[2] * m[6]) / d;
  r[5] = (m[2] * m[3] - m[0] * m[5]) / d;
  r[6] = (m[3] * m[7] - m[4] * m[6]) / d;
  r[7] = (m[1] * m[6] - m[0] * m[7]) / d;
  r[8] = (m[0] * m[4] - m[1] * m[3]) / d;
}

// P (row-major) from g (row-major, g[i*3+j] = du_i/dX_j).
void first_piola(int kind, double lam, double mu, const double* g, double* P) {
  if (kind == 0) {
    const double tr = g[0] + g[4] + g[8];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        P[i * 3 + j] = mu * (g[i * 3 + j] + g[j * 3 + i]) + (i == j ? lam * tr : 0.0);
    return;
  }
  double F[9], C[9], Ci[9], S[9];
  for (int k = 0; k < 9; ++k) F[k] = g[k] + (k % 4 == 0 ? 1.0 : 0.0);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double c = 0;
      for (int k = 0; k < 3; ++k) c += F[k * 3 + i] * F[k * 3 + j];
      C[i * 3 + j] = c;
    }
  const double J = det3(F);
  inv3(C, Ci);
  const double lnJ = std::log(J);
  for (int k = 0; k < 9; ++k) S[k] = mu * ((k % 4 == 0 ? 1.0 : 0.0) - Ci[k]) + lam * lnJ * Ci[k];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double c = 0;
      for (int k = 0; k < 3; ++k) c += F[i * 3 + k] * S[k * 3 + j];
      P[i * 3 + j] = c;
    }
}

// Smallest eigenvalue of a symmetric 3x3 matrix (trigonometric solution of
// the characteristic cubic, O. K. Smith, Comm. ACM 4(4):168, 1961).
double smallest_eigenvalue(const double* A) {
  const double p1 = A[1] * A[1] + A[2] * A[2] + A[5] * A[5];
  const double q = (A[0] + A[4] + A[8]) / 3.0;
  const double p2 = (A[0] - q) * (A[0] - q) + (A[4] - q) * (A[4] - q) +
                    (A[8] - q) * (A[8] - q) + 2.0 * p1;
  if (p2 <= 0.0) return q;
  const double p = std::sqrt(p2 / 6.0);
  double Bm[9];
  for (int k = 0; k < 9; ++k) Bm[k] = (A[k] - (k % 4 == 0 ? q : 0.0)) / p;
  double r = det3(Bm) / 2.0;
  r = std::min(1.0, std::max(-1.0, r));
  const double phi = std::acos(r) / 3.0;
  return q + 2.0 * p * std::cos(phi + 2.0 * M_PI / 3.0);
}

struct Rve {
  int n;
  double L, h;
  const uint8_t* vm;
  const double *lam, *mu;
  const int32_t* kind;
  double B[8 * 8 * 3];
  double H[9];  // row-major
};

inline int node_of(int n, int ex, int ey, int ez, int a) {
  return (ex + kOx[a]) % n + n * ((ey + kOy[a]) % n + n * ((ez + kOz[a]) % n));
}

// Internal force f (n^3 x 3, reference sign: -sum P grad N w detJ) and the
// sum of w detJ P over the RVE (row-major).
void forces(const Rve& R, const double* w, double* f, double* Psum) {
  const int n = R.n, nn = n * n * n;
  const double wq = R.h * R.h * R.h / 8.0;
  std::fill(f, f + 3 * nn, 0.0);
  if (Psum) std::fill(Psum, Psum + 9, 0.0);
  for (int ez = 0; ez < n; ++ez)
    for (int ey = 0; ey < n; ++ey)
      for (int ex = 0; ex < n; ++ex) {
        const int e = ex + n * (ey + n * ez);
        const int m = R.vm[e];
        int nd[8];
        for (int a = 0; a < 8; ++a) nd[a] = node_of(n, ex, ey, ez, a);
        double fe[24] = {0};
        for (int q = 0; q < 8; ++q) {
          const double* Bq = R.B + q * 24;
          double g[9];
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
              double c = R.H[i * 3 + j];
              for (int a = 1; a < 8; ++a) c += (w[nd[a] * 3 + i] - w[nd[0] * 3 + i]) * Bq[a * 3 + j];
              g[i * 3 + j] = c;
            }
          double P[9];
          first_piola(R.kind[m], R.lam[m], R.mu[m], g, P);
          for (int a = 0; a < 8; ++a)
            for (int i = 0; i < 3; ++i) {
              double c = 0;
              for (int j = 0; j < 3; ++j) c += P[i * 3 + j] * Bq[a * 3 + j];
              fe[a * 3 + i] += wq * c;
            }
          if (Psum)
            for (int k = 0; k < 9; ++k) Psum[k] += wq * P[k];
        }
        for (int a = 0; a < 8; ++a)
          for (int i = 0; i < 3; ++i) f[nd[a] * 3 + i] -= fe[a * 3 + i];
      }
}

void setup(Rve& R, int n, double L, const uint8_t* vm, const double* lam, const double* mu,
           const int32_t* kind, const double* grad_u) {
  R.n = n;
  R.L = L;
  R.h = L / n;
  R.vm = vm;
  R.lam = lam;
  R.mu = mu;
  R.kind = kind;
  voxel_gradients(R.h, R.B);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) R.H[i * 3 + j] = grad_u[i + 3 * j];
}

}  // namespace

extern "C" {

void oracle_rve_parameters(int32_t n, double L, int32_t nb_materials, const double* lambda,
                           const double* mu, const int32_t* kind, const double* grad_u,
                           double time_step_factor, double damping_factor, double* dt,
                           double* damping) {
  double F[9], C[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) F[i * 3 + j] = grad_u[i + 3 * j] + (i == j ? 1.0 : 0.0);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double c = 0;
      for (int k = 0; k < 3; ++k) c += F[k * 3 + i] * F[k * 3 + j];
      C[i * 3 + j] = c;
    }
  const double J = det3(F);
  const double smin = std::sqrt(std::max(smallest_eigenvalue(C), 0.0));
  const double stiff = J > 0 ? std::max(0.0, -std::log(J)) : 0.0;
  double c2 = 0.0, cs = 1e300;
  for (int m = 0; m < nb_materials; ++m) {
    const double m2 = lambda[m] + 2.0 * mu[m];  // fictitious density: unit P-wave speed
    const double t = kind[m] == 1 ? (m2 + 2.0 * lambda[m] * stiff) / m2 : 1.0;
    c2 = std::max(c2, t);
    cs = std::min(cs, std::sqrt(mu[m] / m2));
  }
  const double h = L / n;
  *dt = time_step_factor * h * smin / std::sqrt(c2);
  *damping = damping_factor * 2.0 * (2.0 * M_PI / L) * cs;
}

void oracle_rve_stress(int32_t n, double L, const uint8_t* voxel_material,
                       const double* lambda, const double* mu, const int32_t* kind,
                       const double* grad_u, const double* fluct, double* stress,
                       double* internal_force) {
  Rve R;
  setup(R, n, L, voxel_material, lambda, mu, kind, grad_u);
  std::vector<double> f(3 * (size_t)n * n * n);
  double Ps[9];
  forces(R, fluct, f.data(), Ps);
  const double V = L * L * L;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) stress[i + 3 * j] = Ps[i * 3 + j] / V;
  if (internal_force) std::copy(f.begin(), f.end(), internal_force);
}

int32_t oracle_rve_solve(int32_t n, double L, const uint8_t* voxel_material,
                         int32_t nb_materials, const double* lambda, const double* mu,
                         const int32_t* kind, const double* grad_u, double* fluct,
                         int32_t max_iterations, int32_t check_interval, double tolerance,
                         double time_step_factor, double damping_factor, double* stress,
                         double* residual) {
  Rve R;
  setup(R, n, L, voxel_material, lambda, mu, kind, grad_u);
  const int nn = n * n * n;
  const double h = R.h;
  // lumped fictitious mass: rho_e = lambda_e + 2 mu_e, h^3/8 per corner
  std::vector<double> mass(nn, 0.0);
  for (int ez = 0; ez < n; ++ez)
    for (int ey = 0; ey < n; ++ey)
      for (int ex = 0; ex < n; ++ex) {
        const int m = voxel_material[ex + n * (ey + n * ez)];
        for (int a = 0; a < 8; ++a)
          mass[node_of(n, ex, ey, ez, a)] += (lambda[m] + 2.0 * mu[m]) * h * h * h / 8.0;
      }
  double dt, cd;
  oracle_rve_parameters(n, L, nb_materials, lambda, mu, kind, grad_u, time_step_factor,
                        damping_factor, &dt, &cd);
  double hmax = 0, mumax = 0;
  for (int k = 0; k < 9; ++k) hmax = std::max(hmax, std::fabs(grad_u[k]));
  for (int m = 0; m < nb_materials; ++m) mumax = std::max(mumax, mu[m]);
  const double fscale = h * h * mumax * std::max(hmax, 1e-6);
  // an attempt whose residual turns non-finite or exceeds 1e4 restarts from
  // the initial state with a 0.6x time step, at most 3 times
  const std::vector<double> start(fluct, fluct + 3 * nn);
  std::vector<double> f(3 * nn), v(3 * nn);
  int total = 0, k = 0;
  double r = 0, tsf = 1.0;
  for (int attempt = 0;; ++attempt, tsf *= 0.6) {
    std::copy(start.begin(), start.end(), fluct);
    std::fill(v.begin(), v.end(), 0.0);
    const double dta = tsf * dt;
    const double a1 = 1.0 - 0.5 * cd * dta, a2 = 1.0 + 0.5 * cd * dta;
    bool diverged = false;
    for (k = 0;; ++k) {
      forces(R, fluct, f.data(), nullptr);
      const bool last = k >= max_iterations;
      if (last || (check_interval > 0 && k % check_interval == 0)) {
        double fm = 0;
        for (double x : f) fm = std::isfinite(x) ? std::max(fm, std::fabs(x)) : INFINITY;
        r = fm / fscale;
        diverged = !(r <= 1e4);
        if (last || diverged || (tolerance >= 0 && r <= tolerance)) break;
      }
      for (int a = 0; a < nn; ++a)
        for (int i = 0; i < 3; ++i) {
          const int idx = a * 3 + i;
          v[idx] = (a1 * v[idx] + dta * f[idx] / mass[a]) / a2;
          fluct[idx] += dta * v[idx];
        }
    }
    total += k;
    if (!diverged || attempt >= 3) break;
  }
  oracle_rve_stress(n, L, voxel_material, lambda, mu, kind, grad_u, fluct, stress, nullptr);
  *residual = r;
  return total;
}

}  // extern "C"

// ------------------------------------------------------------------- MLP
namespace {

float bf16_round(float f) {  // round to nearest even, BF16 kept in a float
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  u &= 0xFFFF0000u;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

struct MlpShape {
  int nl, nin, nout, width;
  std::vector<int> K, N;
  std::vector<int64_t> woff, boff;
};

MlpShape mlp_shape(int nin, int nout, int width, int nhidden) {
  MlpShape s;
  s.nl = nhidden + 1;
  s.nin = nin;
  s.nout = nout;
  s.width = width;
  int64_t off = 0;
  for (int l = 0; l < s.nl; ++l) {
    s.K.push_back(l == 0 ? nin : width);
    s.N.push_back(l == s.nl - 1 ? nout : width);
    s.woff.push_back(off);
    off += (int64_t)s.K[l] * s.N[l];
    s.boff.push_back(off);
    off += s.N[l];
  }
  return s;
}

// Forward of one sample; keeps per-layer inputs (as consumed) and
// pre-activations for the backward pass.
void mlp_sample(const MlpShape& S, const float* P, const float* sc, const double* x, bool bf,
                std::vector<std::vector<double>>& in, std::vector<std::vector<double>>& z,
                std::vector<double>& out) {
  auto R = [&](double v) { return bf ? (double)bf16_round((float)v) : v; };
  auto F = [&](double v) { return bf ? (double)(float)v : v; };
  in.assign(S.nl, {});
  z.assign(S.nl, {});
  in[0].resize(S.nin);
  for (int j = 0; j < S.nin; ++j) in[0][j] = R((double)(float)((x[j] - sc[j]) * sc[S.nin + j]));
  for (int l = 0; l < S.nl; ++l) {
    z[l].resize(S.N[l]);
    for (int o = 0; o < S.N[l]; ++o) {
      double acc = 0;
      for (int k = 0; k < S.K[l]; ++k) acc += R(P[S.woff[l] + (int64_t)o * S.K[l] + k]) * in[l][k];
      z[l][o] = F(F(acc) + P[S.boff[l] + o]);
    }
    if (l < S.nl - 1) {
      in[l + 1].resize(S.N[l]);
      for (int o = 0; o < S.N[l]; ++o) in[l + 1][o] = R(z[l][o] / (1.0 + std::exp(-z[l][o])));
    }
  }
  out = z[S.nl - 1];
}

}  // namespace

extern "C" {

void oracle_mlp_forward(int32_t nin, int32_t nout, int32_t width, int32_t nhidden,
                        const float* params, const float* scaling, int64_t nb, const double* x,
                        double* y, int32_t emulate_bf16) {
  const MlpShape S = mlp_shape(nin, nout, width, nhidden);
  const float* osh = scaling + 2 * nin;
  const float* osc = scaling + 2 * nin + nout;
  std::vector<std::vector<double>> in, z;
  std::vector<double> out;
  for (int64_t r = 0; r < nb; ++r) {
    mlp_sample(S, params, scaling, x + r * nin, emulate_bf16 != 0, in, z, out);
    for (int j = 0; j < nout; ++j) y[r * nout + j] = out[j] * osc[j] + osh[j];
  }
}

double oracle_mlp_gradients(int32_t nin, int32_t nout, int32_t width, int32_t nhidden,
                            const float* params, const float* scaling, int64_t nb,
                            const double* x, const double* target, double* grad,
                            int32_t emulate_bf16) {
  const MlpShape S = mlp_shape(nin, nout, width, nhidden);
  const bool bf = emulate_bf16 != 0;
  auto R = [&](double v) { return bf ? (double)bf16_round((float)v) : v; };
  const float* osh = scaling + 2 * nin;
  const float* osc = scaling + 2 * nin + nout;
  const int64_t np = S.boff[S.nl - 1] + S.N[S.nl - 1];
  std::fill(grad, grad + np, 0.0);
  double loss = 0;
  const double scale = 2.0 / ((double)nb * nout);
  std::vector<std::vector<double>> in, z;
  std::vector<double> out;
  for (int64_t r = 0; r < nb; ++r) {
    mlp_sample(S, params, scaling, x + r * nin, bf, in, z, out);
    std::vector<double> d(nout);
    for (int j = 0; j < nout; ++j) {
      const double t = bf ? (double)(float)((target[r * nout + j] - osh[j]) / osc[j])
                          : (target[r * nout + j] - osh[j]) / osc[j];
      const double e = out[j] - t;
      loss += e * e;
      d[j] = R(bf ? (double)((float)scale * (float)e) : scale * e);
    }
    for (int l = S.nl - 1; l >= 0; --l) {
      for (int o = 0; o < S.N[l]; ++o) {
        grad[S.boff[l] + o] += d[o];
        for (int k = 0; k < S.K[l]; ++k) grad[S.woff[l] + (int64_t)o * S.K[l] + k] += d[o] * in[l][k];
      }
      if (l == 0) break;
      std::vector<double> dp(S.K[l]);
      for (int k = 0; k < S.K[l]; ++k) {
        double acc = 0;
        for (int o = 0; o < S.N[l]; ++o) acc += d[o] * R(params[S.woff[l] + (int64_t)o * S.K[l] + k]);
        const double zz = z[l - 1][k];
        const double sg = 1.0 / (1.0 + std::exp(-zz));
        dp[k] = R(acc * sg * (1.0 + zz * (1.0 - sg)));
      }
      d.swap(dp);
    }
  }
  return loss / ((double)nb * nout);
}

}  // extern "C"
