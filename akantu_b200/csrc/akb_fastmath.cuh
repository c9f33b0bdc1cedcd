// akb_fastmath.cuh -- element arithmetic of the fast paths (FMA allowed).
//
// Same mathematics as the reference's FE engine (element_class_tmpl.hh:270-355,
// shape_lagrange_inline_impl.hh:355-423, integrator_gauss_inline_impl.hh:426-455,
// material_elastic_inline_impl.hh:41-63, material_neohookean_inline_impl.hh:46-65),
// written for registers: geometry recomputed from the coordinates, differences
// to the element's first node taken in FP64 before any FP32 rounding, the
// internal force written as f_a = sum_q w_q det J_q P_q grad N_a with P = sigma
// (small strain) or P = F S (finite strain), which equals B^T sigma_voigt and
// (B_L0 + B_L2)^T S_voigt of material.cc:178-230 and 637-722.
#pragma once

#include "akb_internal.cuh"

namespace akb {
namespace fast {

// Central-difference predictor and corrector of one free DOF
// (newmark-beta.cc:73-81 and 186-200 with alpha = 0, beta = 1/2), with every
// rounding spelled out so that every kernel computing them agrees bitwise.
__device__ inline void predict(double dt, double& u, double& v, double a) {
  const double dta = __dmul_rn(dt, a);
  u = __dadd_rn(u, __fma_rn(0.5 * dt, dta, __dmul_rn(dt, v)));
  v = __dadd_rn(v, dta);
}
// x = (f_ext + f_int) / M - a; v += dt/2 x; a += x; u += 0 x (only matters
// when x is not finite).
__device__ inline void correct(double dt, double r, double inv_m, double& u, double& v,
                               double& a) {
  const double x = __fma_rn(r, inv_m, -a);
  v = __fma_rn(0.5 * dt, x, v);
  a = __dadd_rn(a, x);
  if (!isfinite(x)) u += 0.0 * x;
}

// dN_a/dxi_k at quadrature point q (k-th row), reference element tables.
template <int T, typename S>
__device__ inline S dN(int k, int a, int q) {
  if (T == AKB_SEGMENT_2) return a == 0 ? S(-0.5) : S(0.5);
  if (T == AKB_TRIANGLE_3) {
    if (a == 0) return S(-1);
    return (a == k + 1) ? S(1) : S(0);
  }
  if (T == AKB_TETRAHEDRON_4) {
    if (a == 0) return S(-1);
    return (a == k + 1) ? S(1) : S(0);
  }
  // hexahedron_8: corners (sx, sy, sz), Gauss point (+-g)^3, g = 1/sqrt(3)
  const int sx[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
  const int sy[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
  const int sz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
  const S g = S(0.57735026918962576451);
  const S cx = (q & 1) ? g : -g, cy = (q & 2) ? g : -g, cz = (q & 4) ? g : -g;
  const S ax = S(1) + sx[a] * cx, ay = S(1) + sy[a] * cy, az = S(1) + sz[a] * cz;
  if (k == 0) return S(0.125) * sx[a] * ay * az;
  if (k == 1) return S(0.125) * sy[a] * ax * az;
  return S(0.125) * sz[a] * ax * ay;
}

template <int T> __host__ __device__ constexpr double weight() {
  return T == AKB_SEGMENT_2 ? 2.0 : T == AKB_TRIANGLE_3 ? 0.5 : T == AKB_TETRAHEDRON_4 ? 1.0 / 6.0 : 1.0;
}

template <int d, typename S>
__device__ inline S det(const S* J) {
  if (d == 1) return J[0];
  if (d == 2) return J[0] * J[3] - J[1] * J[2];
  return J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
         J[2] * (J[3] * J[7] - J[4] * J[6]);
}

// row-major d x d inverse times det (adjugate); returns det
template <int d, typename S>
__device__ inline S adjugate(const S* J, S* A) {
  if (d == 1) {
    A[0] = S(1);
    return J[0];
  }
  if (d == 2) {
    A[0] = J[3]; A[1] = -J[1]; A[2] = -J[2]; A[3] = J[0];
    return J[0] * J[3] - J[1] * J[2];
  }
  A[0] = J[4] * J[8] - J[5] * J[7];
  A[1] = J[2] * J[7] - J[1] * J[8];
  A[2] = J[1] * J[5] - J[2] * J[4];
  A[3] = J[5] * J[6] - J[3] * J[8];
  A[4] = J[0] * J[8] - J[2] * J[6];
  A[5] = J[2] * J[3] - J[0] * J[5];
  A[6] = J[3] * J[7] - J[4] * J[6];
  A[7] = J[1] * J[6] - J[0] * J[7];
  A[8] = J[0] * J[4] - J[1] * J[3];
  return J[0] * A[0] + J[1] * A[3] + J[2] * A[6];
}

// Stress at one point; g is row-major grad u (g[i*d+j] = du_i/dX_j); returns
// P (first Piola for finite strain, Cauchy for small strain), row-major.
template <int d, typename S>
__device__ inline void stress_P(const MatParams& p, const S* g, S* P) {
  const S lam = S(p.lambda), mu = S(p.mu);
  if (d == 1 && !p.finite) {
    P[0] = S(p.E) * g[0];
    return;
  }
  if (!p.finite) {
    S tr = 0;
#pragma unroll
    for (int i = 0; i < d; ++i) tr += g[i * d + i];
#pragma unroll
    for (int i = 0; i < d; ++i)
#pragma unroll
      for (int j = 0; j < d; ++j) P[i * d + j] = mu * (g[i * d + j] + g[j * d + i]) + (i == j ? lam * tr : S(0));
    return;
  }
  if (d == 3 && p.kind == AKB_MATERIAL_NEOHOOKEAN) {
    // P = F S = mu (F - F^-T) + lambda ln J F^-T (F C^-1 = F^-T), written
    // without O(1) terms that cancel near F = I: with t = tr g,
    // I2 = (t^2 - tr g^2)/2, J - 1 = t + I2 + det g,
    // adj(F) = (1 + t + I2) I - (1 + t) g + g^2, F^-T = adj(F)^T / J and
    // F - F^-T = g + (det(g) I + (1 + t) g^T - (g^T)^2) / J.
    S gg[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j)
        gg[i * 3 + j] = g[i * 3] * g[j] + g[i * 3 + 1] * g[3 + j] + g[i * 3 + 2] * g[6 + j];
    const S t = g[0] + g[4] + g[8];
    const S I2 = S(0.5) * (t * t - (gg[0] + gg[4] + gg[8]));
    const S dg = det<3, S>(g);
    const S jm1 = t + I2 + dg;
    const S iJ = S(1) / (S(1) + jm1);
    const S a = mu * iJ, b = lam * log1p(jm1) * iJ, c = S(1) + t;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const S gt = g[j * 3 + i], ggt = gg[j * 3 + i];
        const S adjT = (i == j ? c + I2 : S(0)) - c * gt + ggt;
        const S dev = (i == j ? dg : S(0)) + c * gt - ggt;
        P[i * 3 + j] = mu * g[i * 3 + j] + a * dev + b * adjT;
      }
    return;
  }
  // Written in terms of grad u so that no O(1) quantity cancels near F = I
  // (in FP32, C - I computed as C minus the identity loses eps/strain):
  //   E2 = C - I = g + g^T + g^T g
  //   neo-Hookean S = mu I + (lambda ln J - mu) C^-1 = C^-1 (mu E2 + lambda ln J I)
  //   with J - 1 = I1 + I2 + I3 of g and ln J = log1p(J - 1);
  //   St-Venant-Kirchhoff S = lambda tr(E2)/2 I + mu E2.
  S E2[9], Sk[9];
#pragma unroll
  for (int i = 0; i < d; ++i)
#pragma unroll
    for (int j = 0; j < d; ++j) {
      S c = g[i * d + j] + g[j * d + i];
#pragma unroll
      for (int k = 0; k < d; ++k) c += g[k * d + i] * g[k * d + j];
      E2[i * d + j] = c;
    }
  if (p.kind == AKB_MATERIAL_NEOHOOKEAN) {
    S tr = 0;
#pragma unroll
    for (int i = 0; i < d; ++i) tr += g[i * d + i];
    S Jm1 = tr;
    if (d == 2) Jm1 += g[0] * g[3] - g[1] * g[2];
    if (d == 3) {
      S tr2 = 0;
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k) tr2 += g[i * 3 + k] * g[k * 3 + i];
      Jm1 += S(0.5) * (tr * tr - tr2) + det<3, S>(g);
    }
    const S lnJ = log1p(Jm1);
    const S J = S(1) + Jm1;
    S C[9], Ca[9], M[9];
#pragma unroll
    for (int k = 0; k < d * d; ++k) C[k] = E2[k];
#pragma unroll
    for (int i = 0; i < d; ++i) C[i * d + i] += S(1);
    adjugate<d, S>(C, Ca);
    const S idetC = S(1) / (J * J);
#pragma unroll
    for (int k = 0; k < d * d; ++k) M[k] = mu * E2[k];
#pragma unroll
    for (int i = 0; i < d; ++i) M[i * d + i] += lam * lnJ;
#pragma unroll
    for (int i = 0; i < d; ++i)
#pragma unroll
      for (int j = 0; j < d; ++j) {
        S c = 0;
#pragma unroll
        for (int k = 0; k < d; ++k) c += Ca[i * d + k] * M[k * d + j];
        Sk[i * d + j] = c * idetC;
      }
  } else {
    S trE = 0;
#pragma unroll
    for (int i = 0; i < d; ++i) trE += S(0.5) * E2[i * d + i];
#pragma unroll
    for (int i = 0; i < d; ++i)
#pragma unroll
      for (int j = 0; j < d; ++j) Sk[i * d + j] = mu * E2[i * d + j] + (i == j ? lam * trE : S(0));
  }
  S F[9];
#pragma unroll
  for (int i = 0; i < d; ++i)
#pragma unroll
    for (int j = 0; j < d; ++j) F[i * d + j] = g[i * d + j] + (i == j ? S(1) : S(0));
#pragma unroll
  for (int i = 0; i < d; ++i)
#pragma unroll
    for (int j = 0; j < d; ++j) {
      S c = 0;
#pragma unroll
      for (int k = 0; k < d; ++k) c += F[i * d + k] * Sk[k * d + j];
      P[i * d + j] = c;
    }
}

// Simplex (triangle_3, tetrahedron_4) internal force. The natural
// derivatives are constant (dN_a/dxi_k = delta(a, k+1) - delta(a, 0)), so the
// rows of J are X_a - X_0 (a >= 1) and w det J grad N_a = w adj(J)[:, a-1]:
//   g = (1/det J) sum_a (u_a - u_0) (x) adj(J)[:, a-1],
//   fe_a = w P adj(J)[:, a-1] (a >= 1), fe_0 = -(fe_1 + ... + fe_d).
template <int T, typename S>
__device__ inline void simplex_force(const MatParams& p, const S* dX, const S* du, S* fe) {
  constexpr int d = ET<T>::dim;
  S J[9], A[9];
#pragma unroll
  for (int k = 0; k < d; ++k)
#pragma unroll
    for (int j = 0; j < d; ++j) J[k * d + j] = dX[(k + 1) * d + j];
  const S detJ = adjugate<d, S>(J, A);
  const S idet = S(1) / detJ;
  S g[9];
#pragma unroll
  for (int i = 0; i < d; ++i)
#pragma unroll
    for (int j = 0; j < d; ++j) {
      S c = du[1 * d + i] * A[j * d + 0];
#pragma unroll
      for (int a = 2; a <= d; ++a) c += du[a * d + i] * A[j * d + (a - 1)];
      g[i * d + j] = c * idet;
    }
  S P[9];
  stress_P<d, S>(p, g, P);
  const S w = S(weight<T>());
#pragma unroll
  for (int k = 0; k < d * d; ++k) P[k] *= w;
#pragma unroll
  for (int i = 0; i < d; ++i) fe[i] = 0;
#pragma unroll
  for (int a = 1; a <= d; ++a)
#pragma unroll
    for (int i = 0; i < d; ++i) {
      S c = P[i * d + 0] * A[0 * d + (a - 1)];
#pragma unroll
      for (int j = 1; j < d; ++j) c += P[i * d + j] * A[j * d + (a - 1)];
      fe[a * d + i] = c;
      fe[i] -= c;
    }
}

// Physical shape gradients at quadrature point q: B[a*d + j] = dN_a/dX_j,
// returns det J (dX[a*d+i] = X_a - X_0).
template <int T, typename S>
__device__ inline S shape_gradients(const S* dX, int q, S* B) {
  constexpr int d = ET<T>::dim, n = ET<T>::nnpe;
  S J[9];
#pragma unroll
  for (int k = 0; k < d; ++k)
#pragma unroll
    for (int j = 0; j < d; ++j) {
      S c = 0;
#pragma unroll
      for (int a = 1; a < n; ++a) c += dN<T, S>(k, a, q) * dX[a * d + j];
      J[k * d + j] = c;
    }
  S A[9];
  const S detJ = adjugate<d, S>(J, A);
  const S idet = S(1) / detJ;
#pragma unroll
  for (int a = 0; a < n; ++a)
#pragma unroll
    for (int j = 0; j < d; ++j) {
      S c = 0;
#pragma unroll
      for (int k = 0; k < d; ++k) c += A[j * d + k] * dN<T, S>(k, a, q);
      B[a * d + j] = c * idet;
    }
  return detJ;
}

// Hexahedron force at quadrature point q, without forming the shape
// gradients: with H = du/dxi (H[i*3+k] = sum_a du_a,i dN(k, a, q)) and A the
// adjugate of J, grad u = H A^T / det J, and the corner forces
// w det J P grad N_a = (w P A) dN_a: Q = w P A, fe_a,i += sum_k Q_ik dN(k, a, q).
template <int T, typename S>
__device__ inline void hex_qp_force(const MatParams& p, const S* du, const S* A, S idet, int q,
                                    S* fe) {
  constexpr int d = 3, n = 8;
  S H[9];
#pragma unroll
  for (int i = 0; i < d; ++i)
#pragma unroll
    for (int k = 0; k < d; ++k) {
      S c = 0;
#pragma unroll
      for (int a = 1; a < n; ++a) c += du[a * d + i] * dN<T, S>(k, a, q);
      H[i * d + k] = c;
    }
  S g[9];
#pragma unroll
  for (int i = 0; i < d; ++i)
#pragma unroll
    for (int j = 0; j < d; ++j)
      g[i * d + j] = (H[i * d] * A[j * d] + H[i * d + 1] * A[j * d + 1] + H[i * d + 2] * A[j * d + 2]) * idet;
  S P[9];
  stress_P<d, S>(p, g, P);
  const S w = S(weight<T>());
  S Q[9];
#pragma unroll
  for (int i = 0; i < d; ++i)
#pragma unroll
    for (int k = 0; k < d; ++k)
      Q[i * d + k] = w * (P[i * d] * A[k] + P[i * d + 1] * A[d + k] + P[i * d + 2] * A[2 * d + k]);
#pragma unroll
  for (int a = 0; a < n; ++a)
#pragma unroll
    for (int i = 0; i < d; ++i)
      fe[a * d + i] += Q[i * d] * dN<T, S>(0, a, q) + Q[i * d + 1] * dN<T, S>(1, a, q) +
                       Q[i * d + 2] * dN<T, S>(2, a, q);
}

// Element internal force (without the -1 of the assembly):
// fe[a*d + i] = sum_q w_q det J_q sum_j P_ij dN_a/dx_j.
// dX[a*d+i] = X_a - X_0, du[a*d+i] = u_a - u_0 (entry a = 0 is zero).
template <int T, typename S>
__device__ inline void element_force(const MatParams& p, const S* dX, const S* du, S* fe) {
  if (T == AKB_TRIANGLE_3 || T == AKB_TETRAHEDRON_4) {
    simplex_force<T, S>(p, dX, du, fe);
    return;
  }
  if (T == AKB_HEXAHEDRON_8) {
    constexpr int d = 3, n = 8, nq = 8;
#pragma unroll
    for (int k = 0; k < d * n; ++k) fe[k] = 0;
    // a parallelepiped (the trilinear terms of x(xi) vanish to 1e-12 of the
    // element's extent) has one Jacobian at every point: formed once
    const int sx[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
    const int sy[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
    const int sz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
    S ext = 0, bend = 0;
#pragma unroll
    for (int j = 0; j < d; ++j) {
      S cxy = 0, cxz = 0, cyz = 0, cxyz = 0;
#pragma unroll
      for (int a = 1; a < n; ++a) {
        const S x = dX[a * d + j];
        cxy += S(sx[a] * sy[a]) * x;
        cxz += S(sx[a] * sz[a]) * x;
        cyz += S(sy[a] * sz[a]) * x;
        cxyz += S(sx[a] * sy[a] * sz[a]) * x;
        ext = fmax(ext, fabs(x));
      }
      bend = fmax(bend, fmax(fmax(fabs(cxy), fabs(cxz)), fmax(fabs(cyz), fabs(cxyz))));
    }
    if (bend <= S(1e-12) * ext) {
      S J[9];
#pragma unroll
      for (int k = 0; k < d; ++k)
#pragma unroll
        for (int j = 0; j < d; ++j) {
          S c = 0;
#pragma unroll
          for (int a = 1; a < n; ++a) {
            const int s = k == 0 ? sx[a] : k == 1 ? sy[a] : sz[a];
            c += S(0.125 * s) * dX[a * d + j];
          }
          J[k * d + j] = c;
        }
      S A[9];
      const S idet = S(1) / adjugate<d, S>(J, A);
#pragma unroll 1
      for (int q = 0; q < nq; ++q) hex_qp_force<T, S>(p, du, A, idet, q, fe);
      return;
    }
#pragma unroll 1
    for (int q = 0; q < nq; ++q) {
      S J[9];
#pragma unroll
      for (int k = 0; k < d; ++k)
#pragma unroll
        for (int j = 0; j < d; ++j) {
          S c = 0;
#pragma unroll
          for (int a = 1; a < n; ++a) c += dN<T, S>(k, a, q) * dX[a * d + j];
          J[k * d + j] = c;
        }
      S A[9];
      const S idet = S(1) / adjugate<d, S>(J, A);
      hex_qp_force<T, S>(p, du, A, idet, q, fe);
    }
    return;
  }
  // segment_2: one point, B = +-1 / length
  constexpr int d = ET<T>::dim, n = ET<T>::nnpe, nq = ET<T>::nqp;
#pragma unroll
  for (int k = 0; k < d * n; ++k) fe[k] = 0;
#pragma unroll 1
  for (int q = 0; q < nq; ++q) {
    // J[k*d + j] = dx_j/dxi_k
    S J[9];
#pragma unroll
    for (int k = 0; k < d; ++k)
#pragma unroll
      for (int j = 0; j < d; ++j) {
        S c = 0;
#pragma unroll
        for (int a = 1; a < n; ++a) c += dN<T, S>(k, a, q) * dX[a * d + j];
        J[k * d + j] = c;
      }
    S A[9];
    const S detJ = adjugate<d, S>(J, A);
    const S idet = S(1) / detJ;
    // grad N_a (physical): B[a*d + j] = sum_k Jinv[j][k] dN(k, a)
    S B[3 * 8];
#pragma unroll
    for (int a = 0; a < n; ++a)
#pragma unroll
      for (int j = 0; j < d; ++j) {
        S c = 0;
#pragma unroll
        for (int k = 0; k < d; ++k) c += A[j * d + k] * dN<T, S>(k, a, q);
        B[a * d + j] = c * idet;
      }
    S g[9];
#pragma unroll
    for (int i = 0; i < d; ++i)
#pragma unroll
      for (int j = 0; j < d; ++j) {
        S c = 0;
#pragma unroll
        for (int a = 1; a < n; ++a) c += du[a * d + i] * B[a * d + j];
        g[i * d + j] = c;
      }
    S P[9];
    stress_P<d, S>(p, g, P);
    const S wq = S(weight<T>()) * detJ;
#pragma unroll
    for (int a = 0; a < n; ++a)
#pragma unroll
      for (int i = 0; i < d; ++i) {
        S c = 0;
#pragma unroll
        for (int j = 0; j < d; ++j) c += P[i * d + j] * B[a * d + j];
        fe[a * d + i] += wq * c;
      }
  }
}

}  // namespace fast
}  // namespace akb
