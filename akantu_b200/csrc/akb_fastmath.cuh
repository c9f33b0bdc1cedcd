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
    // with u = (1 + t) g^T - (g^T)^2: dev = det(g) I + u, adj(F)^T =
    // (1 + t + I2) I - u, so P = mu g + (a - b) u + (a det g + b (1 + t + I2)) I
    const S amb = a - b, diag = a * dg + b * (c + I2);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const S u = c * g[j * 3 + i] - gg[j * 3 + i];
        P[i * 3 + j] = mu * g[i * 3 + j] + amb * u + (i == j ? diag : S(0));
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

// A constant carried as hi + lo in the element precision: for FP32, hi is
// the constant rounded to float and lo its remainder, so that products with
// it are as accurate as with the FP64 constant up to the rounding of the
// result; for FP64, lo is zero and unused.
template <typename S> struct Split {
  S hi, lo;
};
template <typename S>
__device__ inline Split<S> split(double x) {
  if constexpr (sizeof(S) == 8) {
    return {x, 0.0};
  } else {
    const float h = (float)x;
    return {h, (float)(x - (double)h)};
  }
}
// x c
template <typename S>
__device__ inline S mulc(S x, const Split<S>& c) {
  if constexpr (sizeof(S) == 8)
    return x * c.hi;
  else
    return fmaf(x, c.hi, x * c.lo);
}
// acc + x c
template <typename S>
__device__ inline S fmac(S x, const Split<S>& c, S acc) {
  if constexpr (sizeof(S) == 8)
    return fma(x, c.hi, acc);
  else
    return fmaf(x, c.hi, fmaf(x, c.lo, acc));
}

// Hexahedron force for a parallelepiped (one Jacobian at every point),
// without rounding any quantity that stays the same from step to step:
//  - J, its adjugate A and 1 / det J in FP64 from FP64 coordinate
//    differences, A and 1 / det J then carried as Split constants;
//  - the Gauss points' shape derivatives (2 x 2 x 2 rule, c = +-1/sqrt(3),
//    element_class_hexahedron_8_inline_impl.hh:118-215) never formed:
//    dN_a/dxi_k = 1/8 s_k(a) (1 + s_m(a) c_m) (1 + s_n(a) c_n) ({k, m, n} the
//    three directions), so at a point
//      H_ik = du_i/dxi_k = 1/8 (E_k + c_m E_km + c_n E_kn + c_m c_n E_xyz)
//    with E the signed corner sums of du (once per element), and the corner
//    forces sum_q Q(q) dN(., a, q) come from four signed sums over the
//    points of Q = w P A; c = +-g and c_m c_n = +-1/3 enter as Split
//    constants, once per element.
// In FP32 the element arithmetic then only rounds quantities that change
// every step (its errors do not accumulate into a frequency shift); in FP64
// it takes fewer operations than the point-by-point shape derivatives.
template <typename S>
__device__ inline void hex_parallelepiped_force(const MatParams& p, const double* dX, const S* du,
                                                S* fe) {
  constexpr int d = 3, n = 8;
  const int sg[3][8] = {{-1, 1, 1, -1, -1, 1, 1, -1},
                        {-1, -1, 1, 1, -1, -1, 1, 1},
                        {-1, -1, -1, -1, 1, 1, 1, 1}};
  double J[9];
#pragma unroll
  for (int k = 0; k < d; ++k)
#pragma unroll
    for (int j = 0; j < d; ++j) {
      double c = 0;
#pragma unroll
      for (int a = 1; a < n; ++a) c += (0.125 * sg[k][a]) * dX[a * d + j];
      J[k * d + j] = c;
    }
  double A64[9];
  const double det = adjugate<d, double>(J, A64);
  const Split<S> idet = split<S>(1.0 / det);
  Split<S> A[9];
#pragma unroll
  for (int t = 0; t < 9; ++t) A[t] = split<S>(A64[t] * weight<AKB_HEXAHEDRON_8>());
  // signed corner sums of du: E0[k] (s_k), Ep[.] (s_x s_y, s_x s_z, s_y s_z),
  // E3 (s_x s_y s_z); then g Ep and E3 / 3
  S E0[3][3], Fp[3][3], F3[3];
  const Split<S> gc = split<S>(0.57735026918962576451), third = split<S>(1.0 / 3.0);
#pragma unroll
  for (int i = 0; i < d; ++i) {
    S e0x = 0, e0y = 0, e0z = 0, exy = 0, exz = 0, eyz = 0, exyz = 0;
#pragma unroll
    for (int a = 1; a < n; ++a) {
      const S v = du[a * d + i];
      e0x += S(sg[0][a]) * v;
      e0y += S(sg[1][a]) * v;
      e0z += S(sg[2][a]) * v;
      exy += S(sg[0][a] * sg[1][a]) * v;
      exz += S(sg[0][a] * sg[2][a]) * v;
      eyz += S(sg[1][a] * sg[2][a]) * v;
      exyz += S(sg[0][a] * sg[1][a] * sg[2][a]) * v;
    }
    // the 1/8 of the trilinear derivatives folded in (exact: a power of two)
    E0[0][i] = S(0.125) * e0x;
    E0[1][i] = S(0.125) * e0y;
    E0[2][i] = S(0.125) * e0z;
    Fp[0][i] = S(0.125) * mulc(exy, gc);
    Fp[1][i] = S(0.125) * mulc(exz, gc);
    Fp[2][i] = S(0.125) * mulc(eyz, gc);
    F3[i] = S(0.125) * mulc(exyz, third);
  }
  // pair index of directions (k, m): xy 0, xz 1, yz 2
  auto pair = [](int k, int m) { return k + m - 1; };
  // per (i, k): sums over the points of Q, s_m Q, s_n Q, s_m s_n Q
  S T0[9], Tm[9], Tn[9], Tmn[9];
#pragma unroll
  for (int t = 0; t < 9; ++t) T0[t] = Tm[t] = Tn[t] = Tmn[t] = 0;
#pragma unroll 2  // two points in flight: independent FP64 chains hide each other's latency
  for (int q = 0; q < 8; ++q) {
    const S sq[3] = {(q & 1) ? S(1) : S(-1), (q & 2) ? S(1) : S(-1), (q & 4) ? S(1) : S(-1)};
    S H[9];
#pragma unroll
    for (int k = 0; k < d; ++k) {
      const int m = k == 0 ? 1 : 0, nn = k == 2 ? 1 : 2;
#pragma unroll
      for (int i = 0; i < d; ++i)
        H[i * d + k] = E0[k][i] + sq[m] * Fp[pair(k, m)][i] + sq[nn] * Fp[pair(k, nn)][i] +
                       (sq[m] * sq[nn]) * F3[i];
    }
    // grad u = H A^T / det J
    S g[9];
#pragma unroll
    for (int i = 0; i < d; ++i)
#pragma unroll
      for (int j = 0; j < d; ++j) {
        S c = 0;
#pragma unroll
        for (int k = 0; k < d; ++k) c = fmac(H[i * d + k], A[j * d + k], c);
        g[i * d + j] = mulc(c, idet);
      }
    S P[9];
    stress_P<d, S>(p, g, P);
#pragma unroll
    for (int i = 0; i < d; ++i)
#pragma unroll
      for (int k = 0; k < d; ++k) {
        const int m = k == 0 ? 1 : 0, nn = k == 2 ? 1 : 2;
        S Q = 0;  // (w P A)_ik
#pragma unroll
        for (int j = 0; j < d; ++j) Q = fmac(P[i * d + j], A[j * d + k], Q);
        const int t = i * d + k;
        T0[t] += Q;
        Tm[t] += sq[m] * Q;
        Tn[t] += sq[nn] * Q;
        Tmn[t] += (sq[m] * sq[nn]) * Q;
      }
  }
#pragma unroll
  for (int t = 0; t < 9; ++t) {
    Tm[t] = mulc(Tm[t], gc);
    Tn[t] = mulc(Tn[t], gc);
    Tmn[t] = mulc(Tmn[t], third);
  }
#pragma unroll
  for (int a = 0; a < n; ++a)
#pragma unroll
    for (int i = 0; i < d; ++i) {
      S f = 0;
#pragma unroll
      for (int k = 0; k < d; ++k) {
        const int m = k == 0 ? 1 : 0, nn = k == 2 ? 1 : 2;
        const int t = i * d + k;
        const S sm = S(sg[m][a]), sn = S(sg[nn][a]);
        f += S(sg[k][a]) * (T0[t] + sm * Tm[t] + sn * Tn[t] + (sm * sn) * Tmn[t]);
      }
      fe[a * d + i] = S(0.125) * f;
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
// dX64[a*d+i] = X_a - X_0 in FP64, du[a*d+i] = u_a - u_0 (entry a = 0 is
// zero).
template <int T, typename S>
__device__ inline void element_force(const MatParams& p, const double* dX64, const S* du, S* fe) {
  constexpr int nd = ET<T>::dim * ET<T>::nnpe;
  S dX[nd];
#pragma unroll
  for (int k = 0; k < nd; ++k) dX[k] = S(dX64[k]);
  if (T == AKB_TRIANGLE_3 || T == AKB_TETRAHEDRON_4) {
    simplex_force<T, S>(p, dX, du, fe);
    return;
  }
  if (T == AKB_HEXAHEDRON_8) {
    constexpr int d = 3, n = 8, nq = 8;
    // a parallelepiped (the trilinear terms of x(xi) vanish to 1e-12 of the
    // element's extent) has one Jacobian at every point: formed once
    const int sx[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
    const int sy[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
    const int sz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
    // (tested on the FP64 differences: rounded to FP32 they are not a
    // parallelepiped to 1e-12)
    double ext = 0, bend = 0;
#pragma unroll
    for (int j = 0; j < d; ++j) {
      double cxy = 0, cxz = 0, cyz = 0, cxyz = 0;
#pragma unroll
      for (int a = 1; a < n; ++a) {
        const double x = dX64[a * d + j];
        cxy += double(sx[a] * sy[a]) * x;
        cxz += double(sx[a] * sz[a]) * x;
        cyz += double(sy[a] * sz[a]) * x;
        cxyz += double(sx[a] * sy[a] * sz[a]) * x;
        ext = fmax(ext, fabs(x));
      }
      bend = fmax(bend, fmax(fmax(fabs(cxy), fabs(cxz)), fmax(fabs(cyz), fabs(cxyz))));
    }
    if (bend <= 1e-12 * ext) {
      hex_parallelepiped_force<S>(p, dX64, du, fe);
      return;
    }
#pragma unroll
    for (int k = 0; k < d * n; ++k) fe[k] = 0;
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
