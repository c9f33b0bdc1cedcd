// akb_refmath.cuh -- element arithmetic in the reference's operation order.
//
// Included only by translation units compiled with --fmad=false, so each
// product and sum is rounded where Akantu's C++ rounds it. Layouts follow the
// reference: Matrix column-major (aka_types.hh:929-944), shape derivatives
// B(j, a) = dN_a/dx_j at [j + a*d], element vectors [i + a*d].
#pragma once

#include "akb_internal.cuh"

namespace akb {
namespace ref {

// Gauss points and weights (gauss_integration.cc:52-56, 72-73, 122-123;
// tensor-product order of gauss_integration_tmpl.hh:160-196, xi fastest).
template <int T>
__host__ __device__ inline void qp_coords(int q, double* c) {
  if (T == AKB_SEGMENT_2) {
    c[0] = 0.;
  } else if (T == AKB_TRIANGLE_3) {
    c[0] = 1. / 3.; c[1] = 1. / 3.;
  } else if (T == AKB_TETRAHEDRON_4) {
    c[0] = 1. / 4.; c[1] = 1. / 4.; c[2] = 1. / 4.;
  } else {
    const double m = -1. / sqrt(3.), p = 1. / sqrt(3.);
    c[0] = (q & 1) ? p : m;
    c[1] = (q & 2) ? p : m;
    c[2] = (q & 4) ? p : m;
  }
}
template <int T>
__host__ __device__ inline double qp_weight(int) {
  return T == AKB_SEGMENT_2 ? 2. : T == AKB_TRIANGLE_3 ? 1. / 2. : T == AKB_TETRAHEDRON_4 ? 1. / 6. : 1. * 1. * 1.;
}

// Shape functions (element_class_*_inline_impl.hh computeShapes).
template <int T>
__host__ __device__ inline void shapes(const double* c, double* N) {
  if (T == AKB_SEGMENT_2) {
    N[0] = 0.5 * (1 - c[0]);
    N[1] = 0.5 * (1 + c[0]);
  } else if (T == AKB_TRIANGLE_3) {
    N[0] = 1 - c[0] - c[1];
    N[1] = c[0];
    N[2] = c[1];
  } else if (T == AKB_TETRAHEDRON_4) {
    N[0] = 1 - c[0] - c[1] - c[2];
    N[1] = c[1];
    N[2] = c[2];
    N[3] = c[0];
  } else {
    N[0] = .125 * (1 - c[0]) * (1 - c[1]) * (1 - c[2]);
    N[1] = .125 * (1 + c[0]) * (1 - c[1]) * (1 - c[2]);
    N[2] = .125 * (1 + c[0]) * (1 + c[1]) * (1 - c[2]);
    N[3] = .125 * (1 - c[0]) * (1 + c[1]) * (1 - c[2]);
    N[4] = .125 * (1 - c[0]) * (1 - c[1]) * (1 + c[2]);
    N[5] = .125 * (1 + c[0]) * (1 - c[1]) * (1 + c[2]);
    N[6] = .125 * (1 + c[0]) * (1 + c[1]) * (1 + c[2]);
    N[7] = .125 * (1 - c[0]) * (1 + c[1]) * (1 + c[2]);
  }
}

// dN/dxi, nat x n column-major (computeDNDS).
template <int T>
__host__ __device__ inline void dnds(const double* c, double* D) {
  if (T == AKB_SEGMENT_2) {
    D[0] = -.5; D[1] = .5;
  } else if (T == AKB_TRIANGLE_3) {
    D[0 + 0 * 2] = -1.; D[0 + 1 * 2] = 1.; D[0 + 2 * 2] = 0.;
    D[1 + 0 * 2] = -1.; D[1 + 1 * 2] = 0.; D[1 + 2 * 2] = 1.;
  } else if (T == AKB_TETRAHEDRON_4) {
    D[0 + 0 * 3] = -1.; D[0 + 1 * 3] = 1.; D[0 + 2 * 3] = 0.; D[0 + 3 * 3] = 0.;
    D[1 + 0 * 3] = -1.; D[1 + 1 * 3] = 0.; D[1 + 2 * 3] = 1.; D[1 + 3 * 3] = 0.;
    D[2 + 0 * 3] = -1.; D[2 + 1 * 3] = 0.; D[2 + 2 * 3] = 0.; D[2 + 3 * 3] = 1.;
  } else {
    D[0 + 0 * 3] = -.125 * (1 - c[1]) * (1 - c[2]);
    D[0 + 1 * 3] = .125 * (1 - c[1]) * (1 - c[2]);
    D[0 + 2 * 3] = .125 * (1 + c[1]) * (1 - c[2]);
    D[0 + 3 * 3] = -.125 * (1 + c[1]) * (1 - c[2]);
    D[0 + 4 * 3] = -.125 * (1 - c[1]) * (1 + c[2]);
    D[0 + 5 * 3] = .125 * (1 - c[1]) * (1 + c[2]);
    D[0 + 6 * 3] = .125 * (1 + c[1]) * (1 + c[2]);
    D[0 + 7 * 3] = -.125 * (1 + c[1]) * (1 + c[2]);
    D[1 + 0 * 3] = -.125 * (1 - c[0]) * (1 - c[2]);
    D[1 + 1 * 3] = -.125 * (1 + c[0]) * (1 - c[2]);
    D[1 + 2 * 3] = .125 * (1 + c[0]) * (1 - c[2]);
    D[1 + 3 * 3] = .125 * (1 - c[0]) * (1 - c[2]);
    D[1 + 4 * 3] = -.125 * (1 - c[0]) * (1 + c[2]);
    D[1 + 5 * 3] = -.125 * (1 + c[0]) * (1 + c[2]);
    D[1 + 6 * 3] = .125 * (1 + c[0]) * (1 + c[2]);
    D[1 + 7 * 3] = .125 * (1 - c[0]) * (1 + c[2]);
    D[2 + 0 * 3] = -.125 * (1 - c[0]) * (1 - c[1]);
    D[2 + 1 * 3] = -.125 * (1 + c[0]) * (1 - c[1]);
    D[2 + 2 * 3] = -.125 * (1 + c[0]) * (1 + c[1]);
    D[2 + 3 * 3] = -.125 * (1 - c[0]) * (1 + c[1]);
    D[2 + 4 * 3] = .125 * (1 - c[0]) * (1 - c[1]);
    D[2 + 5 * 3] = .125 * (1 + c[0]) * (1 - c[1]);
    D[2 + 6 * 3] = .125 * (1 + c[0]) * (1 + c[1]);
    D[2 + 7 * 3] = .125 * (1 - c[0]) * (1 + c[1]);
  }
}

// Math::matrix_matrix / matrixt_matrix / matrix_matrixt (aka_math_tmpl.hh:98-195).
template <int IM, int IN, int IK>
__device__ inline void mm(const double* A, const double* B, double* C, double alpha = 1.) {
#pragma unroll
  for (int j = 0; j < IN; ++j)
#pragma unroll
    for (int i = 0; i < IM; ++i) {
      double c = 0.;
#pragma unroll
      for (int l = 0; l < IK; ++l) c += A[i + l * IM] * B[l + j * IK];
      C[i + j * IM] = c * alpha;
    }
}
template <int IM, int IN, int IK>
__device__ inline void mtm(const double* A, const double* B, double* C, double alpha = 1.) {
#pragma unroll
  for (int j = 0; j < IN; ++j)
#pragma unroll
    for (int i = 0; i < IM; ++i) {
      double c = 0.;
#pragma unroll
      for (int l = 0; l < IK; ++l) c += A[l + i * IK] * B[l + j * IK];
      C[i + j * IM] = c * alpha;
    }
}
template <int IM, int IN, int IK>
__device__ inline void mmt(const double* A, const double* B, double* C, double alpha = 1.) {
#pragma unroll
  for (int j = 0; j < IN; ++j)
#pragma unroll
    for (int i = 0; i < IM; ++i) {
      double c = 0.;
#pragma unroll
      for (int l = 0; l < IK; ++l) c += A[i + l * IM] * B[j + l * IN];
      C[i + j * IM] = c * alpha;
    }
}

// Math::det2/det3, inv2/inv3 (aka_math_tmpl.hh:330-455).
template <int D>
__device__ inline double det(const double* m) {
  if (D == 1) return m[0];
  if (D == 2) return m[0] * m[3] - m[1] * m[2];
  return m[0] * (m[4] * m[8] - m[7] * m[5]) - m[3] * (m[1] * m[8] - m[7] * m[2]) +
         m[6] * (m[1] * m[5] - m[4] * m[2]);
}
template <int D>
__device__ inline void inv(const double* m, double* r) {
  if (D == 1) {
    r[0] = 1. / m[0];
  } else if (D == 2) {
    double d = det<2>(m);
    r[0] = m[3] / d;
    r[1] = -m[1] / d;
    r[2] = -m[2] / d;
    r[3] = m[0] / d;
  } else {
    double d = det<3>(m);
    r[0] = (m[4] * m[8] - m[7] * m[5]) / d;
    r[1] = (m[2] * m[7] - m[8] * m[1]) / d;
    r[2] = (m[1] * m[5] - m[4] * m[2]) / d;
    r[3] = (m[5] * m[6] - m[8] * m[3]) / d;
    r[4] = (m[0] * m[8] - m[6] * m[2]) / d;
    r[5] = (m[2] * m[3] - m[5] * m[0]) / d;
    r[6] = (m[3] * m[7] - m[6] * m[4]) / d;
    r[7] = (m[1] * m[6] - m[7] * m[0]) / d;
    r[8] = (m[0] * m[4] - m[3] * m[1]) / d;
  }
}

// computeShapeDerivativesOnCPointsByElement (shape_lagrange_inline_impl.hh:64-82)
// and computeJacobian * weight (integrator_gauss_inline_impl.hh:380-423).
template <int T>
__device__ inline void geometry(const double* Xel, int q, double* B, double* jac) {
  constexpr int d = ET<T>::dim, n = ET<T>::nnpe;
  double c[3], D[3 * 8], J[9], Ji[9];
  qp_coords<T>(q, c);
  dnds<T>(c, D);
  mmt<d, d, n>(D, Xel, J);  // J = dnds * X^T
  *jac = det<d>(J);
  inv<d>(J, Ji);
  mm<d, n, d>(Ji, D, B);
  *jac = *jac * qp_weight<T>(q);
}

// MaterialElastic::computeStressOnQuad (material_elastic_inline_impl.hh:41-63)
// with the MaterialThermal term at alpha = 0 (material_thermal.hh:99-108).
template <int d>
__device__ inline void elastic_stress(const MatParams& p, const double* g, double* s) {
  const double sigma_th = (d == 1) ? -p.E * 0. * 0. : -p.E / (1. - 2. * p.nu) * 0. * 0.;
  if (d == 1) {
    s[0] = p.E * g[0] + sigma_th;
    return;
  }
  double trace = 0.;
#pragma unroll
  for (int i = 0; i < d; ++i) trace += g[i + i * d];
#pragma unroll
  for (int i = 0; i < d; ++i)
#pragma unroll
    for (int j = 0; j < d; ++j)
      s[i + j * d] = double(i == j) * p.lambda * trace + p.mu * (g[i + j * d] + g[j + i * d]) +
                     double(i == j) * sigma_th;
}

// gradUToE (material_inline_impl.hh:118-127) + elastic law on E.
template <int d>
__device__ inline void svk_stress(const MatParams& p, const double* g, double* s) {
  double E[9];
  mtm<d, d, d>(g, g, E, .5);
#pragma unroll
  for (int i = 0; i < d; ++i)
#pragma unroll
    for (int j = 0; j < d; ++j) E[i + j * d] += 0.5 * (g[i + j * d] + g[j + i * d]);
  elastic_stress<d>(p, E, s);
}

// MaterialNeohookean::computeStressOnQuad (material_neohookean_inline_impl.hh:46-65).
template <int d>
__device__ inline void neohookean_stress(const MatParams& p, const double* g, double* S) {
  double F[9], C[9], Ci[9];
#pragma unroll
  for (int i = 0; i < d; ++i)
#pragma unroll
    for (int j = 0; j < d; ++j) F[i + j * d] = double(i == j);
#pragma unroll
  for (int i = 0; i < d; ++i)
#pragma unroll
    for (int j = 0; j < d; ++j) F[i + j * d] += g[i + j * d];
  mtm<d, d, d>(F, F, C);
  double J = det<d>(F) * sqrt(1.0);
  inv<d>(C, Ci);
  const double f = p.lambda * log(J) - p.mu;
#pragma unroll
  for (int i = 0; i < d; ++i)
#pragma unroll
    for (int j = 0; j < d; ++j) S[i + j * d] = double(i == j) * p.mu + f * Ci[i + j * d];
}

template <int d>
__device__ inline void stress(const MatParams& p, const double* g, double* s) {
  if (p.kind == AKB_MATERIAL_NEOHOOKEAN)
    neohookean_stress<d>(p, g, s);
  else if (p.finite)
    svk_stress<d>(p, g, s);
  else
    elastic_stress<d>(p, g, s);
}

// Per-QP force vector r (d*n), small strain: Bt_D = sigma * B
// (shape_lagrange_inline_impl.hh:383-423); finite strain: r = (B_L0 + B_L2)^T S_voigt
// (material.cc:686-718, aka_voigthelper_tmpl.hh:103-228).
template <int T>
__device__ inline void qp_force(const MatParams& p, const double* B, const double* g,
                                const double* s, double* r) {
  constexpr int d = ET<T>::dim, n = ET<T>::nnpe;
  if (!p.finite) {
    mm<d, n, d>(s, B, r);
    return;
  }
  constexpr int vs = d == 1 ? 1 : (d == 2 ? 3 : 6);
  auto G = [&](int i, int j) { return g[i + j * d]; };
  auto dN = [&](int i, int a) { return B[i + a * d]; };
  double sv[6];
  if (d == 1) {
    sv[0] = s[0];
  } else if (d == 2) {
    sv[0] = s[0]; sv[1] = s[3]; sv[2] = s[0 + 1 * 2];
  } else {
    sv[0] = s[0]; sv[1] = s[4]; sv[2] = s[8];
    sv[3] = s[1 + 2 * 3]; sv[4] = s[0 + 2 * 3]; sv[5] = s[0 + 1 * 3];
  }
  // column c = a*d + k of the (vs x d*n) matrix B_L0 + B_L2, contracted with S_voigt
#pragma unroll
  for (int a = 0; a < n; ++a) {
#pragma unroll
    for (int k = 0; k < d; ++k) {
      double col[6];
      // B_L0 (transferBMatrixToSymVoigtBMatrix)
#pragma unroll
      for (int I = 0; I < vs; ++I) col[I] = 0.;
      col[k] = dN(k, a);
      if (d == 2) {
        if (k == 1) col[2] = dN(0, a);
        if (k == 0) col[2] = dN(1, a);
      }
      if (d == 3) {
        if (k == 1) col[3] = dN(2, a);
        if (k == 2) col[3] = dN(1, a);
        if (k == 0) col[4] = dN(2, a);
        if (k == 2) col[4] = dN(0, a);
        if (k == 0) col[5] = dN(1, a);
        if (k == 1) col[5] = dN(0, a);
      }
      // B_L2 (transferBMatrixToBL2)
      double b2[6];
      if (d == 1) {
        b2[0] = G(0, 0) * dN(0, a);
      } else if (d == 2) {
        b2[0] = G(k, 0) * dN(0, a);
        b2[1] = G(k, 1) * dN(1, a);
        double t = 0.;
#pragma unroll
        for (int m = 0; m < 2; ++m) t += G(k, m) * dN(1 - m, a);
        b2[2] = t;
      } else {
#pragma unroll
        for (int I = 0; I < 3; ++I) b2[I] = G(k, I) * dN(I, a);
#pragma unroll
        for (int Iv = 3; Iv < 6; ++Iv) {
          const int aux = Iv - 3;
          double t = 0.;
#pragma unroll
          for (int m = 0; m < 3; ++m)
            if (m != aux) t += G(k, m) * dN(3 - m - aux, a);
          b2[Iv] = t;
        }
      }
#pragma unroll
      for (int I = 0; I < vs; ++I) col[I] += b2[I];
      // r.mul<true,false>(B_tensor, S_voigt)
      double acc = 0.;
#pragma unroll
      for (int I = 0; I < vs; ++I) acc += col[I] * sv[I];
      r[k + a * d] = acc;
    }
  }
}

// Potential energy density (material_elastic_inline_impl.hh:104-108,
// Math::matrixDoubleDot22/33 aka_math_tmpl.hh:520-532;
// material_neohookean_inline_impl.hh:146-158).
template <int d>
__device__ inline double energy_density(const MatParams& p, const double* g, const double* s) {
  if (p.kind == AKB_MATERIAL_NEOHOOKEAN) {
    double F[9], C[9];
    for (int i = 0; i < d; ++i)
      for (int j = 0; j < d; ++j) F[i + j * d] = double(i == j);
    for (int i = 0; i < d; ++i)
      for (int j = 0; j < d; ++j) F[i + j * d] += g[i + j * d];
    mtm<d, d, d>(F, F, C);
    double J = det<d>(F);
    double trC = 0.;
    for (int i = 0; i < d; ++i) trC += C[i + i * d];
    double lj = log(J);
    return 0.5 * p.lambda * pow(lj, 2.) + p.mu * (-lj + 0.5 * (trC - d));
  }
  double e[9];
  const double* other = g;
  if (p.finite) {
    mtm<d, d, d>(g, g, e, .5);
    for (int i = 0; i < d; ++i)
      for (int j = 0; j < d; ++j) e[i + j * d] += 0.5 * (g[i + j * d] + g[j + i * d]);
    other = e;
  }
  double dd = s[0] * other[0];
  for (int k = 1; k < d * d; ++k) dd = dd + s[k] * other[k];
  return .5 * dd;
}

}  // namespace ref
}  // namespace akb
