// akb_oracle.cc -- CPU restatement of Akantu's explicit central-difference
// step with lumped mass (SolidMechanicsModel + MaterialElastic +
// MaterialNeohookean on segment_2 / triangle_3 / tetrahedron_4 /
// hexahedron_8).
//
// TEST INFRASTRUCTURE ONLY: the checker for libakb.so and the timed CPU
// baseline. Compiled with -ffp-contract=off so that every product and sum is
// rounded exactly where the reference's C++ rounds it. All citations are
// file:line within the Akantu 3.1.0 tree.
//
// Storage mirrors the reference: Array<Real> rows, Matrix column-major
// (aka_types.hh:929-944), shape derivatives stored per quadrature point as a
// d x n column-major matrix (shape_lagrange_inline_impl.hh:206-252) and
// jacobians stored as det(J)*w (integrator_gauss_inline_impl.hh:380-423).
#include "akb_oracle.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

namespace {

struct Material {
  int kind;
  bool plane_stress;
  bool finite;
  double rho, E, nu;
  double lambda, mu;
};

// MaterialElastic::updateInternalParameters (material_elastic.cc:83-107),
// MaterialElastic::initMaterial sets nu = 0 in 1D (material_elastic.cc:74-81),
// MaterialNeohookean::updateInternalParameters (material_neohookean.cc:83-89).
Material make_material(const akb_material_desc& d, int dim) {
  Material m;
  m.kind = d.kind;
  m.plane_stress = d.plane_stress != 0;
  m.finite = (d.kind == AKB_MATERIAL_NEOHOOKEAN) || d.finite_deformation != 0;
  m.rho = d.rho;
  m.E = d.E;
  m.nu = (dim == 1) ? 0. : d.nu;
  m.lambda = m.nu * m.E / ((1 + m.nu) * (1 - 2 * m.nu));
  m.mu = m.E / (2 * (1 + m.nu));
  if (dim == 2 && m.plane_stress && d.kind == AKB_MATERIAL_ELASTIC)
    m.lambda = m.nu * m.E / ((1 + m.nu) * (1 - m.nu));
  return m;
}

// getPushWaveSpeed (material_elastic.cc:164-167, material_neohookean.cc:253-257).
double celerity(const Material& m) {
  return std::sqrt((m.lambda + 2 * m.mu) / m.rho);
}

struct ElementInfo {
  int nat;   // natural dimension
  int nnpe;  // nodes per element
  int nqp;   // quadrature points
  double qpos[8][3];
  double qw[8];
};

// Gauss tables (gauss_integration.cc:52-56, 72-73, 122-123) with the
// tensor-product ordering of gauss_integration_tmpl.hh:160-196 (xi fastest).
ElementInfo element_info(int type) {
  ElementInfo e{};
  switch (type) {
  case AKB_SEGMENT_2:
    e.nat = 1; e.nnpe = 2; e.nqp = 1;
    e.qpos[0][0] = 0.; e.qw[0] = 2.;
    break;
  case AKB_TRIANGLE_3:
    e.nat = 2; e.nnpe = 3; e.nqp = 1;
    e.qpos[0][0] = 1. / 3.; e.qpos[0][1] = 1. / 3.; e.qw[0] = 1. / 2.;
    break;
  case AKB_TETRAHEDRON_4:
    e.nat = 3; e.nnpe = 4; e.nqp = 1;
    e.qpos[0][0] = e.qpos[0][1] = e.qpos[0][2] = 1. / 4.; e.qw[0] = 1. / 6.;
    break;
  case AKB_HEXAHEDRON_8: {
    e.nat = 3; e.nnpe = 8; e.nqp = 8;
    const double p[2] = {-1. / std::sqrt(3.), 1. / std::sqrt(3.)};
    for (int q = 0; q < 8; ++q) {
      e.qpos[q][0] = p[q & 1];
      e.qpos[q][1] = p[(q >> 1) & 1];
      e.qpos[q][2] = p[(q >> 2) & 1];
      e.qw[q] = 1. * 1. * 1.;
    }
    break;
  }
  default:
    e.nat = 0;
  }
  return e;
}

// Shape functions N(xi) (element_class_*_inline_impl.hh computeShapes).
// The tetrahedron keeps the reference's ordering (1-xi-eta-zeta, eta, zeta, xi)
// (element_class_tetrahedron_4_inline_impl.hh:69-85).
void compute_shapes(int type, const double* c, double* N) {
  switch (type) {
  case AKB_SEGMENT_2:
    N[0] = 0.5 * (1 - c[0]);
    N[1] = 0.5 * (1 + c[0]);
    break;
  case AKB_TRIANGLE_3:
    N[0] = 1 - c[0] - c[1];
    N[1] = c[0];
    N[2] = c[1];
    break;
  case AKB_TETRAHEDRON_4:
    N[0] = 1 - c[0] - c[1] - c[2];
    N[1] = c[1];
    N[2] = c[2];
    N[3] = c[0];
    break;
  case AKB_HEXAHEDRON_8:
    N[0] = .125 * (1 - c[0]) * (1 - c[1]) * (1 - c[2]);
    N[1] = .125 * (1 + c[0]) * (1 - c[1]) * (1 - c[2]);
    N[2] = .125 * (1 + c[0]) * (1 + c[1]) * (1 - c[2]);
    N[3] = .125 * (1 - c[0]) * (1 + c[1]) * (1 - c[2]);
    N[4] = .125 * (1 - c[0]) * (1 - c[1]) * (1 + c[2]);
    N[5] = .125 * (1 + c[0]) * (1 - c[1]) * (1 + c[2]);
    N[6] = .125 * (1 + c[0]) * (1 + c[1]) * (1 + c[2]);
    N[7] = .125 * (1 - c[0]) * (1 + c[1]) * (1 + c[2]);
    break;
  }
}

// dN/dxi as a nat x n column-major matrix, dnds(i, a) at [i + a * nat]
// (element_class_*_inline_impl.hh computeDNDS).
void compute_dnds(int type, const double* c, double* D) {
  auto at = [&](int i, int a, int nat) -> double& { return D[i + a * nat]; };
  switch (type) {
  case AKB_SEGMENT_2:
    at(0, 0, 1) = -.5;
    at(0, 1, 1) = .5;
    break;
  case AKB_TRIANGLE_3:
    at(0, 0, 2) = -1.; at(0, 1, 2) = 1.; at(0, 2, 2) = 0.;
    at(1, 0, 2) = -1.; at(1, 1, 2) = 0.; at(1, 2, 2) = 1.;
    break;
  case AKB_TETRAHEDRON_4:
    at(0, 0, 3) = -1.; at(0, 1, 3) = 1.; at(0, 2, 3) = 0.; at(0, 3, 3) = 0.;
    at(1, 0, 3) = -1.; at(1, 1, 3) = 0.; at(1, 2, 3) = 1.; at(1, 3, 3) = 0.;
    at(2, 0, 3) = -1.; at(2, 1, 3) = 0.; at(2, 2, 3) = 0.; at(2, 3, 3) = 1.;
    break;
  case AKB_HEXAHEDRON_8:
    at(0, 0, 3) = -.125 * (1 - c[1]) * (1 - c[2]);
    at(0, 1, 3) = .125 * (1 - c[1]) * (1 - c[2]);
    at(0, 2, 3) = .125 * (1 + c[1]) * (1 - c[2]);
    at(0, 3, 3) = -.125 * (1 + c[1]) * (1 - c[2]);
    at(0, 4, 3) = -.125 * (1 - c[1]) * (1 + c[2]);
    at(0, 5, 3) = .125 * (1 - c[1]) * (1 + c[2]);
    at(0, 6, 3) = .125 * (1 + c[1]) * (1 + c[2]);
    at(0, 7, 3) = -.125 * (1 + c[1]) * (1 + c[2]);
    at(1, 0, 3) = -.125 * (1 - c[0]) * (1 - c[2]);
    at(1, 1, 3) = -.125 * (1 + c[0]) * (1 - c[2]);
    at(1, 2, 3) = .125 * (1 + c[0]) * (1 - c[2]);
    at(1, 3, 3) = .125 * (1 - c[0]) * (1 - c[2]);
    at(1, 4, 3) = -.125 * (1 - c[0]) * (1 + c[2]);
    at(1, 5, 3) = -.125 * (1 + c[0]) * (1 + c[2]);
    at(1, 6, 3) = .125 * (1 + c[0]) * (1 + c[2]);
    at(1, 7, 3) = .125 * (1 - c[0]) * (1 + c[2]);
    at(2, 0, 3) = -.125 * (1 - c[0]) * (1 - c[1]);
    at(2, 1, 3) = -.125 * (1 + c[0]) * (1 - c[1]);
    at(2, 2, 3) = -.125 * (1 + c[0]) * (1 + c[1]);
    at(2, 3, 3) = -.125 * (1 - c[0]) * (1 + c[1]);
    at(2, 4, 3) = .125 * (1 - c[0]) * (1 - c[1]);
    at(2, 5, 3) = .125 * (1 + c[0]) * (1 - c[1]);
    at(2, 6, 3) = .125 * (1 + c[0]) * (1 + c[1]);
    at(2, 7, 3) = .125 * (1 - c[0]) * (1 + c[1]);
    break;
  }
}

// Math::matrix_matrix / matrixt_matrix / matrix_matrixt without BLAS
// (aka_math_tmpl.hh:98-195): C starts at 0, products accumulate in l order,
// then C *= alpha.
void mm(int im, int in, int ik, const double* A, const double* B, double* C,
        double alpha = 1.) {
  std::memset(C, 0, sizeof(double) * im * in);
  for (int j = 0; j < in; ++j)
    for (int i = 0; i < im; ++i) {
      for (int l = 0; l < ik; ++l) C[i + j * im] += A[i + l * im] * B[l + j * ik];
      C[i + j * im] *= alpha;
    }
}
void mtm(int im, int in, int ik, const double* A, const double* B, double* C,
         double alpha = 1.) {
  std::memset(C, 0, sizeof(double) * im * in);
  for (int j = 0; j < in; ++j)
    for (int i = 0; i < im; ++i) {
      for (int l = 0; l < ik; ++l) C[i + j * im] += A[l + i * ik] * B[l + j * ik];
      C[i + j * im] *= alpha;
    }
}
void mmt(int im, int in, int ik, const double* A, const double* B, double* C,
         double alpha = 1.) {
  std::memset(C, 0, sizeof(double) * im * in);
  for (int j = 0; j < in; ++j)
    for (int i = 0; i < im; ++i) {
      for (int l = 0; l < ik; ++l) C[i + j * im] += A[i + l * im] * B[j + l * in];
      C[i + j * im] *= alpha;
    }
}

// Math::det2/det3, inv2/inv3 (aka_math_tmpl.hh:330-455).
double det2(const double* m) { return m[0] * m[3] - m[1] * m[2]; }
double det3(const double* m) {
  return m[0] * (m[4] * m[8] - m[7] * m[5]) - m[3] * (m[1] * m[8] - m[7] * m[2]) +
         m[6] * (m[1] * m[5] - m[4] * m[2]);
}
double detn(int n, const double* m) {
  return n == 1 ? m[0] : (n == 2 ? det2(m) : det3(m));
}
void invn(int n, const double* m, double* inv) {
  if (n == 1) {
    inv[0] = 1. / m[0];
  } else if (n == 2) {
    double d = det2(m);
    inv[0] = m[3] / d;
    inv[1] = -m[1] / d;
    inv[2] = -m[2] / d;
    inv[3] = m[0] / d;
  } else {
    double d = det3(m);
    inv[0] = (m[4] * m[8] - m[7] * m[5]) / d;
    inv[1] = (m[2] * m[7] - m[8] * m[1]) / d;
    inv[2] = (m[1] * m[5] - m[4] * m[2]) / d;
    inv[3] = (m[5] * m[6] - m[8] * m[3]) / d;
    inv[4] = (m[0] * m[8] - m[6] * m[2]) / d;
    inv[5] = (m[2] * m[3] - m[5] * m[0]) / d;
    inv[6] = (m[3] * m[7] - m[6] * m[4]) / d;
    inv[7] = (m[1] * m[6] - m[7] * m[0]) / d;
    inv[8] = (m[0] * m[4] - m[3] * m[1]) / d;
  }
}

// Element inradius (fe_engine_inline_impl.hh:45-55): triangle and
// tetrahedron 2*r_in (aka_math_tmpl.hh:568-587, 650-...), hexahedron the
// shortest edge (element_class_hexahedron_8_inline_impl.hh:219-246),
// segment the length (element_class_segment_2_inline_impl.hh).
double dist(const double* x, const double* y, int d) {
  double s = 0;
  if (d == 2) return std::sqrt((y[0] - x[0]) * (y[0] - x[0]) + (y[1] - x[1]) * (y[1] - x[1]));
  if (d == 3)
    return std::sqrt((y[0] - x[0]) * (y[0] - x[0]) + (y[1] - x[1]) * (y[1] - x[1]) +
                     (y[2] - x[2]) * (y[2] - x[2]));
  for (int i = 0; i < d; ++i) s += (y[i] - x[i]) * (y[i] - x[i]);
  return std::sqrt(s);
}
double tet_volume(const double* c1, const double* c2, const double* c3, const double* c4) {
  double xx[9], vol;
  auto fill = [&](const double* a, const double* b, const double* c) {
    xx[0] = a[0]; xx[1] = a[1]; xx[2] = a[2];
    xx[3] = b[0]; xx[4] = b[1]; xx[5] = b[2];
    xx[6] = c[0]; xx[7] = c[1]; xx[8] = c[2];
  };
  fill(c2, c3, c4); vol = det3(xx);
  fill(c1, c3, c4); vol -= det3(xx);
  fill(c1, c2, c4); vol += det3(xx);
  fill(c1, c2, c3); vol -= det3(xx);
  vol /= 6;
  return vol;
}
double inradius(int type, const double* X /* d x n col-major */, int d) {
  switch (type) {
  case AKB_SEGMENT_2:
    return std::abs(X[0] - X[1]);
  case AKB_TRIANGLE_3: {
    double a = dist(X + 0, X + 2, 2), b = dist(X + 2, X + 4, 2), c = dist(X + 0, X + 4, 2);
    double s = (a + b + c) * 0.5;
    return 2. * std::sqrt((s - a) * (s - b) * (s - c) / s);
  }
  case AKB_TETRAHEDRON_4: {
    const double *c1 = X, *c2 = X + 3, *c3 = X + 6, *c4 = X + 9;
    double l12 = dist(c1, c2, 3), l13 = dist(c1, c3, 3), l14 = dist(c1, c4, 3);
    double l23 = dist(c2, c3, 3), l24 = dist(c2, c4, 3), l34 = dist(c3, c4, 3);
    double s1 = (l12 + l23 + l13) * 0.5;
    s1 = std::sqrt(s1 * (s1 - l12) * (s1 - l23) * (s1 - l13));
    double s2 = (l12 + l24 + l14) * 0.5;
    s2 = std::sqrt(s2 * (s2 - l12) * (s2 - l24) * (s2 - l14));
    double s3 = (l23 + l34 + l24) * 0.5;
    s3 = std::sqrt(s3 * (s3 - l23) * (s3 - l34) * (s3 - l24));
    double s4 = (l13 + l34 + l14) * 0.5;
    s4 = std::sqrt(s4 * (s4 - l13) * (s4 - l34) * (s4 - l14));
    double volume = tet_volume(c1, c2, c3, c4);
    return 2. * (3 * volume / (s1 + s2 + s3 + s4));
  }
  case AKB_HEXAHEDRON_8: {
    const int e[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {0, 4}, {1, 5},
                          {2, 6}, {3, 7}, {4, 5}, {5, 6}, {6, 7}, {7, 4}};
    double p = std::numeric_limits<double>::max();
    for (auto& k : e) p = std::min(p, dist(X + 3 * k[0], X + 3 * k[1], 3));
    return p;
  }
  }
  return 0;
}

}  // namespace

struct oracle_model {
  int dim, type;
  ElementInfo info;
  int64_t nn, ne;
  std::vector<double> X;
  std::vector<uint32_t> conn;
  std::vector<Material> mats;
  std::vector<uint32_t> mat_of;
  // precomputed FE data (ShapeLagrange / IntegratorGauss)
  std::vector<double> B;    // [e*q][d*n], B(j,a) at [j + a*d]
  std::vector<double> jac;  // [e*q] det(J) * w
  std::vector<double> N;    // [q][n] shapes (identical for every element)
  // nodal fields
  std::vector<double> u, v, a, fext, fint, mass, lumped, residual, solution;
  std::vector<uint8_t> blocked;
  // per-QP internal fields (Material gradu / stress or piola_kirchhoff_2)
  std::vector<double> gradu, stress;
  double dt = 0;
  bool mass_assembled = false;
  // multi-threaded variant: element vectors + node -> (element, corner) CSR
  int threads = 1;
  std::vector<double> fe;
  std::vector<int64_t> node_ptr;
  std::vector<int64_t> node_ent;
};

namespace {

// SolidMechanicsModel::assembleMassLumped (solid_mechanics_model_mass.cc:58-133)
// -> assembleFieldLumped / assembleLumpedRowSum (fe_engine_template_tmpl_field.hh:111-199):
// Ntb = rho * N per QP (shape_lagrange_inline_impl.hh:497-533), integrated
// with detJ*w (integrator_gauss_inline_impl.hh:83-96), element-order scatter
// (dof_manager.cc:83-137), then assembleToLumpedMatrix (dof_manager.cc:240-251).
void assemble_mass(oracle_model& m) {
  const int d = m.dim, n = m.info.nnpe, q = m.info.nqp;
  std::vector<double> local(m.nn * d, 0.);
  std::vector<double> ntb(q * d * n), inte(d * n);
  for (int64_t e = 0; e < m.ne; ++e) {
    const Material& mat = m.mats[m.mat_of[e]];
    for (int p = 0; p < q; ++p) {
      double b[3] = {mat.rho, mat.rho, mat.rho};
      // Ntb.mul<false,false>(b (d x 1), N (1 x n))
      mm(d, n, 1, b, &m.N[p * n], &ntb[p * d * n]);
    }
    // integrate: inte[dof] += f[q][dof] * jac[q]
    std::memset(inte.data(), 0, sizeof(double) * d * n);
    for (int p = 0; p < q; ++p)
      for (int k = 0; k < d * n; ++k) inte[k] += ntb[p * d * n + k] * m.jac[e * q + p];
    for (int aa = 0; aa < n; ++aa) {
      uint32_t node = m.conn[e * n + aa];
      for (int i = 0; i < d; ++i) local[node * d + i] += 1. * inte[i + aa * d];
    }
  }
  std::fill(m.lumped.begin(), m.lumped.end(), 0.);
  for (size_t k = 0; k < local.size(); ++k) m.lumped[k] += 1. * local[k];
  m.mass = m.lumped;  // getLumpedMatrixPerDOFs (identity equation numbering)
  m.mass_assembled = true;
}

// MaterialElastic::computeStressOnQuad (material_elastic_inline_impl.hh:41-63),
// with the MaterialThermal contribution sigma_th = -E/(1-2nu)*alpha*dT at
// alpha = 0 (material_thermal.hh:99-108).
void elastic_stress(const Material& mat, int d, const double* g, double* s) {
  const double sigma_th = (d == 1) ? -mat.E * 0. * 0. : -mat.E / (1. - 2. * mat.nu) * 0. * 0.;
  if (d == 1) {
    s[0] = mat.E * g[0] + sigma_th;
    return;
  }
  double trace = 0.;
  for (int i = 0; i < d; ++i) trace += g[i + i * d];
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j)
      s[i + j * d] = double(i == j) * mat.lambda * trace + mat.mu * (g[i + j * d] + g[j + i * d]) +
                     double(i == j) * sigma_th;
}

// Finite-deformation elastic (St-Venant-Kirchhoff): gradUToE
// (material_inline_impl.hh:118-127) then computeStressOnQuad on E.
void svk_stress(const Material& mat, int d, const double* g, double* s) {
  double E[9];
  mtm(d, d, d, g, g, E, .5);
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j) E[i + j * d] += 0.5 * (g[i + j * d] + g[j + i * d]);
  elastic_stress(mat, d, E, s);
}

// MaterialNeohookean::computeStressOnQuad (material_neohookean_inline_impl.hh:46-65):
// F = I + grad_u, C = F^T F, J = det F, S = mu I + (lambda ln J - mu) C^-1.
void neohookean_stress(const Material& mat, int d, const double* g, double* S) {
  double F[9] = {0}, C[9], Ci[9];
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j) F[i + j * d] = double(i == j);
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j) F[i + j * d] += g[i + j * d];
  mtm(d, d, d, F, F, C);
  double J = detn(d, F) * std::sqrt(1.0);
  invn(d, C, Ci);
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j)
      S[i + j * d] = double(i == j) * mat.mu + (mat.lambda * std::log(J) - mat.mu) * Ci[i + j * d];
}

void material_stress(const Material& mat, int d, const double* g, double* s) {
  if (mat.kind == AKB_MATERIAL_NEOHOOKEAN)
    neohookean_stress(mat, d, g, s);
  else if (mat.finite)
    svk_stress(mat, d, g, s);
  else
    elastic_stress(mat, d, g, s);
}

// Material::computeAllStresses (material.cc:254-279): gradient
// (shape_functions_inline_impl.hh:383-390: nabla_u.mul<false,true>(u_el, B)),
// minus eigengradu (zero), then computeStress per QP.
void compute_all_stresses(oracle_model& m) {
  const int d = m.dim, n = m.info.nnpe, q = m.info.nqp;
  double uel[24];
  for (int64_t e = 0; e < m.ne; ++e) {
    for (int aa = 0; aa < n; ++aa)
      for (int i = 0; i < d; ++i) uel[i + aa * d] = m.u[m.conn[e * n + aa] * d + i];
    const Material& mat = m.mats[m.mat_of[e]];
    for (int p = 0; p < q; ++p) {
      double* g = &m.gradu[(e * q + p) * d * d];
      mmt(d, d, n, uel, &m.B[(e * q + p) * d * n], g);
      for (int k = 0; k < d * d; ++k) g[k] -= 0.;  // eigengradu
      material_stress(mat, d, g, &m.stress[(e * q + p) * d * d]);
    }
  }
}

// Voigt B matrices (aka_voigthelper_tmpl.hh:103-228), B_voigt(I, a*d+i)
// stored column-major with `rows` rows.
void b_matrix_sym_voigt(int d, int n, const double* B, double* Bv, int rows) {
  std::memset(Bv, 0, sizeof(double) * rows * d * n);
  auto at = [&](int I, int c) -> double& { return Bv[I + c * rows]; };
  for (int i = 0; i < d; ++i)
    for (int a = 0; a < n; ++a) at(i, i + a * d) = B[i + a * d];
  if (d == 2)
    for (int a = 0; a < n; ++a) {
      at(2, 1 + a * 2) = B[0 + a * 2];
      at(2, 0 + a * 2) = B[1 + a * 2];
    }
  if (d == 3)
    for (int a = 0; a < n; ++a) {
      double dndx = B[0 + a * 3], dndy = B[1 + a * 3], dndz = B[2 + a * 3];
      at(3, 1 + a * 3) = dndz;
      at(3, 2 + a * 3) = dndy;
      at(4, 0 + a * 3) = dndz;
      at(4, 2 + a * 3) = dndx;
      at(5, 0 + a * 3) = dndy;
      at(5, 1 + a * 3) = dndx;
    }
}
void b_matrix_bl2(int d, int n, const double* B, const double* g, double* Bv, int rows) {
  std::memset(Bv, 0, sizeof(double) * rows * d * n);
  auto at = [&](int I, int c) -> double& { return Bv[I + c * rows]; };
  auto G = [&](int i, int j) { return g[i + j * d]; };
  auto dN = [&](int i, int a) { return B[i + a * d]; };
  if (d == 1) {
    for (int j = 0; j < n; ++j) at(0, j) = G(0, 0) * dN(0, j);
  } else if (d == 2) {
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < n; ++j)
        for (int k = 0; k < 2; ++k) at(i, j * 2 + k) = G(k, i) * dN(i, j);
    for (int j = 0; j < n; ++j)
      for (int k = 0; k < 2; ++k)
        for (int mm_ = 0; mm_ < 2; ++mm_) at(2, j * 2 + k) += G(k, mm_) * dN(1 - mm_, j);
  } else {
    for (int I = 0; I < 3; ++I)
      for (int a = 0; a < n; ++a)
        for (int i = 0; i < 3; ++i) at(I, a * 3 + i) = G(i, I) * dN(I, a);
    for (int Iv = 3; Iv < 6; ++Iv)
      for (int a = 0; a < n; ++a)
        for (int k = 0; k < 3; ++k) {
          int aux = Iv - 3;
          for (int mm_ = 0; mm_ < 3; ++mm_)
            if (mm_ != aux) at(Iv, a * 3 + k) += G(k, mm_) * dN(3 - mm_ - aux, a);
        }
  }
}

// SolidMechanicsModel::assembleInternalForces (solid_mechanics_model.cc:375-414)
// -> Material::assembleInternalForces small strain (material.cc:178-230:
// computeBtD shape_lagrange_inline_impl.hh:383-423, integrate
// integrator_gauss_inline_impl.hh:426-455, scatter with scale -1
// dof_manager.cc:83-137) or finite strain (material.cc:637-722).
void element_vector(oracle_model& m, int64_t e, double* inte);

void assemble_internal_forces_parallel(oracle_model& m);

void assemble_internal_forces(oracle_model& m) {
  if (m.threads > 1) {
    assemble_internal_forces_parallel(m);
    return;
  }
  const int d = m.dim, n = m.info.nnpe;
  std::fill(m.fint.begin(), m.fint.end(), 0.);
  compute_all_stresses(m);
  std::vector<double> inte(d * n);
  for (int64_t e = 0; e < m.ne; ++e) {
    element_vector(m, e, inte.data());
    for (int aa = 0; aa < n; ++aa) {
      uint32_t node = m.conn[e * n + aa];
      for (int i = 0; i < d; ++i) m.fint[node * d + i] += -1. * inte[i + aa * d];
    }
  }
}

// Multi-threaded variant, bitwise equal to the serial one: element vectors in
// parallel, then each node adds -1 * (its elements' vectors) in ascending
// element order, the order of the serial element-by-element scatter.
void assemble_internal_forces_parallel(oracle_model& m) {
  const int d = m.dim, n = m.info.nnpe, q = m.info.nqp;
  if (m.fe.size() != (size_t)m.ne * n * d) m.fe.assign((size_t)m.ne * n * d, 0.);
  if (m.node_ptr.empty()) {
    m.node_ptr.assign(m.nn + 1, 0);
    m.node_ent.assign((size_t)m.ne * n, 0);
    for (int64_t k = 0; k < m.ne * n; ++k) m.node_ptr[m.conn[k] + 1]++;
    for (int64_t i = 0; i < m.nn; ++i) m.node_ptr[i + 1] += m.node_ptr[i];
    std::vector<int64_t> fill(m.node_ptr.begin(), m.node_ptr.end() - 1);
    for (int64_t k = 0; k < m.ne * n; ++k) m.node_ent[fill[m.conn[k]]++] = k;
  }
  double* uu = m.u.data();
  (void)q;
#pragma omp parallel for schedule(static) num_threads(m.threads)
  for (int64_t e = 0; e < m.ne; ++e) {
    double uel[24];
    for (int aa = 0; aa < n; ++aa)
      for (int i = 0; i < d; ++i) uel[i + aa * d] = uu[m.conn[e * n + aa] * d + i];
    const Material& mat = m.mats[m.mat_of[e]];
    for (int p = 0; p < q; ++p) {
      double* g = &m.gradu[(e * q + p) * d * d];
      mmt(d, d, n, uel, &m.B[(e * q + p) * d * n], g);
      for (int k = 0; k < d * d; ++k) g[k] -= 0.;
      material_stress(mat, d, g, &m.stress[(e * q + p) * d * d]);
    }
    element_vector(m, e, &m.fe[(size_t)e * n * d]);
  }
#pragma omp parallel for schedule(static) num_threads(m.threads)
  for (int64_t node = 0; node < m.nn; ++node) {
    for (int i = 0; i < d; ++i) {
      double f = 0.;
      for (int64_t k = m.node_ptr[node]; k < m.node_ptr[node + 1]; ++k) {
        const int64_t ent = m.node_ent[k];
        const int64_t e = ent / n, aa = ent % n;
        f += -1. * m.fe[(size_t)e * n * d + i + aa * d];
      }
      m.fint[node * d + i] = f;
    }
  }
}

// Element vector of Material::assembleInternalForces (before the -1 scatter).
void element_vector(oracle_model& m, int64_t e, double* inte) {
  const int d = m.dim, n = m.info.nnpe, q = m.info.nqp;
  const int vs = (d == 1) ? 1 : (d == 2 ? 3 : 6);
  double r[8 * 24];
  double Bv[6 * 24], B2[6 * 24];
  {
    const Material& mat = m.mats[m.mat_of[e]];
    for (int p = 0; p < q; ++p) {
      const double* s = &m.stress[(e * q + p) * d * d];
      const double* B = &m.B[(e * q + p) * d * n];
      if (!mat.finite) {
        // Bt_D.mul<false,false>(D, B): (d x d)(d x n)
        mm(d, n, d, s, B, &r[p * d * n]);
      } else {
        const double* g = &m.gradu[(e * q + p) * d * d];
        b_matrix_sym_voigt(d, n, B, Bv, vs);
        b_matrix_bl2(d, n, B, g, B2, vs);
        for (int k = 0; k < vs * d * n; ++k) Bv[k] += B2[k];
        // stressToVoigt (aka_voigthelper.cc:47-64, aka_voigthelper_tmpl.hh:43-49)
        double sv[6];
        if (d == 1) {
          sv[0] = s[0];
        } else if (d == 2) {
          sv[0] = s[0]; sv[1] = s[3]; sv[2] = s[0 + 1 * 2];
        } else {
          sv[0] = s[0 + 0 * 3]; sv[1] = s[1 + 1 * 3]; sv[2] = s[2 + 2 * 3];
          sv[3] = s[1 + 2 * 3]; sv[4] = s[0 + 2 * 3]; sv[5] = s[0 + 1 * 3];
        }
        // r.mul<true,false>(B_tensor, S_voigt)
        mtm(d * n, 1, vs, Bv, sv, &r[p * d * n]);
      }
    }
    std::memset(inte, 0, sizeof(double) * d * n);
    for (int p = 0; p < q; ++p)
      for (int k = 0; k < d * n; ++k) inte[k] += r[p * d * n + k] * m.jac[e * q + p];
  }
}

// One NonLinearSolverLumped::solve (non_linear_solver_lumped.cc:58-82) with
// CentralDifference = NewmarkBeta(alpha = 0, beta = 1/2) (newmark-beta.hh:159-165).
void solve_step(oracle_model& m) {
  const double alpha = 0., beta = 0.5, k = 0., h = 0.;
  const double dt = m.dt;
  const int64_t ndof = (int64_t)m.u.size();
  // NewmarkBeta::predictor (newmark-beta.cc:60-89)
#pragma omp parallel for schedule(static) num_threads(m.threads) if (m.threads > 1)
  for (int64_t i = 0; i < ndof; ++i) {
    if (!m.blocked[i]) {
      double dt_a_n = dt * m.a[i];
      m.u[i] += (1 - k * alpha) * dt * m.v[i] + (.5 - h * alpha * beta) * dt * dt_a_n;
      m.v[i] = (1 - k) * m.v[i] + (1 - h * beta) * dt_a_n;
      m.a[i] = (1 - h) * m.a[i];
    }
  }
  // TimeStepSolverDefault::assembleResidual (time_step_solver_default.cc:270-284)
  if (!m.mass_assembled) assemble_mass(m);
  std::fill(m.residual.begin(), m.residual.end(), 0.);
  assemble_internal_forces(m);
  // SolidMechanicsModel::assembleResidual (solid_mechanics_model.cc:279-293)
  // through DOFManagerDefault::assembleToGlobalArray (dof_manager_default.cc:105-144)
  // (the loops below are element-wise, so fusing them changes no result)
  const double c = 1., dd = beta * dt, ee = alpha * beta * dt * dt;
#pragma omp parallel for schedule(static) num_threads(m.threads) if (m.threads > 1)
  for (int64_t i = 0; i < ndof; ++i) {
    m.residual[i] += 1. * m.fext[i];
    m.residual[i] += 1. * m.fint[i];
    // IntegrationScheme2ndOrder::assembleResidual (integration_scheme_2nd_order.cc:79-102)
    // -> assembleLumpedMatMulVectToResidual (dof_manager_default.cc:271-287)
    double cache = 0.;
    cache += -1. * m.a[i];
    m.residual[i] += m.lumped[i] * cache;
    // solveLumped (non_linear_solver_lumped.cc:85-98), b_a2x = 1
    if (!m.blocked[i]) m.solution[i] = 1. * (m.residual[i] / m.lumped[i]);
  }
  // NewmarkBeta::allCorrector<_acceleration> (newmark-beta.cc:176-210)
#pragma omp parallel for schedule(static) num_threads(m.threads) if (m.threads > 1)
  for (int64_t i = 0; i < ndof; ++i) {
    if (!m.blocked[i]) {
      m.u[i] += ee * m.solution[i];
      m.v[i] += dd * m.solution[i];
      m.a[i] += c * m.solution[i];
    }
  }
}

// Math::reduce (aka_math.cc:224-250): sort, then pairwise sums.
double reduce(std::vector<double> v) {
  size_t nb = v.size();
  if (nb == 0) return 0.;
  size_t half = nb >> 1;
  std::sort(v.begin(), v.end());
  while (half) {
    size_t rem = nb - 2 * half;
    if (rem) v[nb - 2] += v[nb - 1];
    for (size_t i = 0; i < half; ++i) v[i] = v[2 * i] + v[2 * i + 1];
    nb = half;
    half >>= 1;
  }
  return v[0];
}

}  // namespace

extern "C" {

oracle_model* oracle_create(const akb_mesh_desc* mesh, int32_t nb_materials,
                            const akb_material_desc* materials,
                            const uint32_t* element_material, int32_t* status) {
  *status = AKB_OK;
  ElementInfo info = element_info(mesh->element_type);
  int d = mesh->spatial_dimension;
  if (info.nat == 0 || info.nat != d || nb_materials < 1) {
    *status = AKB_ERR_BAD_MESH;
    return nullptr;
  }
  auto* m = new oracle_model;
  m->dim = d;
  m->type = mesh->element_type;
  m->info = info;
  m->nn = mesh->nb_nodes;
  m->ne = mesh->nb_elements;
  const int n = info.nnpe, q = info.nqp;
  m->X.assign(mesh->nodes, mesh->nodes + m->nn * d);
  m->conn.assign(mesh->connectivity, mesh->connectivity + m->ne * n);
  for (auto c : m->conn)
    if (c >= (uint64_t)m->nn) {
      *status = AKB_ERR_BAD_MESH;
      delete m;
      return nullptr;
    }
  for (int k = 0; k < nb_materials; ++k) m->mats.push_back(make_material(materials[k], d));
  m->mat_of.assign(m->ne, 0);
  if (element_material) m->mat_of.assign(element_material, element_material + m->ne);
  const size_t ndof = m->nn * d;
  for (auto* f : {&m->u, &m->v, &m->a, &m->fext, &m->fint, &m->mass, &m->lumped,
                  &m->residual, &m->solution})
    f->assign(ndof, 0.);
  m->blocked.assign(ndof, 0);
  m->gradu.assign(m->ne * q * d * d, 0.);
  m->stress.assign(m->ne * q * d * d, 0.);
  // ShapeLagrange::precomputeShapesOnIntegrationPoints / ...Derivatives...
  // (shape_lagrange_inline_impl.hh:272-307, 206-252) and
  // IntegratorGauss::initIntegrator (integrator_gauss_inline_impl.hh:676-690).
  m->N.assign(q * n, 0.);
  for (int p = 0; p < q; ++p) compute_shapes(m->type, info.qpos[p], &m->N[p * n]);
  m->B.assign(m->ne * q * d * n, 0.);
  m->jac.assign(m->ne * q, 0.);
  double Xel[24], dnds[24], J[9], Ji[9];
  for (int64_t e = 0; e < m->ne; ++e) {
    for (int aa = 0; aa < n; ++aa)
      for (int i = 0; i < d; ++i) Xel[i + aa * d] = m->X[m->conn[e * n + aa] * d + i];
    for (int p = 0; p < q; ++p) {
      compute_dnds(m->type, info.qpos[p], dnds);
      mmt(d, d, n, dnds, Xel, J);  // J = dnds * X^T (element_class_tmpl.hh:283-289)
      double detJ = detn(d, J);
      if (detJ < 0) {
        *status = AKB_ERR_NEGATIVE_JACOBIAN;
        delete m;
        return nullptr;
      }
      m->jac[e * q + p] = detJ * info.qw[p];
      invn(d, J, Ji);
      mm(d, n, d, Ji, dnds, &m->B[(e * q + p) * d * n]);  // (element_class_tmpl.hh:338-346)
    }
  }
  return m;
}

void oracle_destroy(oracle_model* m) { delete m; }

double* oracle_field(oracle_model* m, int32_t field) {
  switch (field) {
  case AKB_FIELD_DISPLACEMENT: return m->u.data();
  case AKB_FIELD_VELOCITY: return m->v.data();
  case AKB_FIELD_ACCELERATION: return m->a.data();
  case AKB_FIELD_EXTERNAL_FORCE: return m->fext.data();
  case AKB_FIELD_INTERNAL_FORCE: return m->fint.data();
  case AKB_FIELD_MASS: return m->mass.data();
  case AKB_FIELD_NODES: return m->X.data();
  case AKB_FIELD_GRAD_U: return m->gradu.data();
  case AKB_FIELD_STRESS: return m->stress.data();
  }
  return nullptr;
}

int64_t oracle_field_size(oracle_model* m, int32_t field) {
  if (field == AKB_FIELD_GRAD_U || field == AKB_FIELD_STRESS)
    return (int64_t)m->gradu.size();
  return m->nn * m->dim;
}

uint8_t* oracle_blocked(oracle_model* m) { return m->blocked.data(); }

void oracle_assemble_mass_lumped(oracle_model* m) { assemble_mass(*m); }

// SolidMechanicsModel::getStableTimeStep (solid_mechanics_model.cc:482-533)
// on the current position X + u (updateCurrentPosition, :442-457).
double oracle_stable_time_step(oracle_model* m) {
  const int d = m->dim, n = m->info.nnpe;
  double min_dt = std::numeric_limits<double>::max();
  double Xel[24];
  for (int64_t e = 0; e < m->ne; ++e) {
    for (int aa = 0; aa < n; ++aa) {
      uint32_t node = m->conn[e * n + aa];
      for (int i = 0; i < d; ++i) {
        double x = m->X[node * d + i];
        x += m->u[node * d + i];
        Xel[i + aa * d] = x;
      }
    }
    double h = inradius(m->type, Xel, d);
    double c = celerity(m->mats[m->mat_of[e]]);
    min_dt = std::min(min_dt, h / c);
  }
  return min_dt;
}

void oracle_set_time_step(oracle_model* m, double dt) { m->dt = dt; }
void oracle_set_threads(oracle_model* m, int32_t threads) { m->threads = threads < 1 ? 1 : threads; }
void oracle_solve_step(oracle_model* m) { solve_step(*m); }
void oracle_solve_steps(oracle_model* m, int64_t n) {
  for (int64_t s = 0; s < n; ++s) solve_step(*m);
}
void oracle_assemble_internal_forces(oracle_model* m) { assemble_internal_forces(*m); }
void oracle_compute_stresses(oracle_model* m) { compute_all_stresses(*m); }

double oracle_energy(oracle_model* m, int32_t kind) {
  const int d = m->dim, q = m->info.nqp;
  if (kind == AKB_ENERGY_KINETIC) {
    // getKineticEnergy (solid_mechanics_model.cc:536-582)
    double ekin = 0.;
    for (int64_t nd = 0; nd < m->nn; ++nd) {
      double mv2 = 0.;
      for (int i = 0; i < d; ++i) {
        double mm_ = m->mass[nd * d + i], vv = m->v[nd * d + i];
        if (mm_ > std::numeric_limits<double>::epsilon()) mv2 += vv * vv * mm_;
      }
      ekin += mv2;
    }
    return ekin * .5;
  }
  if (kind == AKB_ENERGY_EXTERNAL_WORK) {
    // getExternalWork (solid_mechanics_model.cc:615-662)
    double work = 0.;
    for (size_t i = 0; i < m->u.size(); ++i) {
      if (m->blocked[i])
        work -= m->fint[i] * m->v[i];
      else
        work += m->fext[i] * m->v[i];
    }
    return work * m->dt;
  }
  // Material::getPotentialEnergy (material.cc:743-757): per-QP density
  // (elastic 0.5 sigma:grad_u, material_elastic_inline_impl.hh:104-108;
  // neo-Hookean material_neohookean_inline_impl.hh:146-158), integrated per
  // element with detJ*w, summed with Math::reduce. Uses the stresses of the
  // last residual assembly, like the reference.
  std::vector<double> per_element(m->ne);
  for (int64_t e = 0; e < m->ne; ++e) {
    const Material& mat = m->mats[m->mat_of[e]];
    double inte = 0.;
    for (int p = 0; p < q; ++p) {
      const double* g = &m->gradu[(e * q + p) * d * d];
      const double* s = &m->stress[(e * q + p) * d * d];
      double epot;
      if (mat.kind == AKB_MATERIAL_NEOHOOKEAN) {
        double F[9], C[9];
        for (int i = 0; i < d; ++i)
          for (int j = 0; j < d; ++j) F[i + j * d] = double(i == j);
        for (int i = 0; i < d; ++i)
          for (int j = 0; j < d; ++j) F[i + j * d] += g[i + j * d];
        mtm(d, d, d, F, F, C);
        double J = detn(d, F);
        double trC = 0.;
        for (int i = 0; i < d; ++i) trC += C[i + i * d];
        epot = 0.5 * mat.lambda * std::pow(std::log(J), 2.) +
               mat.mu * (-std::log(J) + 0.5 * (trC - d));
      } else {
        double dd = 0.;
        if (mat.finite) {
          double E[9];
          mtm(d, d, d, g, g, E, .5);
          for (int i = 0; i < d; ++i)
            for (int j = 0; j < d; ++j) E[i + j * d] += 0.5 * (g[i + j * d] + g[j + i * d]);
          for (int k = 0; k < d * d; ++k) dd = (k == 0) ? s[0] * E[0] : dd + s[k] * E[k];
        } else {
          for (int k = 0; k < d * d; ++k) dd = (k == 0) ? s[0] * g[0] : dd + s[k] * g[k];
        }
        epot = .5 * dd;
      }
      inte += epot * m->jac[e * q + p];
    }
    per_element[e] = inte;
  }
  return reduce(per_element);
}

double oracle_time_steps(oracle_model* m, int64_t n) {
  auto t0 = std::chrono::steady_clock::now();
  for (int64_t s = 0; s < n; ++s) solve_step(*m);
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

}  // extern "C"
