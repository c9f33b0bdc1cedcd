// akb_reference.cu -- FP64 kernels in the reference's operation order
// (AKB_MODE_FP64_REFERENCE). Compiled with --fmad=false.
//
// Per step (NonLinearSolverLumped::solve, non_linear_solver_lumped.cc:58-82):
//   ref_predictor        NewmarkBeta::predictor (newmark-beta.cc:60-89)
//   ref_element_forces   Material::computeAllStresses + assembleInternalForces
//                        element part (material.cc:178-279, 637-722)
//   ref_gather_correct   element-order assembly (dof_manager.cc:83-137) as a
//                        node-centric CSR gather in ascending element order,
//                        residual (time_step_solver.cc:177-178,
//                        dof_manager_default.cc:105-144, 271-287),
//                        solveLumped (non_linear_solver_lumped.cc:85-98) and
//                        allCorrector<_acceleration> (newmark-beta.cc:176-210).
#include "akb_refmath.cuh"

namespace akb {
namespace {

constexpr int kThreads = 256;

inline int blocks_for(int64_t n) { return (int)((n + kThreads - 1) / kThreads); }

template <int T>
__device__ inline void gather_el(const DevModel& m, int64_t e, const double* field, double* el) {
  constexpr int d = ET<T>::dim, n = ET<T>::nnpe;
#pragma unroll
  for (int a = 0; a < n; ++a) {
    const uint32_t node = m.conn[e * n + a];
#pragma unroll
    for (int i = 0; i < d; ++i) el[i + a * d] = field[(int64_t)node * d + i];
  }
}

template <int T>
__global__ void k_init_geometry(DevModel m, int* negative) {
  constexpr int d = ET<T>::dim, n = ET<T>::nnpe, q = ET<T>::nqp;
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= m.ne) return;
  double Xel[3 * 8];
  gather_el<T>(m, e, m.X, Xel);
  for (int p = 0; p < q; ++p) {
    double jac;
    ref::geometry<T>(Xel, p, &m.B[(e * q + p) * d * n], &jac);
    // checkJacobians (integrator_gauss_inline_impl.hh:183-205) runs on det(J)
    // before the weights are applied; the weights are positive.
    if (jac < 0) atomicExch(negative, 1);
    m.jac[e * q + p] = jac;
  }
}

__global__ void k_predictor(DevModel m, double dt) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m.nn * m.dim) return;
  if (m.blocked[i]) return;
  const double alpha = 0., beta = 0.5, k = 0., h = 0.;
  double u = m.u[i], v = m.v[i], a = m.a[i];
  double dt_a_n = dt * a;
  u += (1 - k * alpha) * dt * v + (.5 - h * alpha * beta) * dt * dt_a_n;
  v = (1 - k) * v + (1 - h * beta) * dt_a_n;
  a = (1 - h) * a;
  m.u[i] = u;
  m.v[i] = v;
  m.a[i] = a;
}

template <int T>
__global__ void k_element_forces(DevModel m) {
  constexpr int d = ET<T>::dim, n = ET<T>::nnpe, q = ET<T>::nqp;
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= m.ne) return;
  const MatParams& p = (m.mat_of ? m.mat_table[m.mat_of[e]] : m.mats[0]);
  double uel[3 * 8], inte[3 * 8], r[3 * 8];
  gather_el<T>(m, e, m.u, uel);
#pragma unroll
  for (int k = 0; k < d * n; ++k) inte[k] = 0.;
  for (int pq = 0; pq < q; ++pq) {
    const double* B = &m.B[(e * q + pq) * d * n];
    double* g = &m.gradu[(e * q + pq) * d * d];
    double* s = &m.stress[(e * q + pq) * d * d];
    double gl[9], sl[9];
    ref::mmt<d, d, n>(uel, B, gl);  // nabla_u.mul<false,true>(u_el, B)
#pragma unroll
    for (int k = 0; k < d * d; ++k) gl[k] -= 0.;  // eigengradu
    ref::stress<d>(p, gl, sl);
#pragma unroll
    for (int k = 0; k < d * d; ++k) {
      g[k] = gl[k];
      s[k] = sl[k];
    }
    ref::qp_force<T>(p, B, gl, sl, r);
    const double jq = m.jac[e * q + pq];
#pragma unroll
    for (int k = 0; k < d * n; ++k) inte[k] += r[k] * jq;
  }
  double* fe = static_cast<double*>(m.fe) + e * d * n;
#pragma unroll
  for (int k = 0; k < d * n; ++k) fe[k] = inte[k];
}

// One thread per DOF: internal force gathered in ascending element order,
// then the residual, the lumped solve and the corrector.
__global__ void k_gather_correct(DevModel m, double dt, bool correct) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int d = m.dim;
  if (i >= m.nn * d) return;
  const int64_t node = i / d;
  const int comp = (int)(i - node * d);
  const double* fe = static_cast<const double*>(m.fe);
  double f = 0.;
  for (int k = m.node_ptr[node]; k < m.node_ptr[node + 1]; ++k) {
    const int32_t ent = m.node_ent[k];
    const int64_t e = ent / m.nnpe;
    const int a = ent - (int)e * m.nnpe;
    f += -1. * fe[e * d * m.nnpe + comp + a * d];
  }
  m.fint[i] = f;
  if (!correct || m.blocked[i]) return;
  const double M = m.mass[i];
  double r = 0.;
  r += 1. * m.fext[i];
  r += 1. * f;
  double a = m.a[i];
  double c = 0.;
  c += -1. * a;
  r += M * c;
  const double x = 1. * (r / M);
  const double alpha = 0., beta = 0.5;
  const double cc = 1., dd = beta * dt, ee = alpha * beta * dt * dt;
  m.u[i] += ee * x;
  m.v[i] += dd * x;
  m.a[i] = a + cc * x;
}

// Lumped mass, element part: rho * N integrated with detJ*w
// (fe_engine_template_tmpl_field.hh:165-199).
template <int T>
__global__ void k_mass_element(DevModel m) {
  constexpr int d = ET<T>::dim, n = ET<T>::nnpe, q = ET<T>::nqp;
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= m.ne) return;
  const MatParams& p = (m.mat_of ? m.mat_table[m.mat_of[e]] : m.mats[0]);
  double inte[3 * 8];
#pragma unroll
  for (int k = 0; k < d * n; ++k) inte[k] = 0.;
  for (int pq = 0; pq < q; ++pq) {
    double c[3], N[8], b[3] = {p.rho, p.rho, p.rho}, ntb[3 * 8];
    ref::qp_coords<T>(pq, c);
    ref::shapes<T>(c, N);
    ref::mm<d, n, 1>(b, N, ntb);  // Ntb.mul<false,false>(b, N)
    const double jq = m.jac[e * q + pq];
#pragma unroll
    for (int k = 0; k < d * n; ++k) inte[k] += ntb[k] * jq;
  }
  double* fe = static_cast<double*>(m.fe) + e * d * n;
#pragma unroll
  for (int k = 0; k < d * n; ++k) fe[k] = inte[k];
}

__global__ void k_mass_gather(DevModel m) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int d = m.dim;
  if (i >= m.nn * d) return;
  const int64_t node = i / d;
  const int comp = (int)(i - node * d);
  const double* fe = static_cast<const double*>(m.fe);
  double local = 0.;
  for (int k = m.node_ptr[node]; k < m.node_ptr[node + 1]; ++k) {
    const int32_t ent = m.node_ent[k];
    const int64_t e = ent / m.nnpe;
    const int a = ent - (int)e * m.nnpe;
    local += 1. * fe[e * d * m.nnpe + comp + a * d];
  }
  double M = 0.;
  M += 1. * local;
  m.mass[i] = M;
  if (comp == 0) m.inv_mass[node] = 1. / M;
}

template <int T>
__global__ void k_compute_stresses(DevModel m, bool recompute_geometry) {
  constexpr int d = ET<T>::dim, n = ET<T>::nnpe, q = ET<T>::nqp;
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= m.ne) return;
  const MatParams& p = (m.mat_of ? m.mat_table[m.mat_of[e]] : m.mats[0]);
  double uel[3 * 8], Xel[3 * 8];
  gather_el<T>(m, e, m.u, uel);
  if (recompute_geometry) gather_el<T>(m, e, m.X, Xel);
  for (int pq = 0; pq < q; ++pq) {
    double Bl[3 * 8], jac, gl[9], sl[9];
    const double* B = Bl;
    if (recompute_geometry)
      ref::geometry<T>(Xel, pq, Bl, &jac);
    else
      B = &m.B[(e * q + pq) * d * n];
    ref::mmt<d, d, n>(uel, B, gl);
#pragma unroll
    for (int k = 0; k < d * d; ++k) gl[k] -= 0.;
    ref::stress<d>(p, gl, sl);
#pragma unroll
    for (int k = 0; k < d * d; ++k) {
      m.gradu[(e * q + pq) * d * d + k] = gl[k];
      m.stress[(e * q + pq) * d * d + k] = sl[k];
    }
  }
}

#define AKB_DISPATCH_TYPE(type, KERNEL, ...)                                       \
  switch (type) {                                                                  \
  case AKB_SEGMENT_2: KERNEL<AKB_SEGMENT_2><<<__VA_ARGS__>>>; break;               \
  case AKB_TRIANGLE_3: KERNEL<AKB_TRIANGLE_3><<<__VA_ARGS__>>>; break;             \
  case AKB_TETRAHEDRON_4: KERNEL<AKB_TETRAHEDRON_4><<<__VA_ARGS__>>>; break;       \
  default: KERNEL<AKB_HEXAHEDRON_8><<<__VA_ARGS__>>>; break;                       \
  }

}  // namespace

cudaError_t ref_init_geometry(const DevModel& m, cudaStream_t s, int* d_negative) {
  if (m.ne == 0) return cudaSuccess;
  switch (m.type) {
  case AKB_SEGMENT_2: k_init_geometry<AKB_SEGMENT_2><<<blocks_for(m.ne), kThreads, 0, s>>>(m, d_negative); break;
  case AKB_TRIANGLE_3: k_init_geometry<AKB_TRIANGLE_3><<<blocks_for(m.ne), kThreads, 0, s>>>(m, d_negative); break;
  case AKB_TETRAHEDRON_4: k_init_geometry<AKB_TETRAHEDRON_4><<<blocks_for(m.ne), kThreads, 0, s>>>(m, d_negative); break;
  default: k_init_geometry<AKB_HEXAHEDRON_8><<<blocks_for(m.ne), kThreads, 0, s>>>(m, d_negative); break;
  }
  return cudaGetLastError();
}

cudaError_t ref_predictor(const DevModel& m, double dt, cudaStream_t s) {
  k_predictor<<<blocks_for(m.nn * m.dim), kThreads, 0, s>>>(m, dt);
  return cudaGetLastError();
}

cudaError_t ref_element_forces(const DevModel& m, cudaStream_t s) {
  if (m.ne == 0) return cudaSuccess;
  switch (m.type) {
  case AKB_SEGMENT_2: k_element_forces<AKB_SEGMENT_2><<<blocks_for(m.ne), kThreads, 0, s>>>(m); break;
  case AKB_TRIANGLE_3: k_element_forces<AKB_TRIANGLE_3><<<blocks_for(m.ne), kThreads, 0, s>>>(m); break;
  case AKB_TETRAHEDRON_4: k_element_forces<AKB_TETRAHEDRON_4><<<blocks_for(m.ne), kThreads, 0, s>>>(m); break;
  default: k_element_forces<AKB_HEXAHEDRON_8><<<blocks_for(m.ne), kThreads, 0, s>>>(m); break;
  }
  return cudaGetLastError();
}

cudaError_t ref_gather_correct(const DevModel& m, double dt, bool correct, cudaStream_t s) {
  k_gather_correct<<<blocks_for(m.nn * m.dim), kThreads, 0, s>>>(m, dt, correct);
  return cudaGetLastError();
}

cudaError_t ref_mass(const DevModel& m, cudaStream_t s) {
  if (m.ne > 0) {
    switch (m.type) {
    case AKB_SEGMENT_2: k_mass_element<AKB_SEGMENT_2><<<blocks_for(m.ne), kThreads, 0, s>>>(m); break;
    case AKB_TRIANGLE_3: k_mass_element<AKB_TRIANGLE_3><<<blocks_for(m.ne), kThreads, 0, s>>>(m); break;
    case AKB_TETRAHEDRON_4: k_mass_element<AKB_TETRAHEDRON_4><<<blocks_for(m.ne), kThreads, 0, s>>>(m); break;
    default: k_mass_element<AKB_HEXAHEDRON_8><<<blocks_for(m.ne), kThreads, 0, s>>>(m); break;
    }
  }
  k_mass_gather<<<blocks_for(m.nn * m.dim), kThreads, 0, s>>>(m);
  return cudaGetLastError();
}

cudaError_t ref_compute_stresses(const DevModel& m, bool recompute_geometry, cudaStream_t s) {
  if (m.ne == 0) return cudaSuccess;
  switch (m.type) {
  case AKB_SEGMENT_2: k_compute_stresses<AKB_SEGMENT_2><<<blocks_for(m.ne), kThreads, 0, s>>>(m, recompute_geometry); break;
  case AKB_TRIANGLE_3: k_compute_stresses<AKB_TRIANGLE_3><<<blocks_for(m.ne), kThreads, 0, s>>>(m, recompute_geometry); break;
  case AKB_TETRAHEDRON_4: k_compute_stresses<AKB_TETRAHEDRON_4><<<blocks_for(m.ne), kThreads, 0, s>>>(m, recompute_geometry); break;
  default: k_compute_stresses<AKB_HEXAHEDRON_8><<<blocks_for(m.ne), kThreads, 0, s>>>(m, recompute_geometry); break;
  }
  return cudaGetLastError();
}

}  // namespace akb
