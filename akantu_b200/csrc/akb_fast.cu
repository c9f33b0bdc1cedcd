// akb_fast.cu -- generic fast-path kernels (AKB_MODE_FP64, AKB_MODE_FP32_BULK)
// for any mesh: one thread per element writes its force vector, one thread
// per node gathers the forces of its elements (CSR, ascending element order,
// deterministic) and applies the lumped solve and the central-difference
// corrector in FP64.
#include "akb_fastmath.cuh"

namespace akb {
namespace {

constexpr int kThreads = 256;
inline int blocks_for(int64_t n) { return (int)((n + kThreads - 1) / kThreads); }

__global__ void k_predictor(DevModel m, double dt) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m.nn * m.dim) return;
  if (m.blocked[i]) return;
  const double a = m.a[i], v = m.v[i];
  const double dta = dt * a;
  m.u[i] += dt * v + 0.5 * dt * dta;
  m.v[i] = v + dta;
}

template <int T, typename S>
__global__ void k_element_forces(DevModel m) {
  constexpr int d = ET<T>::dim, n = ET<T>::nnpe;
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= m.ne) return;
  const MatParams& p = (m.mat_of ? m.mat_table[m.mat_of[e]] : m.mats[0]);
  uint32_t nodes[8];
#pragma unroll
  for (int a = 0; a < n; ++a) nodes[a] = __ldg(&m.conn[e * n + a]);
  double X0[3], u0[3];
#pragma unroll
  for (int i = 0; i < d; ++i) {
    X0[i] = __ldg(&m.X[(int64_t)nodes[0] * d + i]);
    u0[i] = m.u[(int64_t)nodes[0] * d + i];
  }
  double dX[3 * 8];
  S du[3 * 8];
#pragma unroll
  for (int i = 0; i < d; ++i) {
    dX[i] = 0;
    du[i] = 0;
  }
#pragma unroll
  for (int a = 1; a < n; ++a)
#pragma unroll
    for (int i = 0; i < d; ++i) {
      dX[a * d + i] = __ldg(&m.X[(int64_t)nodes[a] * d + i]) - X0[i];
      du[a * d + i] = S(m.u[(int64_t)nodes[a] * d + i] - u0[i]);
    }
  S fe[3 * 8];
  fast::element_force<T, S>(p, dX, du, fe);
  S* out = static_cast<S*>(m.fe) + e * d * n;
#pragma unroll
  for (int k = 0; k < d * n; ++k) out[k] = fe[k];
}

// One thread per node.
template <typename S>
__global__ void k_gather_correct(DevModel m, double dt, bool correct, bool has_fext) {
  int64_t node = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (node >= m.nn) return;
  const int d = m.dim;
  // element vectors are S; their assembly into the nodal force is FP64
  const S* fe = static_cast<const S*>(m.fe);
  double f[3] = {0, 0, 0};
  const int beg = m.node_ptr[node], end = m.node_ptr[node + 1];
  for (int k = beg; k < end; ++k) {
    const int32_t ent = m.node_ent[k];
    const int64_t base = (int64_t)ent * d;  // (e*n + a)*d
    for (int i = 0; i < d; ++i) f[i] -= double(fe[base + i]);
  }
  const double im = m.inv_mass[node];
  for (int i = 0; i < d; ++i) {
    const int64_t idx = node * d + i;
    const double fi = f[i];
    m.fint[idx] = fi;
    if (!correct || m.blocked[idx]) continue;
    double r = fi;
    if (has_fext) r += m.fext[idx];
    const double a = m.a[idx];
    const double x = r * im - a;
    m.a[idx] = a + x;
    m.v[idx] += 0.5 * dt * x;
    if (!isfinite(x)) m.u[idx] += 0.0 * x;  // u += 0*x (newmark-beta.cc:197)
  }
}

template <typename S>
cudaError_t launch_elements(const DevModel& m, cudaStream_t s) {
  switch (m.type) {
  case AKB_SEGMENT_2: k_element_forces<AKB_SEGMENT_2, S><<<blocks_for(m.ne), kThreads, 0, s>>>(m); break;
  case AKB_TRIANGLE_3: k_element_forces<AKB_TRIANGLE_3, S><<<blocks_for(m.ne), kThreads, 0, s>>>(m); break;
  case AKB_TETRAHEDRON_4: k_element_forces<AKB_TETRAHEDRON_4, S><<<blocks_for(m.ne), kThreads, 0, s>>>(m); break;
  default: k_element_forces<AKB_HEXAHEDRON_8, S><<<blocks_for(m.ne), kThreads, 0, s>>>(m); break;
  }
  return cudaGetLastError();
}

// User materials: displacement gradient at every quadrature point (FP64,
// column-major per point, like Material::gradu), one thread per point (the
// points of an element are consecutive threads: their corner loads coincide) ...
template <int T>
__global__ void k_qp_gradu(DevModel m) {
  constexpr int d = ET<T>::dim, n = ET<T>::nnpe, nq = ET<T>::nqp;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= m.ne * nq) return;
  const int64_t e = t / nq;
  const int q = (int)(t - e * nq);
  double dX[3 * 8], du[3 * 8];
  uint32_t nodes[8];
#pragma unroll
  for (int a = 0; a < n; ++a) nodes[a] = m.conn[e * n + a];
#pragma unroll
  for (int a = 0; a < n; ++a)
#pragma unroll
    for (int i = 0; i < d; ++i) {
      dX[a * d + i] = m.X[(int64_t)nodes[a] * d + i] - m.X[(int64_t)nodes[0] * d + i];
      du[a * d + i] = m.u[(int64_t)nodes[a] * d + i] - m.u[(int64_t)nodes[0] * d + i];
    }
  double B[3 * 8];
  fast::shape_gradients<T, double>(dX, q, B);
  double* g = m.gradu + (e * nq + q) * d * d;
#pragma unroll
  for (int i = 0; i < d; ++i)
#pragma unroll
    for (int j = 0; j < d; ++j) {
      double c = 0;
#pragma unroll
      for (int a = 1; a < n; ++a) c += du[a * d + i] * B[a * d + j];
      g[i + j * d] = c;
    }
}

// ... and the element force vectors sum_q w_q det J_q stress_q grad N_a from
// the stresses the caller wrote: one thread per point, the nq points of an
// element in consecutive lanes of one warp, their vectors added by a fixed
// butterfly over those lanes (the element's first lane writes the sum).
template <int T>
__global__ void k_qp_forces(DevModel m) {
  constexpr int d = ET<T>::dim, n = ET<T>::nnpe, nq = ET<T>::nqp;
  static_assert((nq & (nq - 1)) == 0 && nq <= 32, "points per element: a power of two <= 32");
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool valid = t < m.ne * nq;  // every lane takes part in the shuffles
  const int64_t e = t / nq;
  const int q = (int)(t - e * nq);
  double fe[3 * 8];
#pragma unroll
  for (int k = 0; k < d * n; ++k) fe[k] = 0.0;
  if (valid) {
    double dX[3 * 8];
    uint32_t nodes[8];
#pragma unroll
    for (int a = 0; a < n; ++a) nodes[a] = m.conn[e * n + a];
#pragma unroll
    for (int a = 0; a < n; ++a)
#pragma unroll
      for (int i = 0; i < d; ++i)
        dX[a * d + i] = m.X[(int64_t)nodes[a] * d + i] - m.X[(int64_t)nodes[0] * d + i];
    double B[3 * 8];
    const double wq = fast::weight<T>() * fast::shape_gradients<T, double>(dX, q, B);
    const double* P = m.stress + (e * nq + q) * d * d;
#pragma unroll
    for (int a = 0; a < n; ++a)
#pragma unroll
      for (int i = 0; i < d; ++i) {
        double c = 0;
#pragma unroll
        for (int j = 0; j < d; ++j) c += P[i + j * d] * B[a * d + j];
        fe[a * d + i] = wq * c;
      }
  }
#pragma unroll
  for (int off = 1; off < nq; off <<= 1)
#pragma unroll
    for (int k = 0; k < d * n; ++k) fe[k] += __shfl_xor_sync(0xffffffffu, fe[k], off);
  if (valid && q == 0) {
    double* out = static_cast<double*>(m.fe) + e * d * n;
#pragma unroll
    for (int k = 0; k < d * n; ++k) out[k] = fe[k];
  }
}

// comp >= 0: one thread per listed node, that component; comp < 0: one
// thread per (listed node, component), values row per node. Launched with
// programmatic serialization behind the step's last kernel, it waits for
// that grid before touching the node state.
__global__ void k_apply_dirichlet(DevModel m, const uint32_t* nodes, int64_t n, int comp,
                                  const double* values, const uint32_t* perm, double* w) {
  grid_wait();
  grid_launch_dependents();
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int ncomp = comp < 0 ? m.dim : 1;
  if (k >= n * ncomp) return;
  const int64_t q = k / ncomp;
  const int c = comp < 0 ? (int)(k - q * ncomp) : comp;
  uint32_t node = nodes[q];
  if (node >= m.nn) return;  // out-of-range node ids are ignored
  if (perm) node = perm[node];
  const int64_t i = (int64_t)node * m.dim + c;
  m.blocked[i] = 1;
  m.u[i] = values[k];
  if (w) w[i] = values[k];  // a blocked DOF's predicted displacement is its u
}

}  // namespace

cudaError_t apply_dirichlet(const DevModel& m, const uint32_t* nodes, int64_t n, int comp,
                            const double* values, const uint32_t* perm, double* w,
                            cudaStream_t s) {
  return launch_pdl(k_apply_dirichlet, blocks_for(comp < 0 ? n * m.dim : n), kThreads, 0, s, m,
                    nodes, n, comp, values, perm, w);
}

cudaError_t user_qp_gradients(const DevModel& m, cudaStream_t s) {
  if (m.ne == 0) return cudaSuccess;
  switch (m.type) {  // one thread per quadrature point
  case AKB_SEGMENT_2: k_qp_gradu<AKB_SEGMENT_2><<<blocks_for(m.ne), kThreads, 0, s>>>(m); break;
  case AKB_TRIANGLE_3: k_qp_gradu<AKB_TRIANGLE_3><<<blocks_for(m.ne), kThreads, 0, s>>>(m); break;
  case AKB_TETRAHEDRON_4: k_qp_gradu<AKB_TETRAHEDRON_4><<<blocks_for(m.ne), kThreads, 0, s>>>(m); break;
  default: k_qp_gradu<AKB_HEXAHEDRON_8><<<blocks_for(m.ne * 8), kThreads, 0, s>>>(m); break;
  }
  return cudaGetLastError();
}

cudaError_t user_element_forces(const DevModel& m, cudaStream_t s) {
  if (m.ne == 0) return cudaSuccess;
  switch (m.type) {  // one thread per quadrature point
  case AKB_SEGMENT_2: k_qp_forces<AKB_SEGMENT_2><<<blocks_for(m.ne), kThreads, 0, s>>>(m); break;
  case AKB_TRIANGLE_3: k_qp_forces<AKB_TRIANGLE_3><<<blocks_for(m.ne), kThreads, 0, s>>>(m); break;
  case AKB_TETRAHEDRON_4: k_qp_forces<AKB_TETRAHEDRON_4><<<blocks_for(m.ne), kThreads, 0, s>>>(m); break;
  default: k_qp_forces<AKB_HEXAHEDRON_8><<<blocks_for(m.ne * 8), kThreads, 0, s>>>(m); break;
  }
  return cudaGetLastError();
}

cudaError_t fast_predictor(const DevModel& m, double dt, cudaStream_t s) {
  k_predictor<<<blocks_for(m.nn * m.dim), kThreads, 0, s>>>(m, dt);
  return cudaGetLastError();
}

cudaError_t fast_element_forces(const DevModel& m, bool fp32, cudaStream_t s) {
  if (m.ne == 0) return cudaSuccess;
  return fp32 ? launch_elements<float>(m, s) : launch_elements<double>(m, s);
}

cudaError_t fast_gather_correct(const DevModel& m, double dt, bool fp32, bool correct,
                                bool has_fext, cudaStream_t s) {
  if (fp32)
    k_gather_correct<float><<<blocks_for(m.nn), kThreads, 0, s>>>(m, dt, correct, has_fext);
  else
    k_gather_correct<double><<<blocks_for(m.nn), kThreads, 0, s>>>(m, dt, correct, has_fext);
  return cudaGetLastError();
}

}  // namespace akb
