// akb_reduce.cu -- deterministic reductions: stable time step (min over
// elements) and the energies (FP64 sums). Compiled with --fmad=false so the
// per-element terms are the reference's arithmetic.
//
// Each reduction is two launches: a fixed grid writes one partial per block
// into scratch (grid-stride loop in index order, then a fixed-shape tree in
// shared memory), and one block combines the partials in the same fixed
// order. The result is identical from run to run.
#include <cfloat>

#include "akb_refmath.cuh"

namespace akb {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 1184;  // 8 x 148 SMs

enum Op { kSum = 0, kMin = 1 };

template <Op op>
__device__ inline double combine(double a, double b) {
  return op == kSum ? a + b : fmin(a, b);
}

template <Op op>
__device__ inline double block_reduce(double v) {
  __shared__ double sh[kThreads];
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] = combine<op>(sh[threadIdx.x], sh[threadIdx.x + s]);
    __syncthreads();
  }
  return sh[0];
}

// One block; launched behind the kernel that wrote the partials with
// programmatic serialization (sum_partials) it waits for that grid first.
// Each thread combines its partials in index order, eight loads in flight.
template <Op op>
__global__ void k_finish(const double* partial, int n, double scale, double* out) {
  grid_wait();
  grid_launch_dependents();
  double acc = op == kSum ? 0.0 : DBL_MAX;
#pragma unroll 8
  for (int i = threadIdx.x; i < n; i += kThreads) acc = combine<op>(acc, partial[i]);
  acc = block_reduce<op>(acc);
  if (threadIdx.x == 0) *out = op == kSum ? acc * scale : acc;
}

// Element inradius (fe_engine_inline_impl.hh:45-55, aka_math_tmpl.hh:568-650,
// element_class_hexahedron_8_inline_impl.hh:219-246).
__device__ inline double dist(const double* x, const double* y, int d) {
  if (d == 1) return sqrt((y[0] - x[0]) * (y[0] - x[0]));
  if (d == 2) return sqrt((y[0] - x[0]) * (y[0] - x[0]) + (y[1] - x[1]) * (y[1] - x[1]));
  return sqrt((y[0] - x[0]) * (y[0] - x[0]) + (y[1] - x[1]) * (y[1] - x[1]) +
              (y[2] - x[2]) * (y[2] - x[2]));
}

template <int T>
__device__ inline double inradius(const double* X) {
  if (T == AKB_SEGMENT_2) return fabs(X[0] - X[1]);
  if (T == AKB_TRIANGLE_3) {
    double a = dist(X + 0, X + 2, 2), b = dist(X + 2, X + 4, 2), c = dist(X + 0, X + 4, 2);
    double s = (a + b + c) * 0.5;
    return 2. * sqrt((s - a) * (s - b) * (s - c) / s);
  }
  if (T == AKB_TETRAHEDRON_4) {
    const double *c1 = X, *c2 = X + 3, *c3 = X + 6, *c4 = X + 9;
    double l12 = dist(c1, c2, 3), l13 = dist(c1, c3, 3), l14 = dist(c1, c4, 3);
    double l23 = dist(c2, c3, 3), l24 = dist(c2, c4, 3), l34 = dist(c3, c4, 3);
    double s1 = (l12 + l23 + l13) * 0.5;
    s1 = sqrt(s1 * (s1 - l12) * (s1 - l23) * (s1 - l13));
    double s2 = (l12 + l24 + l14) * 0.5;
    s2 = sqrt(s2 * (s2 - l12) * (s2 - l24) * (s2 - l14));
    double s3 = (l23 + l34 + l24) * 0.5;
    s3 = sqrt(s3 * (s3 - l23) * (s3 - l34) * (s3 - l24));
    double s4 = (l13 + l34 + l14) * 0.5;
    s4 = sqrt(s4 * (s4 - l13) * (s4 - l34) * (s4 - l14));
    // Math::tetrahedron_volume (aka_math_tmpl.hh:590-648)
    double xx[9], vol;
    auto fill = [&](const double* a, const double* b, const double* c) {
      xx[0] = a[0]; xx[1] = a[1]; xx[2] = a[2];
      xx[3] = b[0]; xx[4] = b[1]; xx[5] = b[2];
      xx[6] = c[0]; xx[7] = c[1]; xx[8] = c[2];
    };
    fill(c2, c3, c4); vol = ref::det<3>(xx);
    fill(c1, c3, c4); vol -= ref::det<3>(xx);
    fill(c1, c2, c4); vol += ref::det<3>(xx);
    fill(c1, c2, c3); vol -= ref::det<3>(xx);
    vol /= 6;
    return 2. * (3 * vol / (s1 + s2 + s3 + s4));
  }
  const int e[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {0, 4}, {1, 5},
                        {2, 6}, {3, 7}, {4, 5}, {5, 6}, {6, 7}, {7, 4}};
  double p = DBL_MAX;
  for (int k = 0; k < 12; ++k) p = fmin(p, dist(X + 3 * e[k][0], X + 3 * e[k][1], 3));
  return p;
}

template <int T>
__global__ void k_stable_dt(DevModel m, double* partial) {
  constexpr int d = ET<T>::dim, n = ET<T>::nnpe;
  double acc = DBL_MAX;
  for (int64_t e = blockIdx.x * (int64_t)kThreads + threadIdx.x; e < m.ne;
       e += (int64_t)gridDim.x * kThreads) {
    double Xel[3 * 8];
    for (int a = 0; a < n; ++a) {
      const uint32_t node = m.conn[e * n + a];
      for (int i = 0; i < d; ++i) {
        double x = m.X[(int64_t)node * d + i];
        x += m.u[(int64_t)node * d + i];  // updateCurrentPosition
        Xel[a * d + i] = x;
      }
    }
    const double h = inradius<T>(Xel);
    const double c = (m.mat_of ? m.mat_table[m.mat_of[e]] : m.mats[0]).celerity;
    acc = fmin(acc, h / c);
  }
  acc = block_reduce<kMin>(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// getKineticEnergy (solid_mechanics_model.cc:536-582)
__global__ void k_kinetic(DevModel m, double* partial) {
  const int d = m.dim;
  double acc = 0.;
  for (int64_t node = blockIdx.x * (int64_t)kThreads + threadIdx.x; node < m.nn;
       node += (int64_t)gridDim.x * kThreads) {
    double mv2 = 0.;
    for (int i = 0; i < d; ++i) {
      const double mm = m.mass[node * d + i], vv = m.v[node * d + i];
      if (mm > DBL_EPSILON) mv2 += vv * vv * mm;
    }
    acc += mv2;
  }
  acc = block_reduce<kSum>(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// getExternalWork (solid_mechanics_model.cc:615-662)
__global__ void k_work(DevModel m, double* partial) {
  double acc = 0.;
  for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < m.nn * m.dim;
       i += (int64_t)gridDim.x * kThreads) {
    if (m.blocked[i])
      acc -= m.fint[i] * m.v[i];
    else
      acc += m.fext[i] * m.v[i];
  }
  acc = block_reduce<kSum>(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// Material::getPotentialEnergy (material.cc:743-757) on the current
// displacement, geometry recomputed in the reference's arithmetic.
template <int T>
__global__ void k_potential(DevModel m, double* partial) {
  constexpr int d = ET<T>::dim, n = ET<T>::nnpe, q = ET<T>::nqp;
  double acc = 0.;
  for (int64_t e = blockIdx.x * (int64_t)kThreads + threadIdx.x; e < m.ne;
       e += (int64_t)gridDim.x * kThreads) {
    const MatParams& p = (m.mat_of ? m.mat_table[m.mat_of[e]] : m.mats[0]);
    double Xel[3 * 8], uel[3 * 8];
    for (int a = 0; a < n; ++a) {
      const uint32_t node = m.conn[e * n + a];
      for (int i = 0; i < d; ++i) {
        Xel[i + a * d] = m.X[(int64_t)node * d + i];
        uel[i + a * d] = m.u[(int64_t)node * d + i];
      }
    }
    double inte = 0.;
    for (int pq = 0; pq < q; ++pq) {
      double B[3 * 8], jac, g[9], s[9];
      ref::geometry<T>(Xel, pq, B, &jac);
      ref::mmt<d, d, n>(uel, B, g);
      ref::stress<d>(p, g, s);
      inte += ref::energy_density<d>(p, g, s) * jac;
    }
    acc += inte;
  }
  acc = block_reduce<kSum>(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// Batches: block b reduces instance b's elements (or nodes).
template <int T>
__global__ void k_stable_dt_inst(DevModel m, const int64_t* elem_off, double* out) {
  constexpr int d = ET<T>::dim, n = ET<T>::nnpe;
  double acc = DBL_MAX;
  for (int64_t e = elem_off[blockIdx.x] + threadIdx.x; e < elem_off[blockIdx.x + 1]; e += kThreads) {
    double Xel[3 * 8];
    for (int a = 0; a < n; ++a) {
      const uint32_t node = m.conn[e * n + a];
      for (int i = 0; i < d; ++i) {
        double x = m.X[(int64_t)node * d + i];
        x += m.u[(int64_t)node * d + i];
        Xel[a * d + i] = x;
      }
    }
    const double c = (m.mat_of ? m.mat_table[m.mat_of[e]] : m.mats[0]).celerity;
    acc = fmin(acc, inradius<T>(Xel) / c);
  }
  acc = block_reduce<kMin>(acc);
  if (threadIdx.x == 0) out[blockIdx.x] = acc;
}

__global__ void k_kinetic_inst(DevModel m, const int64_t* node_off, double* out) {
  const int d = m.dim;
  double acc = 0.;
  for (int64_t node = node_off[blockIdx.x] + threadIdx.x; node < node_off[blockIdx.x + 1];
       node += kThreads) {
    double mv2 = 0.;
    for (int i = 0; i < d; ++i) {
      const double mm = m.mass[node * d + i], vv = m.v[node * d + i];
      if (mm > DBL_EPSILON) mv2 += vv * vv * mm;
    }
    acc += mv2;
  }
  acc = block_reduce<kSum>(acc);
  if (threadIdx.x == 0) out[blockIdx.x] = acc * 0.5;
}

template <int T>
__global__ void k_potential_inst(DevModel m, const int64_t* elem_off, double* out) {
  constexpr int d = ET<T>::dim, n = ET<T>::nnpe, q = ET<T>::nqp;
  double acc = 0.;
  for (int64_t e = elem_off[blockIdx.x] + threadIdx.x; e < elem_off[blockIdx.x + 1]; e += kThreads) {
    const MatParams& p = (m.mat_of ? m.mat_table[m.mat_of[e]] : m.mats[0]);
    double Xel[3 * 8], uel[3 * 8];
    for (int a = 0; a < n; ++a) {
      const uint32_t node = m.conn[e * n + a];
      for (int i = 0; i < d; ++i) {
        Xel[i + a * d] = m.X[(int64_t)node * d + i];
        uel[i + a * d] = m.u[(int64_t)node * d + i];
      }
    }
    double inte = 0.;
    for (int pq = 0; pq < q; ++pq) {
      double B[3 * 8], jac, g[9], s[9];
      ref::geometry<T>(Xel, pq, B, &jac);
      ref::mmt<d, d, n>(uel, B, g);
      ref::stress<d>(p, g, s);
      inte += ref::energy_density<d>(p, g, s) * jac;
    }
    acc += inte;
  }
  acc = block_reduce<kSum>(acc);
  if (threadIdx.x == 0) out[blockIdx.x] = acc;
}

int grid_for(int64_t n) {
  int64_t b = (n + kThreads - 1) / kThreads;
  if (b < 1) b = 1;
  return (int)(b < kMaxBlocks ? b : kMaxBlocks);
}

}  // namespace

int reduce_blocks(int64_t) { return kMaxBlocks; }

cudaError_t stable_dt(const DevModel& m, double* scratch, int scratch_len, double* out,
                      cudaStream_t s) {
  int g = grid_for(m.ne);
  if (g > scratch_len) g = scratch_len;
  switch (m.type) {
  case AKB_SEGMENT_2: k_stable_dt<AKB_SEGMENT_2><<<g, kThreads, 0, s>>>(m, scratch); break;
  case AKB_TRIANGLE_3: k_stable_dt<AKB_TRIANGLE_3><<<g, kThreads, 0, s>>>(m, scratch); break;
  case AKB_TETRAHEDRON_4: k_stable_dt<AKB_TETRAHEDRON_4><<<g, kThreads, 0, s>>>(m, scratch); break;
  default: k_stable_dt<AKB_HEXAHEDRON_8><<<g, kThreads, 0, s>>>(m, scratch); break;
  }
  k_finish<kMin><<<1, kThreads, 0, s>>>(scratch, g, 1.0, out);
  return cudaGetLastError();
}

cudaError_t sum_partials(const double* partial, int64_t n, double scale, double* out,
                         cudaStream_t s) {
  return launch_pdl(k_finish<kSum>, 1, kThreads, 0, s, partial, (int)n, scale, out);
}

cudaError_t energy(const DevModel& m, int kind, double dt, double* scratch, int scratch_len,
                   double* out, cudaStream_t s) {
  double scale = 1.0;
  int g;
  if (kind == AKB_ENERGY_KINETIC) {
    g = grid_for(m.nn);
    if (g > scratch_len) g = scratch_len;
    k_kinetic<<<g, kThreads, 0, s>>>(m, scratch);
    scale = 0.5;
  } else if (kind == AKB_ENERGY_EXTERNAL_WORK) {
    g = grid_for(m.nn * m.dim);
    if (g > scratch_len) g = scratch_len;
    k_work<<<g, kThreads, 0, s>>>(m, scratch);
    scale = dt;
  } else {
    g = grid_for(m.ne);
    if (g > scratch_len) g = scratch_len;
    switch (m.type) {
    case AKB_SEGMENT_2: k_potential<AKB_SEGMENT_2><<<g, kThreads, 0, s>>>(m, scratch); break;
    case AKB_TRIANGLE_3: k_potential<AKB_TRIANGLE_3><<<g, kThreads, 0, s>>>(m, scratch); break;
    case AKB_TETRAHEDRON_4: k_potential<AKB_TETRAHEDRON_4><<<g, kThreads, 0, s>>>(m, scratch); break;
    default: k_potential<AKB_HEXAHEDRON_8><<<g, kThreads, 0, s>>>(m, scratch); break;
    }
  }
  k_finish<kSum><<<1, kThreads, 0, s>>>(scratch, g, scale, out);
  return cudaGetLastError();
}

}  // namespace akb

namespace akb {

cudaError_t stable_dt_instances(const DevModel& m, const int64_t* elem_off, int ninst,
                                double* out, cudaStream_t s) {
  if (ninst <= 0) return cudaSuccess;
  switch (m.type) {
  case AKB_SEGMENT_2: k_stable_dt_inst<AKB_SEGMENT_2><<<ninst, kThreads, 0, s>>>(m, elem_off, out); break;
  case AKB_TRIANGLE_3: k_stable_dt_inst<AKB_TRIANGLE_3><<<ninst, kThreads, 0, s>>>(m, elem_off, out); break;
  case AKB_TETRAHEDRON_4: k_stable_dt_inst<AKB_TETRAHEDRON_4><<<ninst, kThreads, 0, s>>>(m, elem_off, out); break;
  default: k_stable_dt_inst<AKB_HEXAHEDRON_8><<<ninst, kThreads, 0, s>>>(m, elem_off, out); break;
  }
  return cudaGetLastError();
}

cudaError_t energy_instances(const DevModel& m, int kind, const int64_t* node_off,
                             const int64_t* elem_off, int ninst, double* out, cudaStream_t s) {
  if (ninst <= 0) return cudaSuccess;
  if (kind == AKB_ENERGY_KINETIC) {
    k_kinetic_inst<<<ninst, kThreads, 0, s>>>(m, node_off, out);
  } else {
    switch (m.type) {
    case AKB_SEGMENT_2: k_potential_inst<AKB_SEGMENT_2><<<ninst, kThreads, 0, s>>>(m, elem_off, out); break;
    case AKB_TRIANGLE_3: k_potential_inst<AKB_TRIANGLE_3><<<ninst, kThreads, 0, s>>>(m, elem_off, out); break;
    case AKB_TETRAHEDRON_4: k_potential_inst<AKB_TETRAHEDRON_4><<<ninst, kThreads, 0, s>>>(m, elem_off, out); break;
    default: k_potential_inst<AKB_HEXAHEDRON_8><<<ninst, kThreads, 0, s>>>(m, elem_off, out); break;
    }
  }
  return cudaGetLastError();
}

}  // namespace akb
