// akb_rve.cu -- batched periodic RVE solves (the micro problems of FE^2).
//
// One CTA relaxes one RVE with its whole state on chip: the fluctuation w,
// the velocity and the force of the n^3 periodic nodes (component-major),
// the inverse fictitious mass, the voxel materials and the voxel shape
// gradients live in shared memory (n = 16 in FP32: 170 KB), so an iteration
// reads and writes no global memory. Elements are visited in 8 colours
// (voxel parity in x, y, z; n even keeps them periodic-consistent): voxels
// of one colour share no node, so each thread adds its element's force to
// its 8 corners without atomics and the sum over the 8 colours is in a fixed
// order (deterministic).
//
// Per iteration (leapfrog dynamic relaxation, mass-proportional damping c):
//   f = -sum_e sum_q w_q P(H + grad w) grad N_a     (voxel force, 8 Gauss pts)
//   v = ((1 - c dt / 2) v + dt f / m) / (1 + c dt / 2);  w += dt v
// with m the lumped mass of density lambda + 2 mu (unit P-wave speed in every
// voxel), dt = factor h s_min(F) / c_J (s_min the smallest singular value of
// F, c_J the P-wave speed raised by compression, ln J < 0) and
// c = factor 2 (2 pi / L) min sqrt(mu / (lambda + 2 mu)) (critical damping of
// the lowest shear mode). Strain concentrates in the soft phase beyond what
// F shows, so an attempt whose residual turns non-finite or explodes is
// restarted from its initial state with a 0.6x time step (at most 3 times).
// The homogenised stress is sum w_q P / L^3.
#include <algorithm>
#include <cmath>
#include <memory>
#include <mutex>
#include <vector>

#include "../../include/akb_fe2.h"
#include "akb_fastmath.cuh"

struct akb_rve {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool owns_stream = false;
  int mode = AKB_MODE_FP32_BULK;
  int n = 0, nmat = 0;
  double L = 1.0;
  int max_it = 2000, check = 10;
  double tol = 1e-4, tsf = 0.6, dampf = 0.6;
  double lam[8] = {0}, mu[8] = {0};
  int kind[8] = {0};
  double vf[8] = {0};
  uint8_t* d_vmat = nullptr;
  void* d_inv_mass = nullptr;  // float or double per mode
  size_t smem = 0;
};

namespace akb {
namespace {

constexpr int kRveThreads = 256;  // 2 voxels per thread and colour at n = 16; no register spills
constexpr double kDivergence = 1e4;     // relative residual taken as divergence
constexpr double kRestartFactor = 0.6;  // time-step factor of each restart
constexpr int kMaxRestarts = 3;

struct RveArgs {
  int n, nn, nmat, max_it, check;
  int write_fluct;  // write the relaxed fluctuation back
  double L, h, tol, tsf, dampf;
  double lam[8], mu[8];
  int kind[8];
  const uint8_t* vmat;
  const void* inv_mass;
};

__host__ __device__ inline int corner_x(int a) { return ((a & 3) == 1 || (a & 3) == 2) ? 1 : 0; }
__host__ __device__ inline int corner_y(int a) { return (a >> 1) & 1; }
__host__ __device__ inline int corner_z(int a) { return a >> 2; }

// Shared-memory position of node (or voxel) (x, y, z): grouped by parity
// class (x, y, z mod 2), then (x/2, y/2, z/2) lexicographic. A voxel colour
// reaches each of its corners in one parity class, and its threads' voxels
// are consecutive in that class, so the gathers and scatters of a warp hit
// consecutive words (no bank conflicts).
__device__ inline int pidx(int x, int y, int z, int n) {
  const int hn = n >> 1;
  return ((x & 1) | ((y & 1) << 1) | ((z & 1) << 2)) * (hn * hn * hn) + (x >> 1) +
         hn * ((y >> 1) + hn * (z >> 1));
}

__device__ inline double det3d(const double* m) {
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
         m[2] * (m[3] * m[7] - m[4] * m[6]);
}

// Smallest eigenvalue of a symmetric 3x3 matrix (trigonometric solution of
// the characteristic cubic, O. K. Smith, Comm. ACM 4(4):168, 1961).
__device__ double smallest_eigenvalue(const double* A) {
  const double p1 = A[1] * A[1] + A[2] * A[2] + A[5] * A[5];
  const double q = (A[0] + A[4] + A[8]) / 3.0;
  const double p2 = (A[0] - q) * (A[0] - q) + (A[4] - q) * (A[4] - q) +
                    (A[8] - q) * (A[8] - q) + 2.0 * p1;
  if (p2 <= 0.0) return q;
  const double p = sqrt(p2 / 6.0);
  double Bm[9];
  for (int k = 0; k < 9; ++k) Bm[k] = (A[k] - (k % 4 == 0 ? q : 0.0)) / p;
  double r = det3d(Bm) / 2.0;
  r = fmin(1.0, fmax(-1.0, r));
  const double phi = acos(r) / 3.0;
  return q + 2.0 * p * cos(phi + 2.0 * M_PI / 3.0);
}

template <typename S>
struct RveSmem {
  S *u, *v, *f, *im, *B;
  uint8_t* mat;
  double* red;  // 16 warps x 9
  double* par;  // dt, c, fscale, r
};

template <typename S>
__host__ __device__ inline size_t rve_smem_bytes(int nn) {
  size_t b = 9 * (size_t)nn * sizeof(S) + (size_t)nn * sizeof(S) + 192 * sizeof(S);
  b = (b + (size_t)nn + 15) & ~size_t(15);
  return b + (16 * 9 + 8) * sizeof(double);
}

template <typename S>
__device__ inline RveSmem<S> carve(unsigned char* smem, int nn) {
  RveSmem<S> s;
  S* p = reinterpret_cast<S*>(smem);
  s.u = p;
  s.v = p + 3 * nn;
  s.f = p + 6 * nn;
  s.im = p + 9 * nn;
  s.B = p + 10 * nn;
  s.mat = reinterpret_cast<uint8_t*>(p + 10 * nn + 192);
  size_t off = ((size_t)(10 * nn + 192) * sizeof(S) + (size_t)nn + 15) & ~size_t(15);
  s.red = reinterpret_cast<double*>(smem + off);
  s.par = s.red + 16 * 9;
  return s;
}

// First Piola-Kirchhoff stress of a voxel point (row-major, g = grad u):
// neo-Hookean P = mu (F - F^-T) + lambda ln J F^-T (the reference's F S with
// S = mu (I - C^-1) + lambda ln J C^-1, since F C^-1 = F^-T), written without
// O(1) terms that cancel at small strain: with t = tr g, I2 = (t^2 - tr g^2)/2,
//   J - 1 = t + I2 + det g,  adj(F) = (1 + t + I2) I - (1 + t) g + g^2,
//   F - F^-T = g + (det(g) I + (1 + t) g^T - (g^T)^2) / J,  F^-T = adj(F)^T / J,
//   ln J = log1p(J - 1);
// or small-strain elastic sigma.
template <typename S>
__device__ inline void voxel_stress(const MatParams& mp, const S* g, S* P) {
  const S lam = S(mp.lambda), mu = S(mp.mu);
  if (mp.kind != AKB_MATERIAL_NEOHOOKEAN) {
    const S tr = g[0] + g[4] + g[8];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) P[i * 3 + j] = mu * (g[i * 3 + j] + g[j * 3 + i]) + (i == j ? lam * tr : S(0));
    return;
  }
  S gg[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      gg[i * 3 + j] = g[i * 3] * g[j] + g[i * 3 + 1] * g[3 + j] + g[i * 3 + 2] * g[6 + j];
  const S t = g[0] + g[4] + g[8];
  const S I2 = S(0.5) * (t * t - (gg[0] + gg[4] + gg[8]));
  const S dg = g[0] * (g[4] * g[8] - g[5] * g[7]) - g[1] * (g[3] * g[8] - g[5] * g[6]) +
               g[2] * (g[3] * g[7] - g[4] * g[6]);
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
}

// f -= element forces of every voxel (8 colours); PSUM also adds
// sum_q w_q P (row-major) of this thread's voxels to psum.
//
// The voxel is a cube, so its shape gradients factor along its 12 edges:
// with corners o = ox + 2 oy + 4 oz and s(b) = 2 b - 1,
//   dN_o/dx at Gauss point q = s(ox) (1 + s(oy) c_y)(1 + s(oz) c_z) / (4 h),
// so du/dx at q is sum over the 4 x-edges e = oy + 2 oz of
// W[q][x][e] (u(1, oy, oz) - u(0, oy, oz)) (and likewise along y, z), and the
// corner force sum_q w_q P grad N_o is s(ox) T_x[e_x(o)] + s(oy) T_y[e_y(o)]
// + s(oz) T_z[e_z(o)] with the edge sums T_j[e] = sum_q W[q][j][e] w_q P[:, j].
// Same arithmetic content as the shape-gradient form, half the operations.
template <typename S, bool PSUM>
__device__ void voxel_forces(const RveArgs& R, const RveSmem<S>& s, const S* hH,
                             const MatParams* mats, double* psum) {
  const int n = R.n, nn = R.nn, hn = n >> 1, nc = hn * hn * hn;
  const S wq = S(R.h * R.h * R.h / 8.0);
  for (int color = 0; color < 8; ++color) {
    for (int t = threadIdx.x; t < nc; t += blockDim.x) {
      const int ex = 2 * (t % hn) + (color & 1);
      const int ey = 2 * ((t / hn) % hn) + ((color >> 1) & 1);
      const int ez = 2 * (t / (hn * hn)) + (color >> 2);
      const int x1 = ex + 1 == n ? 0 : ex + 1, y1 = ey + 1 == n ? 0 : ey + 1,
                z1 = ez + 1 == n ? 0 : ez + 1;
      int nd[8];
#pragma unroll
      for (int o = 0; o < 8; ++o) nd[o] = pidx((o & 1) ? x1 : ex, (o & 2) ? y1 : ey, (o & 4) ? z1 : ez, n);
      S D[3][4][3];  // edge differences [direction][edge][component]
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        S uc[8];
#pragma unroll
        for (int o = 0; o < 8; ++o) uc[o] = s.u[i * nn + nd[o]];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          // total displacement along the edge: fluctuation + h H e_j (the
          // weights of a direction sum to 1/h, so sum_e W D = H + grad w)
          const int b0 = e & 1, b1 = e >> 1;
          D[0][e][i] = (uc[1 + 2 * b0 + 4 * b1] - uc[2 * b0 + 4 * b1]) + hH[i * 3 + 0];
          D[1][e][i] = (uc[b0 + 2 + 4 * b1] - uc[b0 + 4 * b1]) + hH[i * 3 + 1];
          D[2][e][i] = (uc[b0 + 2 * b1 + 4] - uc[b0 + 2 * b1]) + hH[i * 3 + 2];
        }
      }
      const MatParams& mp = mats[s.mat[pidx(ex, ey, ez, n)]];
      S T[3][4][3];
#pragma unroll
      for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e)
#pragma unroll
          for (int i = 0; i < 3; ++i) T[j][e][i] = 0;
#pragma unroll 1
      for (int q = 0; q < 8; ++q) {
        const S* Wq = s.B + q * 12;  // [direction][edge]
        S g[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            S c = Wq[j * 4] * D[j][0][i];
#pragma unroll
            for (int e = 1; e < 4; ++e) c += Wq[j * 4 + e] * D[j][e][i];
            g[i * 3 + j] = c;
          }
        S P[9];
        voxel_stress<S>(mp, g, P);
#pragma unroll
        for (int k = 0; k < 9; ++k) P[k] *= wq;
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
          for (int e = 0; e < 4; ++e)
#pragma unroll
            for (int i = 0; i < 3; ++i) T[j][e][i] += Wq[j * 4 + e] * P[i * 3 + j];
        if (PSUM)
#pragma unroll
          for (int k = 0; k < 9; ++k) psum[k] += double(P[k]);
      }
#pragma unroll
      for (int o = 0; o < 8; ++o) {
        const int ox = o & 1, oy = (o >> 1) & 1, oz = o >> 2;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const S tx = T[0][oy + 2 * oz][i], ty = T[1][ox + 2 * oz][i], tz = T[2][ox + 2 * oy][i];
          const S fo = (ox ? tx : -tx) + (oy ? ty : -ty) + (oz ? tz : -tz);
          s.f[i * nn + nd[o]] -= fo;
        }
      }
    }
    __syncthreads();
  }
}

__device__ inline double warp_max(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
  return x;
}
__device__ inline double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// One RVE instance, by the whole CTA: relaxation from the instance's
// fluctuation (or zero), homogenised stress, state written back.
template <typename S>
__device__ __forceinline__ void rve_instance(const RveArgs& R, int64_t inst,
                                             const double* __restrict__ grad_u, S* fluct,
                                             double* __restrict__ stress, int32_t* iterations,
                                             double* residual, double* internal_force) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int nn = R.nn, tid = threadIdx.x, bs = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarps = bs >> 5;
  RveSmem<S> s = carve<S>(smem, nn);
  __shared__ MatParams mats[8];

  // the constant tables
  const S* im_g = static_cast<const S*>(R.inv_mass);
  for (int k = tid; k < nn; k += bs) {
    const int q = pidx(k % R.n, (k / R.n) % R.n, k / (R.n * R.n), R.n);
    s.im[q] = im_g[k];
    s.mat[q] = R.vmat[k];
  }
  if (tid < 96) {  // edge weights W[q][direction][edge] (see voxel_forces)
    const int q = tid / 12, j = (tid / 4) % 3, e = tid % 4;
    const double gp = 1.0 / sqrt(3.0);
    const double c[3] = {(q & 1) ? gp : -gp, (q & 2) ? gp : -gp, (q & 4) ? gp : -gp};
    const int d1 = j == 0 ? 1 : 0, d2 = j == 2 ? 1 : 2;  // the two other directions
    const double s1 = 2.0 * (e & 1) - 1.0, s2 = 2.0 * (e >> 1) - 1.0;
    s.B[tid] = S((1.0 + s1 * c[d1]) * (1.0 + s2 * c[d2]) / (4.0 * R.h));
  }
  if (tid < R.nmat) {
    MatParams mp{};
    mp.kind = R.kind[tid];
    mp.finite = R.kind[tid] == AKB_MATERIAL_NEOHOOKEAN;
    mp.lambda = R.lam[tid];
    mp.mu = R.mu[tid];
    mp.E = 1.0;
    mats[tid] = mp;
  }
  __shared__ S hH[9];  // h H, row-major
  double Hd[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) Hd[i * 3 + j] = grad_u[inst * 9 + i + 3 * j];
  if (tid < 9) hH[tid] = S(R.h * Hd[tid]);
  if (tid == 0) {
    // time-step scale, damping and residual scale of this instance
    double F[9], C[9];
    for (int k = 0; k < 9; ++k) F[k] = Hd[k] + (k % 4 == 0 ? 1.0 : 0.0);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        double c = 0;
        for (int k = 0; k < 3; ++k) c += F[k * 3 + i] * F[k * 3 + j];
        C[i * 3 + j] = c;
      }
    const double J = det3d(F);
    const double smin = sqrt(fmax(smallest_eigenvalue(C), 0.0));
    const double stiff = J > 0 ? fmax(0.0, -log(J)) : 0.0;
    double c2 = 0.0, cs = 1e300, mumax = 0.0, hmax = 0.0;
    for (int m = 0; m < R.nmat; ++m) {
      const double m2 = R.lam[m] + 2.0 * R.mu[m];
      const double t = R.kind[m] == AKB_MATERIAL_NEOHOOKEAN ? (m2 + 2.0 * R.lam[m] * stiff) / m2 : 1.0;
      c2 = fmax(c2, t);
      cs = fmin(cs, sqrt(R.mu[m] / m2));
      mumax = fmax(mumax, R.mu[m]);
    }
    for (int k = 0; k < 9; ++k) hmax = fmax(hmax, fabs(Hd[k]));
    s.par[0] = R.h * smin / sqrt(c2);
    s.par[1] = R.dampf * 2.0 * (2.0 * M_PI / R.L) * cs;
    s.par[2] = R.h * R.h * mumax * fmax(hmax, 1e-6);
  }
  __syncthreads();
  const double fscale = s.par[2];

  // Relaxation; an attempt whose residual turns non-finite or exceeds
  // kDivergence restarts from the initial state with a 0.6x time step.
  int total = 0, k = 0;
  double r = 0.0, tsf = R.tsf;
  for (int attempt = 0;; ++attempt, tsf *= kRestartFactor) {
    for (int idx = tid; idx < 3 * nn; idx += bs) {
      const int node = idx / 3, i = idx - 3 * node;
      const int q = pidx(node % R.n, (node / R.n) % R.n, node / (R.n * R.n), R.n);
      s.u[i * nn + q] = fluct ? fluct[inst * 3 * nn + idx] : S(0);
      s.v[idx] = 0;
    }
    const double dtd = tsf * s.par[0];
    const S dt = S(dtd);
    const S a1 = S(1.0 - 0.5 * s.par[1] * dtd), a2 = S(1.0 + 0.5 * s.par[1] * dtd);
    __syncthreads();
    bool diverged = false;
    for (k = 0;; ++k) {
      for (int idx = tid; idx < 3 * nn; idx += bs) s.f[idx] = 0;
      __syncthreads();
      voxel_forces<S, false>(R, s, hH, mats, nullptr);
      const bool last = k >= R.max_it;
      if (last || (R.check > 0 && k % R.check == 0)) {
        double lm = 0.0;
        for (int idx = tid; idx < 3 * nn; idx += bs) {
          const double x = double(s.f[idx]);
          lm = isfinite(x) ? fmax(lm, fabs(x)) : INFINITY;
        }
        lm = warp_max(lm);
        if (lane == 0) s.red[warp] = lm;
        __syncthreads();
        double m = 0.0;
        for (int w = 0; w < nwarps; ++w) m = fmax(m, s.red[w]);
        r = isfinite(m) ? m / fscale : INFINITY;
        __syncthreads();  // s.red is reused
        diverged = !(r <= kDivergence);
        if (last || diverged || (R.tol >= 0 && r <= R.tol)) break;
      }
      for (int idx = tid; idx < 3 * nn; idx += bs) {
        const int node = idx % nn;
        const S vv = (a1 * s.v[idx] + dt * s.f[idx] * s.im[node]) / a2;
        s.v[idx] = vv;
        s.u[idx] += dt * vv;
      }
      __syncthreads();
    }
    total += k;
    if (!diverged || attempt >= kMaxRestarts) break;
    __syncthreads();
  }

  // homogenised stress (and force) of the final state
  for (int idx = tid; idx < 3 * nn; idx += bs) s.f[idx] = 0;
  __syncthreads();
  double ps[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) ps[q] = 0.0;
  voxel_forces<S, true>(R, s, hH, mats, ps);
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    const double x = warp_sum(ps[q]);
    if (lane == 0) s.red[warp * 9 + q] = x;
  }
  __syncthreads();
  if (tid < 9) {
    double t = 0.0;
    for (int w = 0; w < nwarps; ++w) t += s.red[w * 9 + tid];
    const int i = tid / 3, j = tid % 3;
    stress[inst * 9 + i + 3 * j] = t / (R.L * R.L * R.L);
  }
  if (tid == 0) {
    if (iterations) iterations[inst] = total;
    if (residual) residual[inst] = r;
  }
  for (int idx = tid; idx < 3 * nn; idx += bs) {
    const int node = idx / 3, i = idx - 3 * node;
    const int q = pidx(node % R.n, (node / R.n) % R.n, node / (R.n * R.n), R.n);
    if (fluct && R.write_fluct) fluct[inst * 3 * nn + idx] = s.u[i * nn + q];
    if (internal_force) internal_force[inst * 3 * nn + idx] = double(s.f[i * nn + q]);
  }
}

template <typename S>
__global__ void __launch_bounds__(kRveThreads, 1)
    k_rve(RveArgs R, int64_t nb, const double* __restrict__ grad_u, S* fluct,
          double* __restrict__ stress, int32_t* iterations, double* residual,
          double* internal_force) {
  const int64_t inst = blockIdx.x;
  if (inst >= nb) return;
  rve_instance<S>(R, inst, grad_u, fluct, stress, iterations, residual, internal_force);
}

// The instances index[0 .. min(*count, capacity)) of arrays over all points,
// the count read on the device (written by an earlier kernel on the same
// stream): CTAs stride over the list, so a short or empty list costs one
// small launch and no host round trip.
template <typename S>
__global__ void __launch_bounds__(kRveThreads, 1)
    k_rve_indexed(RveArgs R, int64_t capacity, const int32_t* __restrict__ index,
                  const int32_t* __restrict__ count, const double* __restrict__ grad_u, S* fluct,
                  double* __restrict__ stress, int32_t* iterations, double* residual) {
  const int64_t n = min((int64_t)*count, capacity);
  for (int64_t b = blockIdx.x; b < n; b += gridDim.x) {
    const int64_t inst = index[b];
    if (inst < 0 || inst >= capacity) continue;  // uniform over the CTA
    rve_instance<S>(R, inst, grad_u, fluct, stress, iterations, residual, nullptr);
    __syncthreads();  // shared state is reused by the next instance
  }
}

std::mutex g_rve_attr_mutex;

template <typename S>
cudaError_t raise_limit(size_t bytes) {
  std::lock_guard<std::mutex> lock(g_rve_attr_mutex);
  cudaFuncAttributes attr;
  cudaError_t e = cudaFuncGetAttributes(&attr, k_rve<S>);
  if (e != cudaSuccess) return e;
  if ((size_t)attr.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(k_rve<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_rve_indexed<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)bytes);
}

RveArgs args_of(const akb_rve* r, int max_it) {
  RveArgs a{};
  a.n = r->n;
  a.nn = r->n * r->n * r->n;
  a.nmat = r->nmat;
  a.max_it = max_it;
  a.write_fluct = max_it > 0;
  a.check = r->check;
  a.L = r->L;
  a.h = r->L / r->n;
  a.tol = r->tol;
  a.tsf = r->tsf;
  a.dampf = r->dampf;
  for (int m = 0; m < 8; ++m) {
    a.lam[m] = r->lam[m];
    a.mu[m] = r->mu[m];
    a.kind[m] = r->kind[m];
  }
  a.vmat = r->d_vmat;
  a.inv_mass = r->d_inv_mass;
  return a;
}

akb_status launch(akb_rve* r, int max_it, int64_t nb, const double* grad_u, void* fluct,
                  double* stress, int32_t* iterations, double* residual, double* force,
                  void* stream) {
  if (!r) return fail(AKB_ERR_INVALID_ARGUMENT, "null RVE");
  if (nb < 0 || (nb > 0 && (!grad_u || !stress)))
    return fail(AKB_ERR_INVALID_ARGUMENT, "grad_u and stress are required");
  if (nb > INT32_MAX) return fail(AKB_ERR_UNSUPPORTED, "more than 2^31 RVEs in one call");
  if (nb == 0) return AKB_OK;
  AKB_CUDA_TRY(cudaSetDevice(r->device));
  cudaStream_t s = stream ? (cudaStream_t)stream : r->stream;
  const RveArgs a = args_of(r, max_it);
  if (r->mode == AKB_MODE_FP64)
    k_rve<double><<<(unsigned)nb, kRveThreads, r->smem, s>>>(
        a, nb, grad_u, static_cast<double*>(fluct), stress, iterations, residual, force);
  else
    k_rve<float><<<(unsigned)nb, kRveThreads, r->smem, s>>>(
        a, nb, grad_u, static_cast<float*>(fluct), stress, iterations, residual, force);
  AKB_CUDA_TRY(cudaGetLastError());
  return AKB_OK;
}

}  // namespace
}  // namespace akb

using namespace akb;

extern "C" {

akb_status akb_rve_create(const akb_rve_desc* desc, const akb_rve_options* options,
                          akb_rve** out) {
  if (!out) return fail(AKB_ERR_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  if (!desc || !desc->voxel_material || !desc->materials)
    return fail(AKB_ERR_INVALID_ARGUMENT, "RVE description, voxels and materials are required");
  const int n = desc->cells;
  if (n < 2 || n > 64 || (n & 1)) return fail(AKB_ERR_INVALID_ARGUMENT, "cells must be even, 2..64");
  if (desc->nb_materials < 1 || desc->nb_materials > 8)
    return fail(AKB_ERR_INVALID_ARGUMENT, "1..8 materials");
  if (!(desc->length > 0)) return fail(AKB_ERR_INVALID_ARGUMENT, "length must be positive");
  akb_rve_options opt{AKB_MODE_FP32_BULK, 0, nullptr, 0, 0, 0.0, 0.0, 0.0};
  if (options) opt = *options;
  if (opt.precision_mode != AKB_MODE_FP32_BULK && opt.precision_mode != AKB_MODE_FP64)
    return fail(AKB_ERR_UNSUPPORTED, "RVE precision: AKB_MODE_FP32_BULK or AKB_MODE_FP64");
  auto r = std::make_unique<akb_rve>();
  r->mode = opt.precision_mode;
  r->n = n;
  r->nmat = desc->nb_materials;
  r->L = desc->length;
  r->max_it = opt.max_iterations > 0 ? opt.max_iterations : 2000;
  r->check = opt.check_interval > 0 ? opt.check_interval : 10;
  r->tol = opt.tolerance != 0.0 ? opt.tolerance : 1e-4;
  r->tsf = opt.time_step_factor > 0 ? opt.time_step_factor : 0.6;
  r->dampf = opt.damping_factor > 0 ? opt.damping_factor : 0.6;
  for (int m = 0; m < r->nmat; ++m) {
    const akb_material_desc& md = desc->materials[m];
    if (md.kind != AKB_MATERIAL_ELASTIC && md.kind != AKB_MATERIAL_NEOHOOKEAN)
      return fail(AKB_ERR_UNSUPPORTED, "RVE materials: elastic or neo-Hookean");
    if (!(md.E > 0) || !(md.nu > -1.0 && md.nu < 0.5))
      return fail(AKB_ERR_INVALID_ARGUMENT, "RVE material needs E > 0, -1 < nu < 0.5");
    r->kind[m] = md.kind;
    r->lam[m] = md.nu * md.E / ((1 + md.nu) * (1 - 2 * md.nu));
    r->mu[m] = md.E / (2 * (1 + md.nu));
  }
  const int64_t nn = (int64_t)n * n * n;
  for (int64_t e = 0; e < nn; ++e)
    if (desc->voxel_material[e] >= r->nmat)
      return fail(AKB_ERR_INVALID_ARGUMENT, "voxel material index out of range");
  r->smem = r->mode == AKB_MODE_FP64 ? rve_smem_bytes<double>((int)nn) : rve_smem_bytes<float>((int)nn);
  if (r->smem > 227 * 1024)
    return fail(AKB_ERR_UNSUPPORTED, "RVE does not fit in one SM's shared memory (use FP32 or fewer cells)");
  // lumped fictitious mass: density lambda + 2 mu, h^3/8 per voxel corner
  const double h = r->L / n;
  std::vector<double> mass(nn, 0.0);
  for (int ez = 0; ez < n; ++ez)
    for (int ey = 0; ey < n; ++ey)
      for (int ex = 0; ex < n; ++ex) {
        const int m = desc->voxel_material[ex + n * (ey + n * ez)];
        r->vf[m] += 1.0 / (double)nn;
        for (int a = 0; a < 8; ++a) {
          const int x = (ex + corner_x(a)) % n, y = (ey + corner_y(a)) % n, z = (ez + corner_z(a)) % n;
          mass[x + n * (y + n * z)] += (r->lam[m] + 2.0 * r->mu[m]) * h * h * h / 8.0;
        }
      }
  r->device = opt.device;
  AKB_CUDA_TRY(cudaSetDevice(r->device));
  if (opt.stream) {
    r->stream = (cudaStream_t)opt.stream;
  } else {
    AKB_CUDA_TRY(cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking));
    r->owns_stream = true;
  }
  AKB_CUDA_TRY(cudaMalloc((void**)&r->d_vmat, nn));
  AKB_CUDA_TRY(cudaMemcpy(r->d_vmat, desc->voxel_material, nn, cudaMemcpyHostToDevice));
  if (r->mode == AKB_MODE_FP64) {
    std::vector<double> im(nn);
    for (int64_t k = 0; k < nn; ++k) im[k] = 1.0 / mass[k];
    AKB_CUDA_TRY(cudaMalloc(&r->d_inv_mass, nn * sizeof(double)));
    AKB_CUDA_TRY(cudaMemcpy(r->d_inv_mass, im.data(), nn * sizeof(double), cudaMemcpyHostToDevice));
    AKB_CUDA_TRY(raise_limit<double>(r->smem));
  } else {
    std::vector<float> im(nn);
    for (int64_t k = 0; k < nn; ++k) im[k] = (float)(1.0 / mass[k]);
    AKB_CUDA_TRY(cudaMalloc(&r->d_inv_mass, nn * sizeof(float)));
    AKB_CUDA_TRY(cudaMemcpy(r->d_inv_mass, im.data(), nn * sizeof(float), cudaMemcpyHostToDevice));
    AKB_CUDA_TRY(raise_limit<float>(r->smem));
  }
  *out = r.release();
  return AKB_OK;
}

akb_status akb_rve_destroy(akb_rve* r) {
  if (!r) return AKB_OK;
  cudaSetDevice(r->device);
  cudaStreamSynchronize(r->stream);
  cudaFree(r->d_vmat);
  cudaFree(r->d_inv_mass);
  if (r->owns_stream) cudaStreamDestroy(r->stream);
  delete r;
  return AKB_OK;
}

akb_status akb_rve_get_info(const akb_rve* r, akb_rve_info* info) {
  if (!r || !info) return fail(AKB_ERR_INVALID_ARGUMENT, "null argument");
  info->cells = r->n;
  info->precision_mode = r->mode;
  info->nb_nodes = (int64_t)r->n * r->n * r->n;
  for (int m = 0; m < 8; ++m) info->volume_fraction[m] = r->vf[m];
  info->shared_bytes = (int64_t)r->smem;
  return AKB_OK;
}

akb_status akb_rve_solve(akb_rve* r, int64_t nb, const double* grad_u, void* fluctuation,
                         double* stress, int32_t* iterations, double* residual, void* stream) {
  if (!r) return fail(AKB_ERR_INVALID_ARGUMENT, "null RVE");
  return launch(r, r->max_it, nb, grad_u, fluctuation, stress, iterations, residual, nullptr,
                stream);
}

akb_status akb_rve_solve_indexed(akb_rve* r, int64_t capacity, const int32_t* index,
                                 const int32_t* count, const double* grad_u, void* fluctuation,
                                 double* stress, int32_t* iterations, double* residual,
                                 void* stream) {
  if (!r) return fail(AKB_ERR_INVALID_ARGUMENT, "null RVE");
  if (capacity < 0 || (capacity > 0 && (!index || !count || !grad_u || !stress)))
    return fail(AKB_ERR_INVALID_ARGUMENT, "index, count, grad_u and stress are required");
  if (capacity > INT32_MAX) return fail(AKB_ERR_UNSUPPORTED, "more than 2^31 RVEs in one call");
  if (capacity == 0) return AKB_OK;
  AKB_CUDA_TRY(cudaSetDevice(r->device));
  cudaStream_t s = stream ? (cudaStream_t)stream : r->stream;
  int sms = 0;
  AKB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, r->device));
  const unsigned grid = (unsigned)std::min<int64_t>(capacity, std::max(sms, 1));
  const RveArgs a = args_of(r, r->max_it);
  if (r->mode == AKB_MODE_FP64)
    k_rve_indexed<double><<<grid, kRveThreads, r->smem, s>>>(
        a, capacity, index, count, grad_u, static_cast<double*>(fluctuation), stress, iterations,
        residual);
  else
    k_rve_indexed<float><<<grid, kRveThreads, r->smem, s>>>(
        a, capacity, index, count, grad_u, static_cast<float*>(fluctuation), stress, iterations,
        residual);
  AKB_CUDA_TRY(cudaGetLastError());
  return AKB_OK;
}

akb_status akb_rve_stress(akb_rve* r, int64_t nb, const double* grad_u, const void* fluctuation,
                          double* stress, double* internal_force, void* stream) {
  if (!r) return fail(AKB_ERR_INVALID_ARGUMENT, "null RVE");
  if (!fluctuation) return fail(AKB_ERR_INVALID_ARGUMENT, "fluctuation is required");
  // zero updates: the state is only read
  return launch(r, 0, nb, grad_u, const_cast<void*>(fluctuation), stress, nullptr, nullptr,
                internal_force, stream);
}

}  // extern "C"
