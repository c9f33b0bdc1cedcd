// akb_patch.cu -- the fused explicit step (AKB_MODE_FP64, AKB_MODE_FP32_BULK).
//
// k_patch_step: one CTA per patch.
//   1. stage the patch: its local connectivity, sorted slots and runs by TMA
//      bulk copies completing on an mbarrier, while the threads gather the
//      nodes' X, u, v, a and blocked flags and apply the predictor
//      u+ = u + dt v + dt^2/2 a, v* = v + dt a on free DOFs
//      (NewmarkBeta::predictor, newmark-beta.cc:60-89);
//   2. element forces in chunks of blockDim elements from shared memory
//      (akb_fastmath.cuh), written to the chunk's corners sorted by node;
//      one thread per node run adds the run (ascending local element order)
//      to the node accumulators (the -1 scatter of dof_manager.cc:83-137,
//      without atomics);
//   3. nodes of this patch only: residual, lumped solve and corrector
//      (non_linear_solver_lumped.cc:85-98, newmark-beta.cc:176-210) on u+
//      kept in shared memory and v, a re-read, written back; nodes shared
//      with other patches: FP64 partial force to its slot.
// The wait on the staging copies is bounded: past it the CTA flags the
// error (P.err, read by the host on its next synchronisation), waits again
// (bounded) for its copies and skips the patch.
// k_shared_nodes: one thread per shared node adds its partials in patch order
// and applies the same predictor/corrector arithmetic.
#include <mutex>

#include "akb_fastmath.cuh"
#include "akb_patch.cuh"

namespace akb {
namespace {

constexpr int kThreads = 256;

struct SmemLayout {
  size_t xs, us, fs, contrib, lcs, slots, segs, segp, flags, mbar, total;
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

constexpr int kMaxChunks = 33;  // chunks of a patch (8192 elements) + 1

// Shared-memory layout for patch caps L (nodes), E (elements), R (runs).
// Node arrays are component-major ([i][j]); the chunk's element vectors are
// stored at their sorted slots, component-major ([i][slot]).
__host__ __device__ inline SmemLayout layout(int L, int E, int R, int d, int n, int sbytes,
                                             int threads) {
  SmemLayout s;
  const size_t nd = (size_t)L * d * sizeof(double);
  s.xs = 0;
  s.us = align16(s.xs + nd);
  s.fs = align16(s.us + nd);
  s.contrib = align16(s.fs + nd);
  s.lcs = align16(s.contrib + (size_t)threads * n * d * sbytes);
  s.slots = align16(s.lcs + (size_t)E * n * sizeof(uint16_t));
  s.segs = align16(s.slots + (size_t)E * n * sizeof(uint16_t));
  s.segp = align16(s.segs + (size_t)R * sizeof(uint32_t));
  s.flags = align16(s.segp + (size_t)kMaxChunks * sizeof(int32_t));
  s.mbar = align16(s.flags + (size_t)L * d);
  s.total = s.mbar + 16;
  return s;
}

// The n local indices of element el (uint16, n per element): one vector load
// when n * 2 bytes is a power of two (2, 4 and 8 corners), else n loads.
template <int n>
__device__ inline void load_corners(const uint16_t* base, int el, int* out) {
  if (n == 2 || n == 4 || n == 8) {
    uint32_t w[4];
    if (n == 2) {
      w[0] = reinterpret_cast<const uint32_t*>(base)[el];
    } else if (n == 4) {
      const uint2 q = reinterpret_cast<const uint2*>(base)[el];
      w[0] = q.x;
      w[1] = q.y;
    } else {
      const uint4 q = reinterpret_cast<const uint4*>(base)[el];
      w[0] = q.x;
      w[1] = q.y;
      w[2] = q.z;
      w[3] = q.w;
    }
#pragma unroll
    for (int a = 0; a < n; ++a) out[a] = (int)((w[a >> 1] >> (16 * (a & 1))) & 0xffffu);
  } else {
#pragma unroll
    for (int a = 0; a < n; ++a) out[a] = base[el * n + a];
  }
}

// CTAs per SM each instantiation is built for (register budget).
template <int T, typename S> struct PatchOccupancy { static constexpr int value = 3; };
template <> struct PatchOccupancy<AKB_HEXAHEDRON_8, float> { static constexpr int value = 2; };
template <> struct PatchOccupancy<AKB_HEXAHEDRON_8, double> { static constexpr int value = 1; };

// (node, component) items handled per thread per round of the staging and
// finishing loops: their global loads are issued together.
constexpr int kBatch = 4;
constexpr uint32_t kWaitLimit = 1u << 22;

__device__ inline uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ inline void bulk_copy(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}
__device__ inline bool mbar_wait(uint32_t a, uint32_t parity) {
  for (uint32_t it = 0; it < kWaitLimit; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// One patch p, by the whole CTA.
template <int T, typename S, bool FEXT>
__device__ __forceinline__ void patch_body(const DevModel& m, const DevPatches& P, double dt0,
                                           int p, unsigned char* smem, uint32_t parity) {
  constexpr int d = ET<T>::dim, n = ET<T>::nnpe;
  constexpr int CH = kChunk * n;  // sorted slots of one chunk
  static_assert(kChunk == kThreads, "one element per thread per chunk");
  const double dt = P.inst_dt ? P.inst_dt[P.patch_inst[p]] : dt0;
  const int nb = P.node_ptr[p];
  const int L = P.node_ptr[p + 1] - nb;
  const int eb = P.elem_ptr[p];
  const int ne = P.elem_ptr[p + 1] - eb;
  const int nint = P.ninterior[p];
  const int nchunks = (ne + kChunk - 1) / kChunk;
  const int LM = P.max_nodes;  // row stride of the component-major arrays
  const SmemLayout lay = layout(P.max_nodes, P.max_elems, P.max_segs, d, n, sizeof(S), kThreads);
  double* xs = reinterpret_cast<double*>(smem + lay.xs);
  double* us = reinterpret_cast<double*>(smem + lay.us);
  double* fs = reinterpret_cast<double*>(smem + lay.fs);
  S* contrib = reinterpret_cast<S*>(smem + lay.contrib);
  uint16_t* lcs = reinterpret_cast<uint16_t*>(smem + lay.lcs);
  uint16_t* slots = reinterpret_cast<uint16_t*>(smem + lay.slots);
  uint32_t* segs = reinterpret_cast<uint32_t*>(smem + lay.segs);
  int32_t* segp = reinterpret_cast<int32_t*>(smem + lay.segp);
  uint8_t* flags = smem + lay.flags;
  const int tid = threadIdx.x;
  const int items = L * d;

  // 1. stage the patch: local connectivity, sorted slots and runs by TMA
  //    bulk copies (one thread, completing on an mbarrier) while the CTA
  //    gathers per (node, component) X, predicted u, blocked flag
  const uint32_t mb = saddr(smem + lay.mbar);
  {
    const int32_t* gp = P.seg_ptr + P.chunk_base[p];
    const int s0 = gp[0];
    if (tid <= nchunks) segp[tid] = gp[tid] - s0;
    if (tid == 0) {
      const uint32_t blc = ((uint32_t)(ne * n * 2) + 15u) & ~15u;
      const uint32_t bsg = ((uint32_t)((gp[nchunks] - s0) * 4) + 15u) & ~15u;
      asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(mb),
                   "r"(2 * blc + bsg)
                   : "memory");
      bulk_copy(saddr(lcs), P.lconn_pad + P.lc_off[p], blc, mb);
      bulk_copy(saddr(slots), P.cslot_pad + P.lc_off[p], blc, mb);
      if (bsg) bulk_copy(saddr(segs), P.segs_pad + P.sg_off[p], bsg, mb);
    }
  }
  for (int base = 0; base < items; base += kThreads * kBatch) {
    int64_t idx[kBatch];
#pragma unroll
    for (int b = 0; b < kBatch; ++b) {
      const int k = base + b * kThreads + tid;
      const int j = k / d, i = k - j * d;
      idx[b] = k < items ? (int64_t)P.lnodes[nb + j] * d + i : -1;
    }
    double x[kBatch], u[kBatch], v[kBatch], a[kBatch];
    uint8_t bl[kBatch];
#pragma unroll
    for (int b = 0; b < kBatch; ++b)
      if (idx[b] >= 0) {
        x[b] = __ldg(&m.X[idx[b]]);
        u[b] = m.u[idx[b]];
        v[b] = m.v[idx[b]];
        a[b] = m.a[idx[b]];
        bl[b] = m.blocked[idx[b]];
      }
#pragma unroll
    for (int b = 0; b < kBatch; ++b) {
      const int k = base + b * kThreads + tid;
      if (k >= items) continue;
      const int j = k / d, i = k - j * d;
      double uu = u[b], vv = v[b];
      if (!bl[b]) fast::predict(dt, uu, vv, a[b]);
      xs[i * LM + j] = x[b];
      us[i * LM + j] = uu;
      fs[i * LM + j] = 0.0;
      flags[k] = bl[b];
    }
  }
  __syncthreads();
  if (!mbar_wait(mb, parity)) {  // bounded: flag, drain, skip the patch
    if (tid == 0) atomicExch(P.err, 1);
    mbar_wait(mb, parity);
    return;
  }

  // 2. element forces chunk by chunk: each element writes its corner vectors
  //    to the corners' sorted slots, then one thread per node run adds the
  //    run (ascending element order) to that node
  for (int c0 = 0, chunk = 0; c0 < ne; c0 += kChunk, ++chunk) {
    const int el = c0 + tid;
    if (el < ne) {
      int lc[n], sl[n];
      load_corners<n>(lcs, el, lc);
      load_corners<n>(slots, el, sl);
      const MatParams& mp = (P.emat ? m.mat_table[P.emat[(size_t)eb + el]] : m.mats[0]);
      S dX[3 * 8], du[3 * 8];
#pragma unroll
      for (int i = 0; i < d; ++i) {
        dX[i] = 0;
        du[i] = 0;
        const double x0 = xs[i * LM + lc[0]], u0 = us[i * LM + lc[0]];
#pragma unroll
        for (int a = 1; a < n; ++a) {
          dX[a * d + i] = S(xs[i * LM + lc[a]] - x0);
          du[a * d + i] = S(us[i * LM + lc[a]] - u0);
        }
      }
      S fe[3 * 8];
      fast::element_force<T, S>(mp, dX, du, fe);
#pragma unroll
      for (int a = 0; a < n; ++a)
#pragma unroll
        for (int i = 0; i < d; ++i) contrib[i * CH + sl[a]] = fe[a * d + i];
    }
    __syncthreads();
    const int sb = segp[chunk], nrun = segp[chunk + 1] - sb;
    for (int r = tid; r < nrun; r += kThreads) {  // one thread per run, all components
      const uint32_t w = segs[sb + r];
      const int j = (int)(w >> 16), end = (int)(w & 0xffff);
      const int beg = r == 0 ? 0 : (int)(segs[sb + r - 1] & 0xffff);
      double f[3] = {0.0, 0.0, 0.0};
      for (int k = beg; k < end; ++k)
#pragma unroll
        for (int i = 0; i < d; ++i) f[i] += double(contrib[i * CH + k]);
#pragma unroll
      for (int i = 0; i < d; ++i) fs[i * LM + j] -= f[i];
    }
    __syncthreads();
  }

  // 3. finish the nodes of this patch (state re-read, predictor recomputed
  //    bit for bit), hand out the shared ones
  for (int base = 0; base < items; base += kThreads * kBatch) {
    int64_t idx[kBatch];
    double v[kBatch], a[kBatch], im[kBatch], fx[kBatch];
#pragma unroll
    for (int b = 0; b < kBatch; ++b) {
      const int k = base + b * kThreads + tid;
      const int j = k / d, i = k - j * d;
      idx[b] = -1;
      if (k < items && j < nint && !flags[k]) {
        const int64_t g = P.lnodes[nb + j];
        idx[b] = g * d + i;
        im[b] = m.inv_mass[g];
      }
    }
#pragma unroll
    for (int b = 0; b < kBatch; ++b)
      if (idx[b] >= 0) {
        v[b] = m.v[idx[b]];
        a[b] = m.a[idx[b]];
        fx[b] = FEXT ? m.fext[idx[b]] : 0.0;
      }
#pragma unroll
    for (int b = 0; b < kBatch; ++b) {
      const int k = base + b * kThreads + tid;
      if (k >= items) continue;
      const int j = k / d, i = k - j * d;
      const double f = fs[i * LM + j];
      if (j >= nint) {
        P.partial[(int64_t)P.slot[nb + j] * d + i] = f;
      } else if (idx[b] >= 0) {  // blocked DOFs keep u, v, a
        // u+ from the staging, v* recomputed bit for bit
        double uu = us[i * LM + j], vv = __dadd_rn(v[b], __dmul_rn(dt, a[b])), aa = a[b];
        fast::correct(dt, FEXT ? f + fx[b] : f, im[b], uu, vv, aa);
        m.u[idx[b]] = uu;
        m.v[idx[b]] = vv;
        m.a[idx[b]] = aa;
      }
    }
  }
}

// One CTA per patch, or (PERSIST) a grid smaller than the patch count whose
// CTAs stride over the patches. The loop is a separate instantiation: kept
// out of the one-patch kernel it would raise that kernel's register pressure.
template <int T, typename S, bool FEXT, bool PERSIST>
__global__ void __launch_bounds__(kThreads, (PatchOccupancy<T, S>::value))
    k_patch_step(DevModel m, DevPatches P, double dt0) {
  extern __shared__ __align__(16) unsigned char smem[];
  {
    const SmemLayout lay = layout(P.max_nodes, P.max_elems, P.max_segs, ET<T>::dim, ET<T>::nnpe,
                                  sizeof(S), kThreads);
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(smem + lay.mbar)) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
  }
  if constexpr (PERSIST) {
    uint32_t parity = 0;
    for (int p = blockIdx.x; p < P.npatch; p += gridDim.x, parity ^= 1) {
      if (p != (int)blockIdx.x) __syncthreads();  // shared memory of the previous patch is free
      patch_body<T, S, FEXT>(m, P, dt0, p, smem, parity);
    }
  } else {
    patch_body<T, S, FEXT>(m, P, dt0, blockIdx.x, smem, 0);
  }
}

template <int D, bool FEXT>
__global__ void k_shared_nodes(DevModel m, DevPatches P, double dt0) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= P.nshared) return;
  const int64_t g = P.snodes[s];
  const double dt = P.inst_dt ? P.inst_dt[P.snode_inst[s]] : dt0;
  const int k0 = P.sptr[s], k1 = P.sptr[s + 1];
  double f[3] = {0, 0, 0};
  for (int k = k0; k < k1; ++k)
#pragma unroll
    for (int i = 0; i < D; ++i) f[i] += P.partial[(int64_t)k * D + i];
  const double im = m.inv_mass[g];
#pragma unroll
  for (int i = 0; i < D; ++i) {
    const int64_t k = g * D + i;
    if (m.blocked[k]) continue;
    double u = m.u[k], v = m.v[k], a = m.a[k];
    fast::predict(dt, u, v, a);
    double r = f[i];
    if (FEXT) r += m.fext[k];
    fast::correct(dt, r, im, u, v, a);
    m.u[k] = u;
    m.v[k] = v;
    m.a[k] = a;
  }
}

// grid of the patch kernel: one CTA per patch, or a persistent grid of
// P.grid CTAs that stride over the patches
inline int grid_of(const DevPatches& p) {
  return (p.grid > 0 && p.grid < p.npatch) ? p.grid : p.npatch;
}

template <int T, typename S>
cudaError_t launch_patch(const DevModel& m, const DevPatches& p, double dt, bool fext,
                         cudaStream_t s) {
  const SmemLayout lay = layout(p.max_nodes, p.max_elems, p.max_segs, ET<T>::dim, ET<T>::nnpe, sizeof(S), kThreads);
  const int grid = grid_of(p);
  if (grid < p.npatch) {
    if (fext)
      k_patch_step<T, S, true, true><<<grid, kThreads, lay.total, s>>>(m, p, dt);
    else
      k_patch_step<T, S, false, true><<<grid, kThreads, lay.total, s>>>(m, p, dt);
  } else {
    if (fext)
      k_patch_step<T, S, true, false><<<grid, kThreads, lay.total, s>>>(m, p, dt);
    else
      k_patch_step<T, S, false, false><<<grid, kThreads, lay.total, s>>>(m, p, dt);
  }
  return cudaGetLastError();
}

// The dynamic shared memory limit is an attribute of the kernel function in
// the device's context, shared by every model of the process: it is only ever
// raised, so that a model built later with smaller patches cannot lower it
// below what an earlier model launches with.
std::mutex g_attr_mutex;

template <typename K>
cudaError_t raise_smem_limit(K kernel, size_t bytes) {
  cudaFuncAttributes attr;
  cudaError_t e = cudaFuncGetAttributes(&attr, kernel);
  if (e != cudaSuccess) return e;
  if ((size_t)attr.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <int T, typename S>
cudaError_t configure(const DevPatches& p) {
  const SmemLayout lay = layout(p.max_nodes, p.max_elems, p.max_segs, ET<T>::dim, ET<T>::nnpe, sizeof(S), kThreads);
  std::lock_guard<std::mutex> lock(g_attr_mutex);
  cudaError_t e;
  if ((e = raise_smem_limit(k_patch_step<T, S, true, false>, lay.total)) != cudaSuccess) return e;
  if ((e = raise_smem_limit(k_patch_step<T, S, false, false>, lay.total)) != cudaSuccess) return e;
  if ((e = raise_smem_limit(k_patch_step<T, S, true, true>, lay.total)) != cudaSuccess) return e;
  return raise_smem_limit(k_patch_step<T, S, false, true>, lay.total);
}

}  // namespace

size_t patch_smem_bytes(const DevPatches& p, int dim, int nnpe, bool fp32, int threads) {
  return layout(p.max_nodes, p.max_elems, p.max_segs, dim, nnpe, fp32 ? 4 : 8, threads).total;
}

cudaError_t patch_configure(const DevModel& m, const DevPatches& p, bool fp32) {
  switch (m.type) {
  case AKB_SEGMENT_2: return fp32 ? configure<AKB_SEGMENT_2, float>(p) : configure<AKB_SEGMENT_2, double>(p);
  case AKB_TRIANGLE_3: return fp32 ? configure<AKB_TRIANGLE_3, float>(p) : configure<AKB_TRIANGLE_3, double>(p);
  case AKB_TETRAHEDRON_4: return fp32 ? configure<AKB_TETRAHEDRON_4, float>(p) : configure<AKB_TETRAHEDRON_4, double>(p);
  default: return fp32 ? configure<AKB_HEXAHEDRON_8, float>(p) : configure<AKB_HEXAHEDRON_8, double>(p);
  }
}

cudaError_t patch_step(const DevModel& m, const DevPatches& p, double dt, bool fp32,
                       bool fext, cudaStream_t s) {
  if (p.npatch == 0) return cudaSuccess;
  switch (m.type) {
  case AKB_SEGMENT_2:
    return fp32 ? launch_patch<AKB_SEGMENT_2, float>(m, p, dt, fext, s)
                : launch_patch<AKB_SEGMENT_2, double>(m, p, dt, fext, s);
  case AKB_TRIANGLE_3:
    return fp32 ? launch_patch<AKB_TRIANGLE_3, float>(m, p, dt, fext, s)
                : launch_patch<AKB_TRIANGLE_3, double>(m, p, dt, fext, s);
  case AKB_TETRAHEDRON_4:
    return fp32 ? launch_patch<AKB_TETRAHEDRON_4, float>(m, p, dt, fext, s)
                : launch_patch<AKB_TETRAHEDRON_4, double>(m, p, dt, fext, s);
  default:
    return fp32 ? launch_patch<AKB_HEXAHEDRON_8, float>(m, p, dt, fext, s)
                : launch_patch<AKB_HEXAHEDRON_8, double>(m, p, dt, fext, s);
  }
}

cudaError_t patch_shared_nodes(const DevModel& m, const DevPatches& p, double dt, bool fext,
                               cudaStream_t s) {
  if (p.nshared == 0) return cudaSuccess;
  const int blocks = (int)((p.nshared + kThreads - 1) / kThreads);
  switch (m.dim) {
  case 1: fext ? k_shared_nodes<1, true><<<blocks, kThreads, 0, s>>>(m, p, dt)
               : k_shared_nodes<1, false><<<blocks, kThreads, 0, s>>>(m, p, dt); break;
  case 2: fext ? k_shared_nodes<2, true><<<blocks, kThreads, 0, s>>>(m, p, dt)
               : k_shared_nodes<2, false><<<blocks, kThreads, 0, s>>>(m, p, dt); break;
  default: fext ? k_shared_nodes<3, true><<<blocks, kThreads, 0, s>>>(m, p, dt)
                : k_shared_nodes<3, false><<<blocks, kThreads, 0, s>>>(m, p, dt); break;
  }
  return cudaGetLastError();
}

}  // namespace akb
