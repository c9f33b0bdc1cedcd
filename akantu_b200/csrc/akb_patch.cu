// akb_patch.cu -- the fused explicit step (AKB_MODE_FP64, AKB_MODE_FP32_BULK).
//
// k_patch_step: one CTA per patch.
//   1. stage the patch's nodes: the threads gather X, u, v, a and blocked
//      flags to the nodes' planned shared-memory positions and apply the
//      predictor u+ = u + dt v + dt^2/2 a, v* = v + dt a on free DOFs
//      (NewmarkBeta::predictor, newmark-beta.cc:60-89), while a TMA bulk copy
//      brings the first chunk record (corner positions, contribution slots,
//      runs, index blocks: akb_patch.cuh);
//   2. element forces in chunks of blockDim elements from shared memory
//      (akb_fastmath.cuh), each corner vector written to its contribution
//      slot; one thread per node run adds the run (ascending local element
//      order) to the node accumulators (the -1 scatter of
//      dof_manager.cc:83-137, without atomics). The record of the next chunk
//      is copied while this one is used (two buffers, when they fit);
//   3. nodes of this patch only: residual, lumped solve and corrector
//      (non_linear_solver_lumped.cc:85-98, newmark-beta.cc:176-210) on u+
//      kept in shared memory and v, a re-read, written back; nodes shared
//      with other patches: FP64 partial force to its slot.
// Every wait on a chunk copy is bounded: past it the CTA flags the error
// (P.err, read by the host on its next synchronisation), waits again (bounded)
// for the copies it issued and stops.
// k_shared_nodes: one thread per shared DOF adds its partials in patch order
// and applies the same predictor/corrector arithmetic.
#include <mutex>

#include "akb_fastmath.cuh"
#include "akb_patch.cuh"

namespace akb {
namespace {

constexpr int kThreads = 256;

struct SmemLayout {
  size_t xs, us, fs, contrib, scratch, buf, buf_stride, flags, mbar, total;
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }
__host__ __device__ inline size_t align128(size_t x) { return (x + 127) & ~size_t(127); }

// Shared-memory layout: node arrays component-major ([i][position], row
// stride LM), the chunk's element vectors component-major ([i][slot], CH
// slots), FP32 only: FP64 piece sums ([i][piece], PM pieces), nbuf chunk
// record buffers of CB bytes, per-(node, component) blocked flags for up to
// Lmax nodes, one mbarrier per buffer.
__host__ __device__ inline SmemLayout layout(int LM, int CH, int PM, int CB, int Lmax, int d,
                                             int sbytes, int nbuf) {
  SmemLayout s;
  const size_t nd = align16((size_t)LM * d * sizeof(double));
  s.xs = 0;
  s.us = s.xs + nd;
  s.fs = s.us + nd;
  s.contrib = s.fs + nd;
  s.scratch = align16(s.contrib + (size_t)CH * d * sbytes);
  s.buf = align128(s.scratch + (sbytes == 8 ? 0 : (size_t)PM * d * sizeof(double)));
  s.buf_stride = align128((size_t)CB);
  s.flags = s.buf + nbuf * s.buf_stride;
  s.mbar = align16(s.flags + (size_t)Lmax * d);
  s.total = s.mbar + 16;
  return s;
}
__host__ __device__ inline SmemLayout layout(const DevPatches& p, int d, int sbytes, int nbuf) {
  return layout(p.node_stride, p.contrib_slots, p.max_pieces, p.chunk_bytes, p.max_nodes, d, sbytes,
                nbuf);
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
constexpr int kBatch = 5;
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

__device__ inline void expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(mbar),
               "r"(bytes)
               : "memory");
}

// One patch p, by the whole CTA. uses: chunk records this CTA has consumed
// before (it picks the buffer and the mbarrier phase). Returns false when a
// bounded wait gave up.
template <int T, typename S, bool FEXT>
__device__ __forceinline__ bool patch_body(const DevModel& m, const DevPatches& P, double dt0,
                                           int p, unsigned char* smem, uint32_t& uses) {
  constexpr int d = ET<T>::dim, n = ET<T>::nnpe;
  static_assert(kChunk == kThreads, "one element per thread per chunk");
  const double dt = P.inst_dt ? P.inst_dt[P.patch_inst[p]] : dt0;
  const int nb = P.node_ptr[p];
  const int L = P.node_ptr[p + 1] - nb;
  const int eb = P.elem_ptr[p];
  const int ne = P.elem_ptr[p + 1] - eb;
  const int nint = P.ninterior[p];
  const int nchunks = (ne + kChunk - 1) / kChunk;
  const int ch0 = P.chunk_base[p];
  const int LM = P.node_stride, CH = P.contrib_slots;
  const bool two = P.nbuf == 2;  // buffers: 1 or 2
  const SmemLayout lay = layout(P, d, sizeof(S), two ? 2 : 1);
  double* xs = reinterpret_cast<double*>(smem + lay.xs);
  double* us = reinterpret_cast<double*>(smem + lay.us);
  double* fs = reinterpret_cast<double*>(smem + lay.fs);
  S* contrib = reinterpret_cast<S*>(smem + lay.contrib);
  double* scratch = reinterpret_cast<double*>(smem + lay.scratch);  // FP32: piece sums
  const int PM = P.max_pieces;
  uint8_t* flags = smem + lay.flags;
  const int tid = threadIdx.x;
  const int items = L * d;
  const uint32_t mb0 = saddr(smem + lay.mbar);

  // record k (counted over the CTA's chunks) uses buffer k % nbuf, and the
  // (k / nbuf)-th phase of that buffer's mbarrier
  auto buffer = [&](uint32_t k) { return two ? (k & 1u) : 0u; };
  auto phase = [&](uint32_t k) { return (two ? (k >> 1) : k) & 1u; };
  auto issue = [&](int c) {  // chunk c's record, by thread 0
    const uint2 cd = __ldg(reinterpret_cast<const uint2*>(&P.chunks[ch0 + c]));  // off16, bytes
    const uint32_t b = buffer(uses + c), bar = mb0 + 8 * b;
    expect_tx(bar, cd.y);
    bulk_copy(saddr(smem + lay.buf + b * lay.buf_stride), P.cdata + (size_t)cd.x * 8, cd.y, bar);
  };
  if (tid == 0) {
    issue(0);
    if (two && nchunks > 1) issue(1);
  }

  // 1. stage the nodes at their positions
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
      const int pj = P.lpos[nb + j];
      double uu = u[b], vv = v[b];
      if (!bl[b]) fast::predict(dt, uu, vv, a[b]);
      xs[i * LM + pj] = x[b];
      us[i * LM + pj] = uu;
      fs[i * LM + pj] = 0.0;
      flags[k] = bl[b];
    }
  }

  // 2. element forces chunk by chunk: each element writes its corner vectors
  //    to their contribution slots, then one thread per node run adds the
  //    run (ascending element order) to that node
  for (int c = 0; c < nchunks; ++c) {
    // one buffer: chunk c's record goes where chunk c-1's was, once every
    // thread is done with it
    if (!two && c > 0) {
      __syncthreads();
      if (tid == 0) issue(c);
    }
    // with two buffers this barrier also ends chunk c-1: past it no thread
    // reads chunk c-1's record or contributions any more
    const uint32_t b = buffer(uses + c);
    const bool ok = mbar_wait(mb0 + 8 * b, phase(uses + c));
    if (__syncthreads_or(!ok)) {  // bounded: flag, drain what was issued, stop
      if (tid == 0) {
        atomicExch(P.err, 1);
        const int last = min(nchunks - 1, (two && c == 0) ? 1 : c);
        for (int k = c; k <= last; ++k) mbar_wait(mb0 + 8 * buffer(uses + k), phase(uses + k));
      }
      return false;
    }
    if (two && tid == 0 && c > 0 && c + 1 < nchunks) issue(c + 1);  // into chunk c-1's buffer
    const int c0 = c * kChunk, nec = min(kChunk, ne - c0);
    const uint32_t A = (uint32_t)align16((size_t)nec * n * 2);
    if (tid < nec) {
      const uint16_t* lcs = reinterpret_cast<const uint16_t*>(smem + lay.buf + b * lay.buf_stride + 16);
      int lc[n], sl[n];
      load_corners<n>(lcs, tid, lc);
      load_corners<n>(lcs + A / 2, tid, sl);
      const MatParams& mp = (P.emat ? m.mat_table[P.emat[(size_t)eb + c0 + tid]] : m.mats[0]);
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
    // first level: one thread per piece (up to kMaxPiece contributions of
    // one node, ascending element order); a node in one piece is done, the
    // sum of a piece of a node in several is left for the second level. The
    // index loads depend on the header only, so they issue together.
    const unsigned char* buf = smem + lay.buf + b * lay.buf_stride;
    const uint4 hd = *reinterpret_cast<const uint4*>(buf);  // header: 8 x uint16
    {
      const int R1 = (int)(hd.x & 0xffff), rows = (int)(hd.x >> 16);
      const uint32_t* sums = reinterpret_cast<const uint32_t*>(buf + 16 + 2 * A);
      const uint16_t* ixs = reinterpret_cast<const uint16_t*>(buf + (hd.y & 0xffff));
      for (int q = tid; q < R1; q += kThreads) {
        const uint32_t w = sums[q];
        int k[kMaxPiece];
#pragma unroll
        for (int t = 0; t < kMaxPiece; ++t) k[t] = t < rows ? ixs[t * R1 + q] : 0;
        const int len = (int)((w >> 16) & 0xff), jp = (int)(w & 0xffff);
        double f[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int t = 0; t < kMaxPiece; ++t)
          if (t < len)
#pragma unroll
            for (int i = 0; i < d; ++i) f[i] += double(contrib[i * CH + k[t]]);
        if (len == 0) continue;
        if (w >> 24) {  // FP64: over the piece's first slot; FP32: by piece
#pragma unroll
          for (int i = 0; i < d; ++i) {
            if constexpr (sizeof(S) == 8)
              contrib[i * CH + k[0]] = f[i];
            else
              scratch[i * PM + q] = f[i];
          }
        } else {
#pragma unroll
          for (int i = 0; i < d; ++i) fs[i * LM + jp] -= f[i];
        }
      }
    }
    if ((hd.y >> 16) != 0) {  // second level: nodes cut in several pieces
      __syncthreads();
      const int R2 = (int)(hd.y >> 16), rows = (int)(hd.z & 0xffff);
      const uint32_t* sums = reinterpret_cast<const uint32_t*>(buf + (hd.z >> 16));
      const uint16_t* ixs = reinterpret_cast<const uint16_t*>(buf + (hd.w & 0xffff));
      for (int q = tid; q < R2; q += kThreads) {
        const uint32_t w = sums[q];
        constexpr int kUnroll = 4;  // pieces per node read together
        int k[kUnroll];
#pragma unroll
        for (int j = 0; j < kUnroll; ++j) k[j] = j < rows ? ixs[j * R2 + q] : 0;
        const int np = (int)(w >> 16), jp = (int)(w & 0xffff);
        double f[3] = {0.0, 0.0, 0.0};
        auto add = [&](int kk) {
#pragma unroll
          for (int i = 0; i < d; ++i) {
            if constexpr (sizeof(S) == 8)
              f[i] += double(contrib[i * CH + kk]);
            else
              f[i] += scratch[i * PM + kk];
          }
        };
#pragma unroll
        for (int j = 0; j < kUnroll; ++j)
          if (j < np) add(k[j]);
        for (int j = kUnroll; j < np; ++j) add(ixs[j * R2 + q]);
        if (np == 0) continue;
#pragma unroll
        for (int i = 0; i < d; ++i) fs[i * LM + jp] -= f[i];
      }
    }
  }
  __syncthreads();  // the sums of the last chunk are in
  uses += nchunks;

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
      const int pj = P.lpos[nb + j];
      const double f = fs[i * LM + pj];
      if (j >= nint) {
        P.partial[(int64_t)P.slot[nb + j] * d + i] = f;
      } else if (idx[b] >= 0) {  // blocked DOFs keep u, v, a
        // u+ from the staging, v* recomputed bit for bit
        double uu = us[i * LM + pj], vv = __dadd_rn(v[b], __dmul_rn(dt, a[b])), aa = a[b];
        fast::correct(dt, FEXT ? f + fx[b] : f, im[b], uu, vv, aa);
        m.u[idx[b]] = uu;
        m.v[idx[b]] = vv;
        m.a[idx[b]] = aa;
      }
    }
  }
  return true;
}

// One CTA per patch, or (PERSIST) a grid smaller than the patch count whose
// CTAs stride over the patches. The loop is a separate instantiation: kept
// out of the one-patch kernel it would raise that kernel's register pressure.
template <int T, typename S, bool FEXT, bool PERSIST>
__global__ void __launch_bounds__(kThreads, (PatchOccupancy<T, S>::value))
    k_patch_step(DevModel m, DevPatches P, double dt0) {
  extern __shared__ __align__(128) unsigned char smem[];
  {
    const SmemLayout lay = layout(P, ET<T>::dim, sizeof(S), P.nbuf);
    if (threadIdx.x == 0) {
      for (int b = 0; b < P.nbuf; ++b)
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(smem + lay.mbar + 8 * b))
                     : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
  }
  uint32_t uses = 0;
  if constexpr (PERSIST) {
    for (int p = blockIdx.x; p < P.npatch; p += gridDim.x) {
      if (p != (int)blockIdx.x) __syncthreads();  // shared memory of the previous patch is free
      if (!patch_body<T, S, FEXT>(m, P, dt0, p, smem, uses)) return;
    }
  } else {
    patch_body<T, S, FEXT>(m, P, dt0, blockIdx.x, smem, uses);
  }
}

template <int D, bool FEXT>
__global__ void k_shared_nodes(DevModel m, DevPatches P, double dt0) {
  // one thread per (shared node, component): neighbouring threads touch
  // neighbouring words of the partials and of u, v, a
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t ns = P.nshared;
  if (t >= ns * D) return;
  const int64_t s = t / D;
  const int i = (int)(t - s * D);
  const int64_t g = P.snodes[s];
  const int64_t k = g * D + i;
  // every load that depends on the node id is issued before the blocked
  // flag is tested
  const uint8_t bl = m.blocked[k];
  const double im = m.inv_mass[g];
  double u = m.u[k], v = m.v[k], a = m.a[k];
  const double fx = FEXT ? m.fext[k] : 0.0;
  const double dt = P.inst_dt ? P.inst_dt[P.snode_inst[s]] : dt0;
  // partials in patch order: the first two in the dense rows, the others
  // after them (zero for a node of no element)
  const int k0 = P.sptr[s], k1 = P.sptr[s + 1];
  double f = 0.0 + P.partial[s * D + i];
  f += P.partial[(ns + s) * D + i];
  for (int q = k0; q < k1; ++q) f += P.partial[(2 * ns + q) * D + i];
  if (bl) return;
  fast::predict(dt, u, v, a);
  if (FEXT) f += fx;
  fast::correct(dt, f, im, u, v, a);
  m.u[k] = u;
  m.v[k] = v;
  m.a[k] = a;
}

// Interface nodes of a partitioned mesh, one thread per (interface node,
// component): the sum of the node's partials in patch order (export), or the
// total over all parts written as its only partial (import).
__global__ void k_iface_export(DevPatches P, const uint32_t* iface, int64_t n, int d,
                               double* out) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n * d) return;
  const int64_t q = t / d;
  const int i = (int)(t - q * d);
  const int64_t ns = P.nshared, s = iface[q];
  double f = 0.0 + P.partial[s * d + i];
  f += P.partial[(ns + s) * d + i];
  for (int k = P.sptr[s]; k < P.sptr[s + 1]; ++k) f += P.partial[(2 * ns + k) * d + i];
  out[t] = f;
}

__global__ void k_iface_import(DevPatches P, const uint32_t* iface, int64_t n, int d,
                               const double* in) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n * d) return;
  const int64_t q = t / d;
  const int i = (int)(t - q * d);
  const int64_t ns = P.nshared, s = iface[q];
  P.partial[s * d + i] = in[t];
  P.partial[(ns + s) * d + i] = 0.0;
  for (int k = P.sptr[s]; k < P.sptr[s + 1]; ++k) P.partial[(2 * ns + k) * d + i] = 0.0;
}

__global__ void k_mass_export(DevModel m, const uint32_t* nodes, int64_t n, double* out) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n) return;
  out[t] = m.mass[(int64_t)nodes[t] * m.dim];
}

__global__ void k_mass_import(DevModel m, const uint32_t* nodes, int64_t n, const double* in) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int64_t g = nodes[t];
  const double M = in[t];
  for (int c = 0; c < m.dim; ++c) m.mass[g * m.dim + c] = M;
  m.inv_mass[g] = 1. / M;
}

// grid of the patch kernel: one CTA per patch, or a persistent grid of
// P.grid CTAs that stride over the patches
inline int grid_of(const DevPatches& p) {
  return (p.grid > 0 && p.grid < p.npatch) ? p.grid : p.npatch;
}

template <int T, typename S>
cudaError_t launch_patch(const DevModel& m, const DevPatches& p, double dt, bool fext,
                         cudaStream_t s) {
  const SmemLayout lay = layout(p, ET<T>::dim, sizeof(S), p.nbuf);
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
  const SmemLayout lay = layout(p, ET<T>::dim, sizeof(S), p.nbuf);
  std::lock_guard<std::mutex> lock(g_attr_mutex);
  cudaError_t e;
  if ((e = raise_smem_limit(k_patch_step<T, S, true, false>, lay.total)) != cudaSuccess) return e;
  if ((e = raise_smem_limit(k_patch_step<T, S, false, false>, lay.total)) != cudaSuccess) return e;
  if ((e = raise_smem_limit(k_patch_step<T, S, true, true>, lay.total)) != cudaSuccess) return e;
  return raise_smem_limit(k_patch_step<T, S, false, true>, lay.total);
}

}  // namespace

size_t patch_smem_bytes(const DevPatches& p, int dim, int nnpe, bool fp32, int nbuf) {
  (void)nnpe;
  return layout(p, dim, fp32 ? 4 : 8, nbuf).total;
}

int patch_buffers(const DevPatches& p, int type, bool fp32) {
  // CTAs per SM: 228 KB of shared memory, 1 KB reserved per CTA, and the
  // register budget the instantiation is built for
  int regs;
  switch (type) {
  case AKB_HEXAHEDRON_8: regs = fp32 ? PatchOccupancy<AKB_HEXAHEDRON_8, float>::value
                                     : PatchOccupancy<AKB_HEXAHEDRON_8, double>::value; break;
  default: regs = PatchOccupancy<AKB_TETRAHEDRON_4, double>::value; break;
  }
  const int dim = type == AKB_SEGMENT_2 ? 1 : type == AKB_TRIANGLE_3 ? 2 : 3;
  auto ctas = [&](int nbuf) {
    const size_t s = layout(p, dim, fp32 ? 4 : 8, nbuf).total + 1024;
    return std::min<int>(regs, (int)((228 * 1024) / s));
  };
  return ctas(2) >= ctas(1) ? 2 : 1;
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

cudaError_t patch_iface_export(const DevModel& m, const DevPatches& p, const uint32_t* iface,
                               int64_t n, double* out, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const int blocks = (int)((n * m.dim + kThreads - 1) / kThreads);
  k_iface_export<<<blocks, kThreads, 0, s>>>(p, iface, n, m.dim, out);
  return cudaGetLastError();
}

cudaError_t patch_iface_import(const DevModel& m, const DevPatches& p, const uint32_t* iface,
                               int64_t n, const double* in, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const int blocks = (int)((n * m.dim + kThreads - 1) / kThreads);
  k_iface_import<<<blocks, kThreads, 0, s>>>(p, iface, n, m.dim, in);
  return cudaGetLastError();
}

cudaError_t mass_export(const DevModel& m, const uint32_t* nodes, int64_t n, double* out,
                        cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_mass_export<<<(int)((n + kThreads - 1) / kThreads), kThreads, 0, s>>>(m, nodes, n, out);
  return cudaGetLastError();
}

cudaError_t mass_import(const DevModel& m, const uint32_t* nodes, int64_t n, const double* in,
                        cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_mass_import<<<(int)((n + kThreads - 1) / kThreads), kThreads, 0, s>>>(m, nodes, n, in);
  return cudaGetLastError();
}

cudaError_t patch_shared_nodes(const DevModel& m, const DevPatches& p, double dt, bool fext,
                               cudaStream_t s) {
  if (p.nshared == 0) return cudaSuccess;
  const int blocks = (int)((p.nshared * m.dim + kThreads - 1) / kThreads);
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
