// akb_patch.cu -- the fused explicit step (AKB_MODE_FP64, AKB_MODE_FP32_BULK).
//
// k_patch_step: one CTA per patch (akb_patch.cuh for the node order, the
// predicted displacement w and the shared-node protocol).
//   1. stage: thread 0 starts TMA bulk copies of the interior nodes' X and w
//      (two contiguous slices) and of the first chunk records, and prefetches
//      the interior nodes' v, a, 1/M and blocked flags into L2; every thread
//      starts cp.async copies of its shared nodes' X and w and zeroes the
//      force accumulators;
//   2. element forces in chunks of blockDim elements from shared memory
//      (akb_fastmath.cuh), each corner vector written to its contribution
//      slot; one thread per node run adds the run (ascending local element
//      order) to the node's accumulator (the -1 scatter of
//      dof_manager.cc:83-137, without atomics). The record of the next chunk
//      is copied while this one is used (two buffers, when they fit);
//   3. finish: each shared node's partial force goes to its slot; the
//      interior nodes get the residual, lumped solve and corrector
//      (non_linear_solver_lumped.cc:85-98, newmark-beta.cc:176-210) and the
//      next predictor (newmark-beta.cc:60-89), written back as u, v, a and w.
// Every wait on a bulk copy is bounded: past it the CTA flags the error
// (P.err, read by the host on its next synchronisation), waits again (bounded)
// for the copies it issued and stops.
// k_finish_list: one thread per (listed node, component) adds the partials
// of the shared nodes in patch order and finishes them the same way, and the
// nodes of no element (after the exchange between parts, for a partitioned
// mesh).
#include <cfloat>
#include <mutex>

#include "akb_fastmath.cuh"
#include "akb_patch.cuh"

namespace akb {
namespace {

constexpr int kThreads = 256;

struct SmemLayout {
  size_t xs, ws, fs, contrib, sslot, buf, buf_stride, mbar, total;
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }
__host__ __device__ inline size_t align128(size_t x) { return (x + 127) & ~size_t(127); }

// Shared-memory layout: node arrays X and w row-major ([position][i], 16
// bytes of slack in front for the offset of the interior slice), force
// accumulators component-major ([i][position], row stride LM), the chunk's
// element vectors (CH slots, cidx), the partial slot of each shared node
// (SHmax uint32), nbuf chunk record buffers of CB bytes, three mbarriers (two
// record buffers, the node staging).
__host__ __device__ inline SmemLayout layout(int LM, int CH, int CB, int Lmax, int SHmax, int d,
                                             int sbytes, int nbuf) {
  SmemLayout s;
  const size_t nb = align16(16 + (size_t)Lmax * d * sizeof(double));
  s.xs = 0;
  s.ws = s.xs + nb;
  s.fs = s.ws + nb;
  s.contrib = s.fs + align16((size_t)LM * d * sizeof(double));
  s.sslot = align16(s.contrib + (size_t)CH * d * sbytes);
  s.buf = align128(s.sslot + (size_t)SHmax * sizeof(uint32_t));
  s.buf_stride = align128((size_t)CB);
  s.mbar = s.buf + nbuf * s.buf_stride;
  s.total = s.mbar + 24;
  return s;
}
__host__ __device__ inline SmemLayout layout(const DevPatches& p, int d, int sbytes, int nbuf) {
  return layout(p.node_stride, p.contrib_slots, p.chunk_bytes, p.max_nodes, p.max_shared, d, sbytes,
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

// Differences of an element's corner coordinates and predicted
// displacements to its first corner, in FP64 before any rounding to S. Node
// arrays are row-major; in 2D a node's two components are one 16-byte load.
template <int d, int n, typename S>
__device__ inline void gather_differences(const double* xs, const double* ws, const int* lc,
                                          double* dX, S* du) {
  if constexpr (d == 2) {
    const double2 x0 = reinterpret_cast<const double2*>(xs)[lc[0]];
    const double2 u0 = reinterpret_cast<const double2*>(ws)[lc[0]];
    dX[0] = dX[1] = 0.0;
    du[0] = du[1] = S(0);
#pragma unroll
    for (int a = 1; a < n; ++a) {
      const double2 x = reinterpret_cast<const double2*>(xs)[lc[a]];
      const double2 u = reinterpret_cast<const double2*>(ws)[lc[a]];
      dX[a * 2] = x.x - x0.x;
      dX[a * 2 + 1] = x.y - x0.y;
      du[a * 2] = S(u.x - u0.x);
      du[a * 2 + 1] = S(u.y - u0.y);
    }
  } else {
#pragma unroll
    for (int i = 0; i < d; ++i) {
      dX[i] = 0;
      du[i] = 0;
      const double x0 = xs[d * lc[0] + i], u0 = ws[d * lc[0] + i];
#pragma unroll
      for (int a = 1; a < n; ++a) {
        dX[a * d + i] = xs[d * lc[a] + i] - x0;
        du[a * d + i] = S(ws[d * lc[a] + i] - u0);
      }
    }
  }
}

// Where component i of contribution slot k sits: 3D contributions are rows
// of three (one address per slot; 3 is invertible mod 16 and mod 32, so
// slots at distinct residues keep distinct banks), 1D and 2D ones
// component-major ([i][slot], 16-byte loads in 2D would otherwise pair slots
// on one bank group).
template <int d>
__device__ inline int cidx(int k, int i, int CH) {
  return d == 3 ? 3 * k + i : i * CH + k;
}

// CTAs per SM each instantiation is built for (register budget).
template <int T, typename S> struct PatchOccupancy { static constexpr int value = 3; };
template <> struct PatchOccupancy<AKB_HEXAHEDRON_8, float> { static constexpr int value = 2; };
template <> struct PatchOccupancy<AKB_HEXAHEDRON_8, double> { static constexpr int value = 1; };
// FP32-bulk tetrahedra (FP32 contributions, 768-element patches, one record
// buffer: <= 56 KB), 2D and 1D patches of <= 1024 elements take <= 56 KB of
// shared memory: four CTAs per SM when the registers allow it (<= 64 per
// thread; the FP64 tetrahedron at 64 registers measured slower)
template <> struct PatchOccupancy<AKB_TETRAHEDRON_4, float> { static constexpr int value = 4; };
template <typename S> struct PatchOccupancy<AKB_TRIANGLE_3, S> { static constexpr int value = 4; };
template <typename S> struct PatchOccupancy<AKB_SEGMENT_2, S> { static constexpr int value = 4; };

// DOFs handled per thread per round of the finishing loop: their global
// loads are issued together.
constexpr int kBatch = 4;
constexpr uint32_t kWaitLimit = 1u << 22;

__device__ inline uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// The step's kernels are launched with programmatic stream serialization
// (launch_pdl): k_patch_step waits before its first read of the node state,
// k_finish_list before its first read of the partials.
__device__ inline void bulk_copy(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}
// L2 prefetch of [lo, hi) rounded out to 16-byte boundaries (inside the
// allocation: nodal arrays carry 16 bytes of slack at their end).
__device__ inline void prefetch_l2(const void* base, size_t lo, size_t hi) {
  const size_t a = lo & ~size_t(15), b = (hi + 15) & ~size_t(15);
  if (b <= a) return;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"((const char*)base + a),
               "r"((uint32_t)(b - a))
               : "memory");
}
__device__ inline void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(saddr(dst)), "l"(src) : "memory");
}
__device__ inline void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr(dst)), "l"(src) : "memory");
}
__device__ inline void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
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
__device__ inline void arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

// Finishing inputs of a patch's interior nodes [ib, ib + nint): v, a (rows
// of d doubles), 1/M (one double), blocked flags (d bytes), f_ext (d
// doubles, when used). Each slice is bulk-copied from the 16-byte boundary at
// or below its start to the one at or above its end (inside the arrays'
// 16-byte slack); off[k]: where the slice's first item lands, from the
// buffer's start; returns the bytes of all copies.
template <int d, bool FEXT>
__device__ inline uint32_t finish_regions(int ib, int nint, uint32_t* off, uint32_t* lo,
                                          uint32_t* bytes) {
  constexpr int nf = FEXT ? 5 : 4;
  const uint32_t rowb[5] = {8u * d, 8u * d, 8u, (uint32_t)d, 8u * d};
  uint32_t total = 0;
#pragma unroll
  for (int k = 0; k < nf; ++k) {
    const size_t s0 = (size_t)ib * rowb[k], s1 = (size_t)(ib + nint) * rowb[k];
    const size_t c0 = s0 & ~size_t(15), c1 = (s1 + 15) & ~size_t(15);
    off[k] = total + (uint32_t)(s0 - c0);
    lo[k] = (uint32_t)c0;  // (byte offsets below 4 GB: nn x d doubles < 2^32 bytes)
    bytes[k] = (uint32_t)(c1 - c0);
    total += bytes[k];
  }
  return total;
}

// Corrector of one free DOF from its total force r (with f_ext), and the
// next predictor: u = w (the predicted displacement this step's forces were
// evaluated at), v* = v + dt a recomputed bit for bit, then
// x = r / M - a, v = v* + dt/2 x, a += x (u += 0 x only when x is not
// finite); w' = u + dt v + dt^2/2 a.
// M v^2 of one DOF from its inverse lumped mass, for masses above
// DBL_EPSILON (the test of getKineticEnergy, solid_mechanics_model.cc:547-561).
__device__ inline double ke_term(double v, double im) {
  const double M = 1.0 / im;
  return M > DBL_EPSILON ? v * v * M : 0.0;
}

// Sum of the CTA's per-thread values in a fixed order (lanes by an xor
// tree, then warps in order), by thread 0; every thread must call it.
__device__ inline double cta_sum(double x, double* warp_sums) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();  // warp_sums free (a previous use is read)
  if ((threadIdx.x & 31) == 0) warp_sums[w] = x;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < nw; ++k) s += warp_sums[k];
  return s;
}

__device__ inline void finish_dof(double dt, double r, double im, double w, double& v, double& a,
                                  double& u, double& wn) {
  u = w;
  v = __dadd_rn(v, __dmul_rn(dt, a));
  fast::correct(dt, r, im, u, v, a);
  wn = u;
  double vn = v;
  fast::predict(dt, wn, vn, a);
}

// One patch p, by the whole CTA. uses: chunk records this CTA has consumed
// before (it picks the buffer and the mbarrier phase); stages: patches it
// staged before (the phase of the staging mbarrier). Returns false when a
// bounded wait gave up.
template <int T, typename S, bool FEXT>
__device__ __forceinline__ bool patch_body(const DevModel& m, const DevPatches& P, double dt0,
                                           int p, unsigned char* smem, uint32_t& uses,
                                           uint32_t& stages) {
  constexpr int d = ET<T>::dim, n = ET<T>::nnpe;
  static_assert(kChunk == kThreads, "one element per thread per chunk");
  const double dt = P.inst_dt ? P.inst_dt[P.patch_inst[p]] : dt0;
  const int ib = P.ibeg[p], nint = P.nint[p];
  const int s0 = P.sh_ptr[p], nsh = P.sh_ptr[p + 1] - s0;
  const int L = nint + nsh;
  const int eb = P.elem_ptr[p];
  const int ne = P.elem_ptr[p + 1] - eb;
  const int nchunks = (ne + kChunk - 1) / kChunk;
  const int ch0 = P.chunk_base[p];
  const int LM = P.node_stride, CH = P.contrib_slots;
  const bool two = P.nbuf == 2;  // buffers: 1 or 2
  const SmemLayout lay = layout(P, d, sizeof(S), two ? 2 : 1);
  // the interior slice [ib, ib + nint) of X and w is bulk-copied from the
  // 16-byte boundary at or below its start (the bytes before it land in the
  // slack in front of the array; o: the slice's offset in doubles) to the
  // boundary at or below its end; the remaining tail (one double at most)
  // comes by cp.async, so that nothing is written past the slice, where the
  // shared nodes go
  const size_t row = (size_t)d * sizeof(double);
  const size_t s_lo = (size_t)ib * row, s_hi = (size_t)(ib + nint) * row;
  const size_t c_lo = s_lo & ~size_t(15), c_hi = s_hi & ~size_t(15);
  const int o = (int)((s_lo - c_lo) / sizeof(double));
  double* xs = reinterpret_cast<double*>(smem + lay.xs) + o;  // node at position j: xs[d j + i]
  double* ws = reinterpret_cast<double*>(smem + lay.ws) + o;
  double* fs = reinterpret_cast<double*>(smem + lay.fs);      // fs[i LM + j]
  S* contrib = reinterpret_cast<S*>(smem + lay.contrib);
  const int tid = threadIdx.x;
  const uint32_t mb0 = saddr(smem + lay.mbar), mbs = mb0 + 16;

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

  // 1. staging
  // the interior nodes' finishing inputs go to the spare record buffer (the
  // one the next chunk would use) at the start of the last chunk, when two
  // buffers are used and they fit; the finish then reads shared memory
  bool pre;
  {
    uint32_t f_off[5], f_lo[5], f_bytes[5];
    pre = two && nint > 0 &&
          finish_regions<d, FEXT>(ib, nint, f_off, f_lo, f_bytes) <= lay.buf_stride;
  }
  const uint32_t spare = buffer(uses + nchunks);
  auto issue_finish = [&]() {  // by thread 0
    const void* src[5] = {m.v, m.a, m.inv_mass, m.blocked, m.fext};
    uint32_t f_off[5], f_lo[5], f_bytes[5];
    const uint32_t total = finish_regions<d, FEXT>(ib, nint, f_off, f_lo, f_bytes);
    const uint32_t dst = saddr(smem + lay.buf + spare * lay.buf_stride);
    expect_tx(mbs, total);
    uint32_t at = 0;
#pragma unroll
    for (int k = 0; k < (FEXT ? 5 : 4); ++k) {
      bulk_copy(dst + at, reinterpret_cast<const char*>(src[k]) + f_lo[k], f_bytes[k], mbs);
      at += f_bytes[k];
    }
  };
  if (tid == 0) {
    // the previous patch's generic-proxy accesses of these buffers (ordered
    // before this point by the CTA barrier) come before the bulk copies
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (nint > 0 && c_hi > c_lo) {
      const uint32_t bytes = (uint32_t)(c_hi - c_lo);
      expect_tx(mbs, 2 * bytes);
      bulk_copy(saddr(smem + lay.xs), reinterpret_cast<const char*>(m.X) + c_lo, bytes, mbs);
      bulk_copy(saddr(smem + lay.ws), reinterpret_cast<const char*>(P.w) + c_lo, bytes, mbs);
    } else {
      arrive(mbs);
    }
    if (nchunks > 0) issue(0);
    if (two && nchunks > 1) issue(1);
    if (nint > 0 && !pre) {  // inputs of the interior nodes' finish
      prefetch_l2(m.v, s_lo, s_hi);
      prefetch_l2(m.a, s_lo, s_hi);
      prefetch_l2(m.inv_mass, (size_t)ib * 8, (size_t)(ib + nint) * 8);
      prefetch_l2(m.blocked, (size_t)ib * d, (size_t)(ib + nint) * d);
      if (FEXT) prefetch_l2(m.fext, s_lo, s_hi);
    }
  }
  if (tid == kThreads - 1 && nint > 0 && c_hi < s_hi && c_hi >= s_lo) {  // the tail double
    const size_t k = (c_hi - s_lo) / sizeof(double);
    cp_async8(xs + k, m.X + (size_t)ib * d + k);
    cp_async8(ws + k, P.w + (size_t)ib * d + k);
  } else if (tid == kThreads - 1 && nint > 0 && c_hi < s_lo) {  // slice within one 16 bytes
    for (size_t k = 0; k < (size_t)nint * d; ++k) {
      cp_async8(xs + k, m.X + (size_t)ib * d + k);
      cp_async8(ws + k, P.w + (size_t)ib * d + k);
    }
  }
  uint32_t* sslot = reinterpret_cast<uint32_t*>(smem + lay.sslot);
  for (int t = tid; t < nsh; t += kThreads) {
    const int64_t g = P.sgid[s0 + t];
    sslot[t] = P.sslot[s0 + t];  // for the finish
    const int j = nint + t;
    if constexpr (d == 2) {
      cp_async16(xs + 2 * j, m.X + g * 2);
      cp_async16(ws + 2 * j, P.w + g * 2);
    } else {
#pragma unroll
      for (int i = 0; i < d; ++i) {
        cp_async8(xs + d * j + i, m.X + g * d + i);
        cp_async8(ws + d * j + i, P.w + g * d + i);
      }
    }
  }
  for (int k = tid; k < L * d; k += kThreads) {
    const int i = k / L, j = k - i * L;
    fs[i * LM + j] = 0.0;
  }
  cp_async_wait_all();
  {
    const bool ok = mbar_wait(mbs, stages & 1u);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(P.err, 1);
        mbar_wait(mbs, stages & 1u);
        for (int k = 0; k < min(nchunks, two ? 2 : 1); ++k)
          mbar_wait(mb0 + 8 * buffer(uses + k), phase(uses + k));
      }
      return false;
    }
  }
  ++stages;
  if (pre && nchunks <= 1 && tid == 0) issue_finish();  // the second buffer is free already

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
        if (pre && nchunks <= 1) mbar_wait(mbs, stages & 1u);  // the finishing inputs
      }
      return false;
    }
    if (two && tid == 0 && c > 0 && c + 1 < nchunks) issue(c + 1);  // into chunk c-1's buffer
    if (pre && tid == 0 && c > 0 && c + 1 == nchunks) issue_finish();  // ditto
    const int c0 = c * kChunk, nec = min(kChunk, ne - c0);
    const uint32_t A = (uint32_t)align16((size_t)nec * n * 2);
    if (tid < nec) {
      const uint16_t* lcs = reinterpret_cast<const uint16_t*>(smem + lay.buf + b * lay.buf_stride + 16);
      int lc[n], sl[n];
      load_corners<n>(lcs, tid, lc);
      load_corners<n>(lcs + A / 2, tid, sl);
      const MatParams& mp = (P.emat ? m.mat_table[P.emat[(size_t)eb + c0 + tid]] : m.mats[0]);
      double dX[3 * 8];
      S du[3 * 8];
      gather_differences<d, n, S>(xs, ws, lc, dX, du);
      S fe[3 * 8];
      fast::element_force<T, S>(mp, dX, du, fe);
#pragma unroll
      for (int a = 0; a < n; ++a)
#pragma unroll
        for (int i = 0; i < d; ++i) contrib[cidx<d>(sl[a], i, CH)] = fe[a * d + i];
    }
    __syncthreads();
    // one thread per run (a node's contributions of this chunk, ascending
    // element order) adds the run to the node's accumulator; runs are sorted
    // by length, so a warp's threads loop about as long
    const unsigned char* buf = smem + lay.buf + b * lay.buf_stride;
    const uint4 hd = *reinterpret_cast<const uint4*>(buf);  // header: 8 x uint16
    {
      constexpr int G = sizeof(S) == 8 ? 16 : 32;  // runs per group
      // header words: x = R | ng << 16, y = runs | goff << 16, z = idx | G << 16
      const int R = (int)(hd.x & 0xffff);
      const uint32_t* runs = reinterpret_cast<const uint32_t*>(buf + (hd.y & 0xffff));
      const uint16_t* goff = reinterpret_cast<const uint16_t*>(buf + (hd.y >> 16));
      const uint16_t* idx = reinterpret_cast<const uint16_t*>(buf + (hd.z & 0xffff));
      for (int q = tid; q < R; q += kThreads) {
        const uint32_t w = runs[q];
        const int len = (int)(w >> 16), jp = (int)(w & 0xffff);
        if (len == 0) continue;
        const uint16_t* ix = idx + goff[q / G] + (q % G);
        double f[3] = {0.0, 0.0, 0.0};
#pragma unroll 4
        for (int t = 0; t < len; ++t) {
          const int k = ix[t * G];
#pragma unroll
          for (int i = 0; i < d; ++i) f[i] += double(contrib[cidx<d>(k, i, CH)]);
        }
#pragma unroll
        for (int i = 0; i < d; ++i) fs[i * LM + jp] -= f[i];
      }
    }
  }
  {
    // the sums of the last chunk are in (and the finishing inputs)
    const bool ok = !pre || mbar_wait(mbs, stages & 1u);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(P.err, 1);
        mbar_wait(mbs, stages & 1u);
      }
      return false;
    }
  }
  if (pre) ++stages;
  uses += nchunks;
  const unsigned char* fin = smem + lay.buf + spare * lay.buf_stride;
  uint32_t f_off[5];
  {
    uint32_t f_lo[5], f_bytes[5];
    finish_regions<d, FEXT>(ib, nint, f_off, f_lo, f_bytes);
  }

  // 3. finish: the shared nodes' partials to their slots (the second pass
  //    adds them), the interior nodes finished here, one thread per DOF,
  //    contiguous in the global arrays
  grid_launch_dependents();  // the second pass may start launching (it waits for this grid)
  for (int k = tid; k < nsh * d; k += kThreads) {
    const int t = k / d, i = k - t * d;
    P.partial[(size_t)sslot[t] * d + i] = fs[i * LM + nint + t];
  }
  const int items = nint * d;
  double ke = 0.0;  // M v^2 of this thread's DOFs after the step
  for (int base = 0; base < items; base += kThreads * kBatch) {
    double v[kBatch], a[kBatch], im[kBatch], fx[kBatch];
    uint8_t bl[kBatch];
#pragma unroll
    for (int b = 0; b < kBatch; ++b) {
      const int k = base + b * kThreads + tid;
      if (k < items) {
        if (pre) {
          v[b] = *reinterpret_cast<const double*>(fin + f_off[0] + 8 * k);
          a[b] = *reinterpret_cast<const double*>(fin + f_off[1] + 8 * k);
          im[b] = *reinterpret_cast<const double*>(fin + f_off[2] + 8 * (k / d));
          bl[b] = fin[f_off[3] + k];
          fx[b] = FEXT ? *reinterpret_cast<const double*>(fin + f_off[4] + 8 * k) : 0.0;
        } else {
          const int64_t q = (int64_t)ib * d + k;
          bl[b] = m.blocked[q];
          v[b] = m.v[q];
          a[b] = m.a[q];
          im[b] = m.inv_mass[ib + k / d];
          fx[b] = FEXT ? m.fext[q] : 0.0;
        }
      }
    }
#pragma unroll
    for (int b = 0; b < kBatch; ++b) {
      const int k = base + b * kThreads + tid;
      if (k >= items) continue;
      if (!bl[b]) {  // blocked DOFs keep u, v, a (and w = u)
        const int j = k / d, i = k - j * d;
        const int64_t q = (int64_t)ib * d + k;
        const double f = fs[i * LM + j];
        double u, wn;
        finish_dof(dt, FEXT ? f + fx[b] : f, im[b], ws[k], v[b], a[b], u, wn);
        m.u[q] = u;
        m.v[q] = v[b];
        m.a[q] = a[b];
        P.w[q] = wn;
      }
      ke += ke_term(v[b], im[b]);
    }
  }
  if (P.ke_part) {
    __shared__ double warp_sums[kThreads / 32];
    const double s = cta_sum(ke, warp_sums);
    if (tid == 0) P.ke_part[p] = s;
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
      for (int b = 0; b < 3; ++b)
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(smem + lay.mbar + 8 * b))
                     : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
  }
  grid_wait();  // the previous step's (or update's) writes of w, v, a, u
  uint32_t uses = 0, stages = 0;
  if constexpr (PERSIST) {
    for (int p = blockIdx.x; p < P.npatch; p += gridDim.x) {
      if (p != (int)blockIdx.x) __syncthreads();  // shared memory of the previous patch is free
      if (!patch_body<T, S, FEXT>(m, P, dt0, p, smem, uses, stages)) return;
    }
  } else {
    patch_body<T, S, FEXT>(m, P, dt0, blockIdx.x, smem, uses, stages);
  }
}

// Listed nodes, one thread per (entry, component): the sum of the entry's
// partials in rank order (none for a node of no element), then the same
// finish as in the fused step, from the node's stored w; and the block's sum
// of M v^2 after the step (a kinetic-energy partial). The entry's own state
// (v, a, w, 1/M, blocked flag, f_ext) is not written by the fused step, and
// every kernel before the fused step has completed when this grid launches
// (the fused step waited for them before letting it launch): it is loaded
// before waiting for the fused step, through L2 (no L1 line of an earlier
// grid), so only the partials wait.
template <int D, bool FEXT>
__global__ void k_finish_list(DevModel m, DevPatches P, double dt0) {
  constexpr int d = D;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool on = t < P.nlist * d;
  const int64_t e = on ? t / d : 0;
  const int i = (int)(t - e * d);
  const bool sh = on && e < (int64_t)P.nshared;
  int64_t q = 0;
  uint32_t k = 0;
  uint8_t bl = 1;
  double dt = dt0, im = 1.0, w = 0.0, fx = 0.0, v = 0.0, a = 0.0;
  if (on) {
    // a single mesh's shared nodes are one block: no index to load
    const int64_t g = sh && P.shared_contig ? (int64_t)P.shared_base + e : (int64_t)P.list_gid[e];
    q = g * d + i;
    k = P.list_k[e];
    if (P.inst_dt) dt = P.inst_dt[P.list_inst[e]];
    bl = __ldcg(m.blocked + q);
    im = __ldcg(m.inv_mass + g);
    w = __ldcg(P.w + q);
    if (FEXT) fx = __ldcg(m.fext + q);
    v = __ldcg(m.v + q);
    a = __ldcg(m.a + q);
  }
  grid_wait();               // the fused step's partials
  grid_launch_dependents();  // the next step may start launching (it waits for this grid)
  double ke = 0.0;
  if (on) {
    double f = 0.0;
    if (sh) {  // ranks 0 and 1 in the dense rows at known addresses
      const double p0 = P.partial[(size_t)e * d + i];
      const double p1 = P.partial[((size_t)P.nshared + e) * d + i];  // zero when k = 1
      f += p0;
      if (k > 1) f += p1;
      if (k > 2) {
        const uint32_t over = P.list_part[e];
        for (uint32_t r = 2; r < k; ++r) f += P.partial[(size_t)(over + r - 2) * d + i];
      }
    }
    if (!bl) {
      double u, wn;
      finish_dof(dt, FEXT ? f + fx : f, im, w, v, a, u, wn);
      m.u[q] = u;
      m.v[q] = v;
      m.a[q] = a;
      P.w[q] = wn;
    }
    ke = ke_term(v, im);
  }
  if (P.ke_part) {
    __shared__ double warp_sums[kThreads / 32];
    const double s = cta_sum(ke, warp_sums);
    if (threadIdx.x == 0) P.ke_part[P.npatch + blockIdx.x] = s;
  }
}

// w = u + dt v + dt^2/2 a on free DOFs, w = u on blocked ones; one thread per
// DOF (batches: the node's instance by bisection of the node ranges).
__global__ void k_refresh_w(DevModel m, DevPatches P, double dt0) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= m.nn * m.dim) return;
  double u = m.u[q];
  if (!m.blocked[q]) {
    double dt = dt0;
    if (P.inst_dt) {
      const int64_t node = q / m.dim;
      int lo = 0, hi = P.ninst;  // node_off[lo] <= node < node_off[hi]
      while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (P.node_off[mid] <= node) lo = mid; else hi = mid;
      }
      dt = P.inst_dt[lo];
    }
    double v = m.v[q];
    fast::predict(dt, u, v, m.a[q]);
  }
  P.w[q] = u;
}

// Interface nodes of a partitioned mesh, one thread per (node, component):
// the sum of the node's partials in order (export), or the total over all
// parts written as its only partial (import).
// Component i of the partial of rank r of shared node s.
__device__ inline double& partial_of(const DevPatches& P, uint32_t s, uint32_t r, int d, int i) {
  return P.partial[(size_t)partial_slot(P.nshared, s, P.list_part[s], r) * d + i];
}

__global__ void k_iface_export(DevPatches P, const uint32_t* shared, const uint32_t* ks, int64_t n,
                               int d, double* out) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n * d) return;
  const int64_t e = t / d;
  const int i = (int)(t % d);
  const uint32_t s = shared[e], k = ks[e];
  double f = 0.0;
  for (uint32_t r = 0; r < k; ++r) f += partial_of(P, s, r, d, i);
  out[t] = f;
}

__global__ void k_iface_import(DevPatches P, const uint32_t* shared, const uint32_t* ks, int64_t n,
                               int d, const double* in) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n * d) return;
  const int64_t e = t / d;
  const int i = (int)(t % d);
  const uint32_t s = shared[e], k = ks[e];
  for (uint32_t r = 0; r < k; ++r) partial_of(P, s, r, d, i) = r == 0 ? in[t] : 0.0;
}

// One thread per (packed row, component); the own value of a row is the sum
// of its partial slots, as k_iface_export forms it.
__global__ void k_iface_pack(DevPatches P, const uint32_t* shared, const uint32_t* ks,
                             ExchangePlan x, int d, double* out) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= x.n_send * d) return;
  const int64_t j = t / d;
  const int i = (int)(t - j * d);
  const uint32_t e = x.send_rows[j];
  const uint32_t s = shared[e], k = ks[e];
  double f = 0.0;
  for (uint32_t r = 0; r < k; ++r) f += partial_of(P, s, r, d, i);
  out[t] = f;
}

// One thread per (interface row, component): the terms in the plan's order,
// then the total written as the row's only partial.
__global__ void k_iface_sum_import(DevPatches P, const uint32_t* shared, const uint32_t* ks,
                                   ExchangePlan x, int d, const double* recv) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= x.n_rows * d) return;
  const int64_t e = t / d;
  const int i = (int)(t - e * d);
  const uint32_t s = shared[e], k = ks[e];
  double own = 0.0;
  for (uint32_t r = 0; r < k; ++r) own += partial_of(P, s, r, d, i);
  double acc = 0.0;
  for (uint32_t j = x.sum_ptr[e]; j < x.sum_ptr[e + 1]; ++j) {
    const int32_t src = x.sum_src[j];
    acc += src < 0 ? own : recv[(int64_t)src * d + i];
  }
  for (uint32_t r = 0; r < k; ++r) partial_of(P, s, r, d, i) = r == 0 ? acc : 0.0;
}

__global__ void k_mass_pack(DevModel m, const uint32_t* nodes, ExchangePlan x, double* out) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= x.n_send) return;
  out[t] = m.mass[(int64_t)nodes[x.send_rows[t]] * m.dim];
}

__global__ void k_mass_sum_import(DevModel m, const uint32_t* nodes, ExchangePlan x,
                                  const double* recv) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= x.n_rows) return;
  const int64_t g = nodes[e];
  const double own = m.mass[g * m.dim];
  double M = 0.0;
  for (uint32_t j = x.sum_ptr[e]; j < x.sum_ptr[e + 1]; ++j) {
    const int32_t src = x.sum_src[j];
    M += src < 0 ? own : recv[src];
  }
  for (int c = 0; c < m.dim; ++c) m.mass[g * m.dim + c] = M;
  m.inv_mass[g] = 1. / M;
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

template <typename V>
__global__ void k_permute_rows(const uint32_t* perm, int64_t n, int width, const V* in, V* out,
                               bool scatter) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n * width) return;
  const int64_t i = t / width;
  const int c = (int)(t - i * width);
  const int64_t j = perm[i];
  if (scatter)
    out[j * width + c] = in[t];
  else
    out[t] = in[j * width + c];
}

// grid of the patch kernel: one CTA per patch, or a persistent grid of
// P.grid CTAs that stride over the patches
inline int grid_of(const DevPatches& p) {
  return (p.grid > 0 && p.grid < p.npatch) ? p.grid : p.npatch;
}

inline int blocks_of(int64_t n) { return (int)((n + kThreads - 1) / kThreads); }

template <int T, typename S>
cudaError_t launch_patch(const DevModel& m, const DevPatches& p, double dt, bool fext,
                         cudaStream_t s) {
  const SmemLayout lay = layout(p, ET<T>::dim, sizeof(S), p.nbuf);
  const int grid = grid_of(p);
  if (grid < p.npatch)
    return fext ? launch_pdl(k_patch_step<T, S, true, true>, grid, kThreads, lay.total, s, m, p, dt)
                : launch_pdl(k_patch_step<T, S, false, true>, grid, kThreads, lay.total, s, m, p, dt);
  return fext ? launch_pdl(k_patch_step<T, S, true, false>, grid, kThreads, lay.total, s, m, p, dt)
              : launch_pdl(k_patch_step<T, S, false, false>, grid, kThreads, lay.total, s, m, p, dt);
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

size_t patch_smem_bytes(const DevPatches& p, int dim, bool fp32, int nbuf) {
  return layout(p, dim, fp32 ? 4 : 8, nbuf).total;
}

int patch_buffers(const DevPatches& p, int type, bool fp32) {
  // CTAs per SM: 228 KB of shared memory, 1 KB reserved per CTA, and the
  // register budget the instantiation is built for
  int regs;
  switch (type) {
  case AKB_HEXAHEDRON_8: regs = fp32 ? PatchOccupancy<AKB_HEXAHEDRON_8, float>::value
                                     : PatchOccupancy<AKB_HEXAHEDRON_8, double>::value; break;
  case AKB_TETRAHEDRON_4: regs = fp32 ? PatchOccupancy<AKB_TETRAHEDRON_4, float>::value
                                      : PatchOccupancy<AKB_TETRAHEDRON_4, double>::value; break;
  case AKB_TRIANGLE_3: regs = fp32 ? PatchOccupancy<AKB_TRIANGLE_3, float>::value
                                   : PatchOccupancy<AKB_TRIANGLE_3, double>::value; break;
  default: regs = fp32 ? PatchOccupancy<AKB_SEGMENT_2, float>::value
                       : PatchOccupancy<AKB_SEGMENT_2, double>::value; break;
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

cudaError_t patch_finish_list(const DevModel& m, const DevPatches& p, double dt, bool fext,
                              cudaStream_t s) {
  if (p.nlist <= 0) return cudaSuccess;
  const int blocks = blocks_of(p.nlist * m.dim);
  switch (m.dim) {
  case 1: return fext ? launch_pdl(k_finish_list<1, true>, blocks, kThreads, 0, s, m, p, dt)
                      : launch_pdl(k_finish_list<1, false>, blocks, kThreads, 0, s, m, p, dt);
  case 2: return fext ? launch_pdl(k_finish_list<2, true>, blocks, kThreads, 0, s, m, p, dt)
                      : launch_pdl(k_finish_list<2, false>, blocks, kThreads, 0, s, m, p, dt);
  default: return fext ? launch_pdl(k_finish_list<3, true>, blocks, kThreads, 0, s, m, p, dt)
                       : launch_pdl(k_finish_list<3, false>, blocks, kThreads, 0, s, m, p, dt);
  }
}

int64_t patch_ke_parts(const DevPatches& p, int dim) {
  return p.npatch + (p.nlist > 0 ? blocks_of(p.nlist * dim) : 0);
}

cudaError_t patch_refresh_w(const DevModel& m, const DevPatches& p, double dt, cudaStream_t s) {
  if (m.nn == 0) return cudaSuccess;
  k_refresh_w<<<blocks_of(m.nn * m.dim), kThreads, 0, s>>>(m, p, dt);
  return cudaGetLastError();
}

cudaError_t patch_iface_export(const DevModel& m, const DevPatches& p, const uint32_t* shared,
                               const uint32_t* k, int64_t n, double* out, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_iface_export<<<blocks_of(n * m.dim), kThreads, 0, s>>>(p, shared, k, n, m.dim, out);
  return cudaGetLastError();
}

cudaError_t patch_iface_import(const DevModel& m, const DevPatches& p, const uint32_t* shared,
                               const uint32_t* k, int64_t n, const double* in, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_iface_import<<<blocks_of(n * m.dim), kThreads, 0, s>>>(p, shared, k, n, m.dim, in);
  return cudaGetLastError();
}

cudaError_t mass_export(const DevModel& m, const uint32_t* nodes, int64_t n, double* out,
                        cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_mass_export<<<blocks_of(n), kThreads, 0, s>>>(m, nodes, n, out);
  return cudaGetLastError();
}

cudaError_t mass_import(const DevModel& m, const uint32_t* nodes, int64_t n, const double* in,
                        cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_mass_import<<<blocks_of(n), kThreads, 0, s>>>(m, nodes, n, in);
  return cudaGetLastError();
}

cudaError_t patch_iface_pack(const DevModel& m, const DevPatches& p, const uint32_t* shared,
                             const uint32_t* k, const ExchangePlan& x, double* out,
                             cudaStream_t s) {
  if (x.n_send <= 0) return cudaSuccess;
  k_iface_pack<<<blocks_of(x.n_send * m.dim), kThreads, 0, s>>>(p, shared, k, x, m.dim, out);
  return cudaGetLastError();
}

cudaError_t patch_iface_sum_import(const DevModel& m, const DevPatches& p, const uint32_t* shared,
                                   const uint32_t* k, const ExchangePlan& x, const double* recv,
                                   cudaStream_t s) {
  if (x.n_rows <= 0) return cudaSuccess;
  k_iface_sum_import<<<blocks_of(x.n_rows * m.dim), kThreads, 0, s>>>(p, shared, k, x, m.dim, recv);
  return cudaGetLastError();
}

cudaError_t mass_pack(const DevModel& m, const uint32_t* nodes, const ExchangePlan& x,
                      double* out, cudaStream_t s) {
  if (x.n_send <= 0) return cudaSuccess;
  k_mass_pack<<<blocks_of(x.n_send), kThreads, 0, s>>>(m, nodes, x, out);
  return cudaGetLastError();
}

cudaError_t mass_sum_import(const DevModel& m, const uint32_t* nodes, const ExchangePlan& x,
                            const double* recv, cudaStream_t s) {
  if (x.n_rows <= 0) return cudaSuccess;
  k_mass_sum_import<<<blocks_of(x.n_rows), kThreads, 0, s>>>(m, nodes, x, recv);
  return cudaGetLastError();
}

cudaError_t permute_rows(const uint32_t* perm, int64_t n, int width, const double* in,
                         double* out, bool scatter, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_permute_rows<double><<<blocks_of(n * width), kThreads, 0, s>>>(perm, n, width, in, out, scatter);
  return cudaGetLastError();
}

cudaError_t permute_rows_u8(const uint32_t* perm, int64_t n, int width, const uint8_t* in,
                            uint8_t* out, bool scatter, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_permute_rows<uint8_t><<<blocks_of(n * width), kThreads, 0, s>>>(perm, n, width, in, out, scatter);
  return cudaGetLastError();
}

}  // namespace akb
