// akb_mlp.cu -- the learned RVE surrogate: a multilayer perceptron
// (inputs <= 16, L hidden layers of width <= 256 with SiLU, outputs <= 16)
// trained and evaluated with 5th-generation tensor cores.
//
// Every GEMM is a tcgen05.mma (kind::f16, BF16 operands, FP32 accumulators
// in tensor memory), issued by one thread of the CTA, with operands in shared
// memory in the canonical no-swizzle layout: 8 x 8 BF16 core matrices of 128
// contiguous bytes. A row-major (rows, cols) tile is stored core matrix by
// core matrix, row group major:
//   offset(r, c) = ((r / 8) (cols / 8) + c / 8) 128 + (r % 8) 16 + (c % 8) 2,
// which is a K-major operand (rows = M or N, cols = K; leading byte offset
// 128, stride byte offset 16 cols) and, read the other way, an MN-major one
// (MN = cols, K = rows; stride byte offset 128, leading byte offset 16 cols).
// Activations, their gradients and the weights are kept in this layout in
// global memory too, so staging a tile is a flat copy.
//
//   forward  (one CTA per 128 samples): H_l = SiLU(H_{l-1} W_l^T + b_l),
//            A = H_{l-1} (K-major), B = W_l (N x K, K-major);
//   backward (one CTA per 128 samples): dH_{l-1} = dZ_l W_l,
//            A = dZ_l (K-major), B = W_l^T (K-major);
//   weight gradients (a CTA per range of tiles): dW_l = dZ_l^T H_{l-1},
//            A = dZ_l and B = H_{l-1} both MN-major (samples are K);
//   Adam on FP32 master weights, then the BF16 copies are repacked.
// Weights and activation tiles are staged by TMA bulk copies completing on an
// mbarrier (no multicast); in the forward and backward passes the next
// layer's weights are copied while the current layer's epilogue runs. Each
// wait (copy or MMA completion) is bounded: past the limit the kernel raises
// the error flag, waits (bounded) for what is still in flight, frees its
// tensor memory and returns.
#include <cuda_bf16.h>

#include <cmath>
#include <memory>
#include <vector>

#include "../../include/akb_fe2.h"
#include "akb_internal.cuh"

namespace akb {
namespace mlp {

constexpr int kTile = 128;      // samples per CTA (UMMA M)
constexpr int kMaxWidth = 256;  // one TMEM accumulator of 256 FP32 columns
constexpr int kIO = 16;         // padded input / output width
constexpr int kMaxLayers = 6;   // linear layers
constexpr int kThreads = 128;   // weight-gradient kernel: one thread per TMEM lane
constexpr int kFwdThreads = 256;  // forward / backward: two threads per sample row, each
                                  // reading half of the accumulator columns
constexpr uint32_t kWaitLimit = 1u << 20;

struct Net {
  int nl;                       // linear layers
  int nin, nout;                // real input / output counts
  int K[kMaxLayers], N[kMaxLayers];    // padded shapes (K[0] = N[nl-1] = 16)
  int Kr[kMaxLayers], Nr[kMaxLayers];  // real shapes
  const __nv_bfloat16* W[kMaxLayers];  // packed N x K
  const __nv_bfloat16* Wt[kMaxLayers]; // packed K x N
  const float* b[kMaxLayers];          // N (zero past the real outputs)
  float in_shift[kIO], in_scale[kIO], out_shift[kIO], out_scale[kIO];
  int* error;
};

// Training workspace: packed BF16 layer inputs act[l] (act[0] = the
// normalised input, 16 columns), FP32 pre-activations z[l] of the hidden
// layers ([rows][N]), packed BF16 gradients dz[l] of the layers'
// pre-activations (dz[nl-1] = dY), normalised outputs, per-tile losses.
struct Bufs {
  unsigned char* act[kMaxLayers];
  float* z[kMaxLayers];
  unsigned char* dz[kMaxLayers];
  float* ynorm;
  float* loss_tiles;
};

__host__ __device__ inline size_t pk_off(int r, int c, int cols) {
  return ((size_t)(r >> 3) * (cols >> 3) + (c >> 3)) * 128 + (r & 7) * 16 + (c & 7) * 2;
}

// ------------------------------------------------------------ PTX wrappers
__device__ inline uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (no swizzle): start address, leading and
// stride byte offsets, descriptor version 1.
__device__ inline uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: BF16 x BF16 -> FP32, M x N.
__host__ __device__ constexpr uint32_t idesc(int M, int N, bool a_mn, bool b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) |
         ((b_mn ? 1u : 0u) << 16) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ inline void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(id), "r"(acc)
      : "memory");
}
__device__ inline void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}
__device__ inline void mbar_init(uint32_t a) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
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
// One-dimensional bulk copy global -> this CTA's shared memory (TMA engine,
// no multicast), completing `bytes` of transaction on mbarrier `mbar`; the
// issuing thread first arms the barrier with the expected byte count.
__device__ inline void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(mbar),
               "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}
// Two bulk copies on one barrier (both byte counts armed at once).
__device__ inline void bulk_load2(uint32_t d0, const void* s0, uint32_t b0, uint32_t d1,
                                  const void* s1, uint32_t b1, uint32_t mbar) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(mbar),
               "r"(b0 + b1)
               : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d0),
               "l"(s0), "r"(b0), "r"(mbar)
               : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d1),
               "l"(s1), "r"(b1), "r"(mbar)
               : "memory");
}

__device__ inline void tmem_alloc(uint32_t holder, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(holder), "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ inline void tmem_free(uint32_t taddr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}
__device__ inline void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ inline void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ inline void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 (or 16) FP32 columns of this warp's 32 TMEM lanes; the wait is in the
// same statement so no use of the registers can be scheduled before it.
__device__ inline void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
      "%30, %31}, [%32];\n\ttcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}
__device__ inline void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];\n\ttcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// SiLU and its derivative (the result is rounded to BF16 anyway: fast
// division; exp(-z) overflowing gives the limits 0 and 0)
// The logistic function as 1/2 + tanh(z/2)/2 with the hardware tanh
// approximation: one special-function operation per element (the exp and
// reciprocal form takes two), which bounds the epilogue.
__device__ inline float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ inline float sigmoid(float z) { return fmaf(0.5f, tanh_approx(0.5f * z), 0.5f); }
__device__ inline float silu(float z) { return z * sigmoid(z); }
__device__ inline float dsilu(float z) {
  const float s = sigmoid(z);
  return s * (1.0f + z * (1.0f - s));
}

__device__ inline uint32_t pack2(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}

// 8 consecutive values (columns c..c+7, c % 8 == 0) of row r as one 16-byte
// store into a packed tile with `cols` columns.
__device__ inline void store8(unsigned char* tile, int r, int c, int cols, const float* v) {
  uint4 q;
  q.x = pack2(v[0], v[1]);
  q.y = pack2(v[2], v[3]);
  q.z = pack2(v[4], v[5]);
  q.w = pack2(v[6], v[7]);
  *reinterpret_cast<uint4*>(tile + pk_off(r, c, cols)) = q;
}


// Issues A (M x K) times B^T (N x K) into tmem_d, K in steps of 16, both
// K-major packed tiles (A with K columns, B with K columns), then commits.
__device__ inline void gemm_kmajor(uint32_t tmem_d, uint32_t a, uint32_t b, int K, int N) {
  const uint32_t id = idesc(kTile, N, false, false);
  for (int s = 0; s < K / 16; ++s)
    mma(tmem_d, sdesc(a + s * 256, 128, 16 * K), sdesc(b + s * 256, 128, 16 * K), id, s > 0);
}

struct Shared {
  unsigned char* act;  // 128 x 256 packed BF16 (64 KB)
  unsigned char* wgt;  // 256 x 256 packed BF16 (128 KB)
  float* bias;         // forward: every layer's biases (kMaxWidth per layer); backward: 256
  uint64_t* mbar;      // [0] MMA completion, [1] weights landed
  uint32_t* tmem_holder;
  double* hnorm;       // 128: |H| of each row (stress mode)
};

constexpr size_t kActBytes = (size_t)kTile * kMaxWidth * 2;
constexpr size_t kWgtBytes = (size_t)kMaxWidth * kMaxWidth * 2;
// The forward pass stages a layer's weights in slices of output rows (a
// contiguous block of the packed N x K matrix; 64 rows of a 256-wide layer),
// so that its shared memory (~97 KB) lets two CTAs share an SM: one CTA's
// epilogue (TMEM -> bias -> SiLU -> BF16) runs while the other's MMAs use
// the tensor cores.
constexpr size_t kSliceBytes = (size_t)64 * kMaxWidth * 2;
constexpr size_t kTail = kMaxLayers * kMaxWidth * 4 + 64 + kTile * 8;  // biases, barriers, |H|
constexpr size_t kFwdSmem = kActBytes + kSliceBytes + kTail;
constexpr size_t kBwdSmem = kActBytes + kWgtBytes + kTail;

__device__ inline Shared carve(unsigned char* smem, size_t wgt_bytes) {
  Shared s;
  s.act = smem;
  s.wgt = smem + kActBytes;
  unsigned char* t = smem + kActBytes + wgt_bytes;
  s.bias = reinterpret_cast<float*>(t);
  s.mbar = reinterpret_cast<uint64_t*>(t + kMaxLayers * kMaxWidth * 4);
  s.tmem_holder = reinterpret_cast<uint32_t*>(s.mbar + 2);
  s.hnorm = reinterpret_cast<double*>(t + kMaxLayers * kMaxWidth * 4 + 64);
  return s;
}

// Stress mode of the forward pass (MaterialFE2 with the surrogate): the
// inputs are displacement gradients H ([nb][9], column-major per point), the
// features (H / r, log r) with r = max(|H|, kHMin) are formed in the kernel,
// the outputs are P = |H| net(.) ([nb][9], column-major), and the points
// outside the training envelope (max |H_ij| > amplitude or det(I + H) <
// min_det) are appended to index[] (count[0] entries; the caller zeroes it).
constexpr double kHMin = 1e-8;
struct StressArgs {
  double amplitude = 0.0, min_det = 0.0;
  int32_t* index = nullptr;
  int32_t* count = nullptr;
};

__device__ inline double det_i_plus(const double* H) {  // det(I + H), H column-major
  const double a = 1.0 + H[0], b = H[3], c = H[6];
  const double d = H[1], e = 1.0 + H[4], f = H[7];
  const double g = H[2], h = H[5], i = 1.0 + H[8];
  return a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
}

// Forward pass of one tile of 128 samples. x: [nb][nin] FP64 raw inputs.
// TRAIN stores the packed BF16 input and hidden activations (act[l], tile
// major), the pre-activations Z (z[l], [nb_pad][N] FP32) and the normalised
// outputs (ynorm, [nb_pad][16] FP32); otherwise y: [nb][nout] FP64 outputs.
// The normalised inputs of row r of a tile (columns 8 half .. 8 half + 7 of
// 16) into the packed A tile `act`: x's columns, or in stress mode the
// features (H / r, log r) of the row's displacement gradient, whose |H| goes
// to hnorm[r] and whose envelope test (by the half-0 threads, whole warps)
// appends the row to the fallback list.
template <bool STRESS>
__device__ inline void stage_inputs(const Net& net, int64_t nb, const double* __restrict__ x,
                                    unsigned char* act, double* hnorm, int r, int half,
                                    int64_t row, int tid, const StressArgs& sa, float* v) {
  if (STRESS) {
    double H[9], n2 = 0.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      H[k] = row < nb ? x[row * 9 + k] : 0.0;
      n2 += H[k] * H[k];
    }
    const double hn = sqrt(n2), rr = fmax(hn, kHMin);
#pragma unroll
    for (int q = 0; q < 8; ++q) {  // column j = 8 half + q: H_j / r (j < 9), log r (j = 9)
      const int j = 8 * half + q;
      const double f = half == 0 ? H[q] / rr : (q == 0 ? H[8] / rr : (q == 1 ? log(rr) : 0.0));
      v[q] = (j < net.nin && row < nb) ? (float)((f - net.in_shift[j]) * net.in_scale[j]) : 0.0f;
    }
    store8(act, r, 8 * half, 16, v);
    if (half == 0) {  // whole warps: one row per lane
      hnorm[r] = hn;
      if (sa.count) {
        double hmax = 0.0;
#pragma unroll
        for (int k = 0; k < 9; ++k) hmax = fmax(hmax, fabs(H[k]));
        const bool out = row < nb && (hmax > sa.amplitude || det_i_plus(H) < sa.min_det);
        const unsigned mask = __ballot_sync(0xffffffffu, out);
        int base = 0;
        if ((tid & 31) == 0 && mask) base = atomicAdd(sa.count, __popc(mask));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (out) sa.index[base + __popc(mask & ((1u << (tid & 31)) - 1u))] = (int32_t)row;
      }
    }
  } else {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int j = 8 * half + q;
      float t = 0.0f;
      if (j < net.nin && row < nb) t = (float)((x[row * net.nin + j] - net.in_shift[j]) * net.in_scale[j]);
      v[q] = t;
    }
    store8(act, r, 8 * half, 16, v);
  }
}

// Output rows per weight slice of layer l: as many as the buffer holds (a
// multiple of 16: whole row groups, a valid MMA N), at most the layer's N.
__device__ inline int slice_rows(const Net& net, int l) {
  return min(net.N[l], (int)(kSliceBytes / (2 * (size_t)net.K[l])) & ~15);
}
// Rows of slice j of layer l, its bytes and its source (rows [rows0 j, ...)
// of the packed N x K matrix are one contiguous block).
__device__ inline int slice_n(const Net& net, int l, int j) {
  return min(slice_rows(net, l), net.N[l] - slice_rows(net, l) * j);
}
__device__ inline uint32_t slice_bytes(const Net& net, int l, int j) {
  return (uint32_t)(slice_n(net, l, j) * net.K[l] * 2);
}
__device__ inline const void* slice_src(const Net& net, int l, int j) {
  return reinterpret_cast<const unsigned char*>(net.W[l]) +
         (size_t)slice_rows(net, l) * j * net.K[l] * 2;
}

template <bool TRAIN, bool STRESS = false>
__global__ void __launch_bounds__(kFwdThreads, 2)
    k_forward(Net net, int64_t nb, const double* __restrict__ x, double* __restrict__ y,
              Bufs bufs, StressArgs sa = StressArgs{}) {
  extern __shared__ __align__(1024) unsigned char smem[];
  Shared s = carve(smem, kSliceBytes);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int r = tid & (kTile - 1), half = tid >> 7;  // row in the tile, column half
  const int64_t tile = blockIdx.x;
  const int64_t row = tile * kTile + r;
  const uint32_t mb_mma = saddr(s.mbar), mb_w = saddr(s.mbar + 1);
  if (warp == 0) tmem_alloc(saddr(s.tmem_holder), 256);
  if (tid == 0) {
    mbar_init(mb_mma);
    mbar_init(mb_w);
    bulk_load(saddr(s.wgt), slice_src(net, 0, 0), slice_bytes(net, 0, 0), mb_w);
  }
  // every layer's biases, once (the first barrier below publishes them)
  for (int l = 0; l < net.nl; ++l)
    for (int c = tid; c < net.N[l]; c += kFwdThreads) s.bias[l * kMaxWidth + c] = net.b[l][c];
  // inputs, normalised, padded to 16 columns (8 per thread)
  {
    float v[8];
    stage_inputs<STRESS>(net, nb, x, s.act, s.hnorm, r, half, row, tid, sa, v);
    if (TRAIN) store8(bufs.act[0] + tile * (size_t)kTile * 16 * 2, r, 8 * half, 16, v);
  }
  fence_smem_async();  // the A tile, written by this thread, before the MMAs read it
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *s.tmem_holder;
  const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
  // A layer's weights arrive slice by slice (TMA bulk into one buffer):
  // slice j's MMAs write accumulator columns [kSlice j, ...); the next slice
  // (or the next layer's first, during this layer's epilogue) is copied as
  // soon as they completed.
  uint32_t pm = 0, pw = 0;
  bool ok = true, w_pending = true, m_pending = false;
  for (int l = 0; l < net.nl && ok; ++l) {
    const int K = net.K[l], N = net.N[l];
    const int rows0 = slice_rows(net, l);
    const int nslices = (N + rows0 - 1) / rows0;
    const float* bias = s.bias + l * kMaxWidth;
    for (int j = 0; j < nslices && ok; ++j) {
      ok = mbar_wait(mb_w, pw);
      if (!ok) break;
      pw ^= 1;
      w_pending = false;
      if (tid == 0) {
        fence_after();
        gemm_kmajor(tmem + rows0 * j, saddr(s.act), saddr(s.wgt), K, slice_n(net, l, j));
        mma_commit(mb_mma);
      }
      m_pending = true;
      ok = mbar_wait(mb_mma, pm);
      if (!ok) break;
      pm ^= 1;
      m_pending = false;
      fence_after();
      if (j + 1 < nslices) {
        if (tid == 0) bulk_load(saddr(s.wgt), slice_src(net, l, j + 1), slice_bytes(net, l, j + 1), mb_w);
        w_pending = true;
      } else if (l + 1 < net.nl) {
        if (tid == 0) bulk_load(saddr(s.wgt), slice_src(net, l + 1, 0), slice_bytes(net, l + 1, 0), mb_w);
        w_pending = true;
      }
    }
    if (!ok) break;
    const bool last = l == net.nl - 1;
    if (!last) {
      for (int c0 = half * (N >> 1); c0 < (half + 1) * (N >> 1); c0 += 32) {
        float v[32];
        tmem_ld32(tmem + lane_base + c0, v);
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] += bias[c0 + j];
        if (TRAIN && row < nb) {  // the pre-activations: eight 16-byte stores
          float4* z4 = reinterpret_cast<float4*>(bufs.z[l] + (size_t)row * N + c0);
#pragma unroll
          for (int q = 0; q < 8; ++q)
            z4[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        }
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = silu(v[j]);
#pragma unroll
        for (int q = 0; q < 4; ++q) store8(s.act, r, c0 + 8 * q, N, v + 8 * q);
        if (TRAIN) {
          unsigned char* g = bufs.act[l + 1] + tile * (size_t)kTile * N * 2;
#pragma unroll
          for (int q = 0; q < 4; ++q) store8(g, r, c0 + 8 * q, N, v + 8 * q);
        }
      }
    } else if (half == 0) {  // warp-uniform: warps 0-3 read the 16 output columns
      float v[16];
      tmem_ld16(tmem + lane_base, v);
      if (row < nb) {
        const double scale = STRESS ? s.hnorm[r] : 1.0;
        for (int j = 0; j < 16; ++j) {
          const float yy = v[j] + bias[j];
          if (TRAIN) bufs.ynorm[row * 16 + j] = yy;
          if (!TRAIN && j < net.nout)
            y[row * net.nout + j] = scale * ((double)yy * net.out_scale[j] + net.out_shift[j]);
        }
      }
    }
    fence_smem_async();  // the next layer's A tile before its MMAs
    fence_before();
    __syncthreads();  // TMEM read and activations written before the next MMA
  }
  if (!ok) {  // drain the copy / MMA still in flight before leaving (bounded)
    if (w_pending) mbar_wait(mb_w, pw);
    if (m_pending) mbar_wait(mb_mma, pm);
    if (tid == 0) atomicExch(net.error, 1);
  }
  __syncthreads();
  if (warp == 0) tmem_free(tmem, 256);
}

// Backward pass of one tile: dY from the normalised outputs and targets
// (loss = mean over samples and outputs of (y - t)^2), then
// dZ_{l-1} = (dZ_l W_l) * SiLU'(Z_{l-1}) down to the first hidden layer.
// Stores packed BF16 dY (dz[nl-1]) and dZ (dz[l]) tiles and the tile's loss.
__global__ void __launch_bounds__(kFwdThreads, 1)
    k_backward(Net net, int64_t nb, const double* __restrict__ target, Bufs bufs) {
  extern __shared__ __align__(1024) unsigned char smem[];
  Shared s = carve(smem, kWgtBytes);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int r = tid & (kTile - 1), half = tid >> 7;  // row in the tile, column half
  const int64_t tile = blockIdx.x;
  const int64_t row = tile * kTile + r;
  const uint32_t mb_mma = saddr(s.mbar), mb_w = saddr(s.mbar + 1);
  const int L = net.nl;
  if (warp == 0) tmem_alloc(saddr(s.tmem_holder), 256);
  if (tid == 0) {
    mbar_init(mb_mma);
    mbar_init(mb_w);
    bulk_load(saddr(s.wgt), net.Wt[L - 1], (uint32_t)(net.N[L - 1] * net.K[L - 1] * 2), mb_w);
  }
  {
    float d[8];  // 8 of the 16 (padded) outputs per thread
    float sq = 0.0f;
    const float scale = 2.0f / (float)((double)nb * net.nout);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int j = 8 * half + q;
      float e = 0.0f;
      if (row < nb && j < net.nout) {
        const float t = (float)((target[row * net.nout + j] - net.out_shift[j]) / net.out_scale[j]);
        e = bufs.ynorm[row * 16 + j] - t;
        sq += e * e;
      }
      d[q] = scale * e;
    }
    store8(s.act, r, 8 * half, 16, d);
    store8(bufs.dz[L - 1] + tile * (size_t)kTile * 16 * 2, r, 8 * half, 16, d);
    // tile loss: warp sums, then the 8 warps in order
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
    float* red = s.bias;
    if ((tid & 31) == 0) red[warp] = sq;
    __syncthreads();
    if (tid == 0) {
      float t = 0.0f;
      for (int w = 0; w < kFwdThreads / 32; ++w) t += red[w];
      bufs.loss_tiles[tile] = t;
    }
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *s.tmem_holder;
  const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
  uint32_t pm = 0, pw = 0;
  bool ok = true, w_pending = true, m_pending = false;
  for (int l = L - 1; l >= 1 && ok; --l) {
    const int K = net.N[l], N = net.K[l];  // reduce over the layer's outputs
    fence_smem_async();
    __syncthreads();
    ok = mbar_wait(mb_w, pw);
    if (!ok) break;
    pw ^= 1;
    w_pending = false;
    if (tid == 0) {
      fence_after();
      gemm_kmajor(tmem, saddr(s.act), saddr(s.wgt), K, N);
      mma_commit(mb_mma);
    }
    m_pending = true;
    ok = mbar_wait(mb_mma, pm);
    if (!ok) break;
    pm ^= 1;
    m_pending = false;
    fence_after();
    if (l - 1 >= 1) {  // next layer's W^T, copied while this epilogue runs
      if (tid == 0)
        bulk_load(saddr(s.wgt), net.Wt[l - 1], (uint32_t)(net.N[l - 1] * net.K[l - 1] * 2), mb_w);
      w_pending = true;
    }
    unsigned char* g = bufs.dz[l - 1] + tile * (size_t)kTile * N * 2;
    for (int c0 = half * (N >> 1); c0 < (half + 1) * (N >> 1); c0 += 32) {
      float v[32], zz[32];
      tmem_ld32(tmem + lane_base + c0, v);
      if (row < nb) {  // the row's 32 pre-activations: eight 16-byte loads
        const float4* z4 = reinterpret_cast<const float4*>(bufs.z[l - 1] + (size_t)row * N + c0);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const float4 z = z4[q];
          zz[4 * q] = z.x;
          zz[4 * q + 1] = z.y;
          zz[4 * q + 2] = z.z;
          zz[4 * q + 3] = z.w;
        }
      }
#pragma unroll
      for (int j = 0; j < 32; ++j) v[j] = row < nb ? v[j] * dsilu(zz[j]) : 0.0f;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        store8(s.act, r, c0 + 8 * q, N, v + 8 * q);
        store8(g, r, c0 + 8 * q, N, v + 8 * q);
      }
    }
    fence_before();
    __syncthreads();
  }
  if (!ok || w_pending) {  // drain what is still in flight before leaving (bounded)
    if (w_pending) mbar_wait(mb_w, pw);
    if (m_pending) mbar_wait(mb_mma, pm);
    if (!ok && tid == 0) atomicExch(net.error, 1);
  }
  __syncthreads();
  if (warp == 0) tmem_free(tmem, 256);
}

// Partial weight gradients G[m][n] = sum_s A[s][m] B[s][n] over the tiles
// [tile0, tile1) of this CTA: A tiles with ca columns (128 or 256), B tiles
// with cb columns (16..256); written to part[blockIdx.x][ca][cb].
__global__ void __launch_bounds__(kThreads, 1)
    k_wgrad(const unsigned char* __restrict__ A, int ca, const unsigned char* __restrict__ B,
            int cb, int64_t ntiles, int tiles_per_cta, float* part, int* error) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* sa = smem;
  unsigned char* sb = smem + (size_t)kTile * kMaxWidth * 2;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sb + (size_t)kTile * kMaxWidth * 2);
  uint32_t* holder = reinterpret_cast<uint32_t*>(mbar + 2);
  const uint32_t mb_mma = saddr(mbar), mb_t = saddr(mbar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) tmem_alloc(saddr(holder), 512);
  if (tid == 0) {
    mbar_init(mb_mma);
    mbar_init(mb_t);
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *holder;
  const int64_t t0 = (int64_t)blockIdx.x * tiles_per_cta;
  const int64_t t1 = t0 + tiles_per_cta < ntiles ? t0 + tiles_per_cta : ntiles;
  const int halves = ca / kTile;
  const uint32_t id = idesc(kTile, cb, true, true);
  uint32_t pm = 0, pt = 0;
  bool ok = true, t_pending = false, m_pending = false;
  for (int64_t t = t0; t < t1 && ok; ++t) {
    // both tiles by TMA bulk copies (the previous tile's MMAs have completed)
    if (tid == 0)
      bulk_load2(saddr(sa), A + t * (size_t)kTile * ca * 2, (uint32_t)(kTile * ca * 2), saddr(sb),
                 B + t * (size_t)kTile * cb * 2, (uint32_t)(kTile * cb * 2), mb_t);
    t_pending = true;
    ok = mbar_wait(mb_t, pt);
    if (!ok) break;
    pt ^= 1;
    t_pending = false;
    if (tid == 0) {
      fence_after();
      for (int h = 0; h < halves; ++h)
        for (int s = 0; s < kTile / 16; ++s)
          mma(tmem + h * cb,
              sdesc(saddr(sa) + h * (kTile / 8) * 128 + s * 2 * 16 * ca, 16 * ca, 128),
              sdesc(saddr(sb) + s * 2 * 16 * cb, 16 * cb, 128), id, (t > t0 || s > 0) ? 1u : 0u);
      mma_commit(mb_mma);
    }
    m_pending = true;
    ok = mbar_wait(mb_mma, pm);
    if (!ok) break;
    pm ^= 1;
    m_pending = false;
    fence_after();
    __syncthreads();  // shared tiles free for the next copy
  }
  if (ok && t1 > t0) {
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    float* out = part + (size_t)blockIdx.x * ca * cb;
    for (int h = 0; h < halves; ++h)
      for (int c0 = 0; c0 < cb; c0 += 16) {
        float v[16];
        tmem_ld16(tmem + lane_base + h * cb + c0, v);
        const int m = h * kTile + tid;
        float4* o4 = reinterpret_cast<float4*>(out + (size_t)m * cb + c0);  // four 16-byte stores
#pragma unroll
        for (int q = 0; q < 4; ++q)
          o4[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
      }
  } else if (t1 <= t0) {
    float* out = part + (size_t)blockIdx.x * ca * cb;
    for (int k = tid; k < ca * cb; k += kThreads) out[k] = 0.0f;
  }
  if (!ok) {  // drain what is still in flight before leaving (bounded)
    if (t_pending) mbar_wait(mb_t, pt);
    if (m_pending) mbar_wait(mb_mma, pm);
    if (tid == 0) atomicExch(error, 1);
  }
  fence_before();
  __syncthreads();
  if (warp == 0) tmem_free(tmem, 512);
}

// grad[m][n] (real rows/cols, row stride ncols) = sum over CTAs of the
// partials, in CTA order; TRANSPOSE reads part[.][n][m].
__global__ void k_sum_partials(const float* part, int nparts, int ca, int cb, int rows, int cols,
                               bool transpose, float* grad) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= rows * cols) return;
  const int m = k / cols, n = k % cols;
  const size_t idx = transpose ? (size_t)n * cb + m : (size_t)m * cb + n;
  float acc = 0.0f;
  for (int p = 0; p < nparts; ++p) acc += part[(size_t)p * ca * cb + idx];
  grad[k] = acc;
}

// Bias gradient of a layer: sum over samples of the packed BF16 dZ tiles.
__global__ void k_bias_grad(const unsigned char* dz, int cols, int real, int64_t ntiles,
                            float* grad) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= real) return;
  float acc = 0.0f;
  for (int64_t t = 0; t < ntiles; ++t) {
    const unsigned char* tile = dz + t * (size_t)kTile * cols * 2;
    for (int r = 0; r < kTile; ++r)
      acc += __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(tile + pk_off(r, n, cols)));
  }
  grad[n] = acc;
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters.
__global__ void k_adam(float* p, const float* g, float* m1, float* m2, int64_t n, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float gk = g[k];
  const float a = b1 * m1[k] + (1.0f - b1) * gk;
  const float b = b2 * m2[k] + (1.0f - b2) * gk * gk;
  m1[k] = a;
  m2[k] = b;
  p[k] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

// Packed BF16 W (N x K) and W^T (K x N) of one layer from the real FP32
// row-major weights (nr x kr) and bias, zero padded.
__global__ void k_pack(const float* w, const float* bias, int nr, int kr, int N, int K,
                       __nv_bfloat16* W, __nv_bfloat16* Wt, float* b) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < N) b[k] = k < nr ? bias[k] : 0.0f;
  if (k >= N * K) return;
  const int r = k / K, c = k % K;
  const float v = (r < nr && c < kr) ? w[(size_t)r * kr + c] : 0.0f;
  const __nv_bfloat16 h = __float2bfloat16_rn(v);
  *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<unsigned char*>(W) + pk_off(r, c, K)) = h;
  *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<unsigned char*>(Wt) + pk_off(c, r, N)) = h;
}

}  // namespace mlp
}  // namespace akb

using namespace akb;
using namespace akb::mlp;

struct akb_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool owns_stream = false;
  Net net{};
  int64_t nparams = 0;
  std::vector<int64_t> w_off, b_off;
  float *d_params = nullptr, *d_grad = nullptr, *d_m1 = nullptr, *d_m2 = nullptr;
  int* d_error = nullptr;
  std::vector<void*> allocs;  // device memory owned
  int64_t adam_step = 0;
  // training workspace
  int64_t cap_tiles = 0;
  std::vector<void*> work;
  Bufs bufs{};
  float* d_part = nullptr;
  size_t part_cap = 0;
  float* h_loss = nullptr;  // pinned, one float per tile
};

namespace {

template <typename T>
cudaError_t dmalloc(std::vector<void*>& owner, T** p, size_t count) {
  cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T));
  if (e == cudaSuccess) owner.push_back(*p);
  return e;
}

cudaError_t set_smem(const void* fn, size_t bytes) {
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

constexpr size_t kWgradSmem = 2 * (size_t)kTile * kMaxWidth * 2 + 64;  // tiles, 2 barriers, TMEM address

akb_status repack(akb_mlp* m) {
  for (int l = 0; l < m->net.nl; ++l) {
    const Net& n = m->net;
    const int total = n.N[l] * n.K[l];
    k_pack<<<(total + 255) / 256, 256, 0, m->stream>>>(
        m->d_params + m->w_off[l], m->d_params + m->b_off[l], n.Nr[l], n.Kr[l], n.N[l], n.K[l],
        const_cast<__nv_bfloat16*>(n.W[l]), const_cast<__nv_bfloat16*>(n.Wt[l]),
        const_cast<float*>(n.b[l]));
    AKB_CUDA_TRY(cudaGetLastError());
  }
  return AKB_OK;
}

akb_status ensure_workspace(akb_mlp* m, int64_t ntiles) {
  if (ntiles <= m->cap_tiles) return AKB_OK;
  for (void* p : m->work) cudaFree(p);
  m->work.clear();
  const Net& n = m->net;
  const size_t rows = (size_t)ntiles * kTile;
  Bufs b{};
  for (int l = 0; l < n.nl; ++l) {
    AKB_CUDA_TRY(dmalloc(m->work, &b.act[l], rows * n.K[l] * 2));
    AKB_CUDA_TRY(dmalloc(m->work, &b.dz[l], rows * n.N[l] * 2));
    if (l < n.nl - 1) AKB_CUDA_TRY(dmalloc(m->work, &b.z[l], rows * n.N[l]));
  }
  AKB_CUDA_TRY(dmalloc(m->work, &b.ynorm, rows * 16));
  AKB_CUDA_TRY(dmalloc(m->work, &b.loss_tiles, (size_t)ntiles));
  m->bufs = b;
  if (m->h_loss) cudaFreeHost(m->h_loss);
  AKB_CUDA_TRY(cudaMallocHost((void**)&m->h_loss, ntiles * sizeof(float)));
  m->cap_tiles = ntiles;
  return AKB_OK;
}

// Forward, backward and gradient assembly of one batch; *loss = mean
// squared error of the normalised outputs.
akb_status gradients(akb_mlp* m, int64_t nb, const double* x, const double* target, float* loss) {
  const int64_t ntiles = (nb + kTile - 1) / kTile;
  akb_status st;
  if ((st = ensure_workspace(m, ntiles)) != AKB_OK) return st;
  const Net& n = m->net;
  AKB_CUDA_TRY(cudaMemsetAsync(m->d_error, 0, sizeof(int), m->stream));
  k_forward<true><<<(unsigned)ntiles, kFwdThreads, kFwdSmem, m->stream>>>(n, nb, x, nullptr, m->bufs);
  AKB_CUDA_TRY(cudaGetLastError());
  k_backward<<<(unsigned)ntiles, kFwdThreads, kBwdSmem, m->stream>>>(n, nb, target, m->bufs);
  AKB_CUDA_TRY(cudaGetLastError());
  // at least four tiles per CTA: each CTA writes a whole ca x cb partial,
  // so a few more tiles per CTA cost less than more partials to write and sum
  const int tpc = (int)std::min<int64_t>(ntiles, std::max<int64_t>(4, (ntiles + 147) / 148));
  const int nparts = (int)((ntiles + tpc - 1) / tpc);
  for (int l = 0; l < n.nl; ++l) {
    const bool last = l == n.nl - 1;
    // dW_l = dZ_l^T H_l (the output layer as its transpose: M must be 128 or 256)
    const unsigned char* A = last ? m->bufs.act[l] : m->bufs.dz[l];
    const unsigned char* B = last ? m->bufs.dz[l] : m->bufs.act[l];
    const int ca = last ? n.K[l] : n.N[l], cb = last ? n.N[l] : n.K[l];
    const size_t need = (size_t)nparts * ca * cb;
    if (need > m->part_cap) {
      if (m->d_part) cudaFree(m->d_part);
      m->d_part = nullptr;
      AKB_CUDA_TRY(cudaMalloc((void**)&m->d_part, need * sizeof(float)));
      m->part_cap = need;
    }
    k_wgrad<<<nparts, kThreads, kWgradSmem, m->stream>>>(A, ca, B, cb, ntiles, tpc, m->d_part,
                                                         m->d_error);
    AKB_CUDA_TRY(cudaGetLastError());
    const int cnt = n.Nr[l] * n.Kr[l];
    k_sum_partials<<<(cnt + 255) / 256, 256, 0, m->stream>>>(m->d_part, nparts, ca, cb, n.Nr[l],
                                                             n.Kr[l], last, m->d_grad + m->w_off[l]);
    AKB_CUDA_TRY(cudaGetLastError());
    k_bias_grad<<<(n.Nr[l] + 127) / 128, 128, 0, m->stream>>>(m->bufs.dz[l], n.N[l], n.Nr[l],
                                                               ntiles, m->d_grad + m->b_off[l]);
    AKB_CUDA_TRY(cudaGetLastError());
  }
  AKB_CUDA_TRY(cudaMemcpyAsync(m->h_loss, m->bufs.loss_tiles, ntiles * sizeof(float),
                               cudaMemcpyDeviceToHost, m->stream));
  int err = 0;
  AKB_CUDA_TRY(cudaMemcpyAsync(&err, m->d_error, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
  AKB_CUDA_TRY(cudaStreamSynchronize(m->stream));
  if (err) return fail(AKB_ERR_TIMEOUT, "tensor-core MMA completion wait timed out");
  double acc = 0.0;
  for (int64_t t = 0; t < ntiles; ++t) acc += m->h_loss[t];
  if (loss) *loss = (float)(acc / ((double)nb * n.nout));
  return AKB_OK;
}

}  // namespace

extern "C" {

akb_status akb_mlp_create(int32_t nb_inputs, int32_t nb_outputs, int32_t width,
                          int32_t nb_hidden, int32_t device, void* stream, akb_mlp** out) {
  if (!out) return fail(AKB_ERR_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  if (nb_inputs < 1 || nb_inputs > kIO || nb_outputs < 1 || nb_outputs > kIO)
    return fail(AKB_ERR_UNSUPPORTED, "1..16 inputs and outputs");
  if (width != 128 && width != 256) return fail(AKB_ERR_UNSUPPORTED, "hidden width 128 or 256");
  if (nb_hidden < 1 || nb_hidden > kMaxLayers - 1)
    return fail(AKB_ERR_UNSUPPORTED, "1..5 hidden layers");
  auto m = std::make_unique<akb_mlp>();
  Net& n = m->net;
  n.nl = nb_hidden + 1;
  n.nin = nb_inputs;
  n.nout = nb_outputs;
  for (int l = 0; l < n.nl; ++l) {
    n.K[l] = l == 0 ? kIO : width;
    n.N[l] = l == n.nl - 1 ? kIO : width;
    n.Kr[l] = l == 0 ? nb_inputs : width;
    n.Nr[l] = l == n.nl - 1 ? nb_outputs : width;
    m->w_off.push_back(m->nparams);
    m->nparams += (int64_t)n.Nr[l] * n.Kr[l];
    m->b_off.push_back(m->nparams);
    m->nparams += n.Nr[l];
  }
  for (int j = 0; j < kIO; ++j) {
    n.in_shift[j] = n.out_shift[j] = 0.0f;
    n.in_scale[j] = n.out_scale[j] = 1.0f;
  }
  m->device = device;
  AKB_CUDA_TRY(cudaSetDevice(device));
  if (stream) {
    m->stream = (cudaStream_t)stream;
  } else {
    AKB_CUDA_TRY(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
    m->owns_stream = true;
  }
  AKB_CUDA_TRY(dmalloc(m->allocs, &m->d_params, m->nparams));
  AKB_CUDA_TRY(dmalloc(m->allocs, &m->d_grad, m->nparams));
  AKB_CUDA_TRY(dmalloc(m->allocs, &m->d_m1, m->nparams));
  AKB_CUDA_TRY(dmalloc(m->allocs, &m->d_m2, m->nparams));
  AKB_CUDA_TRY(dmalloc(m->allocs, &m->d_error, 1));
  for (int l = 0; l < n.nl; ++l) {
    __nv_bfloat16 *W, *Wt;
    float* b;
    AKB_CUDA_TRY(dmalloc(m->allocs, &W, (size_t)n.N[l] * n.K[l]));
    AKB_CUDA_TRY(dmalloc(m->allocs, &Wt, (size_t)n.N[l] * n.K[l]));
    AKB_CUDA_TRY(dmalloc(m->allocs, &b, (size_t)n.N[l]));
    n.W[l] = W;
    n.Wt[l] = Wt;
    n.b[l] = b;
  }
  n.error = m->d_error;
  AKB_CUDA_TRY(cudaMemsetAsync(m->d_params, 0, m->nparams * sizeof(float), m->stream));
  AKB_CUDA_TRY(cudaMemsetAsync(m->d_m1, 0, m->nparams * sizeof(float), m->stream));
  AKB_CUDA_TRY(cudaMemsetAsync(m->d_m2, 0, m->nparams * sizeof(float), m->stream));
  akb_status st;
  if ((st = repack(m.get())) != AKB_OK) return st;
  AKB_CUDA_TRY(set_smem((const void*)k_forward<true>, kFwdSmem));
  AKB_CUDA_TRY(set_smem((const void*)k_forward<false>, kFwdSmem));
  AKB_CUDA_TRY(set_smem((const void*)k_forward<false, true>, kFwdSmem));
  AKB_CUDA_TRY(set_smem((const void*)k_backward, kBwdSmem));
  AKB_CUDA_TRY(set_smem((const void*)k_wgrad, kWgradSmem));
  AKB_CUDA_TRY(cudaStreamSynchronize(m->stream));
  *out = m.release();
  return AKB_OK;
}

akb_status akb_mlp_destroy(akb_mlp* m) {
  if (!m) return AKB_OK;
  cudaSetDevice(m->device);
  cudaStreamSynchronize(m->stream);
  for (void* p : m->allocs) cudaFree(p);
  for (void* p : m->work) cudaFree(p);
  if (m->d_part) cudaFree(m->d_part);
  if (m->h_loss) cudaFreeHost(m->h_loss);
  if (m->owns_stream) cudaStreamDestroy(m->stream);
  delete m;
  return AKB_OK;
}

akb_status akb_mlp_get_parameter_count(const akb_mlp* m, int64_t* count) {
  if (!m || !count) return fail(AKB_ERR_INVALID_ARGUMENT, "null argument");
  *count = m->nparams;
  return AKB_OK;
}

akb_status akb_mlp_set_parameters(akb_mlp* m, const float* values, int64_t count) {
  if (!m || !values) return fail(AKB_ERR_INVALID_ARGUMENT, "null argument");
  if (count != m->nparams) return fail(AKB_ERR_INVALID_ARGUMENT, "wrong parameter count");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  AKB_CUDA_TRY(cudaMemcpyAsync(m->d_params, values, count * sizeof(float), cudaMemcpyHostToDevice,
                               m->stream));
  AKB_CUDA_TRY(cudaMemsetAsync(m->d_m1, 0, count * sizeof(float), m->stream));
  AKB_CUDA_TRY(cudaMemsetAsync(m->d_m2, 0, count * sizeof(float), m->stream));
  m->adam_step = 0;
  akb_status st;
  if ((st = repack(m)) != AKB_OK) return st;
  AKB_CUDA_TRY(cudaStreamSynchronize(m->stream));
  return AKB_OK;
}

akb_status akb_mlp_get_parameters(akb_mlp* m, float* values, int64_t count) {
  if (!m || !values) return fail(AKB_ERR_INVALID_ARGUMENT, "null argument");
  if (count != m->nparams) return fail(AKB_ERR_INVALID_ARGUMENT, "wrong parameter count");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  AKB_CUDA_TRY(cudaMemcpyAsync(values, m->d_params, count * sizeof(float), cudaMemcpyDeviceToHost,
                               m->stream));
  AKB_CUDA_TRY(cudaStreamSynchronize(m->stream));
  return AKB_OK;
}

akb_status akb_mlp_set_scaling(akb_mlp* m, const float* in_shift, const float* in_scale,
                               const float* out_shift, const float* out_scale) {
  if (!m || !in_shift || !in_scale || !out_shift || !out_scale)
    return fail(AKB_ERR_INVALID_ARGUMENT, "null argument");
  for (int j = 0; j < m->net.nin; ++j) {
    m->net.in_shift[j] = in_shift[j];
    m->net.in_scale[j] = in_scale[j];
  }
  for (int j = 0; j < m->net.nout; ++j) {
    if (!(out_scale[j] != 0.0f)) return fail(AKB_ERR_INVALID_ARGUMENT, "zero output scale");
    m->net.out_shift[j] = out_shift[j];
    m->net.out_scale[j] = out_scale[j];
  }
  return AKB_OK;
}

akb_status akb_mlp_forward(akb_mlp* m, int64_t nb, const double* x, double* y, void* stream) {
  if (!m) return fail(AKB_ERR_INVALID_ARGUMENT, "null network");
  if (nb < 0 || (nb > 0 && (!x || !y))) return fail(AKB_ERR_INVALID_ARGUMENT, "x and y are required");
  if (nb == 0) return AKB_OK;
  const int64_t ntiles = (nb + kTile - 1) / kTile;
  if (ntiles > INT32_MAX) return fail(AKB_ERR_UNSUPPORTED, "too many samples");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  cudaStream_t s = stream ? (cudaStream_t)stream : m->stream;
  k_forward<false><<<(unsigned)ntiles, kFwdThreads, kFwdSmem, s>>>(m->net, nb, x, y, Bufs{});
  AKB_CUDA_TRY(cudaGetLastError());
  return AKB_OK;
}

akb_status akb_mlp_stress(akb_mlp* m, int64_t nb, const double* grad_u, double* stress,
                          double amplitude, double min_det, int32_t* fallback_index,
                          int32_t* fallback_count, void* stream) {
  if (!m) return fail(AKB_ERR_INVALID_ARGUMENT, "null network");
  if (m->net.nin != 10 || m->net.nout != 9)
    return fail(AKB_ERR_INVALID_ARGUMENT, "the stress map needs 10 inputs (H / |H|, log |H|) and 9 outputs");
  if (nb < 0 || (nb > 0 && (!grad_u || !stress)))
    return fail(AKB_ERR_INVALID_ARGUMENT, "grad_u and stress are required");
  if ((fallback_index == nullptr) != (fallback_count == nullptr))
    return fail(AKB_ERR_INVALID_ARGUMENT, "fallback_index and fallback_count go together");
  const int64_t ntiles = (nb + kTile - 1) / kTile;
  if (ntiles > INT32_MAX || nb > INT32_MAX) return fail(AKB_ERR_UNSUPPORTED, "too many samples");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  cudaStream_t s = stream ? (cudaStream_t)stream : m->stream;
  if (fallback_count) AKB_CUDA_TRY(cudaMemsetAsync(fallback_count, 0, sizeof(int32_t), s));
  if (nb == 0) return AKB_OK;
  StressArgs sa;
  sa.amplitude = amplitude;
  sa.min_det = min_det;
  sa.index = fallback_index;
  sa.count = fallback_count;
  k_forward<false, true><<<(unsigned)ntiles, kFwdThreads, kFwdSmem, s>>>(m->net, nb, grad_u,
                                                                         stress, Bufs{}, sa);
  AKB_CUDA_TRY(cudaGetLastError());
  return AKB_OK;
}

akb_status akb_mlp_gradients(akb_mlp* m, int64_t nb, const double* x, const double* target,
                             float* grad, float* loss) {
  if (!m) return fail(AKB_ERR_INVALID_ARGUMENT, "null network");
  if (nb < 1 || !x || !target) return fail(AKB_ERR_INVALID_ARGUMENT, "x and target are required");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  akb_status st;
  if ((st = gradients(m, nb, x, target, loss)) != AKB_OK) return st;
  if (grad) {
    AKB_CUDA_TRY(cudaMemcpyAsync(grad, m->d_grad, m->nparams * sizeof(float),
                                 cudaMemcpyDeviceToHost, m->stream));
    AKB_CUDA_TRY(cudaStreamSynchronize(m->stream));
  }
  return AKB_OK;
}

akb_status akb_mlp_compute_gradients(akb_mlp* m, int64_t nb, const double* x,
                                     const double* target, float* loss) {
  if (!m) return fail(AKB_ERR_INVALID_ARGUMENT, "null network");
  if (nb < 1 || !x || !target) return fail(AKB_ERR_INVALID_ARGUMENT, "x and target are required");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  return gradients(m, nb, x, target, loss);
}

akb_status akb_mlp_gradient_device_pointer(akb_mlp* m, float** grad) {
  if (!m || !grad) return fail(AKB_ERR_INVALID_ARGUMENT, "null argument");
  *grad = m->d_grad;
  return AKB_OK;
}

akb_status akb_mlp_apply_gradients(akb_mlp* m, float learning_rate) {
  if (!m) return fail(AKB_ERR_INVALID_ARGUMENT, "null network");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  m->adam_step += 1;
  const float c1 = 1.0f - std::pow(b1, (float)m->adam_step);
  const float c2 = 1.0f - std::pow(b2, (float)m->adam_step);
  k_adam<<<(unsigned)((m->nparams + 255) / 256), 256, 0, m->stream>>>(
      m->d_params, m->d_grad, m->d_m1, m->d_m2, m->nparams, learning_rate, b1, b2, eps, c1, c2);
  AKB_CUDA_TRY(cudaGetLastError());
  return repack(m);
}

akb_status akb_mlp_train_step(akb_mlp* m, int64_t nb, const double* x, const double* target,
                              float learning_rate, float* loss) {
  akb_status st;
  if ((st = akb_mlp_compute_gradients(m, nb, x, target, loss)) != AKB_OK) return st;
  return akb_mlp_apply_gradients(m, learning_rate);
}

}  // extern "C"
