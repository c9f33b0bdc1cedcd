// akb_static_scratch.cu -- kinetic energy of device-resident arrays without
// any device allocation.
//
// Some callers cannot call cudaMalloc while they step: code that runs inside
// CUDA stream capture (an allocation there breaks or invalidates the capture)
// and applications whose device memory is owned by another allocator with a
// fixed budget (a framework's caching pool, a solver that reserves its memory
// up front). akb_kinetic_energy_static serves them: the caller passes the
// mass and velocity arrays and a device slot for the result; the per-block
// partial sums live in a fixed array compiled into the library
// (g_partials, 16 KiB), which every GPU that loads the library holds until the
// process exits.
//
// Limits and sharing:
//  - at most kMaxNodes nodes (kMaxPartials blocks of kThreads x kNodesPerThread);
//    larger inputs are rejected before anything runs;
//  - every call on a device uses the same g_partials, and the array keeps the
//    last call's partials. Each call overwrites every partial it reads, so
//    nothing has to start at zero; calls that overlap on the GPU (different
//    streams, no ordering between them) race on the array;
//  - the device address of g_partials is looked up again on every call made
//    outside stream capture (so a device reset, which reloads the module,
//    leaves no stale address behind) and cached per device for calls made
//    during a capture; make one call with the device current before the
//    first capture.
#include <mutex>

#include <cfloat>

#include "akb_internal.cuh"

namespace akb {
namespace {

constexpr int kThreads = 256;
constexpr int kNodesPerThread = 16;
constexpr int kMaxPartials = 2048;
constexpr int64_t kMaxNodes = (int64_t)kMaxPartials * kThreads * kNodesPerThread;  // 8 388 608
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_partials[kMaxPartials];

// Block b sums m v^2 over nodes [b * kThreads * kNodesPerThread, ...), the
// per-node terms as getKineticEnergy writes them (solid_mechanics_model.cc:547-561):
// components with m > epsilon, mv2 += v * v * m.
__global__ void k_kinetic_partials(const double* mass, const double* velocity, int64_t nn,
                                   int dim, double* partials) {
  __shared__ double sh[kThreads];
  const int64_t base = (int64_t)blockIdx.x * kThreads * kNodesPerThread;
  double acc = 0.0;
  for (int r = 0; r < kNodesPerThread; ++r) {
    const int64_t node = base + (int64_t)r * kThreads + threadIdx.x;
    if (node >= nn) break;
    double mv2 = 0.0;
    for (int i = 0; i < dim; ++i) {
      const double m = mass[node * dim + i], v = velocity[node * dim + i];
      if (m > DBL_EPSILON) mv2 += v * v * m;
    }
    acc += mv2;
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = sh[0];
}

__global__ void k_kinetic_finish(const double* partials, int nblocks, double* out) {
  __shared__ double sh[kThreads];
  double acc = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += kThreads) acc += partials[b];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = 0.5 * sh[0];
}

std::mutex g_setup_mutex;
double* g_partials_address[kMaxDevices] = {nullptr};

}  // namespace
}  // namespace akb

using namespace akb;

extern "C" akb_status akb_kinetic_energy_static(const double* mass, const double* velocity,
                                                int64_t nb_nodes, int32_t spatial_dimension,
                                                double* result, void* stream) {
  if (!mass || !velocity || !result)
    return fail(AKB_ERR_INVALID_ARGUMENT, "akb_kinetic_energy_static: null pointer");
  if (spatial_dimension < 1 || spatial_dimension > 3)
    return fail(AKB_ERR_INVALID_ARGUMENT, "akb_kinetic_energy_static: dimension must be 1, 2 or 3");
  if (nb_nodes < 1 || nb_nodes > kMaxNodes)
    return fail(AKB_ERR_INVALID_ARGUMENT,
                "akb_kinetic_energy_static: nb_nodes must be in [1, 8388608] (the fixed "
                "scratch holds 2048 partial sums of 4096 nodes each)");
  int dev = 0;
  AKB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices)
    return fail(AKB_ERR_UNSUPPORTED, "akb_kinetic_energy_static: device ordinal >= 64");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  AKB_CUDA_TRY(cudaStreamIsCapturing(s, &capture));
  double* partials = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_partials_address[dev] || capture == cudaStreamCaptureStatusNone) {
      // host code cannot use &g_partials: it is a host-side stand-in, not the
      // device address; ask the runtime for the address on this device
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_partials);
      if (e != cudaSuccess)
        return fail(AKB_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_partials_address[dev] = static_cast<double*>(p);
    }
    partials = g_partials_address[dev];
  }
  const int per_block = kThreads * kNodesPerThread;
  const int nblocks = (int)((nb_nodes + per_block - 1) / per_block);
  k_kinetic_partials<<<nblocks, kThreads, 0, s>>>(mass, velocity, nb_nodes, spatial_dimension,
                                                  partials);
  k_kinetic_finish<<<1, kThreads, 0, s>>>(partials, nblocks, result);
  AKB_CUDA_TRY(cudaGetLastError());
  return AKB_OK;
}
