// akb_internal.cuh -- shared declarations of libakb.so (not installed).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/akb.h"

namespace akb {

constexpr int kMaxMaterials = 8;

#ifdef __CUDACC__
// Programmatic dependent launch: a kernel launched by launch_pdl may start
// while the kernel before it in the stream is finishing. It waits
// (grid_wait: until that grid has completed and its writes are visible)
// before it touches memory that grid may use, and signals
// (grid_launch_dependents) when the kernel after it may start launching.
__device__ inline void grid_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ inline void grid_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
template <typename... K, typename... A>
cudaError_t launch_pdl(void (*kernel)(K...), int grid, int block, size_t smem, cudaStream_t s,
                       A... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}
#endif

// Compile-time element properties (ElementClassProperty, element_class_*.hh).
template <int T> struct ET;
template <> struct ET<AKB_SEGMENT_2> { static constexpr int dim = 1, nnpe = 2, nqp = 1; };
template <> struct ET<AKB_TRIANGLE_3> { static constexpr int dim = 2, nnpe = 3, nqp = 1; };
template <> struct ET<AKB_TETRAHEDRON_4> { static constexpr int dim = 3, nnpe = 4, nqp = 1; };
template <> struct ET<AKB_HEXAHEDRON_8> { static constexpr int dim = 3, nnpe = 8, nqp = 8; };

inline int nnpe_of(int t) { return t == AKB_SEGMENT_2 ? 2 : t == AKB_TRIANGLE_3 ? 3 : t == AKB_TETRAHEDRON_4 ? 4 : 8; }
inline int nqp_of(int t) { return t == AKB_HEXAHEDRON_8 ? 8 : 1; }
inline int dim_of(int t) { return t == AKB_SEGMENT_2 ? 1 : t == AKB_TRIANGLE_3 ? 2 : 3; }

// Material parameters as the reference derives them from (E, nu)
// (material_elastic.cc:83-107, material_neohookean.cc:83-89).
struct MatParams {
  int kind;
  int finite;
  double rho, E, nu, lambda, mu;
  double celerity;  // sqrt((lambda + 2 mu) / rho)
};

// Device-side view of a model: plain pointers, passed by value to kernels.
struct DevModel {
  int dim, type, nnpe, nqp;
  int64_t nn, ne;
  int nmat;
  const double* X;          // nn x dim
  const uint32_t* conn;     // ne x nnpe
  const uint32_t* mat_of;   // ne or null
  double *u, *v, *a, *fext, *fint, *mass, *inv_mass;  // nn x dim (inv_mass: nn)
  uint8_t* blocked;         // nn x dim
  // reference-order path
  double *B, *jac, *gradu, *stress;  // stored shape derivatives / detJ*w / QP fields
  void* fe;                 // ne x nnpe x dim element forces (double or float)
  const int32_t* node_ptr;  // nn + 1, node -> (element, corner) CSR
  const int32_t* node_ent;  // ne * nnpe entries e * nnpe + a, ascending e
  MatParams mats[kMaxMaterials];  // the first materials, by value (kernel parameter space)
  const MatParams* mat_table;     // all nmat materials (device), indexed by mat_of
};

// Thread-local last-error helpers.
void set_error(const std::string& msg);
akb_status fail(akb_status s, const std::string& msg);

#define AKB_CUDA_TRY(expr)                                                  \
  do {                                                                      \
    cudaError_t _e = (expr);                                                \
    if (_e != cudaSuccess)                                                  \
      return ::akb::fail(AKB_ERR_CUDA, std::string(#expr) + ": " +          \
                                           cudaGetErrorString(_e));         \
  } while (0)

// Kernel launchers (reference-order path: akb_reference.cu).
cudaError_t ref_init_geometry(const DevModel& m, cudaStream_t s, int* d_negative);
cudaError_t ref_predictor(const DevModel& m, double dt, cudaStream_t s);
cudaError_t ref_element_forces(const DevModel& m, cudaStream_t s);
cudaError_t ref_gather_correct(const DevModel& m, double dt, bool correct, cudaStream_t s);
cudaError_t ref_mass(const DevModel& m, cudaStream_t s);
cudaError_t ref_compute_stresses(const DevModel& m, bool recompute_geometry, cudaStream_t s);

// Kernel launchers (fast paths: akb_fast.cu).
cudaError_t fast_predictor(const DevModel& m, double dt, cudaStream_t s);
cudaError_t fast_element_forces(const DevModel& m, bool fp32, cudaStream_t s);
cudaError_t fast_gather_correct(const DevModel& m, double dt, bool fp32, bool correct,
                                bool has_fext, cudaStream_t s);

// User materials (akb_fast.cu): grad u at the quadrature points into gradu;
// element force vectors (FP64, into fe) from the caller's stress.
cudaError_t user_qp_gradients(const DevModel& m, cudaStream_t s);
cudaError_t user_element_forces(const DevModel& m, cudaStream_t s);

// Dirichlet values (akb_fast.cu): blocked[node][comp] = 1, u[node][comp] = value
// (and the predicted displacement w, when the model keeps one); comp < 0:
// every component, values row per node; perm (or null) maps the caller's
// node ids to the model's internal order.
cudaError_t apply_dirichlet(const DevModel& m, const uint32_t* nodes, int64_t n, int comp,
                            const double* values, const uint32_t* perm, double* w,
                            cudaStream_t s);

// Reductions (akb_reduce.cu). Scratch holds per-block partial results.
cudaError_t stable_dt(const DevModel& m, double* d_scratch, int scratch_len,
                      double* d_out, cudaStream_t s);
cudaError_t energy(const DevModel& m, int kind, double dt, double* d_scratch,
                   int scratch_len, double* d_out, cudaStream_t s);
int reduce_blocks(int64_t n);
// *out = scale * (sum of partial[0, n)), in a fixed order.
cudaError_t sum_partials(const double* partial, int64_t n, double scale, double* out,
                         cudaStream_t s);
// Per-instance reductions of a batch: one block per instance.
cudaError_t stable_dt_instances(const DevModel& m, const int64_t* elem_off, int ninst,
                                double* d_out, cudaStream_t s);
cudaError_t energy_instances(const DevModel& m, int kind, const int64_t* node_off,
                             const int64_t* elem_off, int ninst, double* d_out, cudaStream_t s);

}  // namespace akb
