// akb_model.cu -- the C ABI of include/akb.h: model lifecycle, fields, the
// explicit step driver and its CUDA-graph replay.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/akb_fe2.h"
#include "akb_internal.cuh"
#include "akb_patch.cuh"

namespace akb {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
akb_status fail(akb_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

}  // namespace akb

using namespace akb;

// Node and element ranges of the instances of a batch, in the union mesh.
struct BatchLayout {
  int32_t ninst = 0;
  std::vector<int64_t> node_off, elem_off;  // ninst + 1 each
};

struct akb_model {
  DevModel dm{};
  int mode = AKB_MODE_FP64_REFERENCE;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool owns_stream = false;
  std::vector<void*> allocations;
  int64_t device_bytes = 0;
  double dt = 0.0;
  bool has_fext = false;
  bool fint_valid = false;
  bool stresses_valid = false;
  // user materials: stresses come from the caller between step_begin/end
  bool user = false;
  bool in_step = false;
  double* d_scratch = nullptr;  // reduction partials
  int scratch_len = 0;
  double* d_result = nullptr;
  double* h_result = nullptr;   // pinned
  // cached graphs of k consecutive steps, keyed by k
  std::map<int64_t, cudaGraphExec_t> graphs;
  double graph_dt = -1.0;
  bool graph_fext = false;
  // fused patch step of the fast modes
  DevPatches patches{};
  bool use_patches = false;
  int opt_patch_elements = 0, opt_patch_nodes = 0, opt_patch_grid = 0;
  // batch of independent instances (akb_batch_create)
  int32_t ninst = 0;
  std::vector<int64_t> node_off, elem_off;
  double* d_inst_dt = nullptr;
  const int64_t* d_node_off = nullptr;
  const int64_t* d_elem_off = nullptr;
  // staging of akb_apply_dirichlet: a ring of pinned host / device buffer
  // pairs (node ids padded to 8 bytes, then values); a slot is refilled only
  // once the kernel that read its previous contents has run
  struct BcSlot {
    unsigned char* host = nullptr;
    unsigned char* dev = nullptr;
    int64_t capacity = 0;  // bytes
    cudaEvent_t copied = nullptr;  // the upload (upload stream) is done
    cudaEvent_t done = nullptr;    // the update kernel (model stream) has run
    bool pending = false;
  };
  static constexpr int kBcSlots = 4;
  BcSlot bc[kBcSlots];
  int bc_next = 0;
  // host <-> device copies of the per-step calls run on streams of their own,
  // ordered against the model's stream by events, so that they overlap the
  // steps' kernels: Dirichlet uploads on upload_stream, energy results on
  // copy_stream (one stream for both would queue step s's upload behind step
  // s-1's result copy, which waits for step s-1's kernels)
  cudaStream_t copy_stream = nullptr;
  cudaStream_t upload_stream = nullptr;
  // akb_get_energy_async: a ring of device result slots; a slot is written
  // again only once the copy of its previous value is done
  static constexpr int kEnergySlots = 32;
  double* d_eres = nullptr;
  cudaEvent_t eres_ready[kEnergySlots] = {};
  cudaEvent_t eres_copied[kEnergySlots] = {};
  bool eres_pending[kEnergySlots] = {};
  int eres_next = 0;
  // part of a partitioned mesh (akb_model_create_part): its interface nodes
  // (shared nodes of the patch plan), finished only once their forces are
  // summed over all parts
  bool part = false;
  bool part_in_step = false;
  int64_t n_iface = 0;
  const uint32_t* d_iface_g = nullptr;     // internal id of each interface node
  const uint32_t* d_iface_part = nullptr;  // its shared node index (partial_slot)
  const uint32_t* d_iface_k = nullptr;     // its partial count
  akb::ExchangePlan xplan;                 // neighbour exchange (akb_part_set_exchange)
  bool has_xplan = false;
  // internal node order of the fused step (akb_patch.cuh): perm[caller's id]
  // = internal id; nodal arrays crossing the C ABI are reordered through
  // d_tmp. Without patches the order is the caller's (d_perm null).
  const uint32_t* d_perm = nullptr;
  std::vector<uint32_t> perm;
  double* d_tmp = nullptr;
  // the predicted displacement of the fused step is current
  bool w_valid = false;
  // the kinetic-energy partials the last fused step wrote describe the
  // current velocities
  bool ke_valid = false;
};

// Interface nodes of a part, in the caller's order.
struct PartLayout {
  const uint32_t* nodes = nullptr;
  int64_t n = 0;
};

namespace {

template <typename T>
akb_status dalloc(akb_model* m, T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? AKB_ERR_OUT_OF_MEMORY : AKB_ERR_CUDA,
                std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  m->allocations.push_back(*p);
  m->device_bytes += count * sizeof(T);
  return AKB_OK;
}

void dfree(akb_model* m, void* p) {
  if (!p) return;
  for (size_t i = 0; i < m->allocations.size(); ++i)
    if (m->allocations[i] == p) {
      m->allocations.erase(m->allocations.begin() + i);
      break;
    }
  cudaFree(p);
}

MatParams make_params(const akb_material_desc& d, int dim) {
  MatParams p{};
  p.kind = d.kind;
  p.finite = (d.kind == AKB_MATERIAL_NEOHOOKEAN) || d.finite_deformation != 0;
  // a user material's E and nu only give the wave speed of the stable step
  p.rho = d.rho;
  p.E = d.E;
  p.nu = dim == 1 ? 0. : d.nu;
  p.lambda = p.nu * p.E / ((1 + p.nu) * (1 - 2 * p.nu));
  p.mu = p.E / (2 * (1 + p.nu));
  if (dim == 2 && d.plane_stress && d.kind == AKB_MATERIAL_ELASTIC)
    p.lambda = p.nu * p.E / ((1 + p.nu) * (1 - p.nu));
  p.celerity = std::sqrt((p.lambda + 2 * p.mu) / p.rho);
  return p;
}

void destroy_graphs(akb_model* m) {
  for (auto& kv : m->graphs) cudaGraphExecDestroy(kv.second);
  m->graphs.clear();
}

bool fp32(const akb_model* m) { return m->mode == AKB_MODE_FP32_BULK; }

// Optional CUDA events recorded before each kernel of a step (and after the
// last one), for akb_time_kernels.
struct StepTimer {
  cudaEvent_t ev[AKB_MAX_KERNEL_SLOTS + 1];
  int n = 0;
};
inline void mark(StepTimer* t, cudaStream_t s) {
  if (t && t->n <= AKB_MAX_KERNEL_SLOTS) cudaEventRecord(t->ev[t->n++], s);
}

const char* const kRefKernels[] = {"ref_predictor", "ref_element_forces", "ref_gather_correct"};
const char* const kFastKernels[] = {"fast_predictor", "fast_element_forces", "fast_gather_correct"};
const char* const kPatchKernels[] = {"patch_step", "patch_finish_list"};

// One NonLinearSolverLumped::solve.
cudaError_t enqueue_step(akb_model* m, StepTimer* t = nullptr) {
  const DevModel& d = m->dm;
  cudaError_t e;
  if (m->mode == AKB_MODE_FP64_REFERENCE) {
    mark(t, m->stream);
    if ((e = ref_predictor(d, m->dt, m->stream)) != cudaSuccess) return e;
    mark(t, m->stream);
    if ((e = ref_element_forces(d, m->stream)) != cudaSuccess) return e;
    mark(t, m->stream);
    e = ref_gather_correct(d, m->dt, true, m->stream);
    mark(t, m->stream);
    return e;
  }
  if (m->use_patches) {
    mark(t, m->stream);
    if ((e = patch_step(d, m->patches, m->dt, fp32(m), m->has_fext, m->stream)) != cudaSuccess)
      return e;
    mark(t, m->stream);
    e = patch_finish_list(d, m->patches, m->dt, m->has_fext, m->stream);
    mark(t, m->stream);
    return e;
  }
  mark(t, m->stream);
  if ((e = fast_predictor(d, m->dt, m->stream)) != cudaSuccess) return e;
  mark(t, m->stream);
  if ((e = fast_element_forces(d, fp32(m), m->stream)) != cudaSuccess) return e;
  mark(t, m->stream);
  e = fast_gather_correct(d, m->dt, fp32(m), true, m->has_fext, m->stream);
  mark(t, m->stream);
  return e;
}

const char* kernel_name(const akb_model* m, int slot) {
  if (m->use_patches) return (slot >= 0 && slot < 2) ? kPatchKernels[slot] : "";
  const char* const* names = m->mode == AKB_MODE_FP64_REFERENCE ? kRefKernels : kFastKernels;
  return (slot >= 0 && slot < 3) ? names[slot] : "";
}

// Patch size of the fused step per element type: elements per patch and the
// local node cap, chosen so three 256-thread CTAs (two for hexahedra) fit an
// SM (measured sweeps on the tet4 cube and the hex8 block).
void patch_params(int type, int* target, int* max_nodes) {
  switch (type) {
  case AKB_SEGMENT_2: *target = 1024; *max_nodes = 1100; break;
  case AKB_TRIANGLE_3: *target = 1024; *max_nodes = 640; break;
  case AKB_TETRAHEDRON_4: *target = 1024; *max_nodes = 400; break;
  default: *target = 512; *max_nodes = 800; break;
  }
}

template <typename T>
akb_status upload(akb_model* m, const std::vector<T>& v, const T** out);

// Patch plan of the fused step on the host (mesh in the caller's node
// order): a single mesh, a partitioned part (its interface nodes forced to
// be finished outside the fused step), or a batch (patches built per
// instance, so that no patch spans two instances, and concatenated).
// patch_inst / orphan_inst: the instance of each patch and node of no
// element (batches only).
akb_status plan_patches(akb_model* m, const akb_mesh_desc* mesh, const BatchLayout* batch,
                        const PartLayout* part, PatchHost& P, std::vector<uint32_t>& patch_inst,
                        std::vector<uint32_t>& orphan_inst) {
  int target, max_nodes;
  patch_params(m->dm.type, &target, &max_nodes);
  if (fp32(m) && m->dm.type == AKB_TETRAHEDRON_4) {
    // FP32 contributions and one record buffer fit 768-element patches in
    // 56 KB, four CTAs per SM: 0.234 against 0.243 ms per step on the
    // 6 M-element cube with 1024-element patches at three
    target = 768;
    max_nodes = 320;
  }
  if (m->opt_patch_elements <= 0) {
    // small meshes: patches of down to one chunk, so that there are about two
    // per SM (measured on the 8000-element plate: 12.7 ms for 1000 steps at
    // 1024 elements per patch, 8.0 ms at 256)
    int sms = 148;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->device) != cudaSuccess) {
      cudaGetLastError();
      sms = 148;
    }
    const int64_t want = 2 * (int64_t)sms;
    if (mesh->nb_elements / target < want) {
      const int64_t per = (mesh->nb_elements / want + kChunk - 1) / kChunk * kChunk;
      const int t = (int)std::max<int64_t>(kChunk, per);
      if (t < target) {
        max_nodes = (int)((int64_t)max_nodes * t / target * 5 / 4);
        target = t;
      }
    }
  }
  if (m->opt_patch_elements > 0) target = std::min(m->opt_patch_elements, 8191);
  if (m->opt_patch_nodes > 0) max_nodes = std::min(m->opt_patch_nodes, 60000);
  const int cbytes = fp32(m) ? 4 : 8;  // element vector precision
  try {
    if (!batch) {
      std::vector<uint8_t> force;
      if (part) {
        force.assign(mesh->nb_nodes, 0);
        for (int64_t i = 0; i < part->n; ++i) force[part->nodes[i]] = 1;
      }
      P = build_patches(mesh->nodes, mesh->connectivity, mesh->nb_nodes, mesh->nb_elements,
                        m->dm.dim, m->dm.nnpe, target, max_nodes, cbytes,
                        part ? force.data() : nullptr);
      return AKB_OK;
    }
    const int dd = m->dm.dim, nn_ = m->dm.nnpe;
    P = PatchHost{};
    P.elem_ptr.push_back(0);
    P.sh_ptr.push_back(0);
    std::vector<uint32_t> lconn;
    for (int i = 0; i < batch->ninst; ++i) {
      const int64_t n0 = batch->node_off[i], e0 = batch->elem_off[i];
      const int64_t nni = batch->node_off[i + 1] - n0, nei = batch->elem_off[i + 1] - e0;
      lconn.assign(mesh->connectivity + e0 * nn_, mesh->connectivity + (e0 + nei) * nn_);
      for (auto& c : lconn) c -= (uint32_t)n0;
      PatchHost Q = build_patches(mesh->nodes + n0 * dd, lconn.data(), nni, nei, dd, nn_, target,
                                  max_nodes, cbytes);
      const int64_t ebase = (int64_t)P.sgid.size();
      const int64_t chbase = (int64_t)P.chunks.size();
      const uint32_t dbase16 = (uint32_t)(P.cdata.size() / 8);
      for (int p = 0; p < Q.npatch; ++p) {
        P.elem_ptr.push_back((int32_t)(e0 + Q.elem_ptr[p + 1]));
        P.ibeg.push_back((int32_t)(n0 + Q.ibeg[p]));
        P.nint.push_back(Q.nint[p]);
        P.sh_ptr.push_back((int32_t)(ebase + Q.sh_ptr[p + 1]));
        P.chunk_base.push_back((int32_t)(chbase + Q.chunk_base[p]));
        patch_inst.push_back((uint32_t)i);
      }
      P.npatch += Q.npatch;
      P.max_nodes = std::max(P.max_nodes, Q.max_nodes);
      P.max_interior = std::max(P.max_interior, Q.max_interior);
      P.max_shared = std::max(P.max_shared, Q.max_shared);
      P.contrib_slots = std::max(P.contrib_slots, Q.contrib_slots);
      P.max_runs = std::max(P.max_runs, Q.max_runs);
      P.chunk_bytes = std::max(P.chunk_bytes, Q.chunk_bytes);
      for (auto g : Q.perm) P.perm.push_back((uint32_t)(g + n0));
      for (auto e : Q.elem_order) P.elem_order.push_back((uint32_t)(e + e0));
      for (auto g : Q.sgid) P.sgid.push_back((uint32_t)(g + n0));
      P.srank.insert(P.srank.end(), Q.srank.begin(), Q.srank.end());
      for (auto c : Q.chunks) {
        c.off16 += dbase16;
        P.chunks.push_back(c);
      }
      P.cdata.insert(P.cdata.end(), Q.cdata.begin(), Q.cdata.end());
      for (auto g : Q.shared_nodes) P.shared_nodes.push_back((uint32_t)(g + n0));
      P.shared_k.insert(P.shared_k.end(), Q.shared_k.begin(), Q.shared_k.end());
      for (auto g : Q.orphans) {
        P.orphans.push_back((uint32_t)(g + n0));
        orphan_inst.push_back((uint32_t)i);
      }
    }
    assign_partial_slots(P, batch->node_off[batch->ninst]);  // dense rows over all instances
    P.chunk_base.push_back((int32_t)P.chunks.size());
    P.node_stride = (P.max_nodes + kBankPairs - 1) / kBankPairs * kBankPairs + 5;
  } catch (const std::exception& ex) {
    return fail(AKB_ERR_UNSUPPORTED, std::string("patch construction: ") + ex.what());
  }
  return AKB_OK;
}

// Device copy of a patch plan; the model's arrays are already in the plan's
// internal node order.
akb_status build_device_patches(akb_model* m, const PatchHost& P,
                                const std::vector<uint32_t>& patch_inst,
                                const std::vector<uint32_t>& orphan_inst,
                                const uint32_t* element_material, const BatchLayout* batch,
                                const PartLayout* part) {
  DevPatches& d = m->patches;
  d = DevPatches{};
  d.npatch = P.npatch;
  d.grid = m->opt_patch_grid > 0 ? m->opt_patch_grid : 0;
  d.max_nodes = P.max_nodes;
  d.max_shared = P.max_shared;
  d.node_stride = P.node_stride;
  d.contrib_slots = P.contrib_slots;
  d.max_runs = P.max_runs;
  d.chunk_bytes = P.chunk_bytes;
  akb_status st;
  if ((st = upload(m, P.elem_ptr, &d.elem_ptr)) != AKB_OK) return st;
  if ((st = upload(m, P.ibeg, &d.ibeg)) != AKB_OK) return st;
  if ((st = upload(m, P.nint, &d.nint)) != AKB_OK) return st;
  if ((st = upload(m, P.sh_ptr, &d.sh_ptr)) != AKB_OK) return st;
  if ((st = upload(m, P.sgid, &d.sgid)) != AKB_OK) return st;
  if ((st = upload(m, P.sslot, &d.sslot)) != AKB_OK) return st;

  if ((st = upload(m, P.chunk_base, &d.chunk_base)) != AKB_OK) return st;
  if ((st = upload(m, P.cdata, &d.cdata)) != AKB_OK) return st;
  {
    static_assert(sizeof(ChunkDesc) == sizeof(uint2), "chunk descriptor is one 8-byte load");
    std::vector<uint2> cd(P.chunks.size());
    std::memcpy(cd.data(), P.chunks.data(), cd.size() * sizeof(uint2));
    if ((st = upload(m, cd, &d.chunks)) != AKB_OK) return st;
  }
  // nodes finished by k_finish_list: the shared nodes (entry s: shared node
  // s, whose ranks 0 and 1 sit in the dense partial rows), then the nodes of
  // no element
  std::vector<uint32_t> lg(P.shared_nodes), lp(P.shared_part), lk(P.shared_k);
  lg.insert(lg.end(), P.orphans.begin(), P.orphans.end());
  lp.insert(lp.end(), P.orphans.size(), 0);
  lk.insert(lk.end(), P.orphans.size(), 0);
  std::vector<uint32_t> li;
  if (batch) {  // instance of each shared node: instances own contiguous node ranges
    for (uint32_t g : P.shared_nodes) {
      const auto it = std::upper_bound(batch->node_off.begin(), batch->node_off.end(), (int64_t)g);
      li.push_back((uint32_t)(it - batch->node_off.begin() - 1));
    }
    li.insert(li.end(), orphan_inst.begin(), orphan_inst.end());
  }
  d.nshared = (uint32_t)P.shared_nodes.size();
  d.shared_base = P.shared_base;
  // a single mesh numbers its shared nodes as one block (a batch per instance)
  d.shared_contig = batch ? 0 : 1;
  for (size_t s = 0; s < P.shared_nodes.size() && d.shared_contig; ++s)
    if (P.shared_nodes[s] != P.shared_base + s) d.shared_contig = 0;
  if (part) {
    std::vector<uint32_t> ig(part->n), ip(part->n), ik(part->n);
    for (int64_t i = 0; i < part->n; ++i) {
      const uint32_t g = P.perm[part->nodes[i]];
      const int64_t s = (int64_t)g - P.shared_base;
      if (s < 0 || s >= (int64_t)P.shared_nodes.size() || P.shared_nodes[s] != g)
        return fail(AKB_ERR_INVALID_ARGUMENT, "interface node is not a node of an element");
      ig[i] = g;
      ip[i] = (uint32_t)s;  // its shared node index (partial_slot)
      ik[i] = P.shared_k[s];
    }
    if ((st = upload(m, ig, &m->d_iface_g)) != AKB_OK) return st;
    if ((st = upload(m, ip, &m->d_iface_part)) != AKB_OK) return st;
    if ((st = upload(m, ik, &m->d_iface_k)) != AKB_OK) return st;
    m->n_iface = part->n;
    m->part = true;
  }
  d.nlist = (int64_t)lg.size();
  if ((st = upload(m, lg, &d.list_gid)) != AKB_OK) return st;
  if ((st = upload(m, lp, &d.list_part)) != AKB_OK) return st;
  if ((st = upload(m, lk, &d.list_k)) != AKB_OK) return st;
  {
    int* e;
    if ((st = dalloc(m, &e, 1)) != AKB_OK) return st;
    AKB_CUDA_TRY(cudaMemsetAsync(e, 0, sizeof(int), m->stream));
    d.err = e;
  }
  d.emat = nullptr;
  if (element_material) {
    std::vector<uint32_t> em(P.elem_order.size());
    for (size_t i = 0; i < em.size(); ++i) em[i] = element_material[P.elem_order[i]];
    if ((st = upload(m, em, &d.emat)) != AKB_OK) return st;
  }
  {
    double* ke;
    if ((st = dalloc(m, &ke, (size_t)patch_ke_parts(d, m->dm.dim))) != AKB_OK) return st;
    d.ke_part = ke;
  }
  const size_t nsl = (size_t)std::max<int64_t>(P.nslots, 1);
  if ((st = dalloc(m, &d.partial, nsl * m->dm.dim)) != AKB_OK) return st;
  AKB_CUDA_TRY(cudaMemsetAsync(d.partial, 0, nsl * m->dm.dim * sizeof(double), m->stream));
  // predicted displacement, with the slack of the other nodal arrays
  if ((st = dalloc(m, &d.w, (size_t)m->dm.nn * m->dm.dim + 2)) != AKB_OK) return st;
  AKB_CUDA_TRY(cudaMemsetAsync(d.w, 0, ((size_t)m->dm.nn * m->dm.dim + 2) * sizeof(double),
                               m->stream));
  m->w_valid = false;
  if ((st = upload(m, P.perm, &m->d_perm)) != AKB_OK) return st;
  m->perm = P.perm;
  d.inst_dt = nullptr;
  d.patch_inst = nullptr;
  d.list_inst = nullptr;
  d.node_off = nullptr;
  d.ninst = 0;
  if (batch) {
    if ((st = upload(m, patch_inst, &d.patch_inst)) != AKB_OK) return st;
    if ((st = upload(m, li, &d.list_inst)) != AKB_OK) return st;
  }
  AKB_CUDA_TRY(cudaStreamSynchronize(m->stream));  // host vectors go out of scope
  d.nbuf = patch_buffers(d, m->dm.type, fp32(m));
  const size_t smem = patch_smem_bytes(d, m->dm.dim, fp32(m), d.nbuf);
  if (smem > 227 * 1024)
    return fail(AKB_ERR_UNSUPPORTED, "patch does not fit in shared memory");
  AKB_CUDA_TRY(patch_configure(m->dm, d, fp32(m)));
  m->use_patches = true;
  return AKB_OK;
}

template <typename T>
akb_status upload(akb_model* m, const std::vector<T>& v, const T** out) {
  T* p;
  akb_status st;
  if ((st = dalloc(m, &p, v.size())) != AKB_OK) return st;
  if (!v.empty())
    AKB_CUDA_TRY(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice,
                                 m->stream));
  *out = p;
  return AKB_OK;
}

// Internal forces at the current displacement, without touching the state.
cudaError_t enqueue_internal_forces(akb_model* m) {
  const DevModel& d = m->dm;
  cudaError_t e;
  if (m->mode == AKB_MODE_FP64_REFERENCE) {
    if ((e = ref_element_forces(d, m->stream)) != cudaSuccess) return e;
    return ref_gather_correct(d, m->dt, false, m->stream);
  }
  if (m->user) {  // from the stresses the caller wrote last
    if ((e = user_element_forces(d, m->stream)) != cudaSuccess) return e;
    return fast_gather_correct(d, m->dt, false, false, m->has_fext, m->stream);
  }
  if ((e = fast_element_forces(d, fp32(m), m->stream)) != cudaSuccess) return e;
  return fast_gather_correct(d, m->dt, fp32(m), false, m->has_fext, m->stream);
}

akb_status check_model(const akb_model* m) {
  if (!m) return fail(AKB_ERR_INVALID_ARGUMENT, "null model");
  return AKB_OK;
}

akb_status sync(akb_model* m) {
  cudaError_t e = cudaStreamSynchronize(m->stream);
  if (e == cudaSuccess && m->copy_stream) e = cudaStreamSynchronize(m->copy_stream);
  if (e == cudaSuccess && m->upload_stream) e = cudaStreamSynchronize(m->upload_stream);
  if (e != cudaSuccess) return fail(AKB_ERR_CUDA, std::string("stream: ") + cudaGetErrorString(e));
  if (m->use_patches && m->patches.err) {  // a bounded wait of the fused step gave up
    int flag = 0;
    e = cudaMemcpy(&flag, m->patches.err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(AKB_ERR_CUDA, std::string("flag: ") + cudaGetErrorString(e));
    if (flag) {
      cudaMemset(m->patches.err, 0, sizeof(int));
      return fail(AKB_ERR_TIMEOUT, "fused step: staging copy did not complete in time");
    }
  }
  return AKB_OK;
}

// getEnergy into a device double: the kinetic energy right after a fused
// step sums the partials the step wrote, anything else reduces the fields.
cudaError_t enqueue_energy(akb_model* m, int32_t kind, double* out) {
  if (kind == AKB_ENERGY_KINETIC && m->use_patches && m->ke_valid)
    return sum_partials(m->patches.ke_part, patch_ke_parts(m->patches, m->dm.dim), 0.5, out,
                        m->stream);
  return energy(m->dm, kind, m->dt, m->d_scratch, m->scratch_len, out, m->stream);
}

akb_status ensure_copy_stream(akb_model* m) {
  if (m->copy_stream) return AKB_OK;
  AKB_CUDA_TRY(cudaStreamCreateWithFlags(&m->copy_stream, cudaStreamNonBlocking));
  AKB_CUDA_TRY(cudaStreamCreateWithFlags(&m->upload_stream, cudaStreamNonBlocking));
  return AKB_OK;
}

akb_status ensure_stress_arrays(akb_model* m) {
  if (m->dm.gradu) return AKB_OK;
  const size_t n = (size_t)m->dm.ne * m->dm.nqp * m->dm.dim * m->dm.dim;
  akb_status s;
  if ((s = dalloc(m, &m->dm.gradu, n)) != AKB_OK) return s;
  if ((s = dalloc(m, &m->dm.stress, n)) != AKB_OK) return s;
  return AKB_OK;
}

double* field_ptr(akb_model* m, int32_t field) {
  switch (field) {
  case AKB_FIELD_DISPLACEMENT: return m->dm.u;
  case AKB_FIELD_VELOCITY: return m->dm.v;
  case AKB_FIELD_ACCELERATION: return m->dm.a;
  case AKB_FIELD_EXTERNAL_FORCE: return m->dm.fext;
  case AKB_FIELD_INTERNAL_FORCE: return m->dm.fint;
  case AKB_FIELD_MASS: return m->dm.mass;
  case AKB_FIELD_NODES: return const_cast<double*>(m->dm.X);
  case AKB_FIELD_GRAD_U: return m->dm.gradu;
  case AKB_FIELD_STRESS: return m->dm.stress;
  }
  return nullptr;
}

int64_t field_count(const akb_model* m, int32_t field) {
  if (field == AKB_FIELD_GRAD_U || field == AKB_FIELD_STRESS)
    return m->dm.ne * m->dm.nqp * m->dm.dim * m->dm.dim;
  return m->dm.nn * m->dm.dim;
}

bool nodal(int32_t field) { return field != AKB_FIELD_GRAD_U && field != AKB_FIELD_STRESS; }

// Staging buffer of the reordered copies (nn x dim doubles).
akb_status ensure_tmp(akb_model* m) {
  if (m->d_tmp) return AKB_OK;
  return dalloc(m, &m->d_tmp, (size_t)m->dm.nn * m->dm.dim);
}

// The predicted displacement w = u + dt v + dt^2/2 a of the fused step,
// recomputed after the caller changed u, v, a, the blocked DOFs or dt.
akb_status ensure_w(akb_model* m) {
  if (!m->use_patches || m->w_valid) return AKB_OK;
  AKB_CUDA_TRY(patch_refresh_w(m->dm, m->patches, m->dt, m->stream));
  m->w_valid = true;
  return AKB_OK;
}

}  // namespace

static akb_status create_model(const akb_mesh_desc* mesh, int32_t nb_materials,
                               const akb_material_desc* materials,
                               const uint32_t* element_material,
                               const akb_model_options* options, const BatchLayout* batch,
                               akb_model** out, const PartLayout* part = nullptr);

extern "C" {

int32_t akb_abi_version(void) { return AKB_ABI_VERSION; }

const char* akb_last_error(void) { return g_last_error.c_str(); }

akb_status akb_model_create(const akb_mesh_desc* mesh, int32_t nb_materials,
                            const akb_material_desc* materials,
                            const uint32_t* element_material,
                            const akb_model_options* options, akb_model** out) {
  if (!out) return fail(AKB_ERR_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  return create_model(mesh, nb_materials, materials, element_material, options, nullptr, out);
}

akb_status akb_model_create_part(const akb_mesh_desc* mesh, int32_t nb_materials,
                                 const akb_material_desc* materials,
                                 const uint32_t* element_material,
                                 const akb_model_options* options,
                                 const uint32_t* interface_nodes, int64_t nb_interface,
                                 akb_model** out) {
  if (!out) return fail(AKB_ERR_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  PartLayout part;
  part.nodes = interface_nodes;
  part.n = nb_interface;
  return create_model(mesh, nb_materials, materials, element_material, options, nullptr, out,
                      &part);
}

}  // extern "C"

// Shared by akb_model_create and akb_batch_create. batch (may be null) gives
// the node and element ranges of independent instances of a union mesh:
// patches are then built per instance and every instance has its own time
// step.
static akb_status create_model(const akb_mesh_desc* mesh, int32_t nb_materials,
                               const akb_material_desc* materials,
                               const uint32_t* element_material,
                               const akb_model_options* options, const BatchLayout* batch,
                               akb_model** out, const PartLayout* part) {
  if (!out) return fail(AKB_ERR_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  if (!mesh || !materials || nb_materials < 1 || nb_materials > (1 << 24))
    return fail(AKB_ERR_INVALID_ARGUMENT, "mesh and 1..2^24 materials are required");
  const int type = mesh->element_type;
  if (type < AKB_SEGMENT_2 || type > AKB_HEXAHEDRON_8)
    return fail(AKB_ERR_UNSUPPORTED, "unsupported element type");
  if (mesh->spatial_dimension != dim_of(type))
    return fail(AKB_ERR_BAD_MESH, "spatial dimension does not match the element type");
  if (mesh->nb_nodes <= 0 || mesh->nb_elements < 0 || !mesh->nodes ||
      (mesh->nb_elements > 0 && !mesh->connectivity))
    return fail(AKB_ERR_BAD_MESH, "empty mesh");
  const int d = mesh->spatial_dimension, n = nnpe_of(type), q = nqp_of(type);
  const int64_t nn = mesh->nb_nodes, ne = mesh->nb_elements;
  if (ne * n >= INT32_MAX) return fail(AKB_ERR_UNSUPPORTED, "more than 2^31 element corners");
  for (int64_t k = 0; k < ne * n; ++k)
    if (mesh->connectivity[k] >= (uint64_t)nn)
      return fail(AKB_ERR_BAD_MESH, "connectivity refers to a node out of range");
  if (element_material)
    for (int64_t e = 0; e < ne; ++e)
      if (element_material[e] >= (uint32_t)nb_materials)
        return fail(AKB_ERR_INVALID_ARGUMENT, "material index out of range");
  int nb_user = 0;
  for (int k = 0; k < nb_materials; ++k) {
    const auto& md = materials[k];
    if (md.kind != AKB_MATERIAL_ELASTIC && md.kind != AKB_MATERIAL_NEOHOOKEAN &&
        md.kind != AKB_MATERIAL_USER)
      return fail(AKB_ERR_UNSUPPORTED, "unsupported material kind");
    nb_user += md.kind == AKB_MATERIAL_USER;
    if (!(md.rho > 0) || !(md.E > 0))
      return fail(AKB_ERR_INVALID_ARGUMENT, "material needs rho > 0 and E > 0");
  }
  akb_model_options opt{AKB_MODE_FP64_REFERENCE, 0, nullptr, 0, 0, 0};
  if (options) opt = *options;
  if (opt.precision_mode < AKB_MODE_FP64_REFERENCE || opt.precision_mode > AKB_MODE_FP32_BULK)
    return fail(AKB_ERR_INVALID_ARGUMENT, "unknown precision mode");
  if (nb_user && (nb_user != nb_materials || opt.precision_mode != AKB_MODE_FP64 || batch))
    return fail(AKB_ERR_UNSUPPORTED,
                "user materials: every material of the model, AKB_MODE_FP64, no batch");
  if (part) {
    if (opt.precision_mode == AKB_MODE_FP64_REFERENCE || nb_user || batch || ne == 0)
      return fail(AKB_ERR_UNSUPPORTED,
                  "partitioned mesh: AKB_MODE_FP64 or AKB_MODE_FP32_BULK, built-in materials, "
                  "elements");
    if (part->n < 0 || (part->n > 0 && !part->nodes))
      return fail(AKB_ERR_INVALID_ARGUMENT, "null interface node array");
    for (int64_t i = 0; i < part->n; ++i)
      if (part->nodes[i] >= (uint64_t)nn)
        return fail(AKB_ERR_INVALID_ARGUMENT, "interface node out of range");
  }

  auto m = std::make_unique<akb_model>();
  m->mode = opt.precision_mode;
  m->user = nb_user > 0;
  m->opt_patch_elements = opt.patch_elements;
  m->opt_patch_nodes = opt.patch_nodes;
  m->opt_patch_grid = opt.patch_grid;
  m->device = opt.device;
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  if (opt.stream) {
    m->stream = (cudaStream_t)opt.stream;
  } else {
    AKB_CUDA_TRY(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
    m->owns_stream = true;
  }
  DevModel& dm = m->dm;
  dm.dim = d;
  dm.type = type;
  dm.nnpe = n;
  dm.nqp = q;
  dm.nn = nn;
  dm.ne = ne;
  dm.nmat = nb_materials;
  akb_status st;
  {
    std::vector<MatParams> table(nb_materials);
    for (int k = 0; k < nb_materials; ++k) table[k] = make_params(materials[k], d);
    for (int k = 0; k < nb_materials && k < kMaxMaterials; ++k) dm.mats[k] = table[k];
    if ((st = upload(m.get(), table, &dm.mat_table)) != AKB_OK) return st;
    AKB_CUDA_TRY(cudaStreamSynchronize(m->stream));
  }

  const size_t ndof = (size_t)nn * d;
  // the fused step of the fast modes works on the mesh in its own node order
  // (akb_patch.cuh): plan the patches first, then store X and the
  // connectivity renumbered
  const bool patched = m->mode != AKB_MODE_FP64_REFERENCE && !m->user && ne > 0;
  PatchHost plan;
  std::vector<uint32_t> patch_inst, orphan_inst;
  std::vector<double> Xr;
  std::vector<uint32_t> Cr;
  const double* mesh_X = mesh->nodes;
  const uint32_t* mesh_C = mesh->connectivity;
  if (patched) {
    if ((st = plan_patches(m.get(), mesh, batch, part, plan, patch_inst, orphan_inst)) != AKB_OK)
      return st;
    Xr.resize(ndof);
    for (int64_t i = 0; i < nn; ++i)
      for (int c = 0; c < d; ++c) Xr[(size_t)plan.perm[i] * d + c] = mesh->nodes[i * d + c];
    Cr.resize((size_t)ne * n);
    for (int64_t k = 0; k < ne * n; ++k) Cr[k] = plan.perm[mesh->connectivity[k]];
    mesh_X = Xr.data();
    mesh_C = Cr.data();
  }
  double* X;
  uint32_t* conn;
  // nodal arrays carry 16 bytes of slack at their end: the fused step's bulk
  // copies and L2 prefetches round node ranges out to 16 bytes
  if ((st = dalloc(m.get(), &X, ndof + 2)) != AKB_OK) return st;
  if ((st = dalloc(m.get(), &conn, (size_t)ne * n)) != AKB_OK) return st;
  dm.X = X;
  dm.conn = conn;
  for (double** f : {&dm.u, &dm.v, &dm.a, &dm.fext, &dm.fint, &dm.mass})
    if ((st = dalloc(m.get(), f, ndof + 2)) != AKB_OK) return st;
  if ((st = dalloc(m.get(), &dm.inv_mass, nn + 2)) != AKB_OK) return st;
  if ((st = dalloc(m.get(), &dm.blocked, ndof + 16)) != AKB_OK) return st;
  AKB_CUDA_TRY(cudaMemcpyAsync(X, mesh_X, ndof * sizeof(double), cudaMemcpyHostToDevice, m->stream));
  if (ne > 0)
    AKB_CUDA_TRY(cudaMemcpyAsync(conn, mesh_C, (size_t)ne * n * sizeof(uint32_t),
                                 cudaMemcpyHostToDevice, m->stream));
  for (double* f : {dm.u, dm.v, dm.a, dm.fext, dm.fint, dm.mass})
    AKB_CUDA_TRY(cudaMemsetAsync(f, 0, ndof * sizeof(double), m->stream));
  AKB_CUDA_TRY(cudaMemsetAsync(dm.blocked, 0, ndof, m->stream));
  if (element_material) {
    uint32_t* mo;
    if ((st = dalloc(m.get(), &mo, ne)) != AKB_OK) return st;
    AKB_CUDA_TRY(cudaMemcpyAsync(mo, element_material, ne * sizeof(uint32_t), cudaMemcpyHostToDevice, m->stream));
    dm.mat_of = mo;
  }

  // node -> (element, corner) CSR in ascending element order: the order in
  // which DOFManager::assembleElementalArrayLocalArray adds element vectors.
  {
    std::vector<int32_t> ptr(nn + 1, 0), ent((size_t)ne * n);
    for (int64_t k = 0; k < ne * n; ++k) ptr[mesh_C[k] + 1]++;
    for (int64_t i = 0; i < nn; ++i) ptr[i + 1] += ptr[i];
    std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
    for (int64_t k = 0; k < ne * n; ++k) ent[fill[mesh_C[k]]++] = (int32_t)k;
    int32_t *dptr, *dent;
    if ((st = dalloc(m.get(), &dptr, nn + 1)) != AKB_OK) return st;
    if ((st = dalloc(m.get(), &dent, (size_t)ne * n)) != AKB_OK) return st;
    AKB_CUDA_TRY(cudaMemcpyAsync(dptr, ptr.data(), (nn + 1) * sizeof(int32_t), cudaMemcpyHostToDevice, m->stream));
    if (ne > 0)
      AKB_CUDA_TRY(cudaMemcpyAsync(dent, ent.data(), (size_t)ne * n * sizeof(int32_t),
                                   cudaMemcpyHostToDevice, m->stream));
    AKB_CUDA_TRY(cudaStreamSynchronize(m->stream));  // host vectors go out of scope
    dm.node_ptr = dptr;
    dm.node_ent = dent;
  }
  // element force buffer
  {
    // FP64 entries in every mode: the lumped-mass assembly writes FP64
    const size_t bytes = (size_t)ne * n * d * 8;
    char* fe;
    if ((st = dalloc(m.get(), &fe, bytes)) != AKB_OK) return st;
    dm.fe = fe;
  }
  // shape derivatives and detJ*w (initShapeFunctions); stored for the
  // reference-order path, temporary otherwise (used for the lumped mass).
  if ((st = dalloc(m.get(), &dm.B, (size_t)ne * q * d * n)) != AKB_OK) return st;
  if ((st = dalloc(m.get(), &dm.jac, (size_t)ne * q)) != AKB_OK) return st;
  if ((st = dalloc(m.get(), &m->d_result, 4)) != AKB_OK) return st;
  int* d_neg = reinterpret_cast<int*>(m->d_result);
  AKB_CUDA_TRY(cudaMemsetAsync(d_neg, 0, sizeof(int), m->stream));
  AKB_CUDA_TRY(ref_init_geometry(dm, m->stream, d_neg));
  int neg = 0;
  AKB_CUDA_TRY(cudaMemcpyAsync(&neg, d_neg, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
  AKB_CUDA_TRY(cudaStreamSynchronize(m->stream));
  if (neg) return fail(AKB_ERR_NEGATIVE_JACOBIAN,
                       "negative jacobian: check the element node ordering");
  // lumped mass depends only on the reference coordinates and rho
  AKB_CUDA_TRY(ref_mass(dm, m->stream));
  if (m->mode == AKB_MODE_FP64_REFERENCE) {
    if ((st = ensure_stress_arrays(m.get())) != AKB_OK) return st;
  } else {
    AKB_CUDA_TRY(cudaStreamSynchronize(m->stream));
    dfree(m.get(), dm.B);
    dfree(m.get(), dm.jac);
    m->device_bytes -= (int64_t)ne * q * d * n * 8 + (int64_t)ne * q * 8;
    dm.B = nullptr;
    dm.jac = nullptr;
  }
  if (m->user) {
    if ((st = ensure_stress_arrays(m.get())) != AKB_OK) return st;
    AKB_CUDA_TRY(cudaMemsetAsync(dm.stress, 0, (size_t)ne * q * d * d * sizeof(double), m->stream));
  } else if (patched) {
    if ((st = build_device_patches(m.get(), plan, patch_inst, orphan_inst, element_material, batch,
                                   part)) != AKB_OK)
      return st;
  }
  if (batch) {
    m->ninst = batch->ninst;
    m->node_off = batch->node_off;
    m->elem_off = batch->elem_off;
    std::vector<double> dts(batch->ninst, 0.0);
    if ((st = upload(m.get(), dts, (const double**)&m->d_inst_dt)) != AKB_OK) return st;
    if ((st = upload(m.get(), batch->elem_off, &m->d_elem_off)) != AKB_OK) return st;
    if ((st = upload(m.get(), batch->node_off, &m->d_node_off)) != AKB_OK) return st;
    m->patches.inst_dt = m->d_inst_dt;
    m->patches.node_off = m->d_node_off;
    m->patches.ninst = batch->ninst;
    m->dt = 1.0;  // the step reads the instances' time steps from the device
    AKB_CUDA_TRY(cudaStreamSynchronize(m->stream));
  }
  m->scratch_len = reduce_blocks(ne);
  if ((st = dalloc(m.get(), &m->d_scratch, m->scratch_len)) != AKB_OK) return st;
  AKB_CUDA_TRY(cudaMallocHost((void**)&m->h_result, 4 * sizeof(double)));
  AKB_CUDA_TRY(cudaStreamSynchronize(m->stream));
  *out = m.release();
  return AKB_OK;
}

extern "C" {

akb_status akb_model_destroy(akb_model* m) {
  if (!m) return AKB_OK;
  cudaSetDevice(m->device);
  cudaStreamSynchronize(m->stream);
  if (m->copy_stream) cudaStreamSynchronize(m->copy_stream);
  if (m->upload_stream) cudaStreamSynchronize(m->upload_stream);
  destroy_graphs(m);
  for (void* p : m->allocations) cudaFree(p);
  if (m->h_result) cudaFreeHost(m->h_result);
  for (auto& b : m->bc) {
    if (b.host) cudaFreeHost(b.host);
    if (b.done) cudaEventDestroy(b.done);
    if (b.copied) cudaEventDestroy(b.copied);
  }
  for (int k = 0; k < akb_model::kEnergySlots; ++k) {
    if (m->eres_ready[k]) cudaEventDestroy(m->eres_ready[k]);
    if (m->eres_copied[k]) cudaEventDestroy(m->eres_copied[k]);
  }
  if (m->copy_stream) cudaStreamDestroy(m->copy_stream);
  if (m->upload_stream) cudaStreamDestroy(m->upload_stream);
  if (m->owns_stream) cudaStreamDestroy(m->stream);
  delete m;
  return AKB_OK;
}

akb_status akb_model_get_info(const akb_model* m, akb_model_info* info) {
  if (!m || !info) return fail(AKB_ERR_INVALID_ARGUMENT, "null argument");
  info->spatial_dimension = m->dm.dim;
  info->element_type = m->dm.type;
  info->nodes_per_element = m->dm.nnpe;
  info->quadrature_points_per_element = m->dm.nqp;
  info->nb_nodes = m->dm.nn;
  info->nb_elements = m->dm.ne;
  info->precision_mode = m->mode;
  info->nb_materials = m->dm.nmat;
  info->device_bytes = m->device_bytes;
  return AKB_OK;
}

akb_status akb_set_field(akb_model* m, int32_t field, const double* values, int64_t count) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (field != AKB_FIELD_DISPLACEMENT && field != AKB_FIELD_VELOCITY &&
      field != AKB_FIELD_ACCELERATION && field != AKB_FIELD_EXTERNAL_FORCE)
    return fail(AKB_ERR_INVALID_ARGUMENT, "field is read-only");
  if (!values || count != field_count(m, field))
    return fail(AKB_ERR_INVALID_ARGUMENT, "wrong number of values");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  if (m->d_perm) {  // into the model's node order
    if ((st = ensure_tmp(m)) != AKB_OK) return st;
    AKB_CUDA_TRY(cudaMemcpyAsync(m->d_tmp, values, count * sizeof(double), cudaMemcpyHostToDevice,
                                 m->stream));
    AKB_CUDA_TRY(permute_rows(m->d_perm, m->dm.nn, m->dm.dim, m->d_tmp, field_ptr(m, field), true,
                              m->stream));
  } else {
    AKB_CUDA_TRY(cudaMemcpyAsync(field_ptr(m, field), values, count * sizeof(double),
                                 cudaMemcpyHostToDevice, m->stream));
  }
  if (field != AKB_FIELD_EXTERNAL_FORCE) m->w_valid = false;
  if (field == AKB_FIELD_VELOCITY) m->ke_valid = false;
  if (field == AKB_FIELD_DISPLACEMENT) {
    m->fint_valid = false;
    m->stresses_valid = false;
  }
  if (field == AKB_FIELD_EXTERNAL_FORCE) {
    bool any = false;
    for (int64_t i = 0; i < count && !any; ++i) any = values[i] != 0.0;
    m->has_fext = any;
  }
  return sync(m);
}

akb_status akb_get_field(akb_model* m, int32_t field, double* values, int64_t count) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (field < AKB_FIELD_DISPLACEMENT || field > AKB_FIELD_STRESS)
    return fail(AKB_ERR_INVALID_ARGUMENT, "unknown field");
  if (!values || count != field_count(m, field))
    return fail(AKB_ERR_INVALID_ARGUMENT, "wrong number of values");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  if (field == AKB_FIELD_INTERNAL_FORCE && !m->fint_valid) {
    AKB_CUDA_TRY(enqueue_internal_forces(m));
    m->fint_valid = true;
  }
  if ((field == AKB_FIELD_GRAD_U || field == AKB_FIELD_STRESS) && !m->stresses_valid && !m->user) {
    if ((st = akb_compute_stresses(m)) != AKB_OK) return st;
  }
  if (m->d_perm && nodal(field)) {  // back to the caller's node order
    if ((st = ensure_tmp(m)) != AKB_OK) return st;
    AKB_CUDA_TRY(permute_rows(m->d_perm, m->dm.nn, m->dm.dim, field_ptr(m, field), m->d_tmp,
                              false, m->stream));
    AKB_CUDA_TRY(cudaMemcpyAsync(values, m->d_tmp, count * sizeof(double), cudaMemcpyDeviceToHost,
                                 m->stream));
  } else {
    AKB_CUDA_TRY(cudaMemcpyAsync(values, field_ptr(m, field), count * sizeof(double),
                                 cudaMemcpyDeviceToHost, m->stream));
  }
  return sync(m);
}

akb_status akb_field_device_pointer(akb_model* m, int32_t field, void** dptr) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (!dptr) return fail(AKB_ERR_INVALID_ARGUMENT, "null output");
  if (field == AKB_FIELD_GRAD_U || field == AKB_FIELD_STRESS) {
    if ((st = ensure_stress_arrays(m)) != AKB_OK) return st;
  }
  *dptr = field_ptr(m, field);
  if (!*dptr) return fail(AKB_ERR_INVALID_ARGUMENT, "unknown field");
  return AKB_OK;
}

akb_status akb_get_node_numbering(const akb_model* m, uint32_t* row_of_node, int64_t count) {
  if (!m || !row_of_node) return fail(AKB_ERR_INVALID_ARGUMENT, "null argument");
  if (count != m->dm.nn) return fail(AKB_ERR_INVALID_ARGUMENT, "wrong number of values");
  for (int64_t i = 0; i < count; ++i)
    row_of_node[i] = m->perm.empty() ? (uint32_t)i : m->perm[i];
  return AKB_OK;
}

akb_status akb_set_blocked_dofs(akb_model* m, const uint8_t* blocked, int64_t count) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (!blocked || count != m->dm.nn * m->dm.dim)
    return fail(AKB_ERR_INVALID_ARGUMENT, "wrong number of values");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  if (m->d_perm) {
    if ((st = ensure_tmp(m)) != AKB_OK) return st;
    uint8_t* t = reinterpret_cast<uint8_t*>(m->d_tmp);
    AKB_CUDA_TRY(cudaMemcpyAsync(t, blocked, count, cudaMemcpyHostToDevice, m->stream));
    AKB_CUDA_TRY(permute_rows_u8(m->d_perm, m->dm.nn, m->dm.dim, t, m->dm.blocked, true, m->stream));
  } else {
    AKB_CUDA_TRY(cudaMemcpyAsync(m->dm.blocked, blocked, count, cudaMemcpyHostToDevice, m->stream));
  }
  m->w_valid = false;
  return sync(m);
}

akb_status akb_get_blocked_dofs(akb_model* m, uint8_t* blocked, int64_t count) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (!blocked || count != m->dm.nn * m->dm.dim)
    return fail(AKB_ERR_INVALID_ARGUMENT, "wrong number of values");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  if (m->d_perm) {
    if ((st = ensure_tmp(m)) != AKB_OK) return st;
    uint8_t* t = reinterpret_cast<uint8_t*>(m->d_tmp);
    AKB_CUDA_TRY(permute_rows_u8(m->d_perm, m->dm.nn, m->dm.dim, m->dm.blocked, t, false, m->stream));
    AKB_CUDA_TRY(cudaMemcpyAsync(blocked, t, count, cudaMemcpyDeviceToHost, m->stream));
  } else {
    AKB_CUDA_TRY(cudaMemcpyAsync(blocked, m->dm.blocked, count, cudaMemcpyDeviceToHost, m->stream));
  }
  return sync(m);
}

akb_status akb_assemble_mass_lumped(akb_model* m) {
  // The lumped mass depends only on the reference coordinates and the
  // densities; it is assembled once in akb_model_create, as the reference
  // assembles it once (need_to_reassemble_lumped_mass,
  // solid_mechanics_model_mass.cc:61-62).
  return check_model(m);
}

akb_status akb_get_stable_time_step(akb_model* m, double* dt) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (!dt) return fail(AKB_ERR_INVALID_ARGUMENT, "null output");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  AKB_CUDA_TRY(stable_dt(m->dm, m->d_scratch, m->scratch_len, m->d_result, m->stream));
  AKB_CUDA_TRY(cudaMemcpyAsync(m->h_result, m->d_result, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  if ((st = sync(m)) != AKB_OK) return st;
  *dt = *m->h_result;
  return AKB_OK;
}

akb_status akb_set_time_step(akb_model* m, double dt) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (!(dt > 0) || !std::isfinite(dt)) return fail(AKB_ERR_INVALID_ARGUMENT, "time step must be > 0");
  if (dt != m->dt) m->w_valid = false;
  m->dt = dt;
  return AKB_OK;
}

akb_status akb_get_time_step(const akb_model* m, double* dt) {
  if (!m || !dt) return fail(AKB_ERR_INVALID_ARGUMENT, "null argument");
  *dt = m->dt;
  return AKB_OK;
}

akb_status akb_solve_step(akb_model* m) { return akb_solve_steps(m, 1); }

static akb_status get_graph(akb_model* m, int64_t k, cudaGraphExec_t* exec) {
  auto it = m->graphs.find(k);
  if (it != m->graphs.end()) {
    *exec = it->second;
    return AKB_OK;
  }
  cudaGraph_t g;
  AKB_CUDA_TRY(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t err = cudaSuccess;
  for (int64_t s = 0; s < k && err == cudaSuccess; ++s) err = enqueue_step(m);
  cudaError_t end = cudaStreamEndCapture(m->stream, &g);
  if (err != cudaSuccess) return fail(AKB_ERR_CUDA, cudaGetErrorString(err));
  if (end != cudaSuccess) return fail(AKB_ERR_CUDA, cudaGetErrorString(end));
  cudaError_t inst = cudaGraphInstantiate(exec, g, 0);
  cudaGraphDestroy(g);
  if (inst != cudaSuccess) return fail(AKB_ERR_CUDA, cudaGetErrorString(inst));
  m->graphs[k] = *exec;
  return AKB_OK;
}

// Graphs of kGraphSteps steps (and of the remainder) for nb_steps steps.
static constexpr int64_t kGraphSteps = 32;
static akb_status prepare_graphs(akb_model* m, int64_t nb_steps, cudaGraphExec_t* full,
                                 cudaGraphExec_t* rest) {
  if (m->graph_dt != m->dt || m->graph_fext != m->has_fext) {
    destroy_graphs(m);
    m->graph_dt = m->dt;
    m->graph_fext = m->has_fext;
  }
  akb_status st;
  const int64_t chunk = nb_steps >= kGraphSteps ? kGraphSteps : nb_steps;
  *full = *rest = nullptr;
  if ((st = get_graph(m, chunk, full)) != AKB_OK) return st;
  const int64_t rem = nb_steps % chunk;
  if (rem && (st = get_graph(m, rem, rest)) != AKB_OK) return st;
  return AKB_OK;
}

akb_status akb_solve_steps(akb_model* m, int64_t nb_steps) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (m->user)
    return fail(AKB_ERR_STATE, "user material: step with akb_step_begin / akb_step_end");
  if (m->part)
    return fail(AKB_ERR_STATE, "partitioned mesh: step with akb_part_step_begin / akb_part_step_end");
  if (nb_steps < 0) return fail(AKB_ERR_INVALID_ARGUMENT, "negative step count");
  if (!(m->dt > 0)) return fail(AKB_ERR_STATE, "time step not set");
  if (nb_steps == 0) return AKB_OK;
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  if ((st = ensure_w(m)) != AKB_OK) return st;
  if (nb_steps == 1) {
    AKB_CUDA_TRY(enqueue_step(m));
  } else {
    cudaGraphExec_t full, rest;
    if ((st = prepare_graphs(m, nb_steps, &full, &rest)) != AKB_OK) return st;
    const int64_t chunk = nb_steps >= kGraphSteps ? kGraphSteps : nb_steps;
    const int64_t reps = nb_steps / chunk;
    for (int64_t r = 0; r < reps; ++r) AKB_CUDA_TRY(cudaGraphLaunch(full, m->stream));
    if (rest) AKB_CUDA_TRY(cudaGraphLaunch(rest, m->stream));
  }
  // the fused patch step keeps the internal force on chip; it is recomputed
  // on demand at the (unchanged) displacement
  m->fint_valid = !m->use_patches;
  m->stresses_valid = false;
  m->ke_valid = m->use_patches;
  return AKB_OK;
}

akb_status akb_time_solve_steps(akb_model* m, int64_t nb_steps, double* elapsed_ms) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (m->user)
    return fail(AKB_ERR_STATE, "user material: step with akb_step_begin / akb_step_end");
  if (m->part)
    return fail(AKB_ERR_STATE, "partitioned mesh: step with akb_part_step_begin / akb_part_step_end");
  if (!elapsed_ms) return fail(AKB_ERR_INVALID_ARGUMENT, "null output");
  if (!(m->dt > 0)) return fail(AKB_ERR_STATE, "time step not set");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  if ((st = ensure_w(m)) != AKB_OK) return st;
  if (nb_steps > 1) {  // instantiate the graphs outside the timed region
    cudaGraphExec_t full, rest;
    if ((st = prepare_graphs(m, nb_steps, &full, &rest)) != AKB_OK) return st;
  }
  cudaEvent_t e0, e1;
  AKB_CUDA_TRY(cudaEventCreate(&e0));
  AKB_CUDA_TRY(cudaEventCreate(&e1));
  AKB_CUDA_TRY(cudaEventRecord(e0, m->stream));
  st = akb_solve_steps(m, nb_steps);
  AKB_CUDA_TRY(cudaEventRecord(e1, m->stream));
  AKB_CUDA_TRY(cudaEventSynchronize(e1));
  float ms = 0;
  AKB_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *elapsed_ms = ms;
  return st;
}

akb_status akb_assemble_internal_forces(akb_model* m) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  AKB_CUDA_TRY(enqueue_internal_forces(m));
  m->fint_valid = true;
  return sync(m);
}

akb_status akb_compute_stresses(akb_model* m) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (m->user) return fail(AKB_ERR_UNSUPPORTED, "user material: the caller computes the stresses");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  if ((st = ensure_stress_arrays(m)) != AKB_OK) return st;
  AKB_CUDA_TRY(ref_compute_stresses(m->dm, m->dm.B == nullptr, m->stream));
  m->stresses_valid = true;
  return sync(m);
}

akb_status akb_get_energy(akb_model* m, int32_t kind, double* value) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (!value) return fail(AKB_ERR_INVALID_ARGUMENT, "null output");
  if (kind < AKB_ENERGY_KINETIC || kind > AKB_ENERGY_EXTERNAL_WORK)
    return fail(AKB_ERR_INVALID_ARGUMENT, "unknown energy");
  if (m->user && kind == AKB_ENERGY_POTENTIAL)
    return fail(AKB_ERR_UNSUPPORTED, "user material: no potential energy");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  if (kind == AKB_ENERGY_EXTERNAL_WORK && !m->fint_valid) {
    AKB_CUDA_TRY(enqueue_internal_forces(m));
    m->fint_valid = true;
  }
  AKB_CUDA_TRY(enqueue_energy(m, kind, m->d_result));
  AKB_CUDA_TRY(cudaMemcpyAsync(m->h_result, m->d_result, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  if ((st = sync(m)) != AKB_OK) return st;
  *value = *m->h_result;
  return AKB_OK;
}

akb_status akb_get_energy_async(akb_model* m, int32_t kind, double* value) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (!value) return fail(AKB_ERR_INVALID_ARGUMENT, "null output");
  if (kind < AKB_ENERGY_KINETIC || kind > AKB_ENERGY_EXTERNAL_WORK)
    return fail(AKB_ERR_INVALID_ARGUMENT, "unknown energy");
  if (m->user && kind == AKB_ENERGY_POTENTIAL)
    return fail(AKB_ERR_UNSUPPORTED, "user material: no potential energy");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  if (kind == AKB_ENERGY_EXTERNAL_WORK && !m->fint_valid) {
    AKB_CUDA_TRY(enqueue_internal_forces(m));
    m->fint_valid = true;
  }
  if ((st = ensure_copy_stream(m)) != AKB_OK) return st;
  if (!m->d_eres && (st = dalloc(m, &m->d_eres, akb_model::kEnergySlots)) != AKB_OK) return st;
  const int k = m->eres_next;
  m->eres_next = (k + 1) % akb_model::kEnergySlots;
  if (!m->eres_ready[k]) {
    AKB_CUDA_TRY(cudaEventCreateWithFlags(&m->eres_ready[k], cudaEventDisableTiming));
    AKB_CUDA_TRY(cudaEventCreateWithFlags(&m->eres_copied[k], cudaEventDisableTiming));
  }
  // the slot's previous value has been copied out before it is written again
  if (m->eres_pending[k]) AKB_CUDA_TRY(cudaStreamWaitEvent(m->stream, m->eres_copied[k], 0));
  AKB_CUDA_TRY(enqueue_energy(m, kind, m->d_eres + k));
  AKB_CUDA_TRY(cudaEventRecord(m->eres_ready[k], m->stream));
  AKB_CUDA_TRY(cudaStreamWaitEvent(m->copy_stream, m->eres_ready[k], 0));
  AKB_CUDA_TRY(cudaMemcpyAsync(value, m->d_eres + k, sizeof(double), cudaMemcpyDefault,
                               m->copy_stream));
  AKB_CUDA_TRY(cudaEventRecord(m->eres_copied[k], m->copy_stream));
  m->eres_pending[k] = true;
  return AKB_OK;
}

akb_status akb_apply_dirichlet(akb_model* m, const uint32_t* nodes, int64_t nb_nodes,
                               int32_t component, const double* values) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (nb_nodes < 0 || (nb_nodes > 0 && (!nodes || !values)))
    return fail(AKB_ERR_INVALID_ARGUMENT, "null node or value array");
  if ((component < 0 && component != AKB_ALL_COMPONENTS) || component >= m->dm.dim)
    return fail(AKB_ERR_INVALID_ARGUMENT, "component out of range");
  const int64_t nvals = component == AKB_ALL_COMPONENTS ? nb_nodes * m->dm.dim : nb_nodes;
  if (nb_nodes == 0) return AKB_OK;
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  // the caller's arrays are copied to a pinned staging slot on the host, so
  // they may be reused as soon as the call returns; the upload and the kernel
  // are queued on the model's stream without waiting for them
  if ((st = ensure_copy_stream(m)) != AKB_OK) return st;
  akb_model::BcSlot& b = m->bc[m->bc_next];
  m->bc_next = (m->bc_next + 1) % akb_model::kBcSlots;
  if (!b.done) {
    AKB_CUDA_TRY(cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming));
    AKB_CUDA_TRY(cudaEventCreateWithFlags(&b.copied, cudaEventDisableTiming));
  }
  if (b.pending) AKB_CUDA_TRY(cudaEventSynchronize(b.done));
  b.pending = false;
  const size_t nbytes = ((size_t)nb_nodes * sizeof(uint32_t) + 7) & ~size_t(7);
  const size_t bytes = nbytes + (size_t)nvals * sizeof(double);
  if ((int64_t)bytes > b.capacity) {
    if (b.host) cudaFreeHost(b.host);
    dfree(m, b.dev);
    b.host = nullptr;
    b.dev = nullptr;
    b.capacity = 0;
    AKB_CUDA_TRY(cudaMallocHost((void**)&b.host, bytes));
    if ((st = dalloc(m, &b.dev, bytes)) != AKB_OK) return st;
    b.capacity = (int64_t)bytes;
  }
  std::memcpy(b.host, nodes, (size_t)nb_nodes * sizeof(uint32_t));
  std::memcpy(b.host + nbytes, values, (size_t)nvals * sizeof(double));
  // the upload runs on the upload stream (overlapping the kernels queued
  // before it); the update kernel waits for it on the model's stream
  AKB_CUDA_TRY(cudaMemcpyAsync(b.dev, b.host, bytes, cudaMemcpyHostToDevice, m->upload_stream));
  AKB_CUDA_TRY(cudaEventRecord(b.copied, m->upload_stream));
  AKB_CUDA_TRY(cudaStreamWaitEvent(m->stream, b.copied, 0));
  AKB_CUDA_TRY(apply_dirichlet(m->dm, reinterpret_cast<const uint32_t*>(b.dev), nb_nodes, component,
                               reinterpret_cast<const double*>(b.dev + nbytes), m->d_perm,
                               m->use_patches ? m->patches.w : nullptr, m->stream));
  AKB_CUDA_TRY(cudaEventRecord(b.done, m->stream));
  b.pending = true;
  m->fint_valid = false;
  m->stresses_valid = false;
  return AKB_OK;
}

akb_status akb_time_kernels(akb_model* m, int64_t nb_steps, double* ms_per_launch,
                            int32_t nb_slots) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (!ms_per_launch || nb_slots < 0 || nb_steps < 1)
    return fail(AKB_ERR_INVALID_ARGUMENT, "bad timing arguments");
  if (m->user)
    return fail(AKB_ERR_STATE, "user material: step with akb_step_begin / akb_step_end");
  if (m->part)
    return fail(AKB_ERR_STATE, "partitioned mesh: step with akb_part_step_begin / akb_part_step_end");
  if (!(m->dt > 0)) return fail(AKB_ERR_STATE, "time step not set");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  if ((st = ensure_w(m)) != AKB_OK) return st;
  StepTimer t;
  for (auto& e : t.ev) AKB_CUDA_TRY(cudaEventCreate(&e));
  double acc[AKB_MAX_KERNEL_SLOTS] = {0};
  int nk = 0;
  for (int64_t s = 0; s < nb_steps; ++s) {
    t.n = 0;
    AKB_CUDA_TRY(enqueue_step(m, &t));
    AKB_CUDA_TRY(cudaEventSynchronize(t.ev[t.n - 1]));
    nk = t.n - 1;
    for (int k = 0; k < nk; ++k) {
      float ms = 0;
      AKB_CUDA_TRY(cudaEventElapsedTime(&ms, t.ev[k], t.ev[k + 1]));
      acc[k] += ms;
    }
  }
  for (auto& e : t.ev) cudaEventDestroy(e);
  for (int k = 0; k < nb_slots; ++k) ms_per_launch[k] = k < nk ? acc[k] / nb_steps : 0.0;
  m->fint_valid = !m->use_patches;
  m->stresses_valid = false;
  m->ke_valid = m->use_patches;
  return AKB_OK;
}

const char* akb_kernel_name(const akb_model* m, int32_t slot) {
  if (!m) return "";
  return kernel_name(m, slot);
}

akb_status akb_batch_create(const akb_batch_desc* batch, const akb_model_options* options,
                            akb_model** out) {
  if (!out) return fail(AKB_ERR_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  if (!batch || batch->nb_instances < 1 || !batch->meshes || !batch->materials)
    return fail(AKB_ERR_INVALID_ARGUMENT, "batch needs at least one mesh and its materials");
  const akb_model_options opt =
      options ? *options : akb_model_options{AKB_MODE_FP64, 0, nullptr, 0, 0, 0};
  if (opt.precision_mode == AKB_MODE_FP64_REFERENCE)
    return fail(AKB_ERR_UNSUPPORTED, "batches run the fast modes (AKB_MODE_FP64 or AKB_MODE_FP32_BULK)");
  const akb_mesh_desc& m0 = batch->meshes[0];
  BatchLayout lay;
  lay.ninst = batch->nb_instances;
  lay.node_off.push_back(0);
  lay.elem_off.push_back(0);
  const int n = nnpe_of(m0.element_type), d = m0.spatial_dimension;
  for (int i = 0; i < lay.ninst; ++i) {
    const akb_mesh_desc& mi = batch->meshes[i];
    if (mi.element_type != m0.element_type || mi.spatial_dimension != d)
      return fail(AKB_ERR_BAD_MESH, "instances of a batch share one element type");
    if (mi.nb_nodes <= 0 || mi.nb_elements <= 0 || !mi.nodes || !mi.connectivity)
      return fail(AKB_ERR_BAD_MESH, "empty instance mesh");
    for (int64_t k = 0; k < mi.nb_elements * n; ++k)
      if (mi.connectivity[k] >= (uint64_t)mi.nb_nodes)
        return fail(AKB_ERR_BAD_MESH, "instance connectivity refers to a node out of range");
    lay.node_off.push_back(lay.node_off.back() + mi.nb_nodes);
    lay.elem_off.push_back(lay.elem_off.back() + mi.nb_elements);
  }
  if (lay.node_off.back() >= (int64_t)UINT32_MAX)
    return fail(AKB_ERR_UNSUPPORTED, "more than 2^32 nodes in a batch");
  std::vector<double> X((size_t)lay.node_off.back() * d);
  std::vector<uint32_t> conn((size_t)lay.elem_off.back() * n), mat(lay.elem_off.back());
  for (int i = 0; i < lay.ninst; ++i) {
    const akb_mesh_desc& mi = batch->meshes[i];
    std::copy(mi.nodes, mi.nodes + mi.nb_nodes * d, X.begin() + lay.node_off[i] * d);
    for (int64_t k = 0; k < mi.nb_elements * n; ++k)
      conn[lay.elem_off[i] * n + k] = (uint32_t)(mi.connectivity[k] + lay.node_off[i]);
    std::fill(mat.begin() + lay.elem_off[i], mat.begin() + lay.elem_off[i + 1], (uint32_t)i);
  }
  akb_mesh_desc um{d, m0.element_type, lay.node_off.back(), lay.elem_off.back(), X.data(),
                   conn.data()};
  return create_model(&um, lay.ninst, batch->materials, mat.data(), &opt, &lay, out);
}

akb_status akb_batch_get_layout(const akb_model* m, int32_t* nb_instances, int64_t* node_offsets,
                                int64_t* element_offsets) {
  if (!m) return fail(AKB_ERR_INVALID_ARGUMENT, "null model");
  if (m->ninst == 0) return fail(AKB_ERR_STATE, "not a batch");
  if (nb_instances) *nb_instances = m->ninst;
  if (node_offsets) std::copy(m->node_off.begin(), m->node_off.end(), node_offsets);
  if (element_offsets) std::copy(m->elem_off.begin(), m->elem_off.end(), element_offsets);
  return AKB_OK;
}

akb_status akb_batch_set_time_steps(akb_model* m, const double* dt) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (m->ninst == 0) return fail(AKB_ERR_STATE, "not a batch");
  if (!dt) return fail(AKB_ERR_INVALID_ARGUMENT, "null time steps");
  for (int i = 0; i < m->ninst; ++i)
    if (!(dt[i] > 0) || !std::isfinite(dt[i]))
      return fail(AKB_ERR_INVALID_ARGUMENT, "time steps must be > 0");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  AKB_CUDA_TRY(cudaMemcpyAsync(m->d_inst_dt, dt, m->ninst * sizeof(double), cudaMemcpyHostToDevice,
                               m->stream));
  m->w_valid = false;
  return sync(m);
}

akb_status akb_batch_get_stable_time_steps(akb_model* m, double* dt) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (m->ninst == 0) return fail(AKB_ERR_STATE, "not a batch");
  if (!dt) return fail(AKB_ERR_INVALID_ARGUMENT, "null output");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  double* out;
  if ((st = dalloc(m, &out, m->ninst)) != AKB_OK) return st;
  cudaError_t e = stable_dt_instances(m->dm, m->d_elem_off, m->ninst, out, m->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dt, out, m->ninst * sizeof(double), cudaMemcpyDeviceToHost, m->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  dfree(m, out);
  if (e != cudaSuccess) return fail(AKB_ERR_CUDA, cudaGetErrorString(e));
  return AKB_OK;
}

akb_status akb_batch_get_energies(akb_model* m, int32_t kind, double* values) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (m->ninst == 0) return fail(AKB_ERR_STATE, "not a batch");
  if (!values) return fail(AKB_ERR_INVALID_ARGUMENT, "null output");
  if (kind != AKB_ENERGY_KINETIC && kind != AKB_ENERGY_POTENTIAL)
    return fail(AKB_ERR_UNSUPPORTED, "per-instance energies: kinetic or potential");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  double* out;
  if ((st = dalloc(m, &out, m->ninst)) != AKB_OK) return st;
  cudaError_t e = energy_instances(m->dm, kind, m->d_node_off, m->d_elem_off, m->ninst, out, m->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(values, out, m->ninst * sizeof(double), cudaMemcpyDeviceToHost, m->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  dfree(m, out);
  if (e != cudaSuccess) return fail(AKB_ERR_CUDA, cudaGetErrorString(e));
  return AKB_OK;
}

akb_status akb_synchronize(akb_model* m) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  return sync(m);
}

akb_status akb_model_get_stream(akb_model* m, void** stream) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (!stream) return fail(AKB_ERR_INVALID_ARGUMENT, "null output");
  *stream = (void*)m->stream;
  return AKB_OK;
}

// The explicit step split around Material::computeStress: predictor and
// grad u (begin), then the caller's stresses, then internal forces, lumped
// solve and corrector (end) -- the order of NonLinearSolverLumped::solve
// (non_linear_solver_lumped.cc:58-82) with computeAllStresses between.
akb_status akb_step_begin(akb_model* m) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (!m->user) return fail(AKB_ERR_STATE, "akb_step_begin needs AKB_MATERIAL_USER materials");
  if (m->in_step) return fail(AKB_ERR_STATE, "akb_step_begin called twice");
  if (!(m->dt > 0)) return fail(AKB_ERR_STATE, "time step not set");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  AKB_CUDA_TRY(fast_predictor(m->dm, m->dt, m->stream));
  AKB_CUDA_TRY(user_qp_gradients(m->dm, m->stream));
  m->in_step = true;
  m->fint_valid = false;
  return AKB_OK;
}

akb_status akb_step_end(akb_model* m) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (!m->in_step) return fail(AKB_ERR_STATE, "akb_step_end without akb_step_begin");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  AKB_CUDA_TRY(user_element_forces(m->dm, m->stream));
  AKB_CUDA_TRY(fast_gather_correct(m->dm, m->dt, false, true, m->has_fext, m->stream));
  m->in_step = false;
  m->fint_valid = true;
  return AKB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Parts of a partitioned mesh (one process and GPU each): the step is split
// around the sum of the interface nodes' forces over all parts.
extern "C" {

static akb_status check_part(akb_model* m) {
  akb_status st;
  if ((st = check_model(m)) != AKB_OK) return st;
  if (!m->part) return fail(AKB_ERR_STATE, "not a partitioned model (akb_model_create_part)");
  return AKB_OK;
}

akb_status akb_part_step_begin(akb_model* m) {
  akb_status st;
  if ((st = check_part(m)) != AKB_OK) return st;
  if (m->part_in_step) return fail(AKB_ERR_STATE, "step already begun");
  if (!(m->dt > 0)) return fail(AKB_ERR_STATE, "time step not set");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  if ((st = ensure_w(m)) != AKB_OK) return st;
  AKB_CUDA_TRY(patch_step(m->dm, m->patches, m->dt, fp32(m), m->has_fext, m->stream));
  m->part_in_step = true;
  return AKB_OK;
}

akb_status akb_part_export_forces(akb_model* m, double* device_out) {
  akb_status st;
  if ((st = check_part(m)) != AKB_OK) return st;
  if (!m->part_in_step) return fail(AKB_ERR_STATE, "no step begun");
  if (m->n_iface > 0 && !device_out) return fail(AKB_ERR_INVALID_ARGUMENT, "null output");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  AKB_CUDA_TRY(patch_iface_export(m->dm, m->patches, m->d_iface_part, m->d_iface_k, m->n_iface,
                                  device_out, m->stream));
  return AKB_OK;
}

akb_status akb_part_step_end(akb_model* m, const double* device_in) {
  akb_status st;
  if ((st = check_part(m)) != AKB_OK) return st;
  if (!m->part_in_step) return fail(AKB_ERR_STATE, "no step begun");
  if (m->n_iface > 0 && !device_in) return fail(AKB_ERR_INVALID_ARGUMENT, "null input");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  AKB_CUDA_TRY(patch_iface_import(m->dm, m->patches, m->d_iface_part, m->d_iface_k, m->n_iface,
                                  device_in, m->stream));
  AKB_CUDA_TRY(patch_finish_list(m->dm, m->patches, m->dt, m->has_fext, m->stream));
  m->part_in_step = false;
  m->ke_valid = true;
  m->fint_valid = false;
  m->stresses_valid = false;
  return AKB_OK;
}

akb_status akb_part_set_exchange(akb_model* m, int64_t nb_send, const uint32_t* send_rows,
                                 int64_t nb_recv, const int64_t* sum_ptr,
                                 const int64_t* sum_src) {
  akb_status st;
  if ((st = check_part(m)) != AKB_OK) return st;
  if (m->part_in_step) return fail(AKB_ERR_STATE, "inside a step");
  const int64_t n = m->n_iface;
  if (nb_send < 0 || nb_recv < 0 || (nb_send > 0 && !send_rows) || !sum_ptr ||
      (n > 0 && !sum_src))
    return fail(AKB_ERR_INVALID_ARGUMENT, "exchange plan: null array or negative size");
  if (nb_send >= INT32_MAX || nb_recv >= INT32_MAX)
    return fail(AKB_ERR_INVALID_ARGUMENT, "exchange plan: more than 2^31 - 1 rows");
  for (int64_t k = 0; k < nb_send; ++k)
    if ((int64_t)send_rows[k] >= n)
      return fail(AKB_ERR_INVALID_ARGUMENT, "exchange plan: send row out of range");
  if (sum_ptr[0] != 0) return fail(AKB_ERR_INVALID_ARGUMENT, "exchange plan: sum_ptr[0] != 0");
  std::vector<uint32_t> ptr(n + 1), rows(send_rows, send_rows + nb_send);
  std::vector<int32_t> src;
  for (int64_t i = 0; i < n; ++i) {
    if (sum_ptr[i + 1] < sum_ptr[i] || sum_ptr[i + 1] >= INT32_MAX)
      return fail(AKB_ERR_INVALID_ARGUMENT, "exchange plan: sum_ptr not ascending");
    int own = 0;
    for (int64_t j = sum_ptr[i]; j < sum_ptr[i + 1]; ++j) {
      const int64_t v = sum_src[j];
      if (v < -1 || v >= nb_recv)
        return fail(AKB_ERR_INVALID_ARGUMENT, "exchange plan: sum term out of range");
      own += v == -1;
      src.push_back((int32_t)v);
    }
    if (own != 1)
      return fail(AKB_ERR_INVALID_ARGUMENT,
                  "exchange plan: every interface row sums its own value exactly once");
    ptr[i + 1] = (uint32_t)sum_ptr[i + 1];
  }
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  akb::ExchangePlan x;
  x.n_send = nb_send;
  x.n_recv = nb_recv;
  x.n_rows = n;
  if (nb_send > 0 && (st = upload(m, rows, &x.send_rows)) != AKB_OK) return st;
  if ((st = upload(m, ptr, &x.sum_ptr)) != AKB_OK) return st;
  if (!src.empty() && (st = upload(m, src, &x.sum_src)) != AKB_OK) return st;
  m->xplan = x;
  m->has_xplan = true;
  return AKB_OK;
}

static akb_status check_xplan(akb_model* m) {
  akb_status st;
  if ((st = check_part(m)) != AKB_OK) return st;
  if (!m->has_xplan) return fail(AKB_ERR_STATE, "no exchange plan (akb_part_set_exchange)");
  return AKB_OK;
}

akb_status akb_part_pack_forces(akb_model* m, double* device_send) {
  akb_status st;
  if ((st = check_xplan(m)) != AKB_OK) return st;
  if (!m->part_in_step) return fail(AKB_ERR_STATE, "no step begun");
  if (m->xplan.n_send > 0 && !device_send) return fail(AKB_ERR_INVALID_ARGUMENT, "null output");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  AKB_CUDA_TRY(patch_iface_pack(m->dm, m->patches, m->d_iface_part, m->d_iface_k, m->xplan,
                                device_send, m->stream));
  return AKB_OK;
}

akb_status akb_part_step_end_exchange(akb_model* m, const double* device_recv) {
  akb_status st;
  if ((st = check_xplan(m)) != AKB_OK) return st;
  if (!m->part_in_step) return fail(AKB_ERR_STATE, "no step begun");
  if (m->xplan.n_recv > 0 && !device_recv) return fail(AKB_ERR_INVALID_ARGUMENT, "null input");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  AKB_CUDA_TRY(patch_iface_sum_import(m->dm, m->patches, m->d_iface_part, m->d_iface_k,
                                      m->xplan, device_recv, m->stream));
  AKB_CUDA_TRY(patch_finish_list(m->dm, m->patches, m->dt, m->has_fext, m->stream));
  m->part_in_step = false;
  m->ke_valid = true;
  m->fint_valid = false;
  m->stresses_valid = false;
  return AKB_OK;
}

akb_status akb_part_pack_mass(akb_model* m, double* device_send) {
  akb_status st;
  if ((st = check_xplan(m)) != AKB_OK) return st;
  if (m->xplan.n_send > 0 && !device_send) return fail(AKB_ERR_INVALID_ARGUMENT, "null output");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  AKB_CUDA_TRY(mass_pack(m->dm, m->d_iface_g, m->xplan, device_send, m->stream));
  return AKB_OK;
}

akb_status akb_part_import_mass_exchange(akb_model* m, const double* device_recv) {
  akb_status st;
  if ((st = check_xplan(m)) != AKB_OK) return st;
  if (m->part_in_step) return fail(AKB_ERR_STATE, "inside a step");
  if (m->xplan.n_recv > 0 && !device_recv) return fail(AKB_ERR_INVALID_ARGUMENT, "null input");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  AKB_CUDA_TRY(mass_sum_import(m->dm, m->d_iface_g, m->xplan, device_recv, m->stream));
  m->ke_valid = false;
  return AKB_OK;
}

akb_status akb_part_export_mass(akb_model* m, double* device_out) {
  akb_status st;
  if ((st = check_part(m)) != AKB_OK) return st;
  if (m->n_iface > 0 && !device_out) return fail(AKB_ERR_INVALID_ARGUMENT, "null output");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  AKB_CUDA_TRY(mass_export(m->dm, m->d_iface_g, m->n_iface, device_out, m->stream));
  return AKB_OK;
}

akb_status akb_part_import_mass(akb_model* m, const double* device_in) {
  akb_status st;
  if ((st = check_part(m)) != AKB_OK) return st;
  if (m->part_in_step) return fail(AKB_ERR_STATE, "inside a step");
  if (m->n_iface > 0 && !device_in) return fail(AKB_ERR_INVALID_ARGUMENT, "null input");
  AKB_CUDA_TRY(cudaSetDevice(m->device));
  AKB_CUDA_TRY(mass_import(m->dm, m->d_iface_g, m->n_iface, device_in, m->stream));
  m->ke_valid = false;
  return AKB_OK;
}

}  // extern "C"
