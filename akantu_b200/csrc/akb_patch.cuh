// akb_patch.cuh -- element patches of the fused explicit step.
//
// The mesh is cut into patches of spatially close elements (recursive
// coordinate bisection of the element centroids, Morton order inside a
// patch). One CTA owns one patch: it stages the patch's nodes in shared
// memory, computes the element forces and adds them per node in a fixed
// order (static per-chunk runs, so the sum is deterministic without float
// atomics). Where node values and element contributions sit in shared memory
// is planned at build time so that the corner gathers, the contribution
// scatter and the per-node sums are (nearly) free of bank conflicts.
//
// Node numbering. The model stores its nodes in an internal order chosen
// here: the nodes touched by one patch only ("interior" nodes) of patch p
// are the contiguous range [ibeg[p], ibeg[p] + nint[p]), in the order of
// their shared-memory positions, so the CTA stages them with bulk copies of
// contiguous slices; the nodes touched by several patches ("shared") follow
// all interior nodes, then the nodes of no element. perm maps the caller's
// node id to the internal one.
//
// Predicted displacement. Besides u, v, a the model keeps
// w = u + dt v + dt^2/2 a (w = u on blocked DOFs), the displacement the next
// step's forces are evaluated at (NewmarkBeta::predictor, newmark-beta.cc:
// 60-89); a step only stages X and w, and whoever finishes a node writes its
// new u, v, a and the next w.
//
// Shared nodes. Each patch touching a shared node writes its partial force
// to the node's slot of rank r (its position among the node's k patches in
// patch order); a second pass (k_finish_list), one thread per DOF over the
// shared nodes, adds the k partials in rank order and finishes the node. The
// slots of ranks 0 and 1 form two dense rows indexed by the shared node (s,
// ns + s; almost every shared node has two patches), ranks 2 and up follow
// node by node, so the second pass reads a node's first two partials at
// addresses it knows without loading any index. The same pass finishes the
// nodes of no element; for a partitioned mesh the interface nodes' sums are
// exchanged between parts before it.
#pragma once

#include <stdint.h>

#include <vector>

#include "akb_internal.cuh"

namespace akb {

// Elements per chunk: the CTA computes one element per thread per chunk.
constexpr int kChunk = 256;
// Shared-memory bank pairs (8-byte words): a half-warp reading 8-byte words
// at 16 distinct (word index mod 16) takes one wavefront.
constexpr int kBankPairs = 16;

// Node positions are planned so that the CTA's corner gathers hit distinct
// banks: for dim 1 and 3 (8-byte loads of one component; node arrays are
// row-major with an odd row length, so distinct positions mod 16 give
// distinct bank pairs), 16 elements per group and residues mod 16; for
// dim 2 (16-byte loads of a node's two components) 8 elements and mod 8.
inline int place_group(int dim) { return dim == 2 ? 8 : 16; }

// Chunk record: one contiguous, 16-byte aligned block per chunk, staged into
// shared memory by one TMA bulk copy. Contents (uint16 units unless noted;
// every section starts on 16 bytes):
//   header      8 x uint16: R, ng, runs, goff, idx, G, 0, 0 (R: run count
//               padded to a multiple of G; ng = R / G groups; runs, goff,
//               idx: byte offsets)
//   corners     per element, the nnpe shared-memory positions of its corner
//               nodes (at 16 bytes)
//   slots       per element corner, its slot in the chunk's contribution
//               array (after the corners, 16-byte aligned)
//   runs        R uint32: per run (a node's contributions in ascending
//               element order), position | length << 16; runs by descending
//               length, G consecutive runs forming a group
//   goff        ng uint16: where group g's index block starts (in entries)
//   idx         per group, Lg rows (its longest run) of G entries: entry t of
//               the group's run l at goff[g] + t G + l is that contribution's
//               slot
// One thread sums one run. The slots are a colouring: corner a of G
// consecutive elements (one scatter instruction) and entry t of a group's
// runs (one sum instruction) hit G different banks (G = 16 for 8-byte
// contributions, 32 for 4-byte ones), and the runs of a group have their
// nodes at distinct positions mod 16 where the build could arrange it.
// Partial slot of rank r of shared node s (ns shared nodes; over: the node's
// first slot for ranks >= 2).
__host__ __device__ inline uint32_t partial_slot(uint32_t ns, uint32_t s, uint32_t over,
                                                 uint32_t r) {
  return r == 0 ? s : (r == 1 ? ns + s : over + r - 2);
}

struct ChunkDesc {
  uint32_t off16;  // record start in the chunk data, in 16-byte units
  uint32_t bytes;  // record size (multiple of 16)
};

struct PatchHost {
  int npatch = 0;
  int max_nodes = 0;      // largest local node count of a patch
  int max_interior = 0;   // largest interior node count of a patch
  int max_shared = 0;     // largest shared node count of a patch
  int node_stride = 0;    // row stride of the component-major force accumulators
  int contrib_slots = 0;  // largest contribution array of a chunk (per component)
  int max_runs = 0;       // largest padded run count of a chunk
  int chunk_bytes = 0;    // largest chunk record
  std::vector<uint32_t> perm;        // caller's node id -> internal id
  std::vector<int32_t> elem_ptr;     // npatch + 1, into element order
  std::vector<uint32_t> elem_order;  // patch-ordered position -> original element
  std::vector<int32_t> ibeg;         // npatch: internal id of the first interior node
  std::vector<int32_t> nint;         // npatch: interior node count
  std::vector<int32_t> sh_ptr;       // npatch + 1, into the shared entries
  // shared entries, per patch in position order (entry t <-> position nint + t)
  std::vector<uint32_t> sgid;        // internal node id
  std::vector<uint32_t> srank;       // this patch's rank among the node's patches
  std::vector<uint32_t> sslot;       // this patch's partial slot of the node
  std::vector<int32_t> chunk_base;   // npatch + 1: first chunk of each patch
  std::vector<ChunkDesc> chunks;     // per chunk
  std::vector<uint16_t> cdata;       // chunk records (multiple of 8 uint16 each)
  // per shared node s (internal id order; one block starting at shared_base
  // for a single mesh): internal id, first slot of its ranks >= 2, k
  uint32_t shared_base = 0;
  std::vector<uint32_t> shared_nodes, shared_part, shared_k;
  std::vector<uint32_t> orphans;     // internal ids of nodes of no element
  int64_t nslots = 0;
};

// Builds the patches and the internal node order. target_elems: elements per
// patch; max_nodes: local node cap (<= 60000); contrib_bytes: element vector
// precision (8: FP64, 4: FP32); force_shared (per node, or null): nodes treated as shared
// (finished by the second pass from their partials) even when one patch holds
// them (the interface nodes of a partitioned mesh).
PatchHost build_patches(const double* X, const uint32_t* conn, int64_t nn, int64_t ne, int dim,
                        int nnpe, int target_elems, int max_nodes, int contrib_bytes,
                        const uint8_t* force_shared = nullptr);

// Device copy of a PatchHost.
struct DevPatches {
  int npatch;
  int grid;  // 0: one CTA per patch; > 0: persistent grid of that many CTAs
  int nbuf;  // chunk record buffers in shared memory (2: next chunk prefetched)
  int max_nodes, max_shared, node_stride, contrib_slots, max_runs, chunk_bytes;
  const int32_t* elem_ptr;
  const int32_t* ibeg;
  const int32_t* nint;
  const int32_t* sh_ptr;
  const uint32_t* sgid;
  const uint32_t* sslot;
  const int32_t* chunk_base;
  const uint2* chunks;     // ChunkDesc per chunk
  const uint16_t* cdata;   // chunk records (16-byte aligned)
  const uint32_t* emat;    // material of each patch-ordered element, or null
  int* err;                // set when a bounded wait gave up
  double* partial;         // nslots x dim
  double* w;               // nn x dim predicted displacement
  // per patch, then per finishing-list block: sum over the DOFs finished
  // there (blocked ones included) of M v^2 after the step, M > DBL_EPSILON
  // only (getKineticEnergy, solid_mechanics_model.cc:547-561)
  double* ke_part;
  // nodes finished by k_finish_list: the shared nodes (entry s: shared node
  // s), then the nodes of no element; entry i: node, first slot of its ranks
  // >= 2, k (0 for a node of no element)
  int64_t nlist;
  uint32_t nshared;      // shared nodes (the dense partial rows' length)
  uint32_t shared_base;  // with shared_contig: shared node s is node shared_base + s
  int shared_contig;
  const uint32_t* list_gid;
  const uint32_t* list_part;
  const uint32_t* list_k;
  // batches: per-instance time step, instance of each patch / list entry
  const double* inst_dt;       // null for a single model (scalar dt)
  const uint32_t* patch_inst;
  const uint32_t* list_inst;
  // batches: instance node ranges (ninst + 1), for the w refresh
  const int64_t* node_off;
  int ninst;
};

// Partial slots of a plan's shared entries (sslot), its shared nodes' first
// overflow slots (shared_part) and nslots, from sgid, srank, shared_nodes and
// shared_k (run after building, and again after merging the plans of a
// batch).
void assign_partial_slots(PatchHost& P, int64_t nn);

size_t patch_smem_bytes(const DevPatches& p, int dim, bool fp32, int nbuf);
// Chunk record buffers (1 or 2) that keep the most CTAs per SM.
int patch_buffers(const DevPatches& p, int type, bool fp32);
cudaError_t patch_configure(const DevModel& m, const DevPatches& p, bool fp32);
// The fused step: every interior node finished, the shared nodes' partials
// written.
cudaError_t patch_step(const DevModel& m, const DevPatches& p, double dt, bool fp32,
                       bool has_fext, cudaStream_t s);
// Finishes the listed nodes from their partials (the step's second pass).
cudaError_t patch_finish_list(const DevModel& m, const DevPatches& p, double dt, bool has_fext,
                              cudaStream_t s);
// Number of kinetic-energy partials a step writes (patches + list blocks).
int64_t patch_ke_parts(const DevPatches& p, int dim);
// w = u + dt v + dt^2/2 a on free DOFs, w = u on blocked ones.
cudaError_t patch_refresh_w(const DevModel& m, const DevPatches& p, double dt, cudaStream_t s);
// Partitioned meshes, per interface node i (shared node shared[i], k[i]
// partials): out[i] = the sum of its partials (per component); import writes
// in[i] as its only partial. Masses: out[i] = lumped mass of internal node nodes[i];
// import sets it (and 1/M).
cudaError_t patch_iface_export(const DevModel& m, const DevPatches& p, const uint32_t* shared,
                               const uint32_t* k, int64_t n, double* out, cudaStream_t s);
cudaError_t patch_iface_import(const DevModel& m, const DevPatches& p, const uint32_t* shared,
                               const uint32_t* k, int64_t n, const double* in, cudaStream_t s);
cudaError_t mass_export(const DevModel& m, const uint32_t* nodes, int64_t n, double* out,
                        cudaStream_t s);
cudaError_t mass_import(const DevModel& m, const uint32_t* nodes, int64_t n, const double* in,
                        cudaStream_t s);
// Neighbour exchange of a part. An ExchangePlan lists the interface rows
// packed for the neighbours (send_rows, the neighbours' blocks concatenated)
// and, per interface row i, the terms of its sum in ascending part order:
// sum_src[sum_ptr[i] .. sum_ptr[i+1]), -1 for this part's own value, else a
// row of the received buffer. Every part holding a node adds the same terms
// in the same order, so all copies of the sum are equal.
struct ExchangePlan {
  int64_t n_send = 0, n_recv = 0, n_rows = 0;
  const uint32_t* send_rows = nullptr;
  const uint32_t* sum_ptr = nullptr;
  const int32_t* sum_src = nullptr;
};
// out[k] = this part's force on interface row send_rows[k] (d per row)
cudaError_t patch_iface_pack(const DevModel& m, const DevPatches& p, const uint32_t* shared,
                             const uint32_t* k, const ExchangePlan& x, double* out,
                             cudaStream_t s);
// every interface row's force = its ordered sum, imported as its only partial
cudaError_t patch_iface_sum_import(const DevModel& m, const DevPatches& p, const uint32_t* shared,
                                   const uint32_t* k, const ExchangePlan& x, const double* recv,
                                   cudaStream_t s);
// the same for the lumped masses (one value per row) of internal nodes nodes[i]
cudaError_t mass_pack(const DevModel& m, const uint32_t* nodes, const ExchangePlan& x,
                      double* out, cudaStream_t s);
cudaError_t mass_sum_import(const DevModel& m, const uint32_t* nodes, const ExchangePlan& x,
                            const double* recv, cudaStream_t s);
// Caller order <-> internal order of nodal arrays (rows of `width` items):
// gather: out[i] = in[perm[i]]; scatter: out[perm[i]] = in[i].
cudaError_t permute_rows(const uint32_t* perm, int64_t n, int width, const double* in,
                         double* out, bool scatter, cudaStream_t s);
cudaError_t permute_rows_u8(const uint32_t* perm, int64_t n, int width, const uint8_t* in,
                            uint8_t* out, bool scatter, cudaStream_t s);

}  // namespace akb
