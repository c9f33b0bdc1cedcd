// akb_patch.cuh -- element patches of the fused explicit step.
//
// The mesh is cut into patches of spatially close elements (Morton order of
// element centroids). One CTA owns one patch: it stages the patch's nodes in
// shared memory, applies the central-difference predictor there, computes
// the element forces and adds them per node in ascending local element order
// (a static per-patch CSR, so the sum is deterministic without atomics).
// Nodes touched by one patch only ("interior") are finished by that CTA;
// nodes shared by several patches write one FP64 partial per (node, patch) to
// slots laid out node-major, and a second kernel adds them in patch order and
// finishes those nodes.
#pragma once

#include <stdint.h>

#include <vector>

#include "akb_internal.cuh"

namespace akb {

struct PatchHost {
  int npatch = 0;
  int max_nodes = 0;    // largest local node count of a patch
  int max_elems = 0;    // largest element count of a patch
  int max_segs = 0;     // largest run count of a patch (all its chunks)
  std::vector<int32_t> elem_ptr;   // npatch + 1, into element order
  std::vector<int32_t> node_ptr;   // npatch + 1, into lnodes
  std::vector<int32_t> ninterior;  // npatch
  std::vector<uint32_t> lnodes;    // global node ids: interior first, then shared
  std::vector<uint32_t> elem_order;  // patch-ordered position -> original element
  std::vector<uint16_t> lconn;     // per element (patch order) nnpe local indices
  // per chunk of kChunk consecutive elements of a patch: the slot of each
  // element corner once the chunk's corners are sorted by (local node,
  // element, corner), and the runs of equal local node in that order
  std::vector<uint16_t> cslot;     // per element corner (patch order)
  std::vector<uint32_t> segs;      // per run: (local node << 16) | end slot
  std::vector<int32_t> seg_ptr;    // nchunks + 1
  std::vector<int32_t> chunk_base; // npatch: index of the patch's first chunk
  std::vector<uint32_t> slot;      // per local node: partial slot (0xffffffff if interior)
  std::vector<uint32_t> snodes;    // shared nodes, ascending
  std::vector<int32_t> sptr;       // nshared + 1, partial slots of each shared node
  int64_t nslots = 0;
};

// Elements per chunk: the CTA computes one element per thread per chunk.
constexpr int kChunk = 256;

// Builds the patches. target_elems: elements per patch; max_nodes: local node
// cap (<= 65535).
PatchHost build_patches(const double* X, const uint32_t* conn, int64_t nn, int64_t ne, int dim,
                        int nnpe, int target_elems, int max_nodes);

// Device copy of a PatchHost.
struct DevPatches {
  int npatch;
  int grid;  // 0: one CTA per patch; > 0: persistent grid of that many CTAs
  int max_nodes, max_elems, max_segs;
  int64_t nshared;
  const int32_t* elem_ptr;
  const int32_t* node_ptr;
  const int32_t* ninterior;
  const uint32_t* lnodes;
  const int32_t* seg_ptr;
  const int32_t* chunk_base;
  const uint32_t* slot;
  const uint32_t* snodes;
  const int32_t* sptr;
  const uint32_t* emat;  // material of each patch-ordered element, or null
  // per-patch local connectivity, sorted corner slots and runs, each patch's
  // slice padded to 16 bytes: the sources of the TMA bulk staging
  const uint16_t* lconn_pad;
  const uint16_t* cslot_pad;
  const uint32_t* segs_pad;
  const uint32_t* lc_off;  // per patch, in uint16 (multiple of 8)
  const uint32_t* sg_off;  // per patch, in uint32 (multiple of 4)
  int* err;                // set when a bounded wait gave up
  double* partial;       // nslots x dim
  // batches: per-instance time step, instance of each patch and shared node
  const double* inst_dt;       // null for a single model (scalar dt)
  const uint32_t* patch_inst;
  const uint32_t* snode_inst;
};

size_t patch_smem_bytes(const DevPatches& p, int dim, int nnpe, bool fp32, int threads);
cudaError_t patch_step(const DevModel& m, const DevPatches& p, double dt, bool fp32,
                       bool has_fext, cudaStream_t s);
cudaError_t patch_shared_nodes(const DevModel& m, const DevPatches& p, double dt,
                               bool has_fext, cudaStream_t s);
cudaError_t patch_configure(const DevModel& m, const DevPatches& p, bool fp32);

}  // namespace akb
