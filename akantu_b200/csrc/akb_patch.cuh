// akb_patch.cuh -- element patches of the fused explicit step.
//
// The mesh is cut into patches of spatially close elements (recursive
// coordinate bisection of the element centroids, Morton order inside a
// patch). One CTA owns one patch: it stages the patch's nodes in
// shared memory, applies the central-difference predictor there, computes
// the element forces and adds them per node in ascending local element order
// (static per-chunk runs, so the sum is deterministic without atomics).
// Where node values and element contributions sit in shared memory is planned
// at build time so that the corner gathers, the contribution scatter and the
// per-node sums are (nearly) free of bank conflicts.
// Nodes touched by one patch only ("interior") are finished by that CTA;
// nodes shared by several patches write one FP64 partial per (node, patch)
// (the first two of every node in two dense rows, the others node-major), and
// a second kernel adds them in patch order and finishes those nodes.
#pragma once

#include <stdint.h>

#include <vector>

#include "akb_internal.cuh"

namespace akb {

// Shared-memory banks the fused step's layout is planned for: 32 banks of 4
// bytes. An 8-byte word occupies a bank pair, so 16 threads reading 8-byte
// words at 16 different pair indices (word index mod 16) take one wavefront.
constexpr int kBankPairs = 16;

// Elements per chunk: the CTA computes one element per thread per chunk.
constexpr int kChunk = 256;
// Largest piece (contributions of one node added by one thread).
constexpr int kMaxPiece = 8;

// Chunk record: one contiguous, 16-byte aligned block per chunk, staged into
// shared memory by one TMA bulk copy. Contents (uint16 units unless noted;
// every section starts on 16 bytes):
//   header      8 x uint16: R1, rows1, ix1, R2, rows2, r2, ix2, 0 (R: padded
//               counts, multiples of 32; ix1, r2, ix2: byte offsets)
//   corners     per element, the nnpe shared-memory positions of its corner
//               nodes (at 16 bytes)
//   slots       per element corner, its slot in the chunk's contribution
//               array (after the corners, 16-byte aligned)
//   sums 1      R1 uint32 (at 16 + 2 align16(2 ne_c nnpe) bytes): per piece,
//               position | count << 16 | (node cut in several pieces) << 24;
//               a piece is up to `piece` consecutive contributions of one node
//               (ascending element order), pieces by descending count
//   index 1     rows1 x R1 (at ix1): row t, column q = the slot of entry t of
//               piece q
//   sums 2      R2 uint32 (at r2): per node cut in several pieces,
//               position | piece count << 16
//   index 2     rows2 x R2 (at ix2): row j, column q = where the sum of piece
//               j of node q is (FP64: its first entry's slot; FP32: the
//               piece's index in sums 1)
// The slots are a colouring: corner a of G consecutive elements (one scatter
// instruction) and row t of G consecutive pieces (one sum instruction) hit G
// different banks (G = 16 for 8-byte contributions, 32 for 4-byte ones).
struct ChunkDesc {
  uint32_t off16;  // record start in the chunk data, in 16-byte units
  uint32_t bytes;  // record size (multiple of 16)
};

struct PatchHost {
  int npatch = 0;
  int max_nodes = 0;      // largest local node count of a patch
  int node_stride = 0;    // row stride of the shared-memory node arrays
  int contrib_slots = 0;  // largest contribution array of a chunk (per component)
  int max_pieces = 0;     // largest padded first-level piece count of a chunk
  int chunk_bytes = 0;    // largest chunk record
  std::vector<int32_t> elem_ptr;   // npatch + 1, into element order
  std::vector<int32_t> node_ptr;   // npatch + 1, into lnodes
  std::vector<int32_t> ninterior;  // npatch
  std::vector<uint32_t> lnodes;    // global node ids: interior first, then shared
  std::vector<uint16_t> lpos;      // per local node: position in the node arrays
  std::vector<uint32_t> elem_order;  // patch-ordered position -> original element
  std::vector<int32_t> chunk_base; // npatch + 1: first chunk of each patch
  std::vector<ChunkDesc> chunks;   // per chunk
  std::vector<uint16_t> cdata;     // chunk records (multiple of 8 uint16 each)
  std::vector<uint32_t> slot;      // per local node: partial slot (0xffffffff if interior)
  std::vector<uint32_t> snodes;    // shared nodes, ascending
  std::vector<int32_t> sptr;       // nshared + 1, partial slots of each shared node (CSR)
  int64_t nslots = 0;
};

// Builds the patches. target_elems: elements per patch; max_nodes: local node
// cap (<= 60000); contrib_bytes: element vector precision (8: FP64, 4:
// FP32); piece: contributions one thread adds (<= kMaxPiece); force_shared
// (per node, or null): nodes finished by the shared-node pass even when one
// patch holds them (the interface nodes of a partitioned mesh).
PatchHost build_patches(const double* X, const uint32_t* conn, int64_t nn, int64_t ne, int dim,
                        int nnpe, int target_elems, int max_nodes, int contrib_bytes,
                        int piece, const uint8_t* force_shared = nullptr);

// Device copy of a PatchHost.
struct DevPatches {
  int npatch;
  int grid;  // 0: one CTA per patch; > 0: persistent grid of that many CTAs
  int nbuf;  // chunk record buffers in shared memory (2: next chunk prefetched)
  int max_nodes, node_stride, contrib_slots, max_pieces, chunk_bytes;
  int64_t nshared;
  const int32_t* elem_ptr;
  const int32_t* node_ptr;
  const int32_t* ninterior;
  const uint32_t* lnodes;
  const uint16_t* lpos;
  const int32_t* chunk_base;
  const uint2* chunks;     // ChunkDesc per chunk
  const uint16_t* cdata;   // chunk records (16-byte aligned)
  const uint32_t* slot;
  const uint32_t* snodes;
  // partial slots: shared node s has its first two at s and nshared + s, the
  // others at 2 nshared + [sptr[s], sptr[s + 1])
  const int32_t* sptr;
  const uint32_t* emat;  // material of each patch-ordered element, or null
  int* err;              // set when a bounded wait gave up
  double* partial;       // nslots x dim
  // batches: per-instance time step, instance of each patch and shared node
  const double* inst_dt;       // null for a single model (scalar dt)
  const uint32_t* patch_inst;
  const uint32_t* snode_inst;
};

size_t patch_smem_bytes(const DevPatches& p, int dim, int nnpe, bool fp32, int nbuf);
// Chunk record buffers (1 or 2) that keep the most CTAs per SM.
int patch_buffers(const DevPatches& p, int type, bool fp32);
cudaError_t patch_step(const DevModel& m, const DevPatches& p, double dt, bool fp32,
                       bool has_fext, cudaStream_t s);
cudaError_t patch_shared_nodes(const DevModel& m, const DevPatches& p, double dt,
                               bool has_fext, cudaStream_t s);
cudaError_t patch_configure(const DevModel& m, const DevPatches& p, bool fp32);
// Partitioned meshes: out[i] = sum of the partials of shared node iface[i]
// (per component); import writes in[i] as that node's only partial. Masses:
// out[i] = lumped mass of node nodes[i]; import sets it (and 1/M).
cudaError_t patch_iface_export(const DevModel& m, const DevPatches& p, const uint32_t* iface,
                               int64_t n, double* out, cudaStream_t s);
cudaError_t patch_iface_import(const DevModel& m, const DevPatches& p, const uint32_t* iface,
                               int64_t n, const double* in, cudaStream_t s);
cudaError_t mass_export(const DevModel& m, const uint32_t* nodes, int64_t n, double* out,
                        cudaStream_t s);
cudaError_t mass_import(const DevModel& m, const uint32_t* nodes, int64_t n, const double* in,
                        cudaStream_t s);

}  // namespace akb
