// akb_patch_build.cu -- host construction of the element patches.
#include <algorithm>
#include <cstring>
#include <numeric>

#include "akb_patch.cuh"

namespace akb {
namespace {

inline uint64_t spread3(uint64_t x) {  // 21 bits -> every third bit
  x &= 0x1fffff;
  x = (x | x << 32) & 0x1f00000000ffffULL;
  x = (x | x << 16) & 0x1f0000ff0000ffULL;
  x = (x | x << 8) & 0x100f00f00f00f00fULL;
  x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
  x = (x | x << 2) & 0x1249249249249249ULL;
  return x;
}
inline uint64_t spread2(uint64_t x) {  // 31 bits -> every second bit
  x &= 0x7fffffff;
  x = (x | x << 16) & 0x0000ffff0000ffffULL;
  x = (x | x << 8) & 0x00ff00ff00ff00ffULL;
  x = (x | x << 4) & 0x0f0f0f0f0f0f0f0fULL;
  x = (x | x << 2) & 0x3333333333333333ULL;
  x = (x | x << 1) & 0x5555555555555555ULL;
  return x;
}

}  // namespace

PatchHost build_patches(const double* X, const uint32_t* conn, int64_t nn, int64_t ne, int dim,
                        int nnpe, int target_elems, int max_nodes) {
  PatchHost P;
  // 1. Morton order of element centroids
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int64_t i = 0; i < nn; ++i)
    for (int k = 0; k < dim; ++k) {
      lo[k] = std::min(lo[k], X[i * dim + k]);
      hi[k] = std::max(hi[k], X[i * dim + k]);
    }
  const int bits = dim == 3 ? 21 : (dim == 2 ? 31 : 62);
  const double scale = (double)((1ULL << std::min(bits, 52)) - 1);
  std::vector<std::pair<uint64_t, uint32_t>> keys(ne);
  for (int64_t e = 0; e < ne; ++e) {
    double c[3] = {0, 0, 0};
    for (int a = 0; a < nnpe; ++a)
      for (int k = 0; k < dim; ++k) c[k] += X[(int64_t)conn[e * nnpe + a] * dim + k];
    uint64_t q[3] = {0, 0, 0};
    for (int k = 0; k < dim; ++k) {
      double ext = hi[k] - lo[k];
      double t = ext > 0 ? (c[k] / nnpe - lo[k]) / ext : 0.0;
      t = std::min(std::max(t, 0.0), 1.0);
      q[k] = (uint64_t)(t * scale);
    }
    uint64_t key = dim == 3 ? (spread3(q[0]) | spread3(q[1]) << 1 | spread3(q[2]) << 2)
                 : dim == 2 ? (spread2(q[0]) | spread2(q[1]) << 1)
                            : q[0];
    keys[e] = {key, (uint32_t)e};
  }
  std::sort(keys.begin(), keys.end());
  P.elem_order.resize(ne);
  for (int64_t i = 0; i < ne; ++i) P.elem_order[i] = keys[i].second;
  keys.clear();
  keys.shrink_to_fit();

  // 2. greedy patches of consecutive elements, capped by elements and nodes
  std::vector<int32_t> stamp(nn, -1);
  P.elem_ptr.push_back(0);
  {
    int cur = 0, cur_nodes = 0, cur_elems = 0;
    for (int64_t i = 0; i < ne; ++i) {
      const uint32_t* c = conn + (int64_t)P.elem_order[i] * nnpe;
      int fresh = 0;
      for (int a = 0; a < nnpe; ++a)
        if (stamp[c[a]] != cur) {
          bool dup = false;
          for (int b = 0; b < a; ++b) dup |= c[b] == c[a];
          fresh += !dup;
        }
      if (cur_elems > 0 && (cur_elems >= target_elems || cur_nodes + fresh > max_nodes)) {
        P.elem_ptr.push_back((int32_t)i);
        ++cur;
        cur_nodes = cur_elems = 0;
        fresh = 0;
        for (int a = 0; a < nnpe; ++a) {
          bool dup = false;
          for (int b = 0; b < a; ++b) dup |= c[b] == c[a];
          fresh += !dup;
        }
      }
      for (int a = 0; a < nnpe; ++a) stamp[c[a]] = cur;
      cur_nodes += fresh;
      ++cur_elems;
    }
    if (ne > 0) P.elem_ptr.push_back((int32_t)ne);
  }
  P.npatch = (int)P.elem_ptr.size() - 1;

  // 3. patches per node
  std::fill(stamp.begin(), stamp.end(), -1);
  std::vector<int32_t> count(nn, 0);
  for (int p = 0; p < P.npatch; ++p)
    for (int32_t i = P.elem_ptr[p]; i < P.elem_ptr[p + 1]; ++i) {
      const uint32_t* c = conn + (int64_t)P.elem_order[i] * nnpe;
      for (int a = 0; a < nnpe; ++a)
        if (stamp[c[a]] != p) {
          stamp[c[a]] = p;
          ++count[c[a]];
        }
    }
  // shared nodes and their node-major partial slots; nodes of no element
  // join them with no slot, so they get the reference's lumped solve with
  // M = 0 (r / M not finite, solid_mechanics_model_mass.cc:79-95)
  std::vector<int64_t> sidx(nn, -1);
  P.sptr.push_back(0);
  for (int64_t i = 0; i < nn; ++i)
    if (count[i] >= 2 || count[i] == 0) {
      sidx[i] = (int64_t)P.snodes.size();
      P.snodes.push_back((uint32_t)i);
      P.sptr.push_back(P.sptr.back() + count[i]);
    }
  P.nslots = P.sptr.back();
  std::vector<int32_t> sfill(P.snodes.size(), 0);

  // 4. per-patch local nodes, local connectivity, CSR, slots
  std::fill(stamp.begin(), stamp.end(), -1);
  std::vector<int32_t> lidx(nn, -1);
  P.node_ptr.push_back(0);
  P.lconn.resize((size_t)ne * nnpe);
  std::vector<uint32_t> local;
  std::vector<uint64_t> keyed;
  P.cslot.resize((size_t)ne * nnpe);
  for (int p = 0; p < P.npatch; ++p) {
    const int32_t eb = P.elem_ptr[p], ee = P.elem_ptr[p + 1];
    local.clear();
    for (int32_t i = eb; i < ee; ++i) {
      const uint32_t* c = conn + (int64_t)P.elem_order[i] * nnpe;
      for (int a = 0; a < nnpe; ++a)
        if (stamp[c[a]] != p) {
          stamp[c[a]] = p;
          local.push_back(c[a]);
        }
    }
    std::sort(local.begin(), local.end(), [&](uint32_t x, uint32_t y) {
      const bool sx = count[x] >= 2, sy = count[y] >= 2;
      return sx != sy ? !sx : x < y;
    });
    int nint = 0;
    for (size_t j = 0; j < local.size(); ++j) {
      lidx[local[j]] = (int32_t)j;
      nint += count[local[j]] < 2;
    }
    P.ninterior.push_back(nint);
    P.max_nodes = std::max(P.max_nodes, (int)local.size());
    P.max_elems = std::max(P.max_elems, (int)(ee - eb));
    for (int32_t i = eb; i < ee; ++i) {
      const uint32_t* c = conn + (int64_t)P.elem_order[i] * nnpe;
      for (int a = 0; a < nnpe; ++a) P.lconn[(size_t)i * nnpe + a] = (uint16_t)lidx[c[a]];
    }
    for (size_t j = 0; j < local.size(); ++j) {
      const int64_t s = sidx[local[j]];
      P.slot.push_back(s < 0 ? 0xffffffffu : (uint32_t)(P.sptr[s] + sfill[s]++));
    }
    // chunks: corners sorted by (local node, element, corner); the sort key
    // orders a node's contributions by ascending element
    P.chunk_base.push_back((int32_t)P.seg_ptr.size());
    const size_t seg_first = P.segs.size();
    for (int32_t c0 = eb; c0 < ee; c0 += kChunk) {
      const int32_t c1 = std::min(ee, c0 + kChunk);
      keyed.clear();
      for (int32_t i = c0; i < c1; ++i)
        for (int a = 0; a < nnpe; ++a) {
          const uint32_t j = P.lconn[(size_t)i * nnpe + a];
          keyed.push_back(((uint64_t)j << 32) | ((uint64_t)(i - c0) << 8) | (uint64_t)a);
        }
      std::sort(keyed.begin(), keyed.end());
      P.seg_ptr.push_back((int32_t)P.segs.size());
      for (size_t k = 0; k < keyed.size(); ++k) {
        const uint32_t j = (uint32_t)(keyed[k] >> 32);
        const int32_t le = (int32_t)((keyed[k] >> 8) & 0xffffff), a = (int32_t)(keyed[k] & 0xff);
        P.cslot[(size_t)(c0 + le) * nnpe + a] = (uint16_t)k;
        if (k + 1 == keyed.size() || (uint32_t)(keyed[k + 1] >> 32) != j)
          P.segs.push_back((j << 16) | (uint32_t)(k + 1));
      }
    }
    P.max_segs = std::max(P.max_segs, (int)(P.segs.size() - seg_first));
    P.lnodes.insert(P.lnodes.end(), local.begin(), local.end());
    P.node_ptr.push_back((int32_t)P.lnodes.size());
  }
  P.seg_ptr.push_back((int32_t)P.segs.size());
  return P;
}

}  // namespace akb
