// akb_patch_build.cu -- host construction of the element patches.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <stdexcept>

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

// Positions of a patch's L local nodes in the shared-memory node arrays:
// local nodes [0, nint) are the interior ones and take positions [0, nint),
// the others positions [nint, L). The CTA reads corner a of G consecutive
// elements in one instruction; each distinct node of such a group should sit
// at its own position mod G (place_group). Greedy in first-touch order: a
// node takes, within its range, the residue least used by the groups it
// belongs to, then the one with the most free positions left.
void place_nodes(const std::vector<uint16_t>& lc, int ne, int nnpe, int L, int nint, int G,
                 uint16_t* pos) {
  const int nhalf = (ne + G - 1) / G;
  std::vector<std::pair<int32_t, int32_t>> mem;  // (node, group), each pair once
  mem.reserve((size_t)ne * nnpe);
  for (int h = 0; h < nhalf; ++h)
    for (int a = 0; a < nnpe; ++a) {
      const int e0 = h * G, e1 = std::min(ne, e0 + G);
      for (int e = e0; e < e1; ++e) {
        const int v = lc[(size_t)e * nnpe + a];
        bool dup = false;
        for (int f = e0; f < e && !dup; ++f) dup = lc[(size_t)f * nnpe + a] == v;
        if (!dup) mem.push_back({v, h * nnpe + a});
      }
    }
  std::sort(mem.begin(), mem.end());
  std::vector<int32_t> gptr(L + 1, 0);
  for (auto& m : mem) ++gptr[m.first + 1];
  for (int v = 0; v < L; ++v) gptr[v + 1] += gptr[v];
  std::vector<int32_t> used((size_t)nhalf * nnpe * G, 0);
  std::vector<int32_t> order;
  order.reserve(L);
  std::vector<char> seen(L, 0);
  for (int e = 0; e < ne; ++e)
    for (int a = 0; a < nnpe; ++a) {
      const int v = lc[(size_t)e * nnpe + a];
      if (!seen[v]) {
        seen[v] = 1;
        order.push_back(v);
      }
    }
  for (int v = 0; v < L; ++v)
    if (!seen[v]) order.push_back(v);
  // free positions per (range, residue): next position and how many are left
  int next[2][kBankPairs], left[2][kBankPairs];
  const int lo[2] = {0, nint}, hi[2] = {nint, L};
  for (int g = 0; g < 2; ++g)
    for (int r = 0; r < G; ++r) {
      const int p0 = lo[g] + ((r - lo[g] % G) + G) % G;
      next[g][r] = p0;
      left[g][r] = p0 < hi[g] ? (hi[g] - 1 - p0) / G + 1 : 0;
    }
  for (int v : order) {
    const int g = v < nint ? 0 : 1;
    int64_t cost[kBankPairs] = {0};
    for (int k = gptr[v]; k < gptr[v + 1]; ++k) {
      const int32_t* u = &used[(size_t)mem[k].second * G];
      for (int r = 0; r < G; ++r) cost[r] += u[r];
    }
    int best = -1;
    for (int r = 0; r < G; ++r) {
      if (left[g][r] == 0) continue;
      if (best < 0 || cost[r] < cost[best] || (cost[r] == cost[best] && left[g][r] > left[g][best]))
        best = r;
    }
    pos[v] = (uint16_t)next[g][best];
    next[g][best] += G;
    --left[g][best];
    for (int k = gptr[v]; k < gptr[v + 1]; ++k) ++used[(size_t)mem[k].second * G + best];
  }
}

// Proper edge colouring of a bipartite multigraph with C colours, C at least
// its largest degree (Koenig's edge-colouring theorem). Edges are added one at
// a time: with a the first colour free at the left end u and b the first free
// at the right end v, an edge takes a if a is free at v, else b if b is free
// at u, else the path from v alternating colours a, b is recoloured (a <-> b),
// which frees a at v; in a bipartite graph that path cannot reach u.
class BipartiteColouring {
 public:
  BipartiteColouring(int nl, int nr, int C)
      : C_(C), at_l_((size_t)nl * C, -1), at_r_((size_t)nr * C, -1) {}
  void add(int u, int v) {
    const int e = (int)eu_.size();
    eu_.push_back(u);
    ev_.push_back(v);
    col_.push_back(-1);
    int a = 0, b = 0;
    while (at_l_[(size_t)u * C_ + a] >= 0) ++a;
    while (at_r_[(size_t)v * C_ + b] >= 0) ++b;
    if (at_r_[(size_t)v * C_ + a] >= 0) {
      if (at_l_[(size_t)u * C_ + b] < 0) {
        a = b;
      } else {
        path_.clear();
        int x = v, c = a;
        bool right = true;
        for (;;) {
          const int f = right ? at_r_[(size_t)x * C_ + c] : at_l_[(size_t)x * C_ + c];
          if (f < 0) break;
          path_.push_back(f);
          x = right ? eu_[f] : ev_[f];
          right = !right;
          c = c == a ? b : a;
        }
        for (int f : path_) {
          at_l_[(size_t)eu_[f] * C_ + col_[f]] = -1;
          at_r_[(size_t)ev_[f] * C_ + col_[f]] = -1;
        }
        for (int f : path_) {
          col_[f] = col_[f] == a ? b : a;
          at_l_[(size_t)eu_[f] * C_ + col_[f]] = f;
          at_r_[(size_t)ev_[f] * C_ + col_[f]] = f;
        }
      }
    }
    col_[e] = a;
    at_l_[(size_t)u * C_ + a] = e;
    at_r_[(size_t)v * C_ + a] = e;
  }
  int colour(int e) const { return col_[e]; }

 private:
  int C_;
  std::vector<int32_t> at_l_, at_r_, eu_, ev_, col_, path_;
};

}  // namespace

PatchHost build_patches(const double* X, const uint32_t* conn, int64_t nn, int64_t ne, int dim,
                        int nnpe, int target_elems, int max_nodes, int contrib_bytes,
                        const uint8_t* force_shared) {
  PatchHost P;
  // 1. element centroids and their Morton keys
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int64_t i = 0; i < nn; ++i)
    for (int k = 0; k < dim; ++k) {
      lo[k] = std::min(lo[k], X[i * dim + k]);
      hi[k] = std::max(hi[k], X[i * dim + k]);
    }
  const int bits = dim == 3 ? 21 : (dim == 2 ? 31 : 62);
  const double scale = (double)((1ULL << std::min(bits, 52)) - 1);
  std::vector<uint64_t> mkey(ne);
  std::vector<double> cen((size_t)ne * 3, 0.0);
  for (int64_t e = 0; e < ne; ++e) {
    double* c = &cen[(size_t)e * 3];
    for (int a = 0; a < nnpe; ++a)
      for (int k = 0; k < dim; ++k) c[k] += X[(int64_t)conn[e * nnpe + a] * dim + k];
    uint64_t q[3] = {0, 0, 0};
    for (int k = 0; k < dim; ++k) {
      c[k] /= nnpe;
      double ext = hi[k] - lo[k];
      double t = ext > 0 ? (c[k] - lo[k]) / ext : 0.0;
      t = std::min(std::max(t, 0.0), 1.0);
      q[k] = (uint64_t)(t * scale);
    }
    mkey[e] = dim == 3 ? (spread3(q[0]) | spread3(q[1]) << 1 | spread3(q[2]) << 2)
            : dim == 2 ? (spread2(q[0]) | spread2(q[1]) << 1)
                       : q[0];
  }

  // 2. patches: recursive coordinate bisection of the centroids (split at
  //    the element count that leaves whole patches of target_elems on each
  //    side, across the longest extent) until a part has at most
  //    target_elems elements and max_nodes nodes; parts in depth-first
  //    order, elements of a part in Morton order. Compact parts share fewer
  //    nodes with their neighbours than cuts of one space-filling curve
  //    (tetrahedral cube, 1024-element parts: 10 % fewer patch-local nodes,
  //    17 % fewer shared-node partials).
  std::vector<int32_t> stamp(nn, -1);
  P.elem_order.resize(ne);
  for (int64_t i = 0; i < ne; ++i) P.elem_order[i] = (uint32_t)i;
  P.elem_ptr.push_back(0);
  {
    uint32_t* ord = P.elem_order.data();
    int32_t tag = 0;
    std::vector<std::pair<int64_t, int64_t>> todo;
    if (ne > 0) todo.push_back({0, ne});
    while (!todo.empty()) {
      const int64_t b = todo.back().first, e = todo.back().second;
      todo.pop_back();
      const int64_t n = e - b;
      bool leaf = n <= target_elems;
      if (leaf && n > 1) {
        int nodes = 0;
        for (int64_t i = b; i < e; ++i)
          for (int a = 0; a < nnpe; ++a) {
            const uint32_t v = conn[(int64_t)ord[i] * nnpe + a];
            if (stamp[v] != tag) {
              stamp[v] = tag;
              ++nodes;
            }
          }
        ++tag;
        leaf = nodes <= max_nodes;
      }
      if (leaf) {
        std::sort(ord + b, ord + e, [&](uint32_t x, uint32_t y) {
          return mkey[x] != mkey[y] ? mkey[x] < mkey[y] : x < y;
        });
        P.elem_ptr.push_back((int32_t)e);
        continue;
      }
      const int64_t parts = std::max<int64_t>(2, (n + target_elems - 1) / target_elems);
      const int64_t k = std::max<int64_t>(1, n * (parts / 2) / parts);
      double clo[3] = {1e300, 1e300, 1e300}, chi[3] = {-1e300, -1e300, -1e300};
      for (int64_t i = b; i < e; ++i)
        for (int d = 0; d < dim; ++d) {
          clo[d] = std::min(clo[d], cen[(size_t)ord[i] * 3 + d]);
          chi[d] = std::max(chi[d], cen[(size_t)ord[i] * 3 + d]);
        }
      int ax = 0;
      for (int d = 1; d < dim; ++d)
        if (chi[d] - clo[d] > chi[ax] - clo[ax]) ax = d;
      std::nth_element(ord + b, ord + b + k, ord + e, [&](uint32_t x, uint32_t y) {
        const double cx = cen[(size_t)x * 3 + ax], cy = cen[(size_t)y * 3 + ax];
        return cx != cy ? cx < cy : x < y;
      });
      todo.push_back({b + k, e});
      todo.push_back({b, b + k});
    }
  }
  mkey.clear();
  mkey.shrink_to_fit();
  cen.clear();
  cen.shrink_to_fit();
  std::fill(stamp.begin(), stamp.end(), -1);
  P.npatch = (int)P.elem_ptr.size() - 1;

  // 3. patches per node: a node of one patch is interior to it, a node of
  //    several (or a forced one) is shared, a node of none is an orphan;
  //    nodes of no element get the reference's lumped solve with M = 0
  //    (r / M not finite, solid_mechanics_model_mass.cc:79-95)
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
  auto is_shared = [&](int64_t v) {
    return count[v] >= 2 || (count[v] == 1 && force_shared && force_shared[v]);
  };

  // 4. per patch: local nodes (interior first), their shared-memory
  //    positions, the internal ids of the interior nodes, the shared entries
  //    and the chunk records
  std::fill(stamp.begin(), stamp.end(), -1);
  P.perm.assign(nn, 0xffffffffu);
  std::vector<int32_t> lidx(nn, -1), rank_fill(nn, 0);
  std::vector<uint32_t> entry_user;  // caller's id of each shared entry
  std::vector<uint32_t> entry_rank;  // the patch's rank among the node's patches
  std::vector<uint32_t> local;
  std::vector<uint16_t> lcl, pos;
  std::vector<uint64_t> keyed;
  struct Run { int32_t node, first, len; };
  std::vector<Run> runs;
  std::vector<int32_t> order, gbase, eslot, cls;
  std::vector<uint16_t> rec;
  // contribution bank groups: 16 bank pairs for 8-byte contributions, 32
  // banks for 4-byte ones
  const int G = contrib_bytes == 8 ? kBankPairs : 32;
  const int GP = place_group(dim);
  uint32_t next_id = 0;
  P.sh_ptr.push_back(0);
  for (int p = 0; p < P.npatch; ++p) {
    const int32_t eb = P.elem_ptr[p], ee = P.elem_ptr[p + 1];
    const int ne_p = ee - eb;
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
      const bool sx = is_shared(x), sy = is_shared(y);
      return sx != sy ? !sx : x < y;
    });
    const int L = (int)local.size();
    int nint = 0;
    for (int j = 0; j < L; ++j) {
      lidx[local[j]] = j;
      nint += !is_shared(local[j]);
    }
    P.max_nodes = std::max(P.max_nodes, L);
    P.max_interior = std::max(P.max_interior, nint);
    P.max_shared = std::max(P.max_shared, L - nint);
    lcl.resize((size_t)ne_p * nnpe);
    for (int32_t i = eb; i < ee; ++i) {
      const uint32_t* c = conn + (int64_t)P.elem_order[i] * nnpe;
      for (int a = 0; a < nnpe; ++a) lcl[(size_t)(i - eb) * nnpe + a] = (uint16_t)lidx[c[a]];
    }
    pos.assign(L, 0);
    place_nodes(lcl, ne_p, nnpe, L, nint, GP, pos.data());
    P.ibeg.push_back((int32_t)next_id);
    P.nint.push_back(nint);
    const size_t e0 = entry_user.size();
    entry_user.resize(e0 + (L - nint));
    entry_rank.resize(e0 + (L - nint));
    for (int j = 0; j < L; ++j) {
      const uint32_t v = local[j];
      if (j < nint) {
        P.perm[v] = next_id + pos[j];
      } else {
        const size_t t = e0 + (pos[j] - nint);
        entry_user[t] = v;
        entry_rank[t] = (uint32_t)rank_fill[v]++;
      }
    }
    next_id += nint;
    P.sh_ptr.push_back((int32_t)entry_user.size());
    P.chunk_base.push_back((int32_t)P.chunks.size());
    for (int c0 = 0; c0 < ne_p; c0 += kChunk) {
      const int nec = std::min(ne_p - c0, kChunk), ncorner = nec * nnpe;
      // runs: the chunk's corners sorted by (local node, element, corner);
      // one run is a node's contributions in ascending element order
      keyed.clear();
      for (int e = 0; e < nec; ++e)
        for (int a = 0; a < nnpe; ++a)
          keyed.push_back(((uint64_t)lcl[(size_t)(c0 + e) * nnpe + a] << 32) |
                          ((uint64_t)e << 8) | (uint64_t)a);
      std::sort(keyed.begin(), keyed.end());
      runs.clear();
      for (int k = 0; k < ncorner; ++k) {
        const int32_t j = (int32_t)(keyed[k] >> 32);
        if (runs.empty() || runs.back().node != j) runs.push_back({j, k, 0});
        ++runs.back().len;
      }
      // run order: by descending length (a warp's threads loop about as
      // long), and within 16 consecutive runs (a half-warp) the nodes'
      // positions at distinct residues mod 16 where possible, so that the
      // read-modify-write of the node accumulators hits distinct bank pairs;
      // the pick looks at the next runs of the sorted list only
      std::vector<int32_t> sorted(runs.size());
      std::iota(sorted.begin(), sorted.end(), 0);
      std::stable_sort(sorted.begin(), sorted.end(),
                       [&](int32_t x, int32_t y) { return runs[x].len > runs[y].len; });
      order.clear();
      {
        std::vector<char> taken(runs.size(), 0);
        size_t head = 0;
        int used[kBankPairs] = {0};
        for (size_t q = 0; q < runs.size(); ++q) {
          if (q % kBankPairs == 0) std::fill(used, used + kBankPairs, 0);
          while (taken[sorted[head]]) ++head;
          size_t pick = head;
          int seen = 0;
          for (size_t c = head; c < sorted.size() && seen < 3 * G; ++c) {
            if (taken[sorted[c]]) continue;
            ++seen;
            if (!used[pos[runs[sorted[c]].node] % kBankPairs]) {
              pick = c;
              break;
            }
          }
          taken[sorted[pick]] = 1;
          ++used[pos[runs[sorted[pick]].node] % kBankPairs];
          order.push_back(sorted[pick]);
        }
      }
      const int R = (int)order.size(), Rp = (R + G - 1) / G * G, ng = Rp / G;
      P.max_runs = std::max(P.max_runs, Rp);
      // index blocks: group g holds Lg rows (its longest run) of G entries;
      // entry t of the group's run l at gbase[g] + t G + l
      gbase.assign(ng + 1, 0);
      for (int g = 0; g < ng; ++g) {
        int Lg = 0;
        for (int l = 0; l < G && g * G + l < R; ++l) Lg = std::max(Lg, runs[order[g * G + l]].len);
        gbase[g + 1] = gbase[g] + Lg * G;
      }
      // colour the (scatter instruction, sum instruction) graph: corner a of
      // G consecutive elements is one scatter instruction, entry t of a
      // group's runs one sum instruction; each has at most G contributions,
      // so G colours suffice (Koenig); a colour is a slot residue
      const int nsg = (nec + G - 1) / G * nnpe;
      BipartiteColouring bc(nsg, std::max(gbase[ng] / G, 1), G);
      std::vector<int32_t> edge_of(ncorner);
      int ne_ = 0;
      for (int q = 0; q < R; ++q) {
        const Run& rn = runs[order[q]];
        for (int t = 0; t < rn.len; ++t) {
          const uint64_t kk = keyed[rn.first + t];
          const int e = (int)((kk >> 8) & 0xffffff), a = (int)(kk & 0xff);
          bc.add((e / G) * nnpe + a, gbase[q / G] / G + t);
          edge_of[e * nnpe + a] = ne_++;
        }
      }
      cls.assign(G, 0);
      eslot.assign(ncorner, 0);
      for (int k = 0; k < ncorner; ++k) {
        const int c = bc.colour(edge_of[k]);
        eslot[k] = c + G * cls[c]++;
      }
      int maxcls = 0;
      for (int c = 0; c < G; ++c) maxcls = std::max(maxcls, cls[c]);
      P.contrib_slots = std::max(P.contrib_slots, G * maxcls);
      // the record (akb_patch.cuh), offsets in uint16
      const int A = (ncorner + 7) / 8 * 8;
      const int o_lc = 8, o_cs = o_lc + A, o_runs = o_cs + A;
      const int o_goff = o_runs + 2 * Rp, o_idx = o_goff + (ng + 7) / 8 * 8;
      const int o_end = o_idx + (gbase[ng] + 7) / 8 * 8;
      if (o_end * 2 > 65535 || gbase[ng] > 65535)
        throw std::length_error("chunk record above 64 KB");
      rec.assign(o_end, 0);
      const int hdr[8] = {Rp, ng, 2 * o_runs, 2 * o_goff, 2 * o_idx, G, 0, 0};
      for (int k = 0; k < 8; ++k) rec[k] = (uint16_t)hdr[k];
      for (int k = 0; k < ncorner; ++k) {
        rec[o_lc + k] = pos[lcl[(size_t)c0 * nnpe + k]];
        rec[o_cs + k] = (uint16_t)eslot[k];
      }
      for (int q = 0; q < R; ++q) {
        const Run& rn = runs[order[q]];
        const uint32_t w = (uint32_t)pos[rn.node] | ((uint32_t)rn.len << 16);
        rec[o_runs + 2 * q] = (uint16_t)(w & 0xffff);
        rec[o_runs + 2 * q + 1] = (uint16_t)(w >> 16);
        for (int t = 0; t < rn.len; ++t) {
          const uint64_t kk = keyed[rn.first + t];
          rec[o_idx + gbase[q / G] + t * G + q % G] =
              (uint16_t)eslot[((kk >> 8) & 0xffffff) * nnpe + (kk & 0xff)];
        }
      }
      for (int g = 0; g < ng; ++g) rec[o_goff + g] = (uint16_t)gbase[g];
      ChunkDesc cd;
      cd.off16 = (uint32_t)(P.cdata.size() / 8);
      cd.bytes = (uint32_t)rec.size() * 2;
      P.chunks.push_back(cd);
      P.cdata.insert(P.cdata.end(), rec.begin(), rec.end());
      P.chunk_bytes = std::max(P.chunk_bytes, (int)cd.bytes);
    }
  }
  P.chunk_base.push_back((int32_t)P.chunks.size());

  // 5. internal ids of the shared nodes (in order of first appearance, so
  //    that the nodes of neighbouring patches stay close) and their partial
  //    slots (one per patch in patch order: partial_slot), then the nodes of
  //    no element
  P.shared_base = next_id;
  for (size_t t = 0; t < entry_user.size(); ++t) {
    const uint32_t v = entry_user[t];
    if (P.perm[v] != 0xffffffffu) continue;
    P.perm[v] = next_id++;
    P.shared_nodes.push_back(P.perm[v]);
    P.shared_k.push_back((uint32_t)count[v]);
  }
  for (int64_t v = 0; v < nn; ++v)
    if (count[v] == 0) {
      P.perm[v] = next_id++;
      P.orphans.push_back(P.perm[v]);
    }
  if ((int64_t)next_id != nn) throw std::logic_error("node numbering is not a bijection");
  P.sgid.resize(entry_user.size());
  P.srank.resize(entry_user.size());
  for (size_t t = 0; t < entry_user.size(); ++t) {
    P.sgid[t] = P.perm[entry_user[t]];
    P.srank[t] = (uint32_t)entry_rank[t];
  }
  assign_partial_slots(P, nn);
  // positions stay below L; a stride of 5 mod 16 puts the components of a
  // node's force accumulator in different bank pairs
  P.node_stride = (P.max_nodes + kBankPairs - 1) / kBankPairs * kBankPairs + 5;
  return P;
}

void assign_partial_slots(PatchHost& P, int64_t nn) {
  const uint32_t ns = (uint32_t)P.shared_nodes.size();
  std::vector<int32_t> sidx((size_t)nn, -1);  // internal id -> shared node
  for (uint32_t s = 0; s < ns; ++s) sidx[P.shared_nodes[s]] = (int32_t)s;
  P.shared_part.assign(ns, 0);
  int64_t slots = 2 * (int64_t)ns;  // the dense rows of ranks 0 and 1
  for (uint32_t s = 0; s < ns; ++s) {
    P.shared_part[s] = (uint32_t)slots;
    slots += P.shared_k[s] > 2 ? P.shared_k[s] - 2 : 0;
  }
  if (slots >= (int64_t)UINT32_MAX) throw std::length_error("too many partial slots");
  P.nslots = slots;
  P.sslot.resize(P.sgid.size());
  for (size_t t = 0; t < P.sgid.size(); ++t) {
    const int32_t s = sidx[P.sgid[t]];
    if (s < 0 || P.srank[t] >= P.shared_k[s]) throw std::logic_error("shared entry without its node");
    P.sslot[t] = partial_slot(ns, (uint32_t)s, P.shared_part[s], P.srank[t]);
  }
}

}  // namespace akb
