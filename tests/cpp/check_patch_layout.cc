// Host check of the fused step's patch records (akb_patch_build.cu), no GPU:
// every shared-memory index the kernel derives from a record stays inside
// the buffers it addresses, the contribution slots of a chunk are a
// bijection, the first- and second-level sums reproduce each node's sum of
// contributions, node positions are distinct, and the coloured accesses (a
// half-warp's scatter, a half-warp's row of piece sums; 16 bank pairs for
// 8-byte contributions, 32 banks for 4-byte ones) hit distinct banks.
// Prints one line per case and exits non-zero on any failure.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <vector>

#include "akb_patch.cuh"

using namespace akb;

namespace {

struct Mesh {
  std::vector<double> X;
  std::vector<uint32_t> C;
  int dim, nnpe;
};

Mesh tet_cube(int n) {
  Mesh m{{}, {}, 3, 4};
  const int N = n + 1;
  for (int k = 0; k < N; ++k)
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < N; ++i) m.X.insert(m.X.end(), {double(i), double(j), double(k)});
  auto id = [&](int i, int j, int k) { return (uint32_t)((k * N + j) * N + i); };
  const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i)
        for (const auto& p : perm) {
          int c[3] = {i, j, k};
          m.C.push_back(id(c[0], c[1], c[2]));
          for (int s = 0; s < 3; ++s) {
            c[p[s]]++;
            m.C.push_back(id(c[0], c[1], c[2]));
          }
        }
  return m;
}

Mesh hex_cube(int n) {
  Mesh m{{}, {}, 3, 8};
  const int N = n + 1;
  for (int k = 0; k < N; ++k)
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < N; ++i) m.X.insert(m.X.end(), {double(i), double(j), double(k)});
  auto id = [&](int i, int j, int k) { return (uint32_t)((k * N + j) * N + i); };
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i)
        m.C.insert(m.C.end(), {id(i, j, k), id(i + 1, j, k), id(i + 1, j + 1, k), id(i, j + 1, k),
                               id(i, j, k + 1), id(i + 1, j, k + 1), id(i + 1, j + 1, k + 1),
                               id(i, j + 1, k + 1)});
  return m;
}

Mesh tri_plate(int nx, int ny) {
  Mesh m{{}, {}, 2, 3};
  for (int j = 0; j <= ny; ++j)
    for (int i = 0; i <= nx; ++i) m.X.insert(m.X.end(), {double(i), double(j)});
  auto id = [&](int i, int j) { return (uint32_t)(j * (nx + 1) + i); };
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      m.C.insert(m.C.end(), {id(i, j), id(i + 1, j), id(i + 1, j + 1)});
      m.C.insert(m.C.end(), {id(i, j), id(i + 1, j + 1), id(i, j + 1)});
    }
  return m;
}

Mesh seg_line(int n) {
  Mesh m{{}, {}, 1, 2};
  for (int i = 0; i <= n; ++i) m.X.push_back(i);
  for (int i = 0; i < n; ++i) m.C.insert(m.C.end(), {(uint32_t)i, (uint32_t)i + 1});
  return m;
}

// the same mesh with its elements in a scrambled order
Mesh shuffled(Mesh m, unsigned seed) {
  srand(seed);
  const int ne = (int)m.C.size() / m.nnpe;
  for (int e = ne - 1; e > 0; --e) {
    const int f = rand() % (e + 1);
    for (int a = 0; a < m.nnpe; ++a) std::swap(m.C[e * m.nnpe + a], m.C[f * m.nnpe + a]);
  }
  return m;
}

// a star: every element shares node 0 (one node with a long run)
Mesh star(int k) {
  Mesh m{{}, {}, 3, 4};
  m.X.insert(m.X.end(), {0, 0, 0});
  for (int i = 0; i < k + 2; ++i) m.X.insert(m.X.end(), {std::cos(i * 0.37), std::sin(i * 0.37), i * 0.1});
  for (int i = 0; i < k; ++i) m.C.insert(m.C.end(), {0u, (uint32_t)i + 1, (uint32_t)i + 2, (uint32_t)i + 3});
  return m;
}

size_t a16(size_t x) { return (x + 15) & ~size_t(15); }

int fails = 0;
#define CHECK(c)                                                                         \
  do {                                                                                   \
    if (!(c) && fails++ < 20)                                                            \
      printf("FAIL %s (line %d, case %s, patch %d, chunk %d)\n", #c, __LINE__, name, p, c_); \
  } while (0)

long max_group(const std::vector<int>& addr, int banks) {
  std::vector<std::set<int>> b(banks);
  for (int x : addr) b[x % banks].insert(x);
  size_t mx = 0;
  for (auto& s : b) mx = std::max(mx, s.size());
  return (long)mx;
}

void check(const char* name, const Mesh& m, int target, int maxn, int cbytes,
           const std::vector<uint8_t>* force = nullptr) {
  const int64_t nn = (int64_t)m.X.size() / m.dim, ne = (int64_t)m.C.size() / m.nnpe;
  PatchHost P = build_patches(m.X.data(), m.C.data(), nn, ne, m.dim, m.nnpe, target, maxn, cbytes,
                              force ? force->data() : nullptr);
  const int n = m.nnpe, G = cbytes == 8 ? 16 : 32, LM = P.node_stride, CH = P.contrib_slots;
  const int GP = place_group(m.dim);
  long worst_scatter = 0, worst_sum = 0, worst_gather = 0, acc_conflicts = 0, acc_groups = 0;
  int p = -1, c_ = -1;
  std::vector<int> elem_seen(ne, 0);
  // the internal numbering is a bijection: interior ranges in patch order,
  // then the shared block, then the nodes of no element
  std::vector<int> hit(nn, 0);
  for (int64_t v = 0; v < nn; ++v) {
    CHECK(P.perm[v] < (uint64_t)nn);
    if (P.perm[v] < (uint64_t)nn) hit[P.perm[v]]++;
  }
  for (int64_t g = 0; g < nn; ++g) CHECK(hit[g] == 1);
  std::vector<int64_t> user_of(nn, -1);
  for (int64_t v = 0; v < nn; ++v)
    if (P.perm[v] < (uint64_t)nn) user_of[P.perm[v]] = v;
  int64_t next = 0;
  for (int q = 0; q < P.npatch; ++q) {
    CHECK(P.ibeg[q] == next);
    next += P.nint[q];
  }
  CHECK(next == (int64_t)P.shared_base);
  CHECK((int64_t)P.shared_base + (int64_t)P.shared_nodes.size() + (int64_t)P.orphans.size() == nn);
  // every shared node: its k patches hold it with ranks 0..k-1 (in patch
  // order), one slot each
  std::map<uint32_t, std::vector<int>> ranks;
  for (int q = 0; q < P.npatch; ++q)
    for (int t = P.sh_ptr[q]; t < P.sh_ptr[q + 1]; ++t) {
      const int64_t s = (int64_t)P.sgid[t] - P.shared_base;
      CHECK(s >= 0 && s < (int64_t)P.shared_nodes.size());
      if (s < 0 || s >= (int64_t)P.shared_nodes.size()) continue;
      const int r = (int)P.srank[t];
      CHECK(r >= 0 && r < (int)P.shared_k[s]);
      CHECK((int)ranks[P.sgid[t]].size() == r);  // patches met in order
      // ranks 0 and 1 in the dense rows, the others after them node by node
      CHECK(P.sslot[t] == akb::partial_slot((uint32_t)P.shared_nodes.size(), (uint32_t)s,
                                            P.shared_part[s], (uint32_t)r));
      ranks[P.sgid[t]].push_back(r);
    }
  // forced (interface) nodes are shared even in one patch
  if (force)
    for (int64_t v = 0; v < nn; ++v)
      if ((*force)[v] && P.perm[v] < P.shared_base) CHECK(false);
  int64_t slots = 2 * (int64_t)P.shared_nodes.size();
  for (size_t s = 0; s < P.shared_nodes.size(); ++s) {
    std::vector<int> r = ranks[P.shared_nodes[s]];
    std::sort(r.begin(), r.end());
    CHECK((int)r.size() == (int)P.shared_k[s]);
    for (int i = 0; i < (int)r.size(); ++i) CHECK(r[i] == i);
    CHECK(P.shared_part[s] == slots);
    slots += P.shared_k[s] > 2 ? P.shared_k[s] - 2 : 0;
  }
  CHECK(slots == P.nslots);
  {  // no two entries share a slot
    std::vector<uint32_t> all(P.sslot);
    std::sort(all.begin(), all.end());
    CHECK(std::adjacent_find(all.begin(), all.end()) == all.end());
    CHECK(all.empty() || (int64_t)all.back() < P.nslots);
  }
  for (p = 0; p < P.npatch; ++p) {
    c_ = -1;
    const int nint = P.nint[p], s0 = P.sh_ptr[p], L = nint + (P.sh_ptr[p + 1] - s0);
    const int eb = P.elem_ptr[p];
    const int nep = P.elem_ptr[p + 1] - eb;
    CHECK(L <= P.max_nodes && nint <= P.max_interior && L - nint <= P.max_shared && nep > 0);
    // internal id of the node at each shared-memory position
    auto id_at = [&](int pos) -> int64_t {
      return pos < nint ? (int64_t)P.ibeg[p] + pos : (int64_t)P.sgid[s0 + pos - nint];
    };
    for (int i = eb; i < eb + nep; ++i) elem_seen[P.elem_order[i]]++;
    const int nch = (nep + kChunk - 1) / kChunk;
    CHECK(P.chunk_base[p + 1] - P.chunk_base[p] == nch);
    for (int c = 0; c < nch; ++c) {
      c_ = c;
      const ChunkDesc& cd = P.chunks[P.chunk_base[p] + c];
      CHECK((int)cd.bytes <= P.chunk_bytes && cd.bytes % 16 == 0);
      CHECK((size_t)cd.off16 * 8 + cd.bytes / 2 <= P.cdata.size());
      const uint16_t* rec = &P.cdata[(size_t)cd.off16 * 8];
      const char* rb = (const char*)rec;
      const int nec = std::min(kChunk, nep - c * kChunk);
      const size_t A = a16((size_t)nec * n * 2);
      const uint16_t* lcs = rec + 8;
      const uint16_t* sl = (const uint16_t*)(rb + 16 + A);
      const int R = rec[0], ng = rec[1], o_runs = rec[2], o_goff = rec[3], o_idx = rec[4];
      {
        // the kernel reads the header as four little-endian 32-bit words
        uint32_t hd[4];
        std::memcpy(hd, rec, 16);
        CHECK((int)(hd[0] & 0xffff) == R && (int)(hd[1] & 0xffff) == o_runs &&
              (int)(hd[1] >> 16) == o_goff && (int)(hd[2] & 0xffff) == o_idx);
      }
      CHECK(rec[5] == G && R % G == 0 && ng * G == R && R <= P.max_runs);
      CHECK(16 + 2 * A <= (size_t)o_runs && o_runs + 4 * R <= o_goff && o_goff + 2 * ng <= o_idx &&
            o_idx <= (int)cd.bytes && o_runs % 4 == 0 && o_goff % 2 == 0 && o_idx % 2 == 0);
      const uint32_t* runs = (const uint32_t*)(rb + o_runs);
      const uint16_t* goff = (const uint16_t*)(rb + o_goff);
      const uint16_t* idx = (const uint16_t*)(rb + o_idx);
      // slots: a bijection onto the chunk's corners
      std::vector<int> owner(CH, -1);
      for (int k = 0; k < nec * n; ++k) {
        CHECK(sl[k] < CH && lcs[k] < L && lcs[k] < LM);
        const uint32_t e = P.elem_order[eb + c * kChunk + k / n];
        if (lcs[k] < L) CHECK(id_at(lcs[k]) == (int64_t)P.perm[m.C[(size_t)e * n + k % n]]);
        if (sl[k] < CH) {
          CHECK(owner[sl[k]] < 0);
          owner[sl[k]] = k;
        }
      }
      // sums: contribution k = k + 1; the runs must give every node the sum
      // of its corners, each contribution read once, a node in one run
      std::map<int, long> expect, got;
      for (int k = 0; k < nec * n; ++k) expect[lcs[k]] += k + 1;
      std::vector<int> reads(CH, 0);
      for (int q = 0; q < R; ++q) {
        const int len = runs[q] >> 16, jp = runs[q] & 0xffff;
        if (!len) continue;
        CHECK(jp < L && got.count(jp) == 0);
        const int base = goff[q / G] + q % G;
        CHECK(q / G + 1 >= ng || base + (len - 1) * G < goff[q / G + 1]);
        CHECK((size_t)o_idx + 2 * (size_t)(base + (len - 1) * G) < cd.bytes);
        long f = 0;
        int prev = -1;
        for (int t = 0; t < len; ++t) {
          const int s = idx[base + t * G];
          CHECK(s < CH && owner[s] >= 0);
          if (s >= CH || owner[s] < 0) continue;
          CHECK(lcs[owner[s]] == jp);       // the run's node
          CHECK(owner[s] / n >= prev);      // ascending element order
          prev = owner[s] / n;
          reads[s]++;
          f += owner[s] + 1;
        }
        got[jp] = f;
      }
      for (int s = 0; s < CH; ++s)
        if (owner[s] >= 0) CHECK(reads[s] == 1);
      CHECK(got == expect);
      // colouring: one scatter instruction (corner a of G elements), entry t
      // of a group's runs: distinct banks; a group's node accumulators
      for (int h = 0; h * G < nec; ++h)
        for (int a = 0; a < n; ++a) {
          std::vector<int> ad;
          for (int e = h * G; e < std::min(nec, h * G + G); ++e) ad.push_back(sl[e * n + a]);
          worst_scatter = std::max(worst_scatter, max_group(ad, G));
        }
      for (int g = 0; g < ng; ++g) {
        int Lg = 0;
        for (int q = g * G; q < g * G + G; ++q) Lg = std::max(Lg, (int)(runs[q] >> 16));
        for (int t = 0; t < Lg; ++t) {
          std::vector<int> ad;
          for (int q = g * G; q < g * G + G; ++q)
            if (t < (int)(runs[q] >> 16)) ad.push_back(idx[goff[g] + t * G + q % G]);
          worst_sum = std::max(worst_sum, max_group(ad, G));
        }
        std::vector<int> acc;
        for (int q = g * G; q < g * G + G; ++q)
          if (runs[q] >> 16) acc.push_back(runs[q] & 0xffff);
        for (int hh = 0; hh < (int)acc.size(); hh += 16) {
          std::vector<int> half(acc.begin() + hh, acc.begin() + std::min((int)acc.size(), hh + 16));
          acc_conflicts += max_group(half, 16) - 1;
          acc_groups++;
        }
      }
      for (int h = 0; h * GP < nec; ++h)
        for (int a = 0; a < n; ++a) {
          std::vector<int> ad;
          for (int e = h * GP; e < std::min(nec, h * GP + GP); ++e) ad.push_back(lcs[e * n + a]);
          worst_gather = std::max(worst_gather, max_group(ad, GP));
        }
    }
  }
  p = c_ = -1;
  for (int64_t e = 0; e < ne; ++e) CHECK(elem_seen[e] == 1);  // every element in one patch
  CHECK(worst_scatter <= 1 && worst_sum <= 1);
  printf("%-28s patches %5d max_nodes %4d contrib %4d chunk_bytes %5d worst bank group "
         "%ld/%ld (node gathers %ld, accumulator conflicts %.2f per half-warp)\n",
         name, P.npatch, P.max_nodes, CH, P.chunk_bytes, worst_scatter, worst_sum, worst_gather,
         acc_groups ? (double)acc_conflicts / acc_groups : 0.0);
}

}  // namespace

int main() {
  check("tet4 cube 20 fp64", tet_cube(20), 1024, 400, 8);
  check("tet4 cube 20 fp32", tet_cube(20), 768, 320, 4);
  check("tet4 shuffled fp64", shuffled(tet_cube(12), 1), 1024, 400, 8);
  check("tet4 shuffled fp32", shuffled(tet_cube(12), 2), 1024, 400, 4);
  check("tet4 odd sizes", tet_cube(7), 300, 150, 8);
  check("tet4 star", star(300), 1024, 400, 8);
  check("hex8 cube fp64", hex_cube(16), 512, 800, 8);
  check("hex8 cube fp32", hex_cube(16), 512, 800, 4);
  check("tri3 plate", tri_plate(200, 20), 1024, 640, 8);
  check("tri3 plate small patches", tri_plate(200, 20), 256, 200, 8);
  check("seg2 line fp64", seg_line(3000), 1024, 1100, 8);
  check("seg2 line fp32", seg_line(3000), 1024, 1100, 4);
  {
    // interface nodes of a partitioned mesh (every node on the plane x = 6)
    Mesh c = tet_cube(12);
    std::vector<uint8_t> force(c.X.size() / 3, 0);
    for (size_t v = 0; v < force.size(); ++v) force[v] = c.X[v * 3] == 6.0;
    check("tet4 forced interface", c, 1024, 400, 8, &force);
  }
  {
    // nodes of no element, placed after the others
    Mesh c = tet_cube(6);
    c.X.insert(c.X.end(), {50, 50, 50, 60, 60, 60});
    check("tet4 with orphan nodes", c, 256, 200, 8);
  }
  printf("fails %d\n", fails);
  return fails != 0;
}
