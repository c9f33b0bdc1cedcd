// akb_msh.cu -- the Gmsh reader of include/akb_mesh.h (host code only).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/akb_mesh.h"
#include "akb_internal.cuh"

using akb::fail;

struct akb_msh {
  int32_t dim = 0;
  int32_t type = 0;
  std::vector<double> nodes;    // nb_nodes x dim
  std::vector<uint32_t> conn;   // elements of the mesh's dimension
  struct Group {
    std::string name;
    std::vector<uint32_t> nodes, elements;
    int32_t facet_nodes = 0;        // nodes per facet (0: no facet, -1: two kinds)
    std::vector<uint32_t> facets;   // elements of dimension dim - 1
  };
  std::vector<Group> groups;
};

namespace {

// Gmsh element types read here: number of nodes, dimension, library type
// (0: carries groups only -- points, and quadrangle_4 as the facet of a 3D
// mesh).
struct MshType {
  int nodes, dim, type;
};
bool msh_type(int t, MshType* out) {
  switch (t) {
  case 1: *out = {2, 1, AKB_SEGMENT_2}; return true;
  case 2: *out = {3, 2, AKB_TRIANGLE_3}; return true;
  case 3: *out = {4, 2, 0}; return true;
  case 4: *out = {4, 3, AKB_TETRAHEDRON_4}; return true;
  case 5: *out = {8, 3, AKB_HEXAHEDRON_8}; return true;
  case 15: *out = {1, 0, 0}; return true;
  default: return false;
  }
}

struct Reader {
  std::istringstream in;
  size_t line_no = 0;
  bool next(std::string& line) {
    while (std::getline(in, line)) {
      ++line_no;
      if (!line.empty() && line.back() == '\r') line.pop_back();
      const size_t b = line.find_first_not_of(" \t");
      if (b == std::string::npos) continue;
      line = line.substr(b);
      const size_t e = line.find_last_not_of(" \t");
      line = line.substr(0, e + 1);
      return true;
    }
    return false;
  }
  std::string where() const { return " (line " + std::to_string(line_no) + ")"; }
};

akb_status parse(const std::string& text, int32_t dim, akb_msh** out) {
  if (dim < 1 || dim > 3) return fail(AKB_ERR_INVALID_ARGUMENT, "spatial dimension must be 1, 2 or 3");
  Reader r;
  r.in.str(text);
  auto m = std::make_unique<akb_msh>();
  m->dim = dim;
  std::unordered_map<long long, uint32_t> node_of;  // file node id -> index
  std::map<long long, std::string> names;           // physical tag -> name
  bool has_names = false, has_format = false;
  struct Elem {
    int type_dim, type;
    long long phys;
    std::vector<uint32_t> nodes;
  };
  std::vector<Elem> elems;
  std::string line;
  while (r.next(line)) {
    if (line[0] != '$') return fail(AKB_ERR_BAD_MESH, "expected a $Block line" + r.where());
    const std::string block = line.substr(1);
    if (block == "MeshFormat") {
      if (!r.next(line)) return fail(AKB_ERR_BAD_MESH, "truncated $MeshFormat");
      std::istringstream s(line);
      double version = 0;
      int format = -1;
      s >> version >> format;
      if (format != 0) return fail(AKB_ERR_UNSUPPORTED, "only ASCII Gmsh files are read" + r.where());
      if (version < 2.0 || version >= 3.0)
        return fail(AKB_ERR_UNSUPPORTED, "only Gmsh format 2.x is read" + r.where());
      has_format = true;
    } else if (block == "PhysicalNames") {
      has_names = true;
      if (!r.next(line)) return fail(AKB_ERR_BAD_MESH, "truncated $PhysicalNames");
      const long n = std::stol(line);
      for (long k = 0; k < n; ++k) {
        if (!r.next(line)) return fail(AKB_ERR_BAD_MESH, "truncated $PhysicalNames");
        std::istringstream s(line);
        int pdim;
        long long id;
        std::string name;
        if (!(s >> pdim >> id >> std::quoted(name)))
          return fail(AKB_ERR_BAD_MESH, "bad physical name" + r.where());
        names[id] = name;
      }
    } else if (block == "Nodes" || block == "NOD") {
      if (!r.next(line)) return fail(AKB_ERR_BAD_MESH, "truncated $Nodes");
      const long long n = std::stoll(line);
      if (n < 0 || n >= (long long)UINT32_MAX) return fail(AKB_ERR_BAD_MESH, "bad node count");
      m->nodes.resize((size_t)n * dim);
      for (long long i = 0; i < n; ++i) {
        if (!r.next(line)) return fail(AKB_ERR_BAD_MESH, "truncated $Nodes");
        std::istringstream s(line);
        long long id;
        double x[3] = {0, 0, 0};
        if (!(s >> id >> x[0] >> x[1] >> x[2])) return fail(AKB_ERR_BAD_MESH, "bad node" + r.where());
        if (!node_of.emplace(id, (uint32_t)i).second)
          return fail(AKB_ERR_BAD_MESH, "node id given twice" + r.where());
        for (int c = 0; c < dim; ++c) m->nodes[(size_t)i * dim + c] = x[c];
      }
    } else if (block == "Elements" || block == "ELM") {
      if (!r.next(line)) return fail(AKB_ERR_BAD_MESH, "truncated $Elements");
      const long long n = std::stoll(line);
      for (long long i = 0; i < n; ++i) {
        if (!r.next(line)) return fail(AKB_ERR_BAD_MESH, "truncated $Elements");
        std::istringstream s(line);
        long long id;
        int t, ntags;
        if (!(s >> id >> t >> ntags) || ntags < 0) return fail(AKB_ERR_BAD_MESH, "bad element" + r.where());
        std::vector<long long> tags(ntags);
        for (auto& g : tags)
          if (!(s >> g)) return fail(AKB_ERR_BAD_MESH, "bad element tags" + r.where());
        MshType mt;
        if (!msh_type(t, &mt)) continue;  // a type off this path: skipped
        Elem e{mt.dim, mt.type, ntags > 0 ? tags[0] : 0, std::vector<uint32_t>(mt.nodes)};
        for (int a = 0; a < mt.nodes; ++a) {
          long long nid;
          if (!(s >> nid)) return fail(AKB_ERR_BAD_MESH, "bad element nodes" + r.where());
          const auto it = node_of.find(nid);
          if (it == node_of.end()) return fail(AKB_ERR_BAD_MESH, "element refers to an unknown node" + r.where());
          e.nodes[a] = it->second;
        }
        elems.push_back(std::move(e));
      }
    } else {
      // a block this reader does not use: skip to its end
      bool closed = false;
      while (r.next(line))
        if (line == "$End" + block) {
          closed = true;
          break;
        }
      if (!closed) return fail(AKB_ERR_BAD_MESH, "unterminated $" + block);
      continue;
    }
    if (!r.next(line) || line != "$End" + block)
      return fail(AKB_ERR_BAD_MESH, "expected $End" + block + r.where());
  }
  if (!has_format) return fail(AKB_ERR_BAD_MESH, "no $MeshFormat block");
  // the mesh: the elements of the requested dimension, of one type
  int type = 0;
  for (const auto& e : elems)
    if (e.type_dim == dim && e.type != 0) {  // (a quadrangle of a 2D mesh: skipped)
      if (type && e.type != type)
        return fail(AKB_ERR_UNSUPPORTED, "elements of several types in the mesh's dimension");
      type = e.type;
    }
  if (!type) return fail(AKB_ERR_BAD_MESH, "no element of the mesh's dimension");
  m->type = type;
  std::map<std::string, size_t> gidx;
  std::vector<std::vector<uint32_t>> gnodes, gelems, gfacets;
  std::vector<int32_t> gfnodes;
  uint32_t ecount = 0;
  for (const auto& e : elems) {
    const bool in_mesh = e.type_dim == dim && e.type != 0;
    if (in_mesh) m->conn.insert(m->conn.end(), e.nodes.begin(), e.nodes.end());
    if (has_names) {
      const auto it = names.find(e.phys);
      const std::string name = it != names.end() ? it->second : std::to_string(e.phys);
      auto g = gidx.find(name);
      if (g == gidx.end()) {
        g = gidx.emplace(name, gnodes.size()).first;
        gnodes.emplace_back();
        gelems.emplace_back();
        gfacets.emplace_back();
        gfnodes.push_back(0);
      }
      gnodes[g->second].insert(gnodes[g->second].end(), e.nodes.begin(), e.nodes.end());
      if (in_mesh) gelems[g->second].push_back(ecount);
      if (dim >= 2 && e.type_dim == dim - 1 && gfnodes[g->second] >= 0) {  // a facet
        const int32_t nf = (int32_t)e.nodes.size();
        if (gfnodes[g->second] && gfnodes[g->second] != nf) {  // two kinds: none kept
          gfnodes[g->second] = -1;
          gfacets[g->second].clear();
        } else {
          gfnodes[g->second] = nf;
          gfacets[g->second].insert(gfacets[g->second].end(), e.nodes.begin(), e.nodes.end());
        }
      }
    }
    if (in_mesh) ++ecount;
  }
  for (const auto& kv : gidx) {
    akb_msh::Group g;
    g.name = kv.first;
    g.nodes = std::move(gnodes[kv.second]);
    std::sort(g.nodes.begin(), g.nodes.end());
    g.nodes.erase(std::unique(g.nodes.begin(), g.nodes.end()), g.nodes.end());
    g.elements = std::move(gelems[kv.second]);
    g.facet_nodes = gfnodes[kv.second];
    g.facets = std::move(gfacets[kv.second]);
    m->groups.push_back(std::move(g));
  }
  *out = m.release();
  return AKB_OK;
}

}  // namespace

extern "C" {

akb_status akb_msh_read(const char* path, int32_t spatial_dimension, akb_msh** mesh) {
  if (!path || !mesh) return fail(AKB_ERR_INVALID_ARGUMENT, "null argument");
  *mesh = nullptr;
  std::ifstream f(path, std::ios::binary);
  if (!f) return fail(AKB_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
  std::stringstream ss;
  ss << f.rdbuf();
  try {
    return parse(ss.str(), spatial_dimension, mesh);
  } catch (const std::exception& ex) {
    return fail(AKB_ERR_BAD_MESH, std::string("mesh file: ") + ex.what());
  }
}

akb_status akb_msh_parse(const char* text, int64_t length, int32_t spatial_dimension,
                         akb_msh** mesh) {
  if (!text || !mesh || length < 0) return fail(AKB_ERR_INVALID_ARGUMENT, "null argument");
  *mesh = nullptr;
  try {
    return parse(std::string(text, (size_t)length), spatial_dimension, mesh);
  } catch (const std::exception& ex) {
    return fail(AKB_ERR_BAD_MESH, std::string("mesh text: ") + ex.what());
  }
}

akb_status akb_msh_destroy(akb_msh* mesh) {
  delete mesh;
  return AKB_OK;
}

akb_status akb_msh_get_mesh(const akb_msh* m, akb_mesh_desc* desc) {
  if (!m || !desc) return fail(AKB_ERR_INVALID_ARGUMENT, "null argument");
  desc->spatial_dimension = m->dim;
  desc->element_type = m->type;
  desc->nb_nodes = (int64_t)(m->nodes.size() / m->dim);
  desc->nb_elements = (int64_t)(m->conn.size() / akb::nnpe_of(m->type));
  desc->nodes = m->nodes.data();
  desc->connectivity = m->conn.data();
  return AKB_OK;
}

akb_status akb_msh_get_nb_groups(const akb_msh* m, int32_t* nb_groups) {
  if (!m || !nb_groups) return fail(AKB_ERR_INVALID_ARGUMENT, "null argument");
  *nb_groups = (int32_t)m->groups.size();
  return AKB_OK;
}

akb_status akb_msh_get_group(const akb_msh* m, int32_t index, const char** name,
                             int64_t* nb_nodes, const uint32_t** nodes, int64_t* nb_elements,
                             const uint32_t** elements) {
  if (!m) return fail(AKB_ERR_INVALID_ARGUMENT, "null mesh");
  if (index < 0 || index >= (int32_t)m->groups.size())
    return fail(AKB_ERR_INVALID_ARGUMENT, "group index out of range");
  const auto& g = m->groups[index];
  if (name) *name = g.name.c_str();
  if (nb_nodes) *nb_nodes = (int64_t)g.nodes.size();
  if (nodes) *nodes = g.nodes.data();
  if (nb_elements) *nb_elements = (int64_t)g.elements.size();
  if (elements) *elements = g.elements.data();
  return AKB_OK;
}

akb_status akb_msh_get_group_facets(const akb_msh* m, int32_t index, int64_t* nb_facets,
                                    int32_t* nodes_per_facet, const uint32_t** facets) {
  if (!m) return fail(AKB_ERR_INVALID_ARGUMENT, "null mesh");
  if (index < 0 || index >= (int32_t)m->groups.size())
    return fail(AKB_ERR_INVALID_ARGUMENT, "group index out of range");
  const auto& g = m->groups[index];
  if (g.facet_nodes < 0)
    return fail(AKB_ERR_UNSUPPORTED, "group '" + g.name + "' has facets of two kinds");
  if (nb_facets) *nb_facets = g.facet_nodes ? (int64_t)(g.facets.size() / g.facet_nodes) : 0;
  if (nodes_per_facet) *nodes_per_facet = g.facet_nodes;
  if (facets) *facets = g.facets.data();
  return AKB_OK;
}

}  // extern "C"

namespace {

// Gauss points of a boundary element in its natural coordinates, with the
// weights and shape functions there: segment_2 (N = (1 -+ xi) / 2) and
// triangle_3 (N = 1 - xi - eta, xi, eta) one point; quadrangle_4 (corners
// (-1,-1), (1,-1), (1,1), (-1,1)) the 2 x 2 rule.
struct FacetPoint {
  double w, N[4], dN[2][4];  // shape values, derivatives in xi and eta
};
std::vector<FacetPoint> facet_rule(int nf) {
  std::vector<FacetPoint> pts;
  if (nf == 2) {
    pts.push_back({2.0, {0.5, 0.5}, {{-0.5, 0.5}}});
  } else if (nf == 3) {
    const double t = 1.0 / 3.0;
    pts.push_back({0.5, {t, t, t}, {{-1.0, 1.0, 0.0}, {-1.0, 0.0, 1.0}}});
  } else {
    const double g = 1.0 / std::sqrt(3.0);
    const double cx[4] = {-1, 1, 1, -1}, cy[4] = {-1, -1, 1, 1};
    for (int q = 0; q < 4; ++q) {
      const double xi = cx[q] * g, eta = cy[q] * g;
      FacetPoint p{1.0, {}, {}};
      for (int a = 0; a < 4; ++a) {
        p.N[a] = 0.25 * (1 + cx[a] * xi) * (1 + cy[a] * eta);
        p.dN[0][a] = 0.25 * cx[a] * (1 + cy[a] * eta);
        p.dN[1][a] = 0.25 * cy[a] * (1 + cx[a] * xi);
      }
      pts.push_back(p);
    }
  }
  return pts;
}

akb_status check_facets(int32_t d, int64_t nb_nodes, const double* X, int64_t nb_facets, int32_t nf,
                        const uint32_t* facets) {
  if (d != 2 && d != 3)
    return fail(AKB_ERR_UNSUPPORTED, "Neumann conditions are defined in 2D and 3D");
  if (nb_facets < 0 || nb_nodes < 0) return fail(AKB_ERR_INVALID_ARGUMENT, "negative count");
  if (nb_facets > 0 && (!X || !facets)) return fail(AKB_ERR_INVALID_ARGUMENT, "null argument");
  if (nb_facets > 0 && ((d == 2 && nf != 2) || (d == 3 && nf != 3 && nf != 4)))
    return fail(AKB_ERR_INVALID_ARGUMENT, "facets must be segments in 2D, triangles or "
                                          "quadrangles in 3D");
  for (int64_t k = 0; k < nb_facets * nf; ++k)
    if (facets[k] >= (uint64_t)nb_nodes)
      return fail(AKB_ERR_INVALID_ARGUMENT, "facet refers to a node out of range");
  return AKB_OK;
}

// At point p of facet c: its coordinates x, unit normal n (the reference's:
// (t_y, -t_x) of a segment's tangent, t_xi x t_eta of a surface facet) and
// w |J|; false for a degenerate facet.
bool facet_point(int d, int nf, const double* X, const uint32_t* c, const FacetPoint& p,
                 double* x, double* n, double* wj) {
  double t0[3] = {0, 0, 0}, t1[3] = {0, 0, 0};
  for (int i = 0; i < d; ++i) x[i] = 0.0;
  for (int a = 0; a < nf; ++a)
    for (int i = 0; i < d; ++i) {
      const double xa = X[(size_t)c[a] * d + i];
      x[i] += p.N[a] * xa;
      t0[i] += p.dN[0][a] * xa;
      if (d == 3) t1[i] += p.dN[1][a] * xa;
    }
  double jac;
  if (d == 2) {
    n[0] = t0[1];
    n[1] = -t0[0];
    jac = std::sqrt(t0[0] * t0[0] + t0[1] * t0[1]);
  } else {
    n[0] = t0[1] * t1[2] - t0[2] * t1[1];
    n[1] = t0[2] * t1[0] - t0[0] * t1[2];
    n[2] = t0[0] * t1[1] - t0[1] * t1[0];
    jac = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  }
  if (!(jac > 0)) return false;
  for (int i = 0; i < d; ++i) n[i] /= jac;
  *wj = p.w * jac;
  return true;
}

}  // namespace

extern "C" {

akb_status akb_neumann_forces(int32_t d, int64_t nb_nodes, const double* X, int64_t nb_facets,
                              int32_t nf, const uint32_t* facets, int32_t kind,
                              const double* value, double* forces) {
  akb_status st = check_facets(d, nb_nodes, X, nb_facets, nf, facets);
  if (st != AKB_OK || nb_facets == 0) return st;
  if (!value || !forces) return fail(AKB_ERR_INVALID_ARGUMENT, "null argument");
  if (kind != AKB_NEUMANN_TRACTION && kind != AKB_NEUMANN_STRESS)
    return fail(AKB_ERR_INVALID_ARGUMENT, "unknown Neumann kind");
  const std::vector<FacetPoint> pts = facet_rule(nf);
  for (int64_t f = 0; f < nb_facets; ++f) {
    const uint32_t* c = facets + f * nf;
    for (const FacetPoint& p : pts) {
      double x[3], n[3], wj;
      if (!facet_point(d, nf, X, c, p, x, n, &wj)) return fail(AKB_ERR_BAD_MESH, "degenerate facet");
      double t[3] = {0, 0, 0};
      for (int i = 0; i < d; ++i) {
        if (kind == AKB_NEUMANN_TRACTION) {
          t[i] = value[i];
        } else {
          for (int j = 0; j < d; ++j) t[i] += value[i + j * d] * n[j];
        }
      }
      for (int a = 0; a < nf; ++a)
        for (int i = 0; i < d; ++i) forces[(size_t)c[a] * d + i] += wj * p.N[a] * t[i];
    }
  }
  return AKB_OK;
}

int32_t akb_facet_points(int32_t nodes_per_facet) {
  return nodes_per_facet == 2 || nodes_per_facet == 3 ? 1 : nodes_per_facet == 4 ? 4 : 0;
}

akb_status akb_facet_quadrature(int32_t d, int64_t nb_nodes, const double* X, int64_t nb_facets,
                                int32_t nf, const uint32_t* facets, double* coords, double* normals,
                                double* weighted_shapes) {
  akb_status st = check_facets(d, nb_nodes, X, nb_facets, nf, facets);
  if (st != AKB_OK || nb_facets == 0) return st;
  if (!coords || !normals || !weighted_shapes)
    return fail(AKB_ERR_INVALID_ARGUMENT, "null argument");
  const std::vector<FacetPoint> pts = facet_rule(nf);
  const size_t nq = pts.size();
  for (int64_t f = 0; f < nb_facets; ++f)
    for (size_t q = 0; q < nq; ++q) {
      const size_t k = (size_t)f * nq + q;
      double wj;
      if (!facet_point(d, nf, X, facets + f * nf, pts[q], coords + k * d, normals + k * d, &wj))
        return fail(AKB_ERR_BAD_MESH, "degenerate facet");
      for (int a = 0; a < nf; ++a) weighted_shapes[k * nf + a] = wj * pts[q].N[a];
    }
  return AKB_OK;
}

}  // extern "C"
