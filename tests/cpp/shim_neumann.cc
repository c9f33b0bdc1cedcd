// shim_neumann.cc -- the C++ shim's Mesh::read and Neumann forces on the host
// (no model, no GPU): for a group of a 2D Gmsh file, prints its facet count,
// the summed nodal forces of FromTraction({0, -2}) and the summed forces of
// FromStress(identity) (the traction is then each facet's unit normal).
#include <cstdio>

#include "akantu_b200/solid_mechanics_model.hh"

using namespace akantu_b200;

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: shim_neumann mesh.msh group\n");
    return 2;
  }
  try {
    Mesh mesh(2);
    mesh.read(argv[1]);
    const NodeGroup& g = mesh.getNodeGroup(argv[2]);
    Array<Real> f(mesh.getNbNodes(), 2), h(mesh.getNbNodes(), 2);
    addNeumannForces(mesh, argv[2], BC::Neumann::FromTraction({0.0, -2.0}), f);
    addNeumannForces(mesh, argv[2], BC::Neumann::FromStress({1.0, 0.0, 0.0, 1.0}), h);
    double s[4] = {0, 0, 0, 0};
    for (UInt i = 0; i < mesh.getNbNodes(); ++i) {
      s[0] += f(i, 0);
      s[1] += f(i, 1);
      s[2] += h(i, 0);
      s[3] += h(i, 1);
    }
    const long nf = g.nodes_per_facet ? (long)(g.facets.size() / g.nodes_per_facet) : 0;
    std::printf("%ld %.17g %.17g %.17g %.17g\n", nf, s[0], s[1], s[2], s[3]);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
