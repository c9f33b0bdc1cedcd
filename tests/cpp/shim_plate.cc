// Drives the explicit path through the C++ shim the way a reference user
// writes it (examples/explicit/explicit_dynamic.cc:38-106): plate of
// triangle_3, left edge fixed by applyBC(FixedValue), sinusoidal initial
// displacement, dt = 0.8 x stable, N steps; prints the displacement.
#include <akantu_b200/solid_mechanics_model.hh>

#include <cmath>
#include <cstdio>
#include <cstdlib>

using namespace akantu_b200;

int main(int argc, char** argv) {
  const int nx = 20, ny = 4, steps = argc > 1 ? std::atoi(argv[1]) : 100;
  const int precision = argc > 2 ? std::atoi(argv[2]) : AKB_MODE_FP64_REFERENCE;
  const Real lx = 1.0, ly = 0.2;
  Mesh mesh(2);
  mesh.setElementType(_triangle_3);
  auto& X = mesh.getNodes();
  X.resize((nx + 1) * (ny + 1), 2);
  for (int j = 0; j <= ny; ++j)
    for (int i = 0; i <= nx; ++i) {
      X(j * (nx + 1) + i, 0) = i * (lx / nx);
      X(j * (nx + 1) + i, 1) = j * (ly / ny);
    }
  auto& C = mesh.getConnectivity();
  C.resize(2 * nx * ny, 3);
  int e = 0;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      uint32_t n00 = j * (nx + 1) + i, n10 = n00 + 1, n01 = n00 + nx + 1, n11 = n01 + 1;
      C(e, 0) = n00; C(e, 1) = n10; C(e, 2) = n11; ++e;
      C(e, 0) = n00; C(e, 1) = n11; C(e, 2) = n01; ++e;
    }
  SolidMechanicsModel model(mesh, precision);
  model.addMaterial(MaterialElastic(7800., 210e9, 0.3));
  model.initFull(_analysis_method = _explicit_lumped_mass);
  std::vector<uint32_t> left;
  for (int j = 0; j <= ny; ++j) left.push_back(j * (nx + 1));
  model.applyBC(BC::Dirichlet::FixedValue(0., _x), left);
  model.applyBC(BC::Dirichlet::FixedValue(0., _y), left);
  auto& u = model.getDisplacement();
  for (UInt n = 0; n < mesh.getNbNodes(); ++n)
    if (X(n, 0) != 0.0) u(n, 0) = 1e-4 * std::sin(M_PI * X(n, 0) / lx);
  model.setTimeStep(0.8 * model.getStableTimeStep());
  for (int s = 0; s < steps; ++s) model.solveStep();
  const auto& d = model.getDisplacement();
  std::printf("%.17g\n", model.getEnergy("kinetic"));
  for (UInt n = 0; n < mesh.getNbNodes(); ++n) std::printf("%.17g %.17g\n", d(n, 0), d(n, 1));
  return 0;
}
