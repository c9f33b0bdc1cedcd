// FE^2 through the C++ shim: a block of hexahedra whose material is a user
// material that asks periodic RVEs (akb_rve_solve, device arrays, the model's
// stream) for the stress at every Gauss point -- the structure of the
// reference's MaterialFE2::computeStress (material_FE2.cc:116-157). With a
// homogeneous neo-Hookean RVE the result must equal the built-in
// neo-Hookean material; the program prints both displacements.
#include <akantu_b200/solid_mechanics_model.hh>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

using namespace akantu_b200;

static void build_block(Mesh& mesh, int n, Real L) {
  mesh.setElementType(_hexahedron_8);
  auto& X = mesh.getNodes();
  X.resize((n + 1) * (n + 1) * (n + 1), 3);
  auto id = [n](int i, int j, int k) { return (uint32_t)(i + (n + 1) * (j + (n + 1) * k)); };
  for (int k = 0; k <= n; ++k)
    for (int j = 0; j <= n; ++j)
      for (int i = 0; i <= n; ++i) {
        X(id(i, j, k), 0) = i * L / n;
        X(id(i, j, k), 1) = j * L / n;
        X(id(i, j, k), 2) = k * L / n;
      }
  auto& C = mesh.getConnectivity();
  C.resize(n * n * n, 8);
  int e = 0;
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i, ++e) {
        const uint32_t c[8] = {id(i, j, k),         id(i + 1, j, k),     id(i + 1, j + 1, k),
                               id(i, j + 1, k),     id(i, j, k + 1),     id(i + 1, j, k + 1),
                               id(i + 1, j + 1, k + 1), id(i, j + 1, k + 1)};
        for (int a = 0; a < 8; ++a) C(e, a) = c[a];
      }
}

static void run(bool fe2, int steps, std::vector<Real>& out) {
  const int n = 3;
  const Real L = 0.03, rho = 1100., E = 1.0857142857142857e6, nu = 0.35714285714285715;
  Mesh mesh(3);
  build_block(mesh, n, L);
  SolidMechanicsModel model(mesh, AKB_MODE_FP64);
  akb_rve* rve = nullptr;
  if (fe2) {
    const uint8_t vox[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    akb_material_desc md{AKB_MATERIAL_NEOHOOKEAN, 0, 1, 0, rho, E, nu};
    akb_rve_desc rd{2, 1, 1.0, vox, &md};
    akb_rve_options ro{AKB_MODE_FP64, 0, nullptr, 0, 0, 0.0, 0.0, 0.0};
    check(akb_rve_create(&rd, &ro, &rve));
    model.addMaterial(MaterialUser(rho, E, nu, [rve](const double* gu, double* st, int64_t np,
                                                     void* stream) {
      check(akb_rve_solve(rve, np, gu, nullptr, st, nullptr, nullptr, stream));
    }));
  } else {
    model.addMaterial(MaterialNeohookean(rho, E, nu));
  }
  model.initFull(_analysis_method = _explicit_lumped_mass);
  std::vector<uint32_t> left;
  const auto& X = mesh.getNodes();
  for (UInt k = 0; k < mesh.getNbNodes(); ++k)
    if (X(k, 0) == 0.0) left.push_back(k);
  for (auto ax : {_x, _y, _z}) model.applyBC(BC::Dirichlet::FixedValue(0., ax), left);
  auto& v = model.getVelocity();
  for (UInt k = 0; k < mesh.getNbNodes(); ++k)
    if (X(k, 0) != 0.0) {
      v(k, 0) = 0.02 * std::sin(7.0 * k);
      v(k, 1) = 0.02 * std::cos(5.0 * k);
      v(k, 2) = 0.01;
    }
  model.setTimeStep(0.5 * model.getStableTimeStep());
  model.solveSteps(steps);
  const auto& u = model.getDisplacement();
  out.assign(u.storage(), u.storage() + u.size() * 3);
  if (rve) akb_rve_destroy(rve);
}

int main(int argc, char** argv) {
  const int steps = argc > 1 ? std::atoi(argv[1]) : 40;
  std::vector<Real> a, b;
  run(false, steps, a);
  run(true, steps, b);
  for (size_t k = 0; k < a.size(); ++k) std::printf("%.17g %.17g\n", a[k], b[k]);
  return 0;
}
