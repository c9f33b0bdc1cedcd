// solid_mechanics_model.hh -- header-only C++ shim over include/akb.h that
// keeps the reference's names for the explicit path, so that code written
// against akantu::SolidMechanicsModel (solid_mechanics_model.hh:58) compiles
// with `using namespace akantu_b200;` and runs on the GPU:
//
//   Mesh mesh(3); ...                               // mesh.hh:100
//   SolidMechanicsModel model(mesh);                // solid_mechanics_model.hh:85-88
//   model.addMaterial(MaterialElastic(rho, E, nu)); // material input file section
//   model.initFull(_analysis_method = _explicit_lumped_mass);  // model.hh:78-99
//   model.setTimeStep(0.8 * model.getStableTimeStep());
//   auto & u = model.getDisplacement();  u(n, 0) = ...;   // Array<Real> rows
//   model.applyBC(BC::Dirichlet::FixedValue(0., _x), nodes);
//   model.solveStep();
//   Real ekin = model.getEnergy("kinetic");
//
// Nodal arrays returned by reference are host mirrors of the device state:
// they are refreshed on every get*() call and written back before the next
// call that uses the state, so in-place edits reach the model as with the
// reference's model-owned arrays. Errors throw akantu_b200::Exception.
#pragma once

#include <cstdint>
#include <functional>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../akb.h"
#include "../akb_fe2.h"
#include "../akb_mesh.h"

namespace akantu_b200 {

using Real = double;
using UInt = unsigned int;

enum AnalysisMethod { _explicit_lumped_mass = 0 };
enum SpatialDirection { _x = 0, _y = 1, _z = 2 };
enum ElementType {
  _segment_2 = AKB_SEGMENT_2,
  _triangle_3 = AKB_TRIANGLE_3,
  _tetrahedron_4 = AKB_TETRAHEDRON_4,
  _hexahedron_8 = AKB_HEXAHEDRON_8
};
struct AnalysisMethodArg {
  AnalysisMethod value;
};
struct AnalysisMethodTag {
  AnalysisMethodArg operator=(AnalysisMethod m) const { return {m}; }
};
static constexpr AnalysisMethodTag _analysis_method{};

class Exception : public std::runtime_error {
 public:
  Exception(akb_status s, const std::string& what) : std::runtime_error(what), status(s) {}
  akb_status status;
};

inline void check(akb_status s) {
  if (s != AKB_OK) throw Exception(s, akb_last_error());
}

// Row-major table with the reference Array<T> accessors (aka_array.hh:139-224).
template <typename T>
class Array {
 public:
  Array() = default;
  Array(UInt rows, UInt cols, T value = T()) : rows_(rows), cols_(cols), v_(rows * cols, value) {}
  T& operator()(UInt i, UInt j = 0) { return v_[i * cols_ + j]; }
  const T& operator()(UInt i, UInt j = 0) const { return v_[i * cols_ + j]; }
  UInt size() const { return rows_; }
  UInt getNbComponent() const { return cols_; }
  T* storage() { return v_.data(); }
  const T* storage() const { return v_.data(); }
  void set(T value) { std::fill(v_.begin(), v_.end(), value); }
  void resize(UInt rows, UInt cols) {
    rows_ = rows;
    cols_ = cols;
    v_.resize(rows * cols);
  }

 private:
  UInt rows_ = 0, cols_ = 0;
  std::vector<T> v_;
};

// A named group of nodes and of the mesh's elements (GroupManager,
// group_manager.hh:63), as Mesh::read builds them from physical names.
struct NodeGroup {
  std::string name;
  std::vector<uint32_t> nodes;
  std::vector<uint32_t> elements;
  // the group's facets (its elements of one dimension less, on which
  // Neumann conditions act): nodes_per_facet node indices each (-1: facets
  // of two kinds, not kept)
  int32_t nodes_per_facet = 0;
  std::vector<uint32_t> facets;
  UInt size() const { return (UInt)nodes.size(); }
  std::vector<uint32_t>::const_iterator begin() const { return nodes.begin(); }
  std::vector<uint32_t>::const_iterator end() const { return nodes.end(); }
};

class Mesh {
 public:
  explicit Mesh(UInt spatial_dimension) : dim_(spatial_dimension), nodes_(0, spatial_dimension) {}
  // Mesh::read (mesh.hh:133) of a Gmsh ASCII 2.x file (include/akb_mesh.h):
  // elements of the spatial dimension, nodes, and one group per physical name.
  void read(const std::string& filename) {
    akb_msh* m = nullptr;
    check(akb_msh_read(filename.c_str(), (int32_t)dim_, &m));
    akb_mesh_desc d;
    akb_status st = akb_msh_get_mesh(m, &d);
    int32_t ng = 0;
    if (st == AKB_OK) st = akb_msh_get_nb_groups(m, &ng);
    if (st != AKB_OK) {
      akb_msh_destroy(m);
      check(st);
    }
    setElementType((ElementType)d.element_type);
    nodes_.resize((UInt)d.nb_nodes, dim_);
    std::copy(d.nodes, d.nodes + d.nb_nodes * dim_, nodes_.storage());
    const UInt n = conn_.getNbComponent();
    conn_.resize((UInt)d.nb_elements, n);
    std::copy(d.connectivity, d.connectivity + d.nb_elements * n, conn_.storage());
    groups_.clear();
    for (int32_t k = 0; k < ng; ++k) {
      const char* name;
      int64_t nn, ne;
      const uint32_t *pn, *pe;
      check(akb_msh_get_group(m, k, &name, &nn, &pn, &ne, &pe));
      NodeGroup g{name, std::vector<uint32_t>(pn, pn + nn), std::vector<uint32_t>(pe, pe + ne), 0,
                  {}};
      int64_t nf;
      const uint32_t* pf;
      const akb_status fs = akb_msh_get_group_facets(m, k, &nf, &g.nodes_per_facet, &pf);
      if (fs == AKB_ERR_UNSUPPORTED) {
        g.nodes_per_facet = -1;  // facets of two kinds: no Neumann condition on it
      } else {
        check(fs);
        g.facets.assign(pf, pf + nf * g.nodes_per_facet);
      }
      groups_[g.name] = std::move(g);
    }
    akb_msh_destroy(m);
  }
  const NodeGroup& getNodeGroup(const std::string& name) const {
    auto it = groups_.find(name);
    if (it == groups_.end()) throw Exception(AKB_ERR_INVALID_ARGUMENT, "no group " + name);
    return it->second;
  }
  const NodeGroup& getElementGroup(const std::string& name) const { return getNodeGroup(name); }
  const std::map<std::string, NodeGroup>& iterateNodeGroups() const { return groups_; }
  Array<Real>& getNodes() { return nodes_; }
  const Array<Real>& getNodes() const { return nodes_; }
  Array<uint32_t>& getConnectivity() { return conn_; }
  const Array<uint32_t>& getConnectivity() const { return conn_; }
  UInt getSpatialDimension() const { return dim_; }
  UInt getNbNodes() const { return nodes_.size(); }
  UInt getNbElement() const { return conn_.size(); }
  ElementType getElementType() const { return type_; }
  void setElementType(ElementType t) {
    type_ = t;
    conn_.resize(conn_.size(), t == _segment_2 ? 2 : t == _triangle_3 ? 3 : t == _tetrahedron_4 ? 4 : 8);
  }

 private:
  UInt dim_;
  ElementType type_ = _triangle_3;
  Array<Real> nodes_;
  Array<uint32_t> conn_;
  std::map<std::string, NodeGroup> groups_;
};

// material elastic [ rho, E, nu, Plane_Stress, finite_deformation ]
struct MaterialElastic {
  MaterialElastic(Real rho, Real E, Real nu, bool plane_stress = false, bool finite = false)
      : desc{AKB_MATERIAL_ELASTIC, plane_stress, finite, 0, rho, E, nu} {}
  akb_material_desc desc;
};
// material neohookean [ rho, E, nu ]
struct MaterialNeohookean {
  MaterialNeohookean(Real rho, Real E, Real nu) : desc{AKB_MATERIAL_NEOHOOKEAN, 0, 1, 0, rho, E, nu} {}
  akb_material_desc desc;
};

// A material written outside the library: the Material::computeStress plugin
// (material.hh:110). computeStress(grad_u, stress, nb_points, stream) gets
// the model's device arrays of Gauss-point displacement gradients and
// stresses (3 x 3 column-major per point, like the reference's Matrix) and
// the CUDA stream the model runs on; it writes the Cauchy stress (small
// strain) or the first Piola-Kirchhoff stress (finite). rho, E, nu give the
// density and the wave speed of getStableTimeStep. All materials of a model
// using it must be user materials.
struct MaterialUser {
  using Compute = std::function<void(const double* grad_u, double* stress, int64_t nb_points,
                                     void* stream)>;
  MaterialUser(Real rho, Real E, Real nu, Compute compute, bool finite = true)
      : desc{AKB_MATERIAL_USER, 0, finite, 0, rho, E, nu}, computeStress(std::move(compute)) {}
  akb_material_desc desc;
  Compute computeStress;
};

namespace BC {
namespace Dirichlet {
// FixedValue (boundary_condition_functor.hh): blocks one component and sets it.
struct FixedValue {
  FixedValue(Real value, SpatialDirection axis) : value(value), axis(axis) {}
  Real value;
  SpatialDirection axis;
};
}  // namespace Dirichlet
namespace Neumann {
// FromTraction (FromSameDim, boundary_condition_functor.hh): a traction
// vector (d values) on the group's facets.
struct FromTraction {
  explicit FromTraction(const std::vector<Real>& traction) : value(traction) {}
  static constexpr int32_t kind = AKB_NEUMANN_TRACTION;
  std::vector<Real> value;
};
// FromStress (FromHigherDim): a stress (d x d, column-major like Matrix<Real>),
// the traction sigma n with n each facet's unit normal from its node order.
struct FromStress {
  explicit FromStress(const std::vector<Real>& stress_column_major) : value(stress_column_major) {}
  static constexpr int32_t kind = AKB_NEUMANN_STRESS;
  std::vector<Real> value;
};
}  // namespace Neumann
}  // namespace BC

// The nodal forces of a Neumann functor on a group's facets
// (boundary_condition_tmpl.hh:95-185), added into forces (N x d).
template <class F>
void addNeumannForces(const Mesh& mesh, const std::string& group, const F& f, Array<Real>& forces) {
  const NodeGroup& g = mesh.getNodeGroup(group);
  if (g.nodes_per_facet < 0)
    throw Exception(AKB_ERR_UNSUPPORTED, "group " + group + " has facets of two kinds");
  const UInt d = mesh.getSpatialDimension();
  if (f.value.size() != (F::kind == AKB_NEUMANN_TRACTION ? d : d * d))
    throw Exception(AKB_ERR_INVALID_ARGUMENT, "Neumann value of the wrong size");
  const int64_t nf = g.nodes_per_facet ? (int64_t)(g.facets.size() / g.nodes_per_facet) : 0;
  check(akb_neumann_forces((int32_t)d, (int64_t)mesh.getNbNodes(), mesh.getNodes().storage(), nf,
                           g.nodes_per_facet, g.facets.data(), F::kind, f.value.data(),
                           forces.storage()));
}

class SolidMechanicsModel {
 public:
  explicit SolidMechanicsModel(Mesh& mesh, int precision = AKB_MODE_FP64, int device = 0)
      : mesh_(mesh), precision_(precision), device_(device) {}
  ~SolidMechanicsModel() {
    if (h_) akb_model_destroy(h_);
  }
  SolidMechanicsModel(const SolidMechanicsModel&) = delete;
  SolidMechanicsModel& operator=(const SolidMechanicsModel&) = delete;

  template <class M>
  void addMaterial(const M& m) {
    mats_.push_back(m.desc);
  }
  void addMaterial(const MaterialUser& m) {
    mats_.push_back(m.desc);
    user_ = m.computeStress;
  }
  void setMaterialIndex(const std::vector<uint32_t>& per_element) { element_material_ = per_element; }

  void initFull(AnalysisMethodArg arg = {_explicit_lumped_mass}) {
    if (arg.value != _explicit_lumped_mass) throw Exception(AKB_ERR_UNSUPPORTED, "explicit only");
    akb_mesh_desc md{(int32_t)mesh_.getSpatialDimension(), (int32_t)mesh_.getElementType(),
                     (int64_t)mesh_.getNbNodes(), (int64_t)mesh_.getNbElement(),
                     mesh_.getNodes().storage(), mesh_.getConnectivity().storage()};
    akb_model_options opt{precision_, device_, nullptr, 0, 0, 0};  // default patches
    check(akb_model_create(&md, (int32_t)mats_.size(), mats_.data(),
                           element_material_.empty() ? nullptr : element_material_.data(), &opt,
                           &h_));
    const UInt n = mesh_.getNbNodes(), d = mesh_.getSpatialDimension();
    for (auto* a : {&u_, &v_, &acc_, &fext_, &fint_, &mass_}) a->resize(n, d);
    blocked_.resize(n, d);
  }

  Real getStableTimeStep() {
    sync_in();
    Real dt;
    check(akb_get_stable_time_step(h_, &dt));
    return dt;
  }
  void setTimeStep(Real dt) { check(akb_set_time_step(h_, dt)); }
  Real getTimeStep() const {
    Real dt;
    check(akb_get_time_step(h_, &dt));
    return dt;
  }
  void solveStep() {
    sync_in();
    if (user_) return userStep();
    check(akb_solve_step(h_));
  }
  void solveSteps(int64_t n) {
    sync_in();
    if (user_) {
      for (int64_t s = 0; s < n; ++s) userStep();
      return;
    }
    check(akb_solve_steps(h_, n));
  }
  void assembleMassLumped() { check(akb_assemble_mass_lumped(h_)); }
  void assembleInternalForces() {
    sync_in();
    check(akb_assemble_internal_forces(h_));
  }

  Array<Real>& getDisplacement() { return pull(AKB_FIELD_DISPLACEMENT, u_, true); }
  Array<Real>& getVelocity() { return pull(AKB_FIELD_VELOCITY, v_, true); }
  Array<Real>& getAcceleration() { return pull(AKB_FIELD_ACCELERATION, acc_, true); }
  Array<Real>& getExternalForce() { return pull(AKB_FIELD_EXTERNAL_FORCE, fext_, true); }
  const Array<Real>& getInternalForce() { return pull(AKB_FIELD_INTERNAL_FORCE, fint_, false); }
  const Array<Real>& getMass() { return pull(AKB_FIELD_MASS, mass_, false); }
  Array<uint8_t>& getBlockedDOFs() {
    sync_in();
    check(akb_get_blocked_dofs(h_, blocked_.storage(), (int64_t)blocked_.size() * blocked_.getNbComponent()));
    blocked_out_ = true;
    return blocked_;
  }

  // applyBC(FixedValue, group) (boundary_condition_tmpl.hh:186-200): by the
  // group's name, or by its node list
  void applyBC(const BC::Dirichlet::FixedValue& f, const std::vector<uint32_t>& nodes) {
    sync_in();
    std::vector<Real> vals(nodes.size(), f.value);
    check(akb_apply_dirichlet(h_, nodes.data(), (int64_t)nodes.size(), f.axis, vals.data()));
  }
  void applyBC(const BC::Dirichlet::FixedValue& f, const std::string& group) {
    applyBC(f, mesh_.getNodeGroup(group).nodes);
  }
  // applyBC(FromTraction / FromStress, group): the nodal forces added to the
  // external force (pushed before the next call that uses the state)
  void applyBC(const BC::Neumann::FromTraction& f, const std::string& group) {
    addNeumannForces(mesh_, group, f, getExternalForce());
  }
  void applyBC(const BC::Neumann::FromStress& f, const std::string& group) {
    addNeumannForces(mesh_, group, f, getExternalForce());
  }

  Real getEnergy(const std::string& id) {
    sync_in();
    int32_t kind = id == "kinetic" ? AKB_ENERGY_KINETIC
                 : id == "potential" ? AKB_ENERGY_POTENTIAL
                 : id == "external work" ? AKB_ENERGY_EXTERNAL_WORK : -1;
    if (kind < 0) throw Exception(AKB_ERR_INVALID_ARGUMENT, "unknown energy " + id);
    Real e;
    check(akb_get_energy(h_, kind, &e));
    return e;
  }

  akb_model* handle() { return h_; }

 private:
  // predictor + grad u, the user's computeStress, then forces and corrector
  void userStep() {
    check(akb_step_begin(h_));
    void *gradu, *stress, *stream;
    check(akb_field_device_pointer(h_, AKB_FIELD_GRAD_U, &gradu));
    check(akb_field_device_pointer(h_, AKB_FIELD_STRESS, &stress));
    check(akb_model_get_stream(h_, &stream));
    akb_model_info info;
    check(akb_model_get_info(h_, &info));
    user_(static_cast<const double*>(gradu), static_cast<double*>(stress),
          info.nb_elements * info.quadrature_points_per_element, stream);
    check(akb_step_end(h_));
  }

  Array<Real>& pull(int32_t field, Array<Real>& a, bool writable) {
    sync_in();
    check(akb_get_field(h_, field, a.storage(), (int64_t)a.size() * a.getNbComponent()));
    if (writable) out_.push_back({field, &a});
    return a;
  }
  void sync_in() {
    for (auto& o : out_)
      check(akb_set_field(h_, o.first, o.second->storage(),
                          (int64_t)o.second->size() * o.second->getNbComponent()));
    out_.clear();
    if (blocked_out_) {
      check(akb_set_blocked_dofs(h_, blocked_.storage(),
                                 (int64_t)blocked_.size() * blocked_.getNbComponent()));
      blocked_out_ = false;
    }
  }

  Mesh& mesh_;
  int precision_, device_;
  akb_model* h_ = nullptr;
  std::vector<akb_material_desc> mats_;
  std::vector<uint32_t> element_material_;
  Array<Real> u_, v_, acc_, fext_, fint_, mass_;
  Array<uint8_t> blocked_;
  bool blocked_out_ = false;
  std::vector<std::pair<int32_t, Array<Real>*>> out_;
  MaterialUser::Compute user_;
};

}  // namespace akantu_b200
