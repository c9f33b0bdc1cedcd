"""Known-answer cases of the reference test suite, restated as drivers that
run either the CPU oracle or the CUDA library through the same calls.

Each driver takes a model factory and returns what the reference test
checks, so one case serves the oracle test (CPU) and the parity test (GPU).
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

from akantu_b200 import _abi
from akantu_b200.mesh import Mesh, bar_segment2

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_json(name):
    with open(os.path.join(GOLDEN, name)) as fh:
        return json.load(fh)


# ---------------------------------------------------------------------------
# test_model_solver_dynamic.cc (EXPLICIT=true) with test_model_solver_my_model.hh
# ---------------------------------------------------------------------------
MODEL_SOLVER = dict(nb_nodes=201, max_steps=400, time_step=0.001, F=-9.81,
                    pulse_width=0.2, A=0.01, E=1.0, rho=1.0)


def model_solver_dynamic_explicit(make_model):
    """Runs the 1D bar of test_model_solver_dynamic.cc:76-205 and returns the
    printed table as floats (401 rows x 7 columns).

    The bar uses segment_2 linear elasticity with E = A = rho = 1, which is
    the model MyModel writes by hand (test_model_solver_my_model.hh:55-430):
    lumped mass rho*A*L/2 per node, f = E*A*(u2-u1)/L. The reference's
    MyModel stores the internal force with the opposite sign of
    SolidMechanicsModel and computes its work increment as
    dt * sum(blocked ? -f_int_mymodel : f_ext) * v
    (test_model_solver_my_model.hh:370-389); it is reproduced here from the
    model fields.

    make_model(mesh, material) must return an object with the fields and
    calls of tests.golden_cases.ModelAdapter."""
    p = MODEL_SOLVER
    mesh = bar_segment2(p["nb_nodes"], 1.0)
    model = make_model(mesh, dict(kind=_abi.MATERIAL_ELASTIC, rho=p["rho"], E=p["E"], nu=0.0))
    x = mesh.nodes[:, 0]
    k = 2 * math.pi / p["pulse_width"]
    v = math.sqrt(p["E"] / p["rho"])
    A = p["A"]

    def sinusoidal(nodes, t):
        # Sinusoidal::operator() (test_model_solver_dynamic.cc:56-63)
        vel = model.get(_abi.FIELD_VELOCITY)
        disp = model.get(_abi.FIELD_DISPLACEMENT)
        for n in nodes:
            xx = x[n]
            vel[n, 0] = k * v * A * math.sin(k * (xx - v * t))
            disp[n, 0] = A * math.cos(k * (xx - v * t))
        model.set(_abi.FIELD_VELOCITY, vel)
        model.set(_abi.FIELD_DISPLACEMENT, disp)

    fext = np.zeros((p["nb_nodes"], 1))
    fext[-1, 0] = p["F"]
    model.set(_abi.FIELD_EXTERNAL_FORCE, fext)
    blocked = np.zeros((p["nb_nodes"], 1), dtype=np.uint8)
    blocked[0, 0] = 1
    model.set_blocked(blocked)
    border = [0, p["nb_nodes"] - 1]
    sinusoidal(range(p["nb_nodes"]), 0.0)       # applyBC(..., "all")
    blocked[border, 0] = 1                       # FlagOnly(_x) on "border"
    model.set_blocked(blocked)
    model.set_time_step(p["time_step"])
    model.assemble_internal_forces()

    rows = []
    u = model.get(_abi.FIELD_DISPLACEMENT)
    rows.append([0.0, 0.0, 0.0, 0.0, 0.0, max(0.0, u.max()), min(0.0, u.min())])
    wext = 0.0
    einit = 0.0
    for i in range(1, p["max_steps"] + 1):
        sinusoidal(border, p["time_step"] * (i - 1))
        model.solve_step()
        epot = model.energy(_abi.ENERGY_POTENTIAL)
        ekin = model.energy(_abi.ENERGY_KINETIC)
        vel = model.get(_abi.FIELD_VELOCITY)[:, 0]
        fint = model.get(_abi.FIELD_INTERNAL_FORCE)[:, 0]
        bl = model.get_blocked()[:, 0].astype(bool)
        # MyModel's internal force is -f_int of SolidMechanicsModel
        incr = np.where(bl, fint, fext[:, 0]) * vel
        wext += float(np.sum(incr)) * p["time_step"]
        etot = ekin + epot - wext - einit
        u = model.get(_abi.FIELD_DISPLACEMENT)
        rows.append([p["time_step"] * i, wext, epot, ekin, etot,
                     max(0.0, u.max()), min(0.0, u.min())])
    return np.array(rows)


def golden_model_solver_table():
    data = load_json("model_solver_dynamic_explicit.json")
    return data["header"], np.array([[float(s) for s in r] for r in data["rows"]])


def compare_model_solver_table(table):
    """Max error per column, relative to the column's largest magnitude,
    after rounding our values to the 7 significant digits the golden file
    prints. Returns (errors, golden)."""
    header, golden = golden_model_solver_table()
    ours = np.array([[float("%e" % v) for v in row] for row in table])
    scale = np.maximum(np.abs(golden).max(axis=0), 1e-300)
    err = (np.abs(ours - golden) / scale).max(axis=0)
    return dict(zip(header, err)), golden


# ---------------------------------------------------------------------------
# patch tests (patch_test_linear_elastic_explicit.cc:33-68 and fixtures)
# ---------------------------------------------------------------------------
PATCH_ALPHA = np.array([[0.01, 0.02, 0.03, 0.04],
                        [0.05, 0.06, 0.07, 0.08],
                        [0.09, 0.10, 0.11, 0.12]])   # patch_test_linear_fixture.hh:167-169
PATCH_TOL = dict(gradient=1e-13, result=1e-13, dofs=1e-15)  # :171-173


def patch_mesh(name):
    d = load_json("patch_meshes.json")["meshes"][name]
    mesh = Mesh(d["spatial_dimension"], d["element_type"], np.array(d["nodes"]),
                np.array(d["connectivity"], dtype=np.uint32))
    mesh.createBoundaryGroupFromGeometry()
    return mesh


def patch_material(which="plane_strain"):
    m = load_json("patch_meshes.json")["materials"][which]
    return dict(kind=_abi.MATERIAL_ELASTIC, rho=m["rho"], E=m["E"], nu=m["nu"],
                plane_stress=bool(m.get("Plane_Stress", False)),
                finite_deformation=bool(m.get("finite_deformation", False)))


def linear_dof(coords, dim):
    """setLinearDOF (patch_test_linear_fixture.hh:125-133)."""
    a = PATCH_ALPHA
    out = np.empty((coords.shape[0], dim))
    for i in range(dim):
        out[:, i] = a[i, 0]
        for j in range(dim):
            out[:, i] += a[i, j + 1] * coords[:, j]
    return out


def facet_area_vectors(mesh, nodes):
    """Outward area vectors of the boundary facets, for the equivalent nodal
    force of a uniform stress (BC::Neumann::FromHigherDim on linear facets)."""
    from akantu_b200.mesh import _FACETS
    counts = {}
    for e, elem in enumerate(mesh.connectivity):
        for f in _FACETS[mesh.element_type]:
            key = tuple(sorted(int(elem[k]) for k in f))
            counts.setdefault(key, []).append((e, tuple(int(elem[k]) for k in f)))
    out = []
    for key, lst in counts.items():
        if len(lst) != 1:
            continue
        e, f = lst[0]
        P = nodes[list(f)]
        centroid = nodes[mesh.connectivity[e].astype(int)].mean(axis=0)
        if mesh.spatial_dimension == 2:
            t = P[1] - P[0]
            nvec = np.array([t[1], -t[0]])
        else:
            if len(f) == 3:
                nvec = 0.5 * np.cross(P[1] - P[0], P[2] - P[0])
            else:
                nvec = 0.5 * np.cross(P[2] - P[0], P[3] - P[1])
        if np.dot(nvec, P.mean(axis=0) - centroid) < 0:
            nvec = -nvec
        out.append((f, nvec))
    return out


def patch_test_explicit(make_model, name):
    """Runs patch_test_linear_elastic_explicit.cc:33-68 and returns the
    quantities the test checks (see check_patch_results)."""
    mesh = patch_mesh(name)
    dim = mesh.spatial_dimension
    model = make_model(mesh, patch_material("plane_strain"))
    boundary = mesh.getNodeGroup("boundary")
    blocked = np.zeros((mesh.getNbNodes(), dim), dtype=np.uint8)
    blocked[boundary, :] = 1
    model.set_blocked(blocked)
    disp = np.zeros((mesh.getNbNodes(), dim))
    disp[boundary] = linear_dof(mesh.nodes[boundary], dim)
    model.set(_abi.FIELD_DISPLACEMENT, disp)
    dt = model.stable_time_step()
    model.set_time_step(0.8 * dt)
    model.set(_abi.FIELD_DISPLACEMENT, linear_dof(mesh.nodes, dim))
    for _ in range(100):
        model.solve_step()
    out = dict(mesh=mesh, dim=dim, dt=dt)
    out["ekin"] = model.energy(_abi.ENERGY_KINETIC)
    out["epot"] = model.energy(_abi.ENERGY_POTENTIAL)
    out["u"] = model.get(_abi.FIELD_DISPLACEMENT)
    model.compute_stresses()
    out["gradu"] = model.get(_abi.FIELD_GRAD_U)
    out["stress"] = model.get(_abi.FIELD_STRESS)
    out["fint"] = model.get(_abi.FIELD_INTERNAL_FORCE)
    return out


def check_patch_results(r, material=None):
    """The assertions of patch_test_linear_solid_mechanics_fixture.hh:48-130
    and patch_test_linear_fixture.hh:95-160. Returns a dict of errors and
    the tolerance each must meet."""
    mat = material or patch_material("plane_strain")
    dim, mesh = r["dim"], r["mesh"]
    errs = {}
    errs["ekin"] = (abs(r["ekin"]), 1e-16)
    ref = linear_dof(mesh.nodes, dim)
    errs["dofs"] = (np.abs(r["u"] - ref).max(), PATCH_TOL["dofs"])
    pgrad = PATCH_ALPHA[:dim, 1:dim + 1]
    g = r["gradu"].reshape(-1, dim, dim, order="F")  # column-major per QP
    gerr = max(np.abs(gq - pgrad).max() / np.abs(gq).max() for gq in g)
    errs["gradient"] = (gerr, PATCH_TOL["gradient"])
    E, nu = mat["E"], mat["nu"]
    strain = 0.5 * (pgrad + pgrad.T)
    lam = nu * E / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    sig_ref = lam * np.trace(strain) * np.eye(dim) + 2 * mu * strain
    s = r["stress"].reshape(-1, dim, dim, order="F")
    serr = max(np.abs(sq - sig_ref).max() / np.abs(sig_ref).max() for sq in s)
    errs["stress"] = (serr, PATCH_TOL["result"])
    fint = r["fint"]
    fnorm = np.abs(fint).max()
    errs["total_force"] = (np.abs(fint.sum(axis=0)).max() / fnorm, 1e-9)
    fext = np.zeros_like(fint)
    for f, nvec in facet_area_vectors(mesh, mesh.nodes):
        t = sig_ref @ nvec
        for node in f:
            fext[node] += t / len(f)
    errs["equilibrium"] = (np.abs(fint + fext).max() / fnorm, 1e-9)
    return errs


def lumped_mass_case(make_model, name):
    """test_lumped_mass.cc:81-101: sum of lumped masses = integral of rho."""
    mesh = patch_mesh(name)
    mat = patch_material("lumped")
    model = make_model(mesh, mat)
    model.assemble_mass_lumped()
    masses = model.get(_abi.FIELD_MASS)
    vol = element_volumes(mesh).sum()
    return masses.sum(axis=0), mat["rho"] * vol


def element_volumes(mesh):
    X = mesh.nodes[mesh.connectivity.astype(np.int64)]
    if mesh.element_type == _abi.TRIANGLE_3:
        a, b = X[:, 1] - X[:, 0], X[:, 2] - X[:, 0]
        return 0.5 * np.abs(a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0])
    if mesh.element_type == _abi.TETRAHEDRON_4:
        a, b, c = X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]
        return np.abs(np.einsum("ei,ei->e", a, np.cross(b, c))) / 6.0
    if mesh.element_type == _abi.HEXAHEDRON_8:
        # split into 6 tets along 0-6
        tets = [(0, 1, 2, 6), (0, 2, 3, 6), (0, 3, 7, 6), (0, 7, 4, 6), (0, 4, 5, 6), (0, 5, 1, 6)]
        v = 0
        for t in tets:
            a, b, c = X[:, t[1]] - X[:, t[0]], X[:, t[2]] - X[:, t[0]], X[:, t[3]] - X[:, t[0]]
            v = v + np.abs(np.einsum("ei,ei->e", a, np.cross(b, c))) / 6.0
        return v
    return np.abs(X[:, 1, 0] - X[:, 0, 0])


class OracleAdapter:
    """Uniform get/set facade over oracle.OracleModel."""

    def __init__(self, mesh, material, fast=False):
        from oracle.oracle import OracleModel, material_desc
        mats = material if isinstance(material, list) else [material]
        self.m = OracleModel(mesh, [material_desc(**mm) for mm in mats], fast=fast)

    def get(self, field):
        return np.array(self.m.field(field))

    def set(self, field, values):
        self.m.field(field)[...] = values

    def get_blocked(self):
        return np.array(self.m.blocked)

    def set_blocked(self, b):
        self.m.blocked[...] = b

    def stable_time_step(self):
        return self.m.stable_time_step()

    def set_time_step(self, dt):
        self.m.set_time_step(dt)

    def solve_step(self):
        self.m.solve_step()

    def solve_steps(self, n):
        self.m.solve_steps(n)

    def assemble_internal_forces(self):
        self.m.assemble_internal_forces()

    def assemble_mass_lumped(self):
        self.m.assemble_mass_lumped()

    def compute_stresses(self):
        self.m.compute_stresses()

    def energy(self, kind):
        return self.m.energy(kind)

    def apply_dirichlet(self, nodes, comp, values):
        self.m.blocked[nodes, comp] = 1
        self.m.displacement[nodes, comp] = values


class GpuAdapter:
    """The same facade over akantu_b200.SolidMechanicsModel (libakb.so)."""

    def __init__(self, mesh, material, precision=_abi.MODE_FP64_REFERENCE,
                 element_material=None):
        from akantu_b200.model import SolidMechanicsModel, material_from_dict
        mats = material if isinstance(material, list) else [material]
        self.m = SolidMechanicsModel(mesh, [material_from_dict(mm) for mm in mats],
                                     element_material=element_material, precision=precision)
        self.m.initFull()

    def get(self, field):
        return np.array(self.m.getField(field))

    def set(self, field, values):
        self.m.setField(field, values)

    def get_blocked(self):
        return np.array(self.m.getBlockedDOFs(), dtype=np.uint8)

    def set_blocked(self, b):
        self.m.setBlockedDOFs(b)

    def stable_time_step(self):
        return self.m.getStableTimeStep()

    def set_time_step(self, dt):
        self.m.setTimeStep(dt)

    def solve_step(self):
        self.m.solveStep()

    def solve_steps(self, n):
        self.m.solveSteps(n)

    def assemble_internal_forces(self):
        self.m.assembleInternalForces()

    def assemble_mass_lumped(self):
        self.m.assembleMassLumped()

    def compute_stresses(self):
        self.m.computeStresses()

    def energy(self, kind):
        name = {_abi.ENERGY_KINETIC: "kinetic", _abi.ENERGY_POTENTIAL: "potential",
                _abi.ENERGY_EXTERNAL_WORK: "external work"}[kind]
        return self.m.getEnergy(name)

    def apply_dirichlet(self, nodes, comp, values):
        self.m.applyDirichlet(nodes, comp, values)
