"""Ports of the reference's own tests of the explicit path, written once
against the model facade of tests/golden_cases.py so that the CPU oracle and
every GPU mode run the same scenario (test infrastructure).

  finite_deformation_invariance  test_finite_deformation.cc:10-110
  elastic_law                    test_elastic_materials.cc:56-290
  plane_wave                     test_solid_mechanics_model_dynamics.cc:39-297
  work_balance                   test_energies/test_solid_mechanics_model_work_dynamics.cc:50-156
  python_fe_truss                test/python_fe (TrussFE, DynamicSolver): trajectories of
                                 the reference's own Python restatement, as the explicit
                                 lumped scheme (tests/golden/make_python_fe.py)

The bar meshes of the last two (patch_tests/data/bar_*.geo: 10 x 1 x 1, mesh
size 0.6, meshed by Gmsh, which is absent) are generated here as structured
bars of the same extent and element size: 17 x 2 x 2 cells, group "BC" = the
boundary nodes.
"""
import json
import math
import os

import numpy as np

from akantu_b200 import _abi
from akantu_b200.mesh import (Mesh, bar_segment2, box_hexahedron8, box_tetrahedron4,
                              plate_triangle3)

HERE = os.path.dirname(os.path.abspath(__file__))
REF_MATS = json.load(open(os.path.join(HERE, "golden", "reference_materials.json")))


def _mat(name, **extra):
    m = REF_MATS[name]
    d = dict(kind=_abi.MATERIAL_ELASTIC, rho=m["rho"], E=m["E"], nu=m["nu"],
             finite_deformation=bool(m.get("finite_deformation", False)))
    d.update(extra)
    return d


# --------------------------------------------------------------------------
def finite_deformation_invariance(make):
    """One tetrahedron (1_tetrahedron.msh), elastic with finite deformation
    (material_finite_deformation.dat), every DOF blocked. u = alpha X
    (alpha columns 1..3 of the test's matrix), internal force f0; then the
    rotated configuration u' = R (X + u) - X (rotation pi/4 about x) must
    give f = R f0. Returns per-node |f - R f0| and |f0|."""
    mesh = Mesh(3)
    mesh.read(os.path.join(HERE, "golden", "msh", "1_tetrahedron.msh"))
    model = make(mesh, _mat("finite_deformation"))
    X = mesh.nodes
    alpha = np.array([[0.00, 0.02, 0.03, 0.04],
                      [0.00, 0.06, 0.07, 0.08],
                      [0.00, 0.10, 0.11, 0.12]])
    u0 = alpha[:, 0] + X @ alpha[:, 1:].T
    model.set_blocked(np.ones_like(X, dtype=np.uint8))
    model.set(_abi.FIELD_DISPLACEMENT, u0)
    model.assemble_internal_forces()
    f0 = model.get(_abi.FIELD_INTERNAL_FORCE)
    th = math.pi / 4
    R = np.array([[1.0, 0.0, 0.0], [0.0, math.cos(th), -math.sin(th)],
                  [0.0, math.sin(th), math.cos(th)]])
    u1 = (X + u0) @ R.T - X
    model.set(_abi.FIELD_DISPLACEMENT, u1)
    model.assemble_internal_forces()
    f1 = model.get(_abi.FIELD_INTERNAL_FORCE)
    return np.linalg.norm(f1 - f0 @ R.T, axis=1), np.linalg.norm(f0, axis=1)


# --------------------------------------------------------------------------
# the materials of the elastic-law tests (FriendMaterial<...>::setParams)
ELASTIC_PARAMS = {1: dict(E=3.0, nu=0.0, rho=2.0), 2: dict(E=1.0, nu=0.3, rho=2.0),
                  3: dict(E=1.0, nu=0.3, rho=2.0)}


def _one_element(dim):
    if dim == 1:
        return bar_segment2(2, 1.0)
    if dim == 2:
        return Mesh(2, _abi.TRIANGLE_3, [[0, 0], [1, 0], [0, 1]], [[0, 1, 2]])
    return Mesh(3, _abi.TETRAHEDRON_4, [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], [[0, 1, 2, 3]])


def composed_strain(dim):
    """getComposedStrain(1): hydrostatic + deviatoric (test_material_fixtures.hh:94-116),
    its upper-left dim x dim block; in 1D the test's eps = 2."""
    s = np.eye(3) + np.array([[0.0, 1.0, 2.0], [1.0, 0.0, 3.0], [2.0, 3.0, 0.0]])
    return np.array([[2.0]]) if dim == 1 else s[:dim, :dim]


def random_rotation(dim, seed=1):
    """A rotation built like getRandomRotation (test_material_fixtures.hh:131-):
    a random unit first axis completed to an orthonormal frame."""
    rng = np.random.default_rng(seed)
    v1 = rng.uniform(size=dim)
    v1 /= np.linalg.norm(v1)
    if dim == 1:
        return np.array([[1.0]])
    if dim == 2:
        return np.array([[v1[0], v1[1]], [-v1[1], v1[0]]])
    v2 = np.cross([0.0, 0.0, 1.0], v1)
    v2 /= np.linalg.norm(v2)
    return np.stack([v1, v2, np.cross(v1, v2)])


def elastic_law(make, dim, plane_stress=False):
    """ComputeStress, EnergyDensity and Celerity of MaterialElastic<dim>
    through a one-element model: u = G X imposes grad u = G exactly.
      stress: G rotated by R (applyRotation R G R^T), the model's stress
        rotated back (reverseRotation R^T s R) against
        2 mu dev(eps) + K tr(eps) I (plane strain, 3D; the test's form),
        lambda* tr(eps) I + 2 mu eps with lambda* = E nu / (1 - nu^2)
        (plane stress, the tangent of testComputeTangentModuli), E eps (1D;
        the reference test adds a thermal stress, which is zero on this path);
      energy: potential energy of eps = sym(G) over the element volume
        against 1/2 sigma : eps V;
      celerity: the stable time step h / c with c = sqrt((K + 4/3 mu) / rho)
        (plane strain, 3D), sqrt((lambda* + 2 mu) / rho) (plane stress:
        getPushWaveSpeed, material_elastic.cc:164-167, with the plane-stress
        lambda of :95-107) or sqrt(E / rho) (1D) and h the element's
        characteristic length (segment: length; triangle, tetrahedron: 2 r_in).
    Returns (stress error, energy error, time step error), relative."""
    p = ELASTIC_PARAMS[dim]
    E, nu, rho = p["E"], p["nu"], p["rho"]
    mesh = _one_element(dim)
    model = make(mesh, dict(kind=_abi.MATERIAL_ELASTIC, rho=rho, E=E, nu=nu,
                            plane_stress=plane_stress))
    X = mesh.nodes
    G = composed_strain(dim)
    R = random_rotation(dim)
    Grot = R @ G @ R.T
    model.set(_abi.FIELD_DISPLACEMENT, X @ Grot.T)
    model.compute_stresses()
    s_rot = model.get(_abi.FIELD_STRESS).reshape(dim, dim).T  # column-major per point
    sigma = R.T @ s_rot @ R
    eps = 0.5 * (G + G.T)
    I = np.eye(dim)
    mu = E / (2 * (1 + nu))
    K = E / (3 * (1 - 2 * nu))
    if dim == 1:
        expected = E * eps
    elif plane_stress:
        expected = E * nu / ((1 + nu) * (1 - nu)) * np.trace(eps) * I + 2 * mu * eps
    else:
        expected = 2 * mu * (eps - np.trace(eps) / 3 * I) + K * np.trace(eps) * I
    err_s = np.abs(sigma - expected).max() / np.abs(expected).max()
    # energy density of eps
    model.set(_abi.FIELD_DISPLACEMENT, X @ eps.T)
    vol = {1: 1.0, 2: 0.5, 3: 1.0 / 6.0}[dim]
    epot = model.energy(_abi.ENERGY_POTENTIAL)
    ref_e = 0.5 * np.sum(expected * eps) * vol
    err_e = abs(epot - ref_e) / abs(ref_e)
    # celerity through the stable time step, at zero displacement
    model.set(_abi.FIELD_DISPLACEMENT, np.zeros_like(X))
    if dim == 1:
        c = math.sqrt(E / rho)
    elif plane_stress:  # getPushWaveSpeed with the plane-stress lambda
        c = math.sqrt((E * nu / ((1 + nu) * (1 - nu)) + 2 * mu) / rho)
    else:
        c = math.sqrt((K + 4.0 / 3.0 * mu) / rho)
    h = {1: 1.0, 2: 2.0 - math.sqrt(2.0), 3: 1.0 / (1.5 + math.sqrt(3.0) / 2)}[dim]
    err_dt = abs(model.stable_time_step() - h / c) / (h / c)
    return err_s, err_e, err_dt


# --------------------------------------------------------------------------
BAR_TYPES = (_abi.SEGMENT_2, _abi.TRIANGLE_3, _abi.TETRAHEDRON_4, _abi.HEXAHEDRON_8)


def bar_mesh(etype):
    """10 x 1 x 1 bar at the element size of bar_*.geo (h = 0.6): 17 cells
    along x, 2 across; node group "BC" = the boundary nodes."""
    if etype == _abi.SEGMENT_2:
        mesh = bar_segment2(18, 10.0)
    elif etype == _abi.TRIANGLE_3:
        mesh = plate_triangle3(17, 2, 10.0, 1.0)
    elif etype == _abi.TETRAHEDRON_4:
        mesh = box_tetrahedron4(17, 2, 2, 10.0, 1.0, 1.0)
    else:
        mesh = box_hexahedron8(17, 2, 2, 10.0, 1.0, 1.0)
    mesh.createNodeGroup("BC", mesh.boundary_nodes())
    return mesh


# plane wave constants (test_solid_mechanics_model_dynamics.cc:39-54)
_A, _E, _POISSON, _RHO = 1e-1, 1.0, 3.0 / 10, 1.0
_LAM = _E * _POISSON / (1 + _POISSON) / (1 - 2 * _POISSON)
_MU = _E / 2 / (1.0 + _POISSON)
_CP, _CS, _C = math.sqrt((_LAM + 2 * _MU) / _RHO), math.sqrt(_MU / _RHO), math.sqrt(_E / _RHO)
_K = np.array([0.5, 0.0, 0.0])


def plane_wave_solution(X, t, consistent=False):
    """Verification<dim>::displacement / velocity (:57-135). As written there,
    the 2D/3D velocity has cos where the derivative of the displacement has
    sin; consistent=True uses the derivative."""
    dim = X.shape[1]
    kn = np.linalg.norm(_K)
    if dim == 1:
        om = _C * _K[0]
        ph = _K[0] * X[:, 0] - om * t
        return _A * np.cos(ph)[:, None], (om * _A * np.sin(ph))[:, None]
    kpush = _K[:dim]
    if dim == 2:
        kshear = np.array([_K[1], _K[0]])
        shear = [kshear]
    else:
        shear = [np.cross(_K, [0.0, 0.0, 1.0]), np.cross(_K, [0.0, 1.0, 0.0])]
    om_p, om_s = kn * _CP, kn * _CS
    ph_p = X @ kpush - om_p * t
    ph_s = X @ kpush - om_s * t
    u = _A * (np.outer(np.cos(ph_p), kpush) + sum(np.outer(np.cos(ph_s), ks) for ks in shear))
    trig = np.sin if consistent else np.cos
    v = _A * (np.outer(om_p * trig(ph_p), kpush) +
              sum(np.outer(om_s * trig(ph_s), ks) for ks in shear))
    return u, v


def plane_wave(make, etype, consistent=False):
    """Bar of the dynamics material (E = 1, nu = 0, rho = 1), initial u and
    v of the analytic plane wave, group "BC" given the analytic x
    displacement every step (SolutionFunctor sets flags(0) only), dt =
    stable / 10, simulation time 5; the error of a step is
    sqrt(sum |u - u_exact|^2) / nb_nodes, the result its maximum over steps
    (the test requires < 2e-3).
    In 2D and 3D the test's material (nu = 0) is not the one its analytic
    solution assumes (nu = 0.3 in cp, cs) and its initial velocity is not
    the derivative of its displacement, so how far the run stays from the
    formula depends on the mesh (Gmsh's, unavailable here).
    consistent=True: material nu = 0.3, the derivative as velocity and every
    component of "BC" prescribed, so that the plane wave is the exact
    solution of the bar and only the discretisation error remains. Returns
    (max error, steps, final displacement)."""
    mesh = bar_mesh(etype)
    model = make(mesh, _mat("dynamics", nu=_POISSON) if consistent else _mat("dynamics"))
    X = mesh.nodes
    u, v = plane_wave_solution(X, 0.0, consistent)
    model.set(_abi.FIELD_DISPLACEMENT, u)
    model.set(_abi.FIELD_VELOCITY, v)
    bc = mesh.getNodeGroup("BC")
    comps = range(X.shape[1]) if consistent else (0,)
    for c in comps:
        model.apply_dirichlet(bc, c, u[bc, c])
    dt = model.stable_time_step() / 10.0
    model.set_time_step(dt)
    max_steps = int(5.0 / dt)
    t, max_err = 0.0, -1.0
    for _ in range(max_steps):
        us, _ = plane_wave_solution(X, t, consistent)
        for c in comps:
            model.apply_dirichlet(bc, c, us[bc, c])
        ud = model.get(_abi.FIELD_DISPLACEMENT)
        max_err = max(max_err, math.sqrt(np.sum((us - ud) ** 2)) / X.shape[0])
        model.solve_step()
        t += dt
    return max_err, max_steps, model.get(_abi.FIELD_DISPLACEMENT)


def _traction_forces(mesh, traction):
    """Nodal forces of a uniform x traction on the face x = max (linear
    elements: each boundary facet's measure shared equally by its nodes,
    BC::Neumann::FromTraction on el_apply_force; 1D: the end node)."""
    X = mesh.nodes
    f = np.zeros_like(X)
    xmax = X[:, 0].max()
    if mesh.spatial_dimension == 1:
        f[X[:, 0] > xmax - 1e-6, 0] = traction
        return f
    from akantu_b200.mesh import _FACETS
    seen = set()
    for elem in mesh.connectivity:
        for fc in _FACETS[mesh.element_type]:
            nodes = [int(elem[k]) for k in fc]
            if not all(X[n, 0] > xmax - 1e-6 for n in nodes):
                continue
            key = tuple(sorted(nodes))
            if key in seen:
                continue
            seen.add(key)
            P = X[nodes]
            if len(nodes) == 2:
                area = np.linalg.norm(P[1] - P[0])
            elif len(nodes) == 3:
                area = 0.5 * np.linalg.norm(np.cross(P[1] - P[0], P[2] - P[0]))
            else:
                area = 0.5 * np.linalg.norm(np.cross(P[2] - P[0], P[3] - P[1]))
            for n in nodes:
                f[n, 0] += traction * area / len(nodes)
    return f


def work_balance(make, etype):
    """Bar of the work material (E = 1, nu = 0, rho = 1), traction 0.5 on the
    face x = max, dt = stable / 10; for u_x = 0, 0.01, -0.01 on the face
    x = min: 25 steps, then 200 steps summing the external work of each step,
    W against the change of kinetic + potential energy (the test requires
    |W - dE| < 5e-2). Returns the three |W - dE|."""
    mesh = bar_mesh(etype)
    model = make(mesh, _mat("work"))
    X = mesh.nodes
    model.set(_abi.FIELD_EXTERNAL_FORCE, _traction_forces(mesh, 0.5))
    fixed = np.nonzero(X[:, 0] < X[:, 0].min() + 1e-6)[0]
    model.set_time_step(model.stable_time_step() * 0.1)
    errs = []
    for u in (0.00, 0.01, -0.01):
        model.apply_dirichlet(fixed, 0, np.full(fixed.size, u))
        model.solve_steps(25)
        e0 = model.energy(_abi.ENERGY_POTENTIAL) + model.energy(_abi.ENERGY_KINETIC)
        W = 0.0
        for _ in range(200):
            model.solve_step()
            W += model.energy(_abi.ENERGY_EXTERNAL_WORK)
        e1 = model.energy(_abi.ENERGY_POTENTIAL) + model.energy(_abi.ENERGY_KINETIC)
        errs.append(abs(W - (e1 - e0)))
    return errs


def python_fe_truss(make):
    """The bars of tests/golden/python_fe_truss.json (segment_2, node 0
    fixed, end load, sinusoidal initial displacement) stepped with the
    stored time step; per case the largest relative difference of the
    displacement over all stored steps to the reference's Python solver."""
    from akantu_b200.mesh import bar_segment2
    g = json.load(open(os.path.join(HERE, "golden", "python_fe_truss.json")))
    errs = []
    for c in g["cases"]:
        mesh = bar_segment2(c["Ne"] + 1, c["L"])
        model = make(mesh, dict(kind=_abi.MATERIAL_ELASTIC, rho=c["rho"], E=c["E"], nu=0.0))
        u0 = np.array(c["u0"])[:, None]
        f = np.zeros_like(u0)
        f[-1, 0] = c["F"]
        model.set(_abi.FIELD_DISPLACEMENT, u0)
        model.set(_abi.FIELD_EXTERNAL_FORCE, f)
        model.apply_dirichlet(np.array([0]), 0, np.array([0.0]))
        model.set_time_step(c["dt"])
        worst = 0.0
        for ref in c["displacement"]:
            model.solve_step()
            ref = np.array(ref)
            u = model.get(_abi.FIELD_DISPLACEMENT)[:, 0]
            worst = max(worst, np.abs(u - ref).max() / np.abs(ref).max())
        errs.append(worst)
    return errs
