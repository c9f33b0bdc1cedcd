"""The CPU oracle against the reference's own golden data (no GPU needed).

Pins the restatement before it is trusted as the checker of libakb.so:
  * the 402-row explicit model-solver table (test_model_solver_dynamic_explicit.verified)
    must match at every printed digit;
  * the explicit linear patch test (patch_test_linear_elastic_explicit.cc:33-68)
    on the reference's own triangle_3 / tetrahedron_4 / hexahedron_8 meshes;
  * the lumped-mass test (test_lumped_mass.cc:81-101).
"""
import numpy as np
import pytest

from akantu_b200 import _abi
from tests.golden_cases import (OracleAdapter, check_patch_results,
                                compare_model_solver_table, lumped_mass_case,
                                model_solver_dynamic_explicit, patch_test_explicit)

PATCH_TYPES = ["_triangle_3", "_tetrahedron_4", "_hexahedron_8"]


def make(mesh, mat):
    return OracleAdapter(mesh, mat)


def test_model_solver_dynamic_explicit_golden_table():
    table = model_solver_dynamic_explicit(make)
    errs, golden = compare_model_solver_table(table)
    assert table.shape == golden.shape == (401, 7)  # header + 401 rows
    # every printed digit of every row agrees
    for col, e in errs.items():
        assert e == 0.0, (col, e)


@pytest.mark.parametrize("name", PATCH_TYPES)
def test_patch_test_explicit(name):
    r = patch_test_explicit(make, name)
    for key, (err, tol) in check_patch_results(r).items():
        assert err <= tol, (name, key, err, tol)


@pytest.mark.parametrize("name", PATCH_TYPES)
def test_lumped_mass(name):
    total, ref = lumped_mass_case(make, name)
    assert np.all(np.abs((total - ref) / ref) <= 2e-15)


def test_negative_jacobian_is_rejected():
    from oracle.oracle import OracleModel, material_desc
    from akantu_b200.mesh import plate_triangle3
    mesh = plate_triangle3(2, 2, 1.0, 1.0)
    mesh.connectivity = mesh.connectivity[:, [0, 2, 1]].copy()  # clockwise
    with pytest.raises(RuntimeError, match="negative jacobian"):
        OracleModel(mesh, [material_desc(rho=1, E=1, nu=0.3)])


def test_stable_time_step_known_answer():
    """Plate of 200x20 squares over 10 m x 1 m, E = 210 GPa, nu = 0.3,
    rho = 7800, plane strain: h = 2 r_in of a right isoceles triangle with
    legs 0.05 m, c_p = sqrt((lambda + 2 mu) / rho)."""
    from akantu_b200.mesh import plate_triangle3
    mesh = plate_triangle3(200, 20, 10.0, 1.0)
    m = OracleAdapter(mesh, dict(kind=_abi.MATERIAL_ELASTIC, rho=7800., E=210e9, nu=0.3))
    E, nu, rho = 210e9, 0.3, 7800.
    lam = nu * E / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    leg = 0.05
    r_in = leg * leg / (2 * leg + leg * np.sqrt(2))
    dt = 2 * r_in / np.sqrt((lam + 2 * mu) / rho)
    assert m.stable_time_step() == pytest.approx(dt, rel=1e-12)


def test_structured_meshes_positive_orientation():
    from oracle.oracle import OracleModel, material_desc
    from akantu_b200.mesh import block_hexahedron8, cube_tetrahedron4, plate_triangle3
    for mesh in (plate_triangle3(4, 3, 2.0, 1.0), cube_tetrahedron4(3), block_hexahedron8(3)):
        OracleModel(mesh, [material_desc(rho=1, E=1, nu=0.3)])  # raises if negative


def test_energy_conservation_neohookean_block():
    """No reference test pins neo-Hookean (test_finite_def_materials.cc:48-84
    are all disabled): the restatement is checked for S(F = I) = 0 and for
    conservation of kinetic + potential energy of a free block."""
    from akantu_b200.mesh import block_hexahedron8
    mesh = block_hexahedron8(3, 1.0)
    mat = dict(kind=_abi.MATERIAL_NEOHOOKEAN, rho=1100., E=1.085714285714286e6,
               nu=0.357142857142857)
    m = OracleAdapter(mesh, mat)
    rng = np.random.default_rng(7)
    m.set(_abi.FIELD_VELOCITY, rng.normal(0, 0.05, (mesh.getNbNodes(), 3)))
    m.assemble_internal_forces()
    assert np.abs(m.get(_abi.FIELD_STRESS)).max() == 0.0
    dt = m.stable_time_step()
    m.set_time_step(0.1 * dt)
    m.assemble_mass_lumped()
    e0 = m.energy(_abi.ENERGY_KINETIC)
    worst = 0.0
    for _ in range(400):
        m.solve_step()
        e1 = m.energy(_abi.ENERGY_KINETIC) + m.energy(_abi.ENERGY_POTENTIAL)
        worst = max(worst, abs(e1 - e0) / e0)
    # central differences conserve a shadow energy; at dt = 0.1 dt_crit the
    # kinetic + potential sum stays within half a percent
    assert worst < 5e-3


def _oracle_P(H, mat):
    """The oracle's first Piola-Kirchhoff stress of the neo-Hookean law at
    F = I + H: one tetrahedron deformed homogeneously (u = H X), its stress
    field (PK2 S, column-major) times F."""
    from akantu_b200.mesh import Mesh
    X = np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    mesh = Mesh(3, _abi.TETRAHEDRON_4, X, np.array([[0, 1, 2, 3]], dtype=np.uint32))
    m = OracleAdapter(mesh, mat)
    m.set(_abi.FIELD_DISPLACEMENT, X @ H.T)
    m.assemble_internal_forces()
    S = np.asarray(m.get(_abi.FIELD_STRESS)).reshape(3, 3).T  # row [i + 3 j] = S_ij
    return (np.eye(3) + H) @ S


def test_neohookean_law_properties():
    """The oracle's neo-Hookean law (material_neohookean_inline_impl.hh:46-65)
    against an independent numpy statement of the same law, and its
    properties: objectivity P(QF) = Q P(F), the small-strain limit (the
    linear elastic law with the same Lame constants)."""
    from tests.fe2_cases import lame, neohookean_P, random_rotation
    mat = dict(kind=_abi.MATERIAL_NEOHOOKEAN, rho=1.0, E=3.0, nu=0.3)
    lam, mu = lame(mat)
    rng = np.random.default_rng(21)
    for _ in range(3):
        H = rng.uniform(-0.2, 0.2, (3, 3))
        P = _oracle_P(H, mat)
        assert np.allclose(P, neohookean_P(H, lam, mu), rtol=0, atol=1e-13 * np.abs(P).max())
        Q = random_rotation(rng)
        PQ = _oracle_P(Q @ (np.eye(3) + H) - np.eye(3), mat)
        assert np.allclose(PQ, Q @ P, rtol=0, atol=1e-12 * np.abs(P).max())
    H = 1e-7 * rng.normal(size=(3, 3))
    eps = 0.5 * (H + H.T)
    lin = lam * np.trace(eps) * np.eye(3) + 2 * mu * eps
    assert np.abs(_oracle_P(H, mat) - lin).max() <= 1e-5 * np.abs(lin).max()
