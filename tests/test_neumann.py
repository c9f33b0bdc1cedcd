"""Neumann conditions on the host (akb_msh_get_group_facets,
akb_neumann_forces; applyBC(FromTraction / FromStress, group) in the
reference, boundary_condition_tmpl.hh:95-185): the facets the Gmsh reader
keeps per group, the nodal forces of a traction or a stress on segments,
triangles and quadrangles (the Gauss rules of the boundary elements, the
normals as the reference forms them from the node order) against hand
integrals, and a closed surface under a uniform stress, whose forces cancel."""
import ctypes as C
import os

import numpy as np
import pytest

import akantu_b200 as aka
from akantu_b200 import _abi
from akantu_b200._lib import AkbError, check, lib
from akantu_b200.mesh import Mesh
from akantu_b200.model import FromStress, FromTraction

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "msh")


def forces(X, facets, kind, value):
    X = np.ascontiguousarray(X, dtype=np.float64)
    facets = np.ascontiguousarray(facets, dtype=np.uint32)
    value = np.ascontiguousarray(value, dtype=np.float64).reshape(-1)
    out = np.zeros_like(X)
    check(lib().akb_neumann_forces(X.shape[1], X.shape[0], X.ctypes.data_as(C.POINTER(C.c_double)),
                                   facets.shape[0], facets.shape[1],
                                   facets.ctypes.data_as(C.POINTER(C.c_uint32)), kind,
                                   value.ctypes.data_as(C.POINTER(C.c_double)),
                                   out.ctypes.data_as(C.POINTER(C.c_double))))
    return out


def colmajor(s):
    return np.asarray(s, dtype=float).T.reshape(-1)


def test_segments():
    X = np.array([[0.0, 0.0], [2.0, 0.0], [2.0, 3.0]])
    f = forces(X, [[0, 1]], _abi.NEUMANN_TRACTION, [1.0, 3.0])
    assert np.allclose(f, [[1.0, 3.0], [1.0, 3.0], [0.0, 0.0]], rtol=0, atol=1e-15)
    # normal of the tangent t = x1 - x0: (t_y, -t_x) / |t|; segment 1 -> 2 points up: n = (1, 0)
    sigma = np.array([[2.0, 0.5], [0.5, 5.0]])
    f = forces(X, [[1, 2]], _abi.NEUMANN_STRESS, colmajor(sigma))
    t = sigma @ np.array([1.0, 0.0])
    assert np.allclose(f[1], 1.5 * t, atol=1e-14) and np.allclose(f[2], 1.5 * t, atol=1e-14)
    # forces are added to what the array holds
    out = np.ones_like(X)
    check(lib().akb_neumann_forces(2, 3, np.ascontiguousarray(X).ctypes.data_as(C.POINTER(C.c_double)),
                                   1, 2, np.array([0, 1], np.uint32).ctypes.data_as(C.POINTER(C.c_uint32)),
                                   _abi.NEUMANN_TRACTION,
                                   np.array([1.0, 0.0]).ctypes.data_as(C.POINTER(C.c_double)),
                                   out.ctypes.data_as(C.POINTER(C.c_double))))
    assert np.allclose(out[:2, 0], 2.0) and np.allclose(out[2], 1.0)


def test_triangles_and_quadrangles():
    X = np.array([[0.0, 0, 0], [2, 0, 0], [0, 1, 0], [2, 1, 0], [0, 0, 1]])
    # triangle 0-1-2 in z = 0, area 1, normal (x1-x0) x (x2-x0) = +z
    f = forces(X, [[0, 1, 2]], _abi.NEUMANN_TRACTION, [0.0, 0.0, 3.0])
    assert np.allclose(f[:3, 2], 1.0) and np.allclose(f[3:], 0.0)
    sigma = np.diag([1.0, 2.0, 7.0])
    f = forces(X, [[0, 1, 2]], _abi.NEUMANN_STRESS, colmajor(sigma))
    assert np.allclose(f[:3], [0.0, 0.0, 7.0 / 3.0])
    f = forces(X, [[0, 2, 1]], _abi.NEUMANN_STRESS, colmajor(sigma))  # reversed: -z
    assert np.allclose(f[:3], [0.0, 0.0, -7.0 / 3.0])
    # rectangle 0-1-3-2 (2 x 1): the bilinear shape functions' integrals A / 4
    f = forces(X, [[0, 1, 3, 2]], _abi.NEUMANN_TRACTION, [1.0, -1.0, 2.0])
    assert np.allclose(f[:4], 0.5 * np.array([1.0, -1.0, 2.0]))
    # a planar trapezoid: the forces add up to traction x area, unevenly
    Y = np.array([[0.0, 0, 0], [4, 0, 0], [3, 2, 0], [1, 2, 0]])
    f = forces(Y, [[0, 1, 2, 3]], _abi.NEUMANN_TRACTION, [0.0, 0.0, 1.0])
    assert f[:, 2].sum() == pytest.approx(6.0, rel=1e-14)
    assert f[0, 2] > f[3, 2]


def unit_cube_surface():
    X = np.array([[x, y, z] for z in (0.0, 1.0) for y in (0.0, 1.0) for x in (0.0, 1.0)])
    idx = lambda x, y, z: int(x + 2 * y + 4 * z)  # noqa: E731
    # the six faces, each ordered so that t_xi x t_eta points out of the cube
    faces = [[idx(0, 0, 0), idx(0, 1, 0), idx(1, 1, 0), idx(1, 0, 0)],   # z = 0, -z
             [idx(0, 0, 1), idx(1, 0, 1), idx(1, 1, 1), idx(0, 1, 1)],   # z = 1, +z
             [idx(0, 0, 0), idx(1, 0, 0), idx(1, 0, 1), idx(0, 0, 1)],   # y = 0, -y
             [idx(0, 1, 0), idx(0, 1, 1), idx(1, 1, 1), idx(1, 1, 0)],   # y = 1, +y
             [idx(0, 0, 0), idx(0, 0, 1), idx(0, 1, 1), idx(0, 1, 0)],   # x = 0, -x
             [idx(1, 0, 0), idx(1, 1, 0), idx(1, 1, 1), idx(1, 0, 1)]]   # x = 1, +x
    return X, faces


def test_closed_surface_under_uniform_stress():
    X, faces = unit_cube_surface()
    rng = np.random.default_rng(4)
    s = rng.normal(size=(3, 3))
    sigma = s + s.T
    f = forces(X, faces, _abi.NEUMANN_STRESS, colmajor(sigma))
    assert np.abs(f.sum(axis=0)).max() <= 1e-14
    # the +x face alone carries sigma e_x over its unit area
    f = forces(X, [faces[5]], _abi.NEUMANN_STRESS, colmajor(sigma))
    assert np.allclose(f.sum(axis=0), sigma[:, 0])
    # the same faces as triangles: the same total on each face
    tris = [[a, b, c] for a, b, c, d in faces] + [[a, c, d] for a, b, c, d in faces]
    f = forces(X, tris, _abi.NEUMANN_STRESS, colmajor(sigma))
    assert np.abs(f.sum(axis=0)).max() <= 1e-14


def test_checks():
    X = np.zeros((2, 2))
    for args in ((_abi.NEUMANN_TRACTION, [[0, 2]]),      # node out of range
                 (7, [[0, 1]])):                          # unknown kind
        kind, facets = args
        with pytest.raises(AkbError):
            forces(X, facets, kind, [1.0, 0.0])
    with pytest.raises(AkbError):  # triangles in 2D
        forces(np.zeros((3, 2)), [[0, 1, 2]], _abi.NEUMANN_TRACTION, [1.0, 0.0])
    with pytest.raises(AkbError):  # no 1D Neumann condition in the reference
        forces(np.zeros((2, 1)), [[0, 1]], _abi.NEUMANN_TRACTION, [1.0])
    with pytest.raises(AkbError):  # a degenerate facet
        forces(np.zeros((2, 2)), [[0, 1]], _abi.NEUMANN_TRACTION, [1.0, 0.0])


def test_reader_keeps_the_groups_facets():
    mesh = Mesh(2)
    mesh.read(os.path.join(GOLDEN, "cohesive_strait_2D.msh"))
    assert set(mesh.facet_groups) == {"fixed", "loading", "insertion"}
    for name in ("fixed", "loading"):
        segs = mesh.getFacetGroup(name)
        assert segs.shape[1] == 2
        assert set(segs.reshape(-1).tolist()) == set(mesh.getNodeGroup(name).tolist())
    # FromTraction on the loading line: the forces add up to traction x length
    segs = mesh.getFacetGroup("loading")
    x = mesh.nodes
    length = np.linalg.norm(x[segs[:, 1]] - x[segs[:, 0]], axis=1).sum()
    f = mesh.neumannForces("loading", FromTraction([0.0, -2.0]))
    assert f.sum(axis=0) == pytest.approx([0.0, -2.0 * length], abs=1e-14)
    assert np.all(f[np.setdiff1d(np.arange(len(x)), mesh.getNodeGroup("loading"))] == 0.0)
    # the body group has no facets (its elements are of the mesh's dimension)
    assert "body" not in mesh.facet_groups
    with pytest.raises(ValueError):
        FromStress(np.eye(3)).akb_value(2)


HEX_WITH_TOP = """$MeshFormat
2.2 0 8
$EndMeshFormat
$PhysicalNames
2
2 1 "top"
3 2 "body"
$EndPhysicalNames
$Nodes
8
1 0 0 0
2 1 0 0
3 1 1 0
4 0 1 0
5 0 0 1
6 1 0 1
7 1 1 1
8 0 1 1
$EndNodes
$Elements
2
1 3 2 1 1 5 6 7 8
2 5 2 2 2 1 2 3 4 5 6 7 8
$EndElements
"""


def test_quadrangle_facets_of_a_hexahedral_mesh():
    mesh = Mesh(3)
    mesh.read_msh_text(HEX_WITH_TOP)
    assert mesh.element_type == _abi.HEXAHEDRON_8 and len(mesh.connectivity) == 1
    assert mesh.getFacetGroup("top").tolist() == [[4, 5, 6, 7]]
    f = mesh.neumannForces("top", FromStress(np.diag([0.0, 0.0, -3.0])))  # n = +z
    assert np.allclose(f[4:], [0.0, 0.0, -0.75]) and np.all(f[:4] == 0.0)
    with pytest.raises(AkbError):  # a 2D mesh of quadrangles: skipped, so no element left
        Mesh(2).read_msh_text(HEX_WITH_TOP.replace("3 2 \"body\"", "2 2 \"body\"")
                              .replace("2 5 2 2 2 1 2 3 4 5 6 7 8", "2 3 2 2 2 1 2 3 4"))


def test_cpp_shim_neumann_forces(tmp_path):
    """The C++ shim's Mesh::read keeps the groups' facets and its
    addNeumannForces (what applyBC(FromTraction / FromStress, group) adds to
    the external force) gives the same forces as the Python layer."""
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("g++ not found")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.join(root, "akantu_b200")
    exe = str(tmp_path / "shim_neumann")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(root, "include"), "-o", exe,
                    os.path.join(root, "tests", "cpp", "shim_neumann.cc"), "-L", libdir, "-lakb",
                    "-Wl,-rpath," + libdir], check=True)
    msh = os.path.join(GOLDEN, "cohesive_strait_2D.msh")
    out = subprocess.run([exe, msh, "loading"], check=True, capture_output=True, text=True).stdout
    nf, fx, fy, hx, hy = out.split()
    mesh = Mesh(2)
    mesh.read(msh)
    assert int(nf) == len(mesh.getFacetGroup("loading"))
    want_f = mesh.neumannForces("loading", FromTraction([0.0, -2.0])).sum(axis=0)
    want_h = mesh.neumannForces("loading", FromStress(np.eye(2))).sum(axis=0)
    assert np.allclose([float(fx), float(fy)], want_f, rtol=0, atol=1e-14)
    assert np.allclose([float(hx), float(hy)], want_h, rtol=0, atol=1e-14)


def test_group_with_facets_of_two_kinds():
    """A group mixing triangles and quadrangles: the file reads, its nodes and
    elements are kept, and only a Neumann condition on it is refused."""
    text = HEX_WITH_TOP.replace("$Elements\n2\n", "$Elements\n3\n0 2 2 1 1 1 2 3\n")
    mesh = Mesh(3)
    mesh.read_msh_text(text)
    assert sorted(mesh.getNodeGroup("top").tolist()) == [0, 1, 2, 4, 5, 6, 7]
    assert "top" not in mesh.facet_groups
    with pytest.raises(ValueError):
        mesh.neumannForces("top", FromTraction([0.0, 0.0, 1.0]))


class PyTraction(aka.NeumannFunctor):
    """A NeumannFunctor written in Python: a constant traction."""

    def __init__(self, t):
        self.t = np.asarray(t, dtype=float)
        self.calls = []

    def __call__(self, quad_point, dual, coord, normals):
        self.calls.append((quad_point.element, quad_point.num_point))
        dual[:] = self.t


class PyStress(aka.NeumannFunctor):
    def __init__(self, s):
        self.s = np.asarray(s, dtype=float)

    def __call__(self, quad_point, dual, coord, normals):
        dual[:] = self.s @ normals


class PyLinear(aka.NeumannFunctor):
    """A traction growing with x: evaluated at each Gauss point."""

    def __call__(self, quad_point, dual, coord, normals):
        dual[:] = 0.0
        dual[-1] = coord[0]


def test_neumann_functors_written_in_python():
    mesh = Mesh(2)
    mesh.read(os.path.join(GOLDEN, "cohesive_strait_2D.msh"))
    t = PyTraction([0.5, -2.0])
    assert np.allclose(mesh.neumannForces("loading", t),
                       mesh.neumannForces("loading", FromTraction([0.5, -2.0])), rtol=0, atol=1e-15)
    assert t.calls == [(f, 0) for f in range(len(mesh.getFacetGroup("loading")))]  # one point each
    sigma = np.array([[1.0, 0.3], [0.3, -2.0]])
    assert np.allclose(mesh.neumannForces("fixed", PyStress(sigma)),
                       mesh.neumannForces("fixed", FromStress(sigma)), rtol=0, atol=1e-15)
    assert np.all(mesh.neumannForces("loading", aka.FreeBoundary()) == 0.0)
    # 2 x 2 points on a quadrangle: a traction linear in x integrates exactly
    hexm = Mesh(3)
    hexm.read_msh_text(HEX_WITH_TOP)
    f = hexm.neumannForces("top", PyLinear())
    assert f[:, 2].sum() == pytest.approx(0.5, rel=1e-14)  # integral of x over the unit square
    assert f[5, 2] > f[4, 2]  # the x = 1 corners carry more
    assert np.allclose(hexm.neumannForces("top", PyStress(np.diag([0.0, 0.0, -3.0]))),
                       hexm.neumannForces("top", FromStress(np.diag([0.0, 0.0, -3.0]))))


def test_dirichlet_functors():
    """FixedValue, IncrementValue and Increment act on a node's flags and
    displacement as boundary_condition_functor_inline_impl.hh states."""
    flags, primal = np.zeros(3, bool), np.array([1.0, 2.0, 3.0])
    aka.FixedValue(5.0, aka._y)(0, flags, primal, np.zeros(3))
    assert flags.tolist() == [False, True, False] and primal.tolist() == [1.0, 5.0, 3.0]
    aka.IncrementValue(0.5, aka._z)(0, flags, primal, np.zeros(3))
    assert flags.tolist() == [False, True, True] and primal.tolist() == [1.0, 5.0, 3.5]
    aka.Increment([1.0, 1.0, -1.0])(0, flags, primal, np.zeros(3))
    assert flags.all() and primal.tolist() == [2.0, 6.0, 2.5]
    with pytest.raises(NotImplementedError):
        aka.DirichletFunctor()(0, flags, primal, np.zeros(3))


def test_apply_bc_dispatch():
    """SolidMechanicsModel.applyBC without a device (its field accessors
    replaced by arrays): FixedValue goes to the device Dirichlet call, other
    Dirichlet functors run node by node on copies that are written back,
    Neumann functors add their forces to the external force."""
    from akantu_b200.model import SolidMechanicsModel
    mesh = Mesh(2)
    mesh.read(os.path.join(GOLDEN, "cohesive_strait_2D.msh"))
    n = mesh.getNbNodes()

    class Arrays(SolidMechanicsModel):
        def __init__(self):
            super().__init__(mesh, [aka.MaterialElastic(rho=1, E=1, nu=0.3)])
            self.u, self.b, self.fext = np.zeros((n, 2)), np.zeros((n, 2), bool), np.ones((n, 2))
            self.dirichlet = []

        def getField(self, field):
            assert field == _abi.FIELD_DISPLACEMENT
            return self.u

        def getBlockedDOFs(self):
            return self.b

        def setField(self, field, values):
            self.u = np.array(values)

        def setBlockedDOFs(self, blocked):
            self.b = np.array(blocked, bool)

        def getExternalForce(self):
            return self.fext

        def applyDirichlet(self, nodes, component, values):
            self.dirichlet.append((sorted(np.asarray(nodes).tolist()), component, values))

    m = Arrays()
    fixed = mesh.getNodeGroup("fixed")
    m.applyBC(aka.FixedValue(0.25, aka._y), "fixed")
    assert m.dirichlet == [(sorted(fixed.tolist()), aka._y, 0.25)]
    m.applyBC(aka.IncrementValue(0.5, aka._x), "fixed")
    m.applyBC(aka.IncrementValue(0.5, aka._x), "fixed")
    assert np.all(m.u[fixed, 0] == 1.0) and np.all(m.b[fixed, 0])
    others = np.setdiff1d(np.arange(n), fixed)
    assert np.all(m.u[others] == 0.0) and not m.b[others].any()
    m.applyBC(aka.FromTraction([0.0, -2.0]), "loading")
    assert np.allclose(m.fext, 1.0 + mesh.neumannForces("loading", FromTraction([0.0, -2.0])))
    with pytest.raises(TypeError):
        m.applyBC(object(), "fixed")


@pytest.mark.parametrize("etype", [_abi.TRIANGLE_3, _abi.TETRAHEDRON_4, _abi.HEXAHEDRON_8],
                         ids=["triangle_3", "tetrahedron_4", "hexahedron_8"])
def test_library_matches_the_work_balance_port(etype):
    """The work-balance port's nodal forces (FromTraction(0.5 e_x) on the
    bar's face x = max, test_solid_mechanics_model_work_dynamics.cc:84-106,
    restated there by sharing each facet's measure equally) against
    akb_neumann_forces on the same facets."""
    from akantu_b200.mesh import _FACETS
    from tests.reference_ports import _traction_forces, bar_mesh
    mesh = bar_mesh(etype)
    X = mesh.nodes
    xmax = X[:, 0].max()
    facets, seen = [], set()
    for elem in mesh.connectivity:
        for fc in _FACETS[mesh.element_type]:
            nodes = [int(elem[k]) for k in fc]
            key = tuple(sorted(nodes))
            if all(X[n, 0] > xmax - 1e-6 for n in nodes) and key not in seen:
                seen.add(key)
                facets.append(nodes)
    d = mesh.spatial_dimension
    got = forces(X, facets, _abi.NEUMANN_TRACTION, [0.5] + [0.0] * (d - 1))
    want = _traction_forces(mesh, 0.5)
    assert np.allclose(got, want, rtol=0, atol=1e-15)
    assert got[:, 0].sum() == pytest.approx(0.5, rel=1e-14)  # the end face's measure is 1


@pytest.mark.parametrize("etype", [_abi.TRIANGLE_3, _abi.TETRAHEDRON_4, _abi.HEXAHEDRON_8],
                         ids=["triangle_3", "tetrahedron_4", "hexahedron_8"])
def test_element_groups_from_node_groups(etype):
    """createElementGroupFromNodeGroup as the work-balance test uses it: the
    nodes of the face x = max, their facets (dimension d - 1) as a group,
    FromTraction on it equal to the port's forces; every boundary facet
    oriented outward (a uniform stress on the closed boundary sums to
    zero, sigma = I pushes the x = max face towards +x)."""
    from tests.reference_ports import _traction_forces, bar_mesh
    mesh = bar_mesh(etype)
    X = mesh.nodes
    d = mesh.spatial_dimension
    end = np.nonzero(X[:, 0] > X[:, 0].max() - 1e-6)[0]
    mesh.createNodeGroup("apply_force", end)
    nodes = mesh.createElementGroupFromNodeGroup("el_apply_force", "apply_force", d - 1)
    assert sorted(nodes.tolist()) == sorted(end.tolist())
    f = mesh.neumannForces("el_apply_force", FromTraction([0.5] + [0.0] * (d - 1)))
    assert np.allclose(f, _traction_forces(mesh, 0.5), rtol=0, atol=1e-15)
    g = mesh.neumannForces("el_apply_force", FromStress(np.eye(d)))
    assert g[:, 0].sum() == pytest.approx(1.0, rel=1e-14)  # outward: +x, unit face
    mesh.createNodeGroup("all", np.arange(len(X)))
    mesh.createElementGroupFromNodeGroup("skin", "all", d - 1)
    rng = np.random.default_rng(8)
    s = rng.normal(size=(d, d))
    h = mesh.neumannForces("skin", FromStress(s + s.T))
    assert np.abs(h.sum(axis=0)).max() <= 1e-12
    # of the spatial dimension: the elements whose nodes are all in the group
    mesh.createElementGroupFromNodeGroup("bulk", "all")
    assert len(mesh.getElementGroup("bulk")) == len(mesh.connectivity)
