"""Host side of the materials written in Python (akantu_b200.material_plugin):
the input-file sections, MaterialFactory and parameter registration, the
layout in which a law sees its quadrature points (the reference's: rows of
column-major d x d matrices, its own elements only) and the quadrature
weights of the potential energy. The bridge runs here on CPU torch tensors
laid out like the device fields; the stepping itself is in
test_gpu_material_plugin.py."""
import numpy as np
import pytest
import torch

from akantu_b200 import _abi
from akantu_b200 import material_plugin as mp
from akantu_b200.mesh import Mesh


def test_input_sections():
    text = """
    # a comment line
    material elastic [
      name = steel
      rho = 7800      # density
      E = 2.1e11
      nu = 0.3
      Plane_Stress = true
    ]
    model solid_mechanics_model [
      material my_law [ name = soft
        rho = 1. ]
    ]
    """
    got = mp.parse_input_text(text)
    assert got == [("elastic", dict(name="steel", rho=7800.0, E=2.1e11, nu=0.3,
                                    Plane_Stress=True)),
                   ("my_law", dict(name="soft", rho=1.0))]
    assert mp.input_sections() == got
    # brackets on their own lines, a vector value, a value closed by the bracket
    got = mp.parse_input_text("material neohookean\n[\n  name = rubber\n  rho = 1100\n"
                              "  direction = [1, 0, -2.5]\n  E = 1e6 ]\n")
    assert got == [("neohookean", dict(name="rubber", rho=1100.0, direction=[1.0, 0.0, -2.5],
                                       E=1e6))]
    assert mp.parse_input_text("") == [] and mp.input_sections() == []  # replaced, and cleared
    for bad in ("material elastic [ rho = 1", "]", "material [ rho = 1 ]", "material elastic [ = 1 ]"):
        with pytest.raises(ValueError):
            mp.parse_input_text(bad)


class Scaled(mp.Material):
    """stress = k grad_u row by row (any layout passes through unchanged)."""

    def __init__(self, model, _id):
        super().__init__(model, _id)
        self.registerParamReal(2.0, "k", mp._pat_readable | mp._pat_parsable, "factor")
        self.registerParamReal("E", mp._pat_readable | mp._pat_parsable, "Young's modulus")
        self.registerParamReal("nu", mp._pat_readable | mp._pat_parsable, "Poisson's ratio")

    def initMaterial(self):
        self.registerInternal("calls", 1)
        super().initMaterial()

    def computeStress(self, el_type, ghost_type=mp._not_ghost):
        self.getStress(el_type, ghost_type)[...] = self.getReal("k") * self.getGradU(el_type)
        self.internals["calls"](el_type)[:, 0] += 1

    def computePotentialEnergy(self, el_type):
        self.getPotentialEnergy(el_type)[:, 0] = self.getGradU(el_type).sum(axis=1)


class Transposing(mp.Material):
    """Reads its arrays reshaped to (n, d, d) in numpy order, as the
    reference's example scripts do, and writes the transpose back."""

    def computeStress(self, el_type, ghost_type=mp._not_ghost):
        g = self.getGradU(el_type)
        n = g.shape[0]
        s = self.getStress(el_type).reshape(n, 2, 2)  # a view: writes reach the array
        s[:, :, :] = g.reshape(n, 2, 2).transpose(0, 2, 1)

    def getPushWaveSpeed(self, element):
        return 3.0


@pytest.fixture
def factory():
    f = mp.MaterialFactory.getInstance()
    f.registerAllocator("scaled", lambda dim, law, model, mid: Scaled(model, mid))
    f.registerAllocator("transposing", lambda dim, law, model, mid: Transposing(model, mid))
    yield f
    mp.parse_input_text("")


def test_input_grammar_of_the_reference_parser():
    """The constructs of the reference's parser test
    (test_io/test_parser/test_parser.cc and its verified output), in an
    input of this test's own: global parameters, expressions over earlier
    parameters with pi and max, a section option, a nested section, a
    vector, a matrix continued over two lines, a random distribution kept as
    text, a name never evaluated."""
    text = """seed = 42
    level = 2
    material elastic opt [
        name = e        # a name, not the constant
        E = 1 + 3 * level
        rho = 2^3
        nested rules [
            E = 7
        ]
    ]
    base = 50
    angle = 2*pi + max(2, base)
    vect = [ 1, 20+5, angle ]
    mat = [[ 1, 2 ], \\
           [ base, 5+8 ]]
    rand = 10 uniform [0.2, 0.5 ]
    """
    got = mp.parse_input_text(text)
    assert got == [("elastic", dict(name="e", E=7.0, rho=8.0))]
    g = mp.input_parameters()
    assert g["seed"] == 42.0 and g["base"] == 50.0
    assert g["angle"] == 2 * np.pi + 50.0  # bit for bit, as the reference's test checks
    assert g["vect"] == [1.0, 25.0, 2 * np.pi + 50.0]
    assert g["mat"] == [[1.0, 2.0], [50.0, 13.0]]
    assert g["rand"] == "10 uniform [0.2, 0.5 ]"


def test_factory_and_parameters(factory):
    m = mp.law_from_section("scaled", dict(name="a", rho=2.0, E=5.0, nu=0.25), 0, 2, None)
    assert (m.name, m.getReal("rho"), m.getReal("k"), m.getReal("E")) == ("a", 2.0, 2.0, 5.0)
    lam, mu = 0.25 * 5.0 / (1.25 * 0.5), 5.0 / 2.5
    assert m.getPushWaveSpeed(None) == pytest.approx(np.sqrt((lam + 2 * mu) / 2.0), rel=1e-15)
    assert mp.law_from_section("transposing", dict(rho=1.0), 3, 2, None).name == "transposing_3"
    with pytest.raises(KeyError):  # a key the law does not register
        mp.law_from_section("scaled", dict(rho=1.0, G=3.0), 0, 2, None)
    with pytest.raises(KeyError):  # neither built in nor registered
        mp.law_from_section("no_such_law", dict(rho=1.0), 0, 2, None)
    with pytest.raises(NotImplementedError):  # no E and nu, no override
        mp.Material(None, "x").getPushWaveSpeed(None)


def device_like(raw, d):
    """The model's view of a column-major quadrature field: (n, d, d)
    [k, i, j] over storage rows [i + j*d]."""
    return raw.view(-1, d, d).transpose(1, 2)


def test_bridge_layout_and_element_filter(factory):
    d, nqp = 2, 1
    em = np.array([0, 1, 0, 1, 1])
    laws = [mp.law_from_section("scaled", dict(rho=1.0, k=3.0), 0, d, None),
            mp.law_from_section("transposing", dict(rho=1.0), 1, d, None)]
    bridge = mp.LawBridge(laws, em, _abi.TRIANGLE_3, nqp, d)
    for law in laws:
        law.initMaterial()
    assert np.array_equal(laws[0].element_filter(_abi.TRIANGLE_3), [0, 2])
    assert np.array_equal(laws[1].element_filter(_abi.TRIANGLE_3), [1, 3, 4])
    raw_g = torch.arange(5 * d * d, dtype=torch.float64).reshape(5, d * d)
    raw_s = torch.zeros(5, d * d, dtype=torch.float64)
    G, S = device_like(raw_g, d), device_like(raw_s, d)
    bridge.stresses(G, S)
    # the law saw the storage rows of its own elements
    assert np.array_equal(laws[0].getGradU(_abi.TRIANGLE_3), raw_g.numpy()[[0, 2]])
    assert np.array_equal(raw_s.numpy()[[0, 2]], 3.0 * raw_g.numpy()[[0, 2]])
    # numpy's (n, d, d) reshape of a column-major row reads, and writes, the
    # transposed matrix: writing back the transpose of what it read stores G^T
    assert torch.equal(S[[1, 3, 4]], G[[1, 3, 4]].transpose(1, 2))
    assert laws[0].internals["calls"](_abi.TRIANGLE_3)[:, 0].tolist() == [1, 1]
    with pytest.raises(ValueError):
        laws[0].getGradU(_abi.TETRAHEDRON_4)
    with pytest.raises(ValueError):
        laws[0].getGradU(_abi.TRIANGLE_3, mp._ghost)


def test_bridge_potential_energy(factory):
    laws = [mp.law_from_section("scaled", dict(rho=1.0), 0, 2, None)]
    bridge = mp.LawBridge(laws, np.zeros(4, int), _abi.TRIANGLE_3, 1, 2)
    laws[0].initMaterial()
    w = np.array([0.5, 1.0, 2.0, 4.0])
    with pytest.raises(RuntimeError):  # no step yet
        bridge.potential_energy(w)
    raw = torch.rand(4, 4, dtype=torch.float64)
    bridge.stresses(device_like(raw, 2), device_like(torch.zeros(4, 4, dtype=torch.float64), 2))
    assert bridge.potential_energy(w) == pytest.approx(float(raw.sum(1).numpy() @ w), rel=1e-15)


def hex_volume_3x3x3(x):
    """Volume of a trilinear hexahedron by the 3-point Gauss rule per axis
    (exact for det J, of degree 2 per axis), corners in the order of
    hexahedron_8."""
    s = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                  [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=float)
    pts, wts = np.array([-np.sqrt(0.6), 0.0, np.sqrt(0.6)]), np.array([5, 8, 5]) / 9.0
    vol = 0.0
    for a, wa in zip(pts, wts):
        for b, wb in zip(pts, wts):
            for c, wc in zip(pts, wts):
                p = np.array([a, b, c])
                dN = np.empty((3, 8))
                for k in range(3):
                    f = s[:, k] / 8.0
                    for m in range(3):
                        if m != k:
                            f = f * (1 + s[:, m] * p[m])
                    dN[k] = f
                vol += wa * wb * wc * np.linalg.det(dN @ x)
    return vol


def test_quadrature_weights():
    tri = Mesh(2, _abi.TRIANGLE_3, np.array([[0.0, 0.0], [2.0, 0.0], [0.0, 1.0]]),
               np.array([[0, 1, 2]], dtype=np.uint32))
    assert mp.qp_weights(tri) == pytest.approx([1.0], rel=1e-15)
    tet = Mesh(3, _abi.TETRAHEDRON_4, np.array([[0.0, 0, 0], [1, 0, 0], [0, 2, 0], [0, 0, 3]]),
               np.array([[0, 1, 2, 3]], dtype=np.uint32))
    assert mp.qp_weights(tet) == pytest.approx([1.0], rel=1e-15)
    seg = Mesh(1, _abi.SEGMENT_2, np.array([[1.0], [3.5]]), np.array([[0, 1]], dtype=np.uint32))
    assert mp.qp_weights(seg) == pytest.approx([2.5], rel=1e-15)
    corners = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                        [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=float)
    box = Mesh(3, _abi.HEXAHEDRON_8, corners * [2.0, 3.0, 0.5], np.arange(8, dtype=np.uint32)[None])
    assert mp.qp_weights(box) == pytest.approx([3.0 / 8] * 8, rel=1e-14)
    # a distorted hexahedron: the eight weights add up to its volume, and the
    # points with bit 0 set (x = +g) carry the larger weights when the
    # element widens towards +x
    rng = np.random.default_rng(3)
    x = corners + rng.uniform(-0.15, 0.15, corners.shape)
    x[[1, 2, 5, 6], 1:] *= 1.5
    w = mp.qp_weights(Mesh(3, _abi.HEXAHEDRON_8, x, np.arange(8, dtype=np.uint32)[None]))
    assert w.sum() == pytest.approx(hex_volume_3x3x3(x), rel=1e-13)
    assert all(w[q | 1] > w[q & ~1] for q in range(8))


def test_material_selector_by_physical_names():
    """test_material_selector.cc on its own mesh: the segments of the
    physical groups chocolate, chewing-gum and candy take the materials of
    those names (material_selector.dat order: chocolate, chewing-gum,
    candy); an element of no named material takes the fallback."""
    import os

    class ModelLike:  # the selector reads the model's mesh only
        mesh = Mesh(1)
    ModelLike.mesh.read(os.path.join(os.path.dirname(__file__), "golden", "msh",
                                     "material_selector.msh"))
    sel = mp.MeshDataMaterialSelectorString("physical_names", ModelLike)
    em = sel.select(["chocolate", "chewing-gum", "candy"])
    first = {k: int(np.nonzero(em == k)[0][0]) for k in range(3)}
    assert first == {0: 0, 1: 1, 2: 2}
    sel.setFallback(1)
    assert sel.select(["chocolate"]).tolist() == [0, 1, 1]
    with pytest.raises(ValueError):
        mp.MeshDataMaterialSelectorString("tag_0", ModelLike)


def test_builtin_material_views():
    """getGradU / getStress of a built-in material: the rows of the model's
    quadrature field (column-major matrices) that belong to its elements,
    every Gauss point of each, in element order."""
    from akantu_b200.model import MaterialElastic

    class ModelLike:
        mesh = Mesh(3, _abi.HEXAHEDRON_8, np.zeros((8, 3)), np.zeros((3, 8), dtype=np.uint32))
        nqp, dim = 8, 3

        @staticmethod
        def getField(field):
            base = 1000.0 if field == _abi.FIELD_STRESS else 0.0
            return base + np.arange(3 * 8 * 9, dtype=float).reshape(3 * 8, 9)

    m = MaterialElastic(rho=1.0, E=1.0, nu=0.3)
    with pytest.raises(RuntimeError):
        m.getGradU(_abi.HEXAHEDRON_8)
    m._model, m._elements = (lambda: ModelLike), np.array([0, 2])  # as the weak reference
    g = m.getGradU(_abi.HEXAHEDRON_8)
    assert g.shape == (16, 9)
    assert np.array_equal(g, ModelLike.getField(_abi.FIELD_GRAD_U)[list(range(8)) + list(range(16, 24))])
    assert np.array_equal(m.getStress(_abi.HEXAHEDRON_8), 1000.0 + g)
    with pytest.raises(ValueError):
        m.getStress(_abi.TETRAHEDRON_4)


def test_initialize_points_to_parse_input():
    import akantu_b200 as aka
    for f in (aka.initialize, aka.finalize):
        with pytest.raises(RuntimeError):
            f("material.dat")
