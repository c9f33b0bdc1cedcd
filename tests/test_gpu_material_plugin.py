"""Materials written in Python in the reference's plugin style, stepped on
the GPU with their stresses computed on the host (B200): a small-strain
isotropic law written against getGradU / getStress, allocated through
MaterialFactory from an input file, against the library's own elastic
material in AKB_MODE_FP64 on the same mesh. The two compute the same
stresses in different operation orders: displacements and energies agree to
<= 1e-10 relative after 100 steps. On distorted hexahedra (det J differs
from Gauss point to Gauss point) the potential energy also checks the order
of the host quadrature weights against the library's points."""
import os

import numpy as np
import pytest

import akantu_b200 as aka
from akantu_b200 import material_plugin as mp
from akantu_b200.mesh import block_hexahedron8

pytestmark = pytest.mark.gpu

MSH = os.path.join(os.path.dirname(__file__), "golden", "msh", "cohesive_strait_2D.msh")


class IsotropicElastic(aka.Material):
    """sigma = lambda tr(eps) I + 2 mu eps on the column-major rows of
    getGradU (the Lame constants from the registered E and nu), energy
    density sigma : eps / 2."""

    def __init__(self, model, _id):
        super().__init__(model, _id)
        self.registerParamReal("E", aka._pat_readable | aka._pat_parsable, "Young's modulus")
        self.registerParamReal("nu", aka._pat_readable | aka._pat_parsable, "Poisson's ratio")

    def initMaterial(self):
        E, nu = self.getReal("E"), self.getReal("nu")
        self.lam = nu * E / ((1 + nu) * (1 - 2 * nu))
        self.mu = E / (2 * (1 + nu))
        super().initMaterial()

    def _strain(self, el_type):
        g = self.getGradU(el_type)
        d = int(round(np.sqrt(g.shape[1])))
        G = g.reshape(-1, d, d).transpose(0, 2, 1)  # [k, i, j] = du_i / dX_j
        return 0.5 * (G + G.transpose(0, 2, 1)), d

    def computeStress(self, el_type, ghost_type=aka._not_ghost):
        eps, d = self._strain(el_type)
        tr = np.trace(eps, axis1=1, axis2=2)
        sig = 2 * self.mu * eps + self.lam * tr[:, None, None] * np.eye(d)
        self.getStress(el_type, ghost_type)[...] = sig.transpose(0, 2, 1).reshape(len(sig), d * d)

    def computePotentialEnergy(self, el_type):
        eps, d = self._strain(el_type)
        sig = self.getStress(el_type).reshape(-1, d, d).transpose(0, 2, 1)
        self.getPotentialEnergy(el_type)[:, 0] = 0.5 * np.einsum("kij,kij->k", sig, eps)


@pytest.fixture(autouse=True)
def registered():
    aka.MaterialFactory.getInstance().registerAllocator(
        "isotropic_elastic", lambda dim, law, model, mid: IsotropicElastic(model, mid))
    yield
    mp.parse_input_text("")  # no sections left for models created later


def rel(x, ref):
    return np.abs(x - ref).max() / np.abs(ref).max()


def run(model, mesh, setup, steps):
    model.initFull(_analysis_method=aka._explicit_lumped_mass)
    setup(model)
    dt = 0.8 * model.getStableTimeStep()
    model.setTimeStep(dt)
    energies = []
    for _ in range(steps):
        model.solveStep()
        energies.append((model.getEnergy("potential"), model.getEnergy("kinetic")))
    out = dt, model.getDisplacement().copy(), model.getVelocity().copy(), np.array(energies)
    model.close()
    return out


def test_input_file_script_on_a_gmsh_mesh(tmp_path):
    """The flow of the reference's custom-material script: parseInput,
    SolidMechanicsModel(mesh) with the law registered in Python, applyBC on
    the mesh's named group, an initial displacement written into
    getDisplacement(), then solveStep with the energies."""
    dat = tmp_path / "material.dat"
    dat.write_text("material isotropic_elastic [\n  name = fictive\n  rho = 1.  # density\n"
                   "  E = 1.\n  nu = .3\n]\n")

    def setup(model):
        model.applyBC(aka.FixedValue(0.0, aka._x), "fixed")
        model.applyBC(aka.FixedValue(0.0, aka._y), "fixed")
        x = model.mesh.getNodes()
        u = model.getDisplacement()
        u[:, 0] = 0.01 * np.sin(x[:, 0] + 2 * x[:, 1])
        u[:, 1] = 0.005 * np.cos(3 * x[:, 0])
        u[model.mesh.getNodeGroup("fixed")] = 0.0

    mesh = aka.Mesh(2)
    mesh.read(MSH)
    aka.parseInput(str(dat))
    python_law = aka.SolidMechanicsModel(mesh)
    got = run(python_law, mesh, setup, 100)
    assert python_law.getMaterial("fictive").getReal("nu") == 0.3
    builtin = aka.SolidMechanicsModel(mesh, [aka.MaterialElastic(rho=1.0, E=1.0, nu=0.3)],
                                      precision=aka.MODE_FP64)
    want = run(builtin, mesh, setup, 100)
    assert got[0] == pytest.approx(want[0], rel=1e-14)  # same push wave speed
    assert rel(got[1], want[1]) <= 1e-10 and rel(got[2], want[2]) <= 1e-10
    assert np.abs(got[3] - want[3]).max() <= 1e-10 * np.abs(want[3]).max()
    assert got[3][:, 0].max() > 0  # the pulse stores elastic energy


def test_distorted_hexahedra():
    mesh = block_hexahedron8(3, 1.0)
    rng = np.random.default_rng(17)
    x = mesh.nodes
    inner = np.all((x > 1e-9) & (x < 1 - 1e-9), axis=1)
    x[inner] += rng.uniform(-0.08, 0.08, (inner.sum(), 3))
    mp.parse_input_text("material isotropic_elastic [ name = steel\n rho = 7800\n E = 2e11\n"
                        " nu = 0.3 ]\n")
    v0 = rng.normal(0.0, 1.0, x.shape)
    bottom = np.isclose(x[:, 2], 0.0)
    v0[bottom] = 0.0

    def setup(model):
        blocked = model.getBlockedDOFs()
        blocked[bottom] = True
        model.getVelocity()[...] = v0

    got = run(aka.SolidMechanicsModel(mesh), mesh, setup, 100)
    want = run(aka.SolidMechanicsModel(mesh, [aka.MaterialElastic(rho=7800, E=2e11, nu=0.3)],
                                       precision=aka.MODE_FP64), mesh, setup, 100)
    assert got[0] == pytest.approx(want[0], rel=1e-14)
    assert rel(got[1], want[1]) <= 1e-10 and rel(got[2], want[2]) <= 1e-10
    assert np.abs(got[3] - want[3]).max() <= 1e-10 * np.abs(want[3]).max()


def test_material_selector_in_a_model():
    """setMaterialSelector with the physical names, as
    test_material_selector.cc (with the densities the library needs): each
    segment of material_selector.msh takes the built-in elastic material of
    its group's name, seen through getMaterial(name).getElementFilter."""
    mesh = aka.Mesh(1)
    mesh.read(os.path.join(os.path.dirname(__file__), "golden", "msh", "material_selector.msh"))
    mp.parse_input_text("material elastic [ name = chocolate\n rho = 1\n E = 2\n nu = 0 ]\n"
                        "material elastic [ name = chewing-gum\n rho = 1\n E = 1\n nu = 0 ]\n"
                        "material elastic [ name = candy\n rho = 1\n E = 3\n nu = 0 ]\n")
    model = aka.SolidMechanicsModel(mesh)
    model.setMaterialSelector(aka.MeshDataMaterialSelectorString("physical_names", model))
    model.initFull(_analysis_method=aka._explicit_lumped_mass)
    for name, element in (("chocolate", 0), ("chewing-gum", 1), ("candy", 2)):
        assert model.getMaterial(name).getElementFilter(aka._segment_2).tolist() == [element]
        assert model.getMaterialIndex(name) == element
    # the stable step: each segment's length over its own material's wave speed
    x = mesh.getNodes()[:, 0]
    lengths = np.abs(x[mesh.connectivity[:, 1]] - x[mesh.connectivity[:, 0]])
    assert model.getStableTimeStep() == pytest.approx((lengths / np.sqrt([2.0, 1.0, 3.0])).min(),
                                                      rel=1e-12)
    model.close()
