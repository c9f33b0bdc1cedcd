"""The fused step's planned shared-memory layout on meshes that stress it,
against the CPU oracle (B200).

The layout (node positions, coloured contribution slots, node sums cut in
pieces of six with a second level for nodes cut in several) is built on the
host from the mesh; these cases reach the parts the structured benchmark
meshes do not:
  - a star of 192 tetrahedra around one node: that node has 192
    contributions in one chunk (32 pieces, the second level's loop past its
    unrolled part) while every other node has at most a few;
  - a tetrahedral cube with randomly permuted node ids, shuffled elements and
    jittered coordinates, with the default patches, one-chunk patches and
    patches of several chunks.
Tolerances as in test_gpu_parity.py: FP64 <= 1e-10, FP32-bulk <= 1e-5 on u
(relative to the field's maximum).
"""
import numpy as np
import pytest

from akantu_b200 import _abi, configs
from akantu_b200.mesh import Mesh, cube_tetrahedron4
from tests.golden_cases import OracleAdapter

pytestmark = pytest.mark.gpu

SEED = 20261203


def rel(x, ref):
    s = np.abs(ref).max()
    return np.abs(x - ref).max() / (s if s > 0 else 1.0)


def star_mesh(k=4):
    """Surface of [-1, 1]^3 cut into k x k squares per face, two triangles per
    square, each joined to the centre node 0 (positive volumes)."""
    pts = {}
    nodes = [(0.0, 0.0, 0.0)]

    def node(p):
        key = tuple(np.round(p, 12))
        if key not in pts:
            pts[key] = len(nodes)
            nodes.append(key)
        return pts[key]
    tets = []
    g = np.linspace(-1.0, 1.0, k + 1)
    for axis in range(3):
        for side in (-1.0, 1.0):
            for i in range(k):
                for j in range(k):
                    quad = []
                    for a, b in ((i, j), (i + 1, j), (i + 1, j + 1), (i, j + 1)):
                        p = np.zeros(3)
                        p[axis] = side
                        p[(axis + 1) % 3] = g[a]
                        p[(axis + 2) % 3] = g[b]
                        quad.append(node(p))
                    for tri in ((quad[0], quad[1], quad[2]), (quad[0], quad[2], quad[3])):
                        t = [0, *tri]
                        x = np.array([nodes[v] for v in t])
                        if np.linalg.det(x[1:] - x[0]) < 0:
                            t[2], t[3] = t[3], t[2]
                        tets.append(t)
    return Mesh(3, _abi.TETRAHEDRON_4, np.array(nodes), np.array(tets, dtype=np.uint32))


def scrambled_cube(n=10):
    """cube_tetrahedron4(n) with permuted node ids, shuffled elements and
    coordinates jittered by up to 0.1 of a cell."""
    base = cube_tetrahedron4(n, 1.0)
    rng = np.random.default_rng(SEED)
    x = base.nodes + rng.uniform(-0.1, 0.1, base.nodes.shape) / n
    perm = rng.permutation(len(x))          # old id -> new id
    nodes = np.empty_like(x)
    nodes[perm] = x
    conn = perm[base.connectivity.astype(np.int64)].astype(np.uint32)
    conn = conn[rng.permutation(len(conn))]
    return Mesh(3, _abi.TETRAHEDRON_4, nodes, conn)


def workload(mesh, fixed):
    rng = np.random.default_rng(SEED + 1)
    x = mesh.nodes
    blocked = np.zeros_like(x, dtype=np.uint8)
    blocked[fixed] = 1
    v0 = rng.normal(0.0, 1.0, x.shape)
    v0[blocked.astype(bool)] = 0.0
    mat = dict(kind=_abi.MATERIAL_ELASTIC, rho=2700.0, E=70e9, nu=0.33)
    return dict(mesh=mesh, materials=[mat], blocked=blocked, u0=np.zeros_like(x), v0=v0,
                dt_factor=0.8)


class Gpu:
    def __init__(self, w, mode, **patch):
        from akantu_b200.model import SolidMechanicsModel, material_from_dict
        self.m = SolidMechanicsModel(w["mesh"], [material_from_dict(mm) for mm in w["materials"]],
                                     precision=mode, **patch)
        self.m.initFull()

    def get(self, f):
        return np.array(self.m.getField(f))

    def set(self, f, v):
        self.m.setField(f, v)

    def set_blocked(self, b):
        self.m.setBlockedDOFs(b)

    def stable_time_step(self):
        return self.m.getStableTimeStep()

    def set_time_step(self, dt):
        self.m.setTimeStep(dt)


def compare(w, mode, steps, **patch):
    cpu = OracleAdapter(w["mesh"], w["materials"])
    dev = Gpu(w, mode, **patch)
    configs.setup_model(cpu, w)
    configs.setup_model(dev, w)
    cpu.solve_steps(steps)
    dev.m.solveSteps(steps)
    tol = 1e-10 if mode == _abi.MODE_FP64 else 1e-5
    for f in (_abi.FIELD_DISPLACEMENT, _abi.FIELD_VELOCITY):
        e = rel(dev.get(f), cpu.get(f))
        assert e <= (tol if f == _abi.FIELD_DISPLACEMENT else 10 * tol), (f, e, patch)
    dev.m.close()


@pytest.mark.parametrize("mode", [_abi.MODE_FP64, _abi.MODE_FP32_BULK], ids=["fp64", "fp32bulk"])
def test_star_of_tetrahedra(mode):
    mesh = star_mesh(4)
    assert len(mesh.connectivity) == 192
    fixed = np.isclose(mesh.nodes[:, 2], -1.0)
    compare(workload(mesh, fixed), mode, 100)


@pytest.mark.parametrize("mode", [_abi.MODE_FP64, _abi.MODE_FP32_BULK], ids=["fp64", "fp32bulk"])
@pytest.mark.parametrize("patch", [dict(), dict(patch_elements=256, patch_nodes=160),
                                   dict(patch_elements=1536, patch_nodes=600)],
                         ids=["default", "one_chunk", "six_chunks"])
def test_scrambled_cube(mode, patch):
    mesh = scrambled_cube(10)
    fixed = mesh.nodes[:, 2] < 0.05
    compare(workload(mesh, fixed), mode, 100, **patch)


@pytest.mark.parametrize("mode", [_abi.MODE_FP64, _abi.MODE_FP32_BULK], ids=["fp64", "fp32bulk"])
def test_single_mesh_schedules_match_a_batch_of_one(mode):
    """A single mesh against a batch holding only that mesh (same patches,
    the batch's per-instance time step and instance lookups): u, v and a bit
    for bit, with one CTA per patch and with a persistent grid of 5 CTAs
    (several patches per CTA, the chunk-record buffers and mbarrier phases
    carried from patch to patch), and the kinetic energy to rounding."""
    from akantu_b200.batch import BatchModel
    mesh = scrambled_cube(10)
    w = workload(mesh, mesh.nodes[:, 2] < 0.05)
    patch = dict(patch_elements=256, patch_nodes=160)
    state = (_abi.FIELD_DISPLACEMENT, _abi.FIELD_VELOCITY, _abi.FIELD_ACCELERATION)
    ref = BatchModel([mesh], w["materials"], precision=mode, **patch)
    ref.initFull()
    ref.setBlockedDOFs(w["blocked"])
    ref.setField(_abi.FIELD_DISPLACEMENT, w["u0"])
    ref.setField(_abi.FIELD_VELOCITY, w["v0"])
    dt = w["dt_factor"] * ref.getStableTimeSteps()
    ref.setTimeSteps(dt)
    ref.solveSteps(100)
    want = {f: np.array(ref.getField(f)) for f in state}
    ek = ref.getEnergies("kinetic")[0]
    ref.close()
    for grid in (0, 5):
        dev = Gpu(w, mode, patch_grid=grid, **patch)
        assert configs.setup_model(dev, w) == dt[0]
        dev.m.solveSteps(100)
        for f in state:
            assert np.array_equal(dev.get(f), want[f]), (grid, f)
        assert abs(dev.m.getEnergy("kinetic") - ek) <= 1e-13 * ek, grid
        dev.m.close()
