"""The synthetic workloads of the explicit path (seeded, fixed sizes).

  plate_tri3     2D plane-strain bar, 200 x 20 squares over 10 m x 1 m split
                 into 8000 triangle_3 (4221 nodes), E = 210 GPa, nu = 0.3,
                 rho = 7800; left edge fixed; u_x = 1e-4 sin(pi x / 10);
                 dt = 0.8 x stable; 1000 steps.
  cube_tet4      100^3 cubes x 6 tetrahedron_4 (6 M elements, 1 030 301
                 nodes) over a 1 m cube, E = 70 GPa, nu = 0.33, rho = 2700;
                 bottom face fixed, top face v_z = 1 m/s; 1000 steps.
  bar_tet4       cube_tet4 stacked nslabs times along z: n x n x (n nslabs)
                 cubes x 6 tetrahedron_4 over 1 m x 1 m x nslabs m, same
                 material, bottom face fixed, top face v_z = 1 m/s; cut into
                 its nslabs cubes along z (one part per GPU, weak scaling).
  block_hex8     128^3 hexahedron_8 (2 097 152 elements, 2 146 689 nodes)
                 over a 1.28 m block, neo-Hookean lambda = 1 MPa, mu = 0.4 MPa
                 (E, nu derived), rho = 1100; face x = 0 fixed; v ~ N(0, 0.05)
                 per component (seed 20261203), zero on fixed DOFs; 2000 steps.

Each builder takes a size parameter so the tests run the same workload at a
size the CPU oracle finishes in seconds.
"""
from __future__ import annotations

import math

import numpy as np

from . import _abi
from .mesh import Mesh, block_hexahedron8, box_tetrahedron4, cube_tetrahedron4, plate_triangle3

SEED = 20261203


def plate_tri3(nx=200, ny=20, lx=10.0, ly=1.0):
    mesh = plate_triangle3(nx, ny, lx, ly)
    x = mesh.nodes
    blocked = np.zeros_like(x, dtype=np.uint8)
    blocked[np.isclose(x[:, 0], 0.0)] = 1
    u0 = np.zeros_like(x)
    u0[:, 0] = 1e-4 * np.sin(math.pi * x[:, 0] / lx)
    u0[blocked.astype(bool)] = 0.0
    mat = dict(kind=_abi.MATERIAL_ELASTIC, rho=7800.0, E=210e9, nu=0.3)
    return dict(name="plate_tri3", mesh=mesh, materials=[mat], blocked=blocked, u0=u0,
                v0=np.zeros_like(x), dt_factor=0.8, steps=1000)


def cube_tet4(n=100, length=1.0):
    mesh = cube_tetrahedron4(n, length)
    x = mesh.nodes
    blocked = np.zeros_like(x, dtype=np.uint8)
    blocked[np.isclose(x[:, 2], 0.0)] = 1
    v0 = np.zeros_like(x)
    v0[np.isclose(x[:, 2], length), 2] = 1.0
    mat = dict(kind=_abi.MATERIAL_ELASTIC, rho=2700.0, E=70e9, nu=0.33)
    return dict(name="cube_tet4", mesh=mesh, materials=[mat], blocked=blocked,
                u0=np.zeros_like(x), v0=v0, dt_factor=0.8, steps=1000)


def bar_tet4(n=100, nslabs=1, length=1.0):
    """The whole bar as one mesh (for sizes a test can hold)."""
    mesh = box_tetrahedron4(n, n, n * nslabs, length, length, length * nslabs)
    x = mesh.nodes
    blocked, v0 = _bar_conditions(x[:, 2], length * nslabs)
    mat = dict(kind=_abi.MATERIAL_ELASTIC, rho=2700.0, E=70e9, nu=0.33)
    return dict(name="bar_tet4", mesh=mesh, materials=[mat], blocked=blocked,
                u0=np.zeros_like(x), v0=v0, dt_factor=0.8, steps=1000)


def _bar_conditions(z, top):
    blocked = np.zeros((len(z), 3), dtype=np.uint8)
    blocked[np.isclose(z, 0.0)] = 1
    v0 = np.zeros((len(z), 3))
    v0[np.isclose(z, top), 2] = 1.0
    return blocked, v0


def bar_tet4_slabs(n, nslabs, here, length=1.0):
    """The parts of bar_tet4(n, nslabs) cut into its nslabs cubes along z
    (part r: the cells r n <= k < (r + 1) n), built directly, without the
    whole mesh: for each part in `here` a decompose.MeshPart with global
    node ids, its local mesh (node coordinates bit-identical to the whole
    mesh's), its interface planes (bottom shared with part r - 1, top with
    part r + 1) and their holders. Also returns the whole mesh's node count
    and its blocked / initial-velocity arrays (whole-mesh, for set_field)."""
    from .decompose import MeshPart
    p = n + 1
    plane = p * p
    lz, nz = length * nslabs, n * nslabs
    h = lz / nz  # the whole mesh's spacing, _grid_nodes_3d
    xs = np.arange(p, dtype=np.float64) * (length / n)
    local = box_tetrahedron4(n, n, n, length, length, length)
    ne = len(local.connectivity)
    parts = []
    for r in here:
        zs = np.arange(r * n, (r + 1) * n + 1, dtype=np.float64) * h
        Z, Y, X = np.meshgrid(zs, xs, xs, indexing="ij")
        coords = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
        mesh = Mesh(3, _abi.TETRAHEDRON_4, coords, local.connectivity)
        nodes = np.arange(r * n * plane, r * n * plane + p * plane, dtype=np.int64)
        lo = np.arange(plane) if r > 0 else np.zeros(0, np.int64)
        hi = n * plane + np.arange(plane) if r < nslabs - 1 else np.zeros(0, np.int64)
        iface = np.concatenate([lo, hi]).astype(np.uint32)
        holders = np.concatenate([np.repeat([[r - 1, r]], len(lo), 0).ravel(),
                                  np.repeat([[r, r + 1]], len(hi), 0).ravel()]).astype(np.int64)
        owned = np.ones(len(nodes), dtype=bool)
        owned[lo] = False  # the bottom plane belongs to the part below
        parts.append(MeshPart(r, np.arange(r * ne, (r + 1) * ne, dtype=np.int64), nodes, mesh,
                              iface, None, owned, np.arange(0, 2 * len(iface) + 1, 2), holders))
    nb_nodes = plane * (nz + 1)
    z = np.repeat(np.arange(nz + 1, dtype=np.float64) * h, plane)
    blocked, v0 = _bar_conditions(z, lz)
    mat = dict(kind=_abi.MATERIAL_ELASTIC, rho=2700.0, E=70e9, nu=0.33)
    return dict(name="bar_tet4", parts=parts, nb_nodes=nb_nodes, materials=[mat],
                blocked=blocked, u0=np.zeros((nb_nodes, 3)), v0=v0, dt_factor=0.8, steps=1000)


def neohookean_from_lame(lam, mu, rho):
    nu = lam / (2 * (lam + mu))
    E = mu * (3 * lam + 2 * mu) / (lam + mu)
    return dict(kind=_abi.MATERIAL_NEOHOOKEAN, rho=rho, E=E, nu=nu)


def block_hex8(n=128, length=1.28, seed=SEED):
    mesh = block_hexahedron8(n, length)
    x = mesh.nodes
    blocked = np.zeros_like(x, dtype=np.uint8)
    blocked[np.isclose(x[:, 0], 0.0)] = 1
    rng = np.random.default_rng(seed)
    v0 = rng.normal(0.0, 0.05, x.shape)
    v0[blocked.astype(bool)] = 0.0
    mat = neohookean_from_lame(1.0e6, 0.4e6, 1100.0)
    return dict(name="block_hex8", mesh=mesh, materials=[mat], blocked=blocked,
                u0=np.zeros_like(x), v0=v0, dt_factor=0.8, steps=2000)


def plates_batch(n_instances=4096, seed=SEED, min_elems=100, max_elems=20000):
    """Independent triangle_3 plane-strain plates of uneven size: element
    counts log-uniform in [min_elems, max_elems], aspect a ~ U[1, 8],
    nx = round(sqrt(n a / 2)), ny = round(sqrt(n / (2 a))) squares of size
    1/ny m (plate 1 m wide, a m long), two triangles per square; E ~ U[1, 200]
    GPa, nu ~ U[0.2, 0.4], rho ~ U[1000, 8000]; left edge fixed; initial
    u_x = 1e-4 L sin(pi x / L); dt = 0.8 x the instance's stable step;
    500 steps."""
    rng = np.random.default_rng(seed)
    n_el = np.exp(rng.uniform(np.log(min_elems), np.log(max_elems), n_instances))
    aspect = rng.uniform(1.0, 8.0, n_instances)
    E = rng.uniform(1e9, 200e9, n_instances)
    nu = rng.uniform(0.2, 0.4, n_instances)
    rho = rng.uniform(1000.0, 8000.0, n_instances)
    meshes, mats, blocked, u0 = [], [], [], []
    for k in range(n_instances):
        nx = max(1, int(round(math.sqrt(n_el[k] * aspect[k] / 2))))
        ny = max(1, int(round(math.sqrt(n_el[k] / (2 * aspect[k])))))
        lx = nx / ny  # square cells of size 1/ny over a 1 m wide plate
        mesh = plate_triangle3(nx, ny, lx, 1.0)
        x = mesh.nodes
        b = np.zeros_like(x, dtype=np.uint8)
        b[np.isclose(x[:, 0], 0.0)] = 1
        u = np.zeros_like(x)
        u[:, 0] = 1e-4 * lx * np.sin(math.pi * x[:, 0] / lx)
        u[b.astype(bool)] = 0.0
        meshes.append(mesh)
        mats.append(dict(kind=_abi.MATERIAL_ELASTIC, rho=float(rho[k]), E=float(E[k]),
                         nu=float(nu[k])))
        blocked.append(b)
        u0.append(u)
    return dict(name="plates_tri3_batch", meshes=meshes, materials=mats, blocked=blocked,
                u0=u0, dt_factor=0.8, steps=500)


def setup_batch(batch, w):
    """Boundary and initial conditions of plates_batch on a BatchModel;
    returns the per-instance time steps."""
    batch.setBlockedDOFs(np.concatenate(w["blocked"]))
    batch.setField(_abi.FIELD_DISPLACEMENT, np.concatenate(w["u0"]))
    batch.setField(_abi.FIELD_VELOCITY, np.zeros((batch.node_offsets[-1], 2)))
    dts = w["dt_factor"] * batch.getStableTimeSteps()
    batch.setTimeSteps(dts)
    return dts


def setup_model(model, w):
    """Applies a workload's boundary and initial conditions to a model facade
    (get/set/set_blocked/stable_time_step/set_time_step) and returns dt."""
    model.set_blocked(w["blocked"])
    model.set(_abi.FIELD_DISPLACEMENT, w["u0"])
    model.set(_abi.FIELD_VELOCITY, w["v0"])
    dt = w["dt_factor"] * model.stable_time_step()
    model.set_time_step(dt)
    return dt
