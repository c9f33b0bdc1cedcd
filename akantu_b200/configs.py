"""The synthetic workloads of the explicit path (seeded, fixed sizes).

  plate_tri3     2D plane-strain bar, 200 x 20 squares over 10 m x 1 m split
                 into 8000 triangle_3 (4221 nodes), E = 210 GPa, nu = 0.3,
                 rho = 7800; left edge fixed; u_x = 1e-4 sin(pi x / 10);
                 dt = 0.8 x stable; 1000 steps.
  cube_tet4      100^3 cubes x 6 tetrahedron_4 (6 M elements, 1 030 301
                 nodes) over a 1 m cube, E = 70 GPa, nu = 0.33, rho = 2700;
                 bottom face fixed, top face v_z = 1 m/s; 1000 steps.
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
from .mesh import block_hexahedron8, cube_tetrahedron4, plate_triangle3

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


def setup_model(model, w):
    """Applies a workload's boundary and initial conditions to a model facade
    (get/set/set_blocked/stable_time_step/set_time_step) and returns dt."""
    model.set_blocked(w["blocked"])
    model.set(_abi.FIELD_DISPLACEMENT, w["u0"])
    model.set(_abi.FIELD_VELOCITY, w["v0"])
    dt = w["dt_factor"] * model.stable_time_step()
    model.set_time_step(dt)
    return dt
