"""Shared FE^2 test cases: RVE microstructures and their oracle twins."""
import numpy as np

from akantu_b200 import _abi, fe2


def lame(m):
    """lambda, mu as libakb derives them from (E, nu) (material_elastic.cc:83-107)."""
    E, nu = m["E"], m["nu"]
    return nu * E / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))


def rve_case(cells=8, homogeneous=False, contrast=10.0):
    vm, vf = fe2.sphere_inclusion_rve(cells)
    if homogeneous:
        vm = np.zeros_like(vm)
    mats = fe2.matrix_inclusion_materials(contrast=contrast)
    return vm, mats


def oracle_rve(cells, vm, mats, length=1.0):
    from oracle.oracle import OracleRVE
    lm = [lame(m) for m in mats]
    return OracleRVE(cells, length, vm, [a for a, _ in lm], [b for _, b in lm],
                     [1 if m["kind"] == _abi.MATERIAL_NEOHOOKEAN else 0 for m in mats])


def neohookean_P(H, lam, mu):
    """First Piola-Kirchhoff stress of the neo-Hookean law at F = I + H."""
    F = np.eye(3) + H
    C = F.T @ F
    Ci = np.linalg.inv(C)
    J = np.linalg.det(F)
    S = mu * (np.eye(3) - Ci) + lam * np.log(J) * Ci
    return F @ S


def random_rotation(rng):
    q, r = np.linalg.qr(rng.normal(size=(3, 3)))
    q = q @ np.diag(np.sign(np.diag(r)))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q
