"""FE^2 building blocks: periodic voxel RVEs and their macroscopic samples.

The micro problem is a cube of n^3 hexahedron_8 voxels with periodic nodes,
loaded by a macroscopic displacement gradient H (F = I + H); its homogenised
first Piola-Kirchhoff stress is what the macroscopic material
(MaterialFE2, extra_packages/extra-materials/src/material_FE2/material_FE2.hh:
40-101 in the reference, which linearises the same micro-macro coupling)
returns at each quadrature point.
"""
from __future__ import annotations

import math

import numpy as np

from . import _abi

SEED = 20261203


def sphere_inclusion_rve(cells=16, volume_fraction=0.2, length=1.0):
    """Voxel materials of a cube with one centred spherical inclusion of the
    given volume fraction (radius (vf 3 / 4 pi)^(1/3) L), voxelised by
    element centroid: 0 = matrix, 1 = inclusion. Returns (voxel_material
    uint8 n^3 with x fastest, actual voxel volume fraction)."""
    n = int(cells)
    r = (volume_fraction * 3.0 / (4.0 * math.pi)) ** (1.0 / 3.0) * length
    c = (np.arange(n) + 0.5) * (length / n) - 0.5 * length
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    inside = (x * x + y * y + z * z) <= r * r
    vm = inside.astype(np.uint8).ravel()  # index x + n (y + n z)
    return vm, float(vm.mean())


def matrix_inclusion_materials(lam=1.0e6, mu=0.4e6, contrast=10.0, rho=1100.0):
    """Neo-Hookean matrix (lambda, mu) and an inclusion `contrast` times
    stiffer, as material descriptors (E, nu derived from the Lame moduli)."""
    def nh(l, m):
        return dict(kind=_abi.MATERIAL_NEOHOOKEAN, rho=rho, E=m * (3 * l + 2 * m) / (l + m),
                    nu=l / (2 * (l + m)), lam=l, mu=m)
    return [nh(lam, mu), nh(contrast * lam, contrast * mu)]


def sample_gradients(count, seed=SEED, amplitude=0.3, min_det=0.5):
    """Macroscopic displacement gradients H with H_ij ~ U[-a, a], rejecting
    det(I + H) < min_det. Returns (count, 3, 3) FP64."""
    rng = np.random.default_rng(seed)
    out = np.empty((0, 3, 3))
    while out.shape[0] < count:
        H = rng.uniform(-amplitude, amplitude, (2 * (count - out.shape[0]) + 16, 3, 3))
        ok = np.linalg.det(np.eye(3) + H) >= min_det
        out = np.concatenate([out, H[ok]])
    return out[:count].copy()


def in_envelope(H, amplitude=0.3, min_det=0.5):
    """The training envelope of the surrogate: |H_ij| <= a and det F >= d."""
    H = np.asarray(H).reshape(-1, 3, 3)
    return (np.abs(H).max(axis=(1, 2)) <= amplitude) & \
           (np.linalg.det(np.eye(3) + H) >= min_det)
